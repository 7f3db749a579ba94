// Blocked triangular solve — replaces mojoBLAS trsm (src/level3/trsm.mojo:20-275).
//
// The reference runs an unblocked, single-threaded substitution per right-hand
// side column (:105-168).  Here the triangle is split recursively at a multiple
// of 64 rows until a diagonal block of at most 64 rows is left:
//     effective lower op(A):  X1 = solve(A11, B1);  B2 -= op(A)21 X1;  X2 = solve(A22, B2)
//     effective upper op(A):  X2 = solve(A22, B2);  B1 -= op(A)12 X2;  X1 = solve(A11, B1)
// The off-diagonal updates are gemm calls in the caller's precision mode (plain
// FP32/FP64, BF16x3/x6 split, or Ozaki int8 slices), so almost all flops run in
// large GEMMs.  Diagonal blocks are solved by `diag_solve_kernel`: the block is
// staged once per CTA in shared memory, and each group of eight lanes owns one
// right-hand-side column, eight rows per lane, broadcasting the pivot with a
// shuffle — the reference's column-axpy substitution (:130-148), scaled by the
// reciprocal of the diagonal, with the same skip of zero pivots.
//
// Right side: X op(A) = alpha B  <=>  op(A)^T X^T = alpha B^T.  B is transposed
// into a workspace (alpha folded in), solved from the left with the transpose
// flag flipped, and transposed back.  This follows Netlib; the reference's
// right-side Trans branches ignore the transpose (:224-273).
//
// Iterative refinement (refine > 0): keep alpha*B, solve, form
// R = alpha*B - op(A) X with the accurate residual product (FP64 / BF16x6 /
// 8-slice Ozaki by recursion, diagonal blocks in the input precision), solve
// op(A) D = R in the caller's mode and add D to X.
//
// Triangular multiply (trmm, src/level3/trmm.mojo:20-305), at the end of this
// file, needs no recursion: it is one GEMM of a dense copy of the triangle with a
// copy of B, each output tile running only the slabs of the reduction where the
// triangle is nonzero.
#include "mbg_internal.cuh"
#include "block_solve.cuh"

#include <vector>

namespace mbg {

namespace {

constexpr int NB = 64;        // diagonal block (leaf) size
using bs::BS_COLS;
using bs::BS_THREADS;
using bs::bs_smem_bytes;
using bs::block_solve_kernel;
constexpr int DS_WARPS = 8;   // columns per CTA in flight

// Solves op(A)[0:nb, 0:nb] X = B[0:nb, :] in place for nb <= 64.
// LOWER: effective op(A) lower triangular (forward), else upper (backward).
// The block is staged once per CTA in shared memory with the reciprocals of its
// diagonal; its rows are stored interleaved (row q*8+j at position j*8+q of the
// column) so that the eight lanes serving one right-hand side read eight
// consecutive words.  Each group of eight lanes owns one column, eight rows per
// lane in registers, and runs the reference's column-axpy substitution
// (src/level3/trsm.mojo:111-148): the pivot x_l is broadcast within the group
// by a shuffle, scaled by 1/a_ll (a multiply: a division would put a long
// software sequence on every step's dependency chain), and every lane updates
// its rows below (above) it.  Zero pivots are skipped as in the reference, by
// predication so the four columns of a warp do not diverge.
template <typename T, bool LOWER, bool TRANS, bool UNIT>
__global__ void __launch_bounds__(DS_WARPS * 32)
diag_solve_kernel(int nb, i64 ncols, const T* __restrict__ A, i64 lda, T* __restrict__ B, i64 ldb) {
    constexpr int LD = NB + 1;
    __shared__ T Ls[NB * LD];
    __shared__ T inv[NB];
    // stage the whole nb x nb block (compile-time 64 x 64 indexing, coalesced);
    // entries of the other triangle are copied but never read
#pragma unroll 4
    for (int e = threadIdx.x; e < NB * NB; e += DS_WARPS * 32) {
        const int fast = e & (NB - 1), slow = e >> 6;  // fast index runs along contiguous memory
        const int i = TRANS ? slow : fast, l = TRANS ? fast : slow;
        if (i < nb && l < nb)
            Ls[l * LD + (i & 7) * 8 + (i >> 3)] = TRANS ? A[l + (i64)i * lda] : A[i + (i64)l * lda];
    }
    __syncthreads();
    for (int l = threadIdx.x; l < nb; l += blockDim.x)
        inv[l] = UNIT ? T(1) : T(1) / Ls[l * LD + (l & 7) * 8 + (l >> 3)];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int q = lane & 7;      // rows q*8 .. q*8+7 of the column
    const int grp = lane >> 3;   // which of the warp's four columns
    const i64 cols_per_cta = DS_WARPS * 4;
    for (i64 j0 = (i64)blockIdx.x * cols_per_cta; j0 < ncols; j0 += (i64)gridDim.x * cols_per_cta) {
        const i64 j = j0 + (threadIdx.x >> 5) * 4 + grp;
        const bool active = j < ncols;
        T* bj = B + (active ? j : 0) * ldb;
        T x[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const int r = q * 8 + s;
            x[s] = (active && r < nb) ? bj[r] : T(0);
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            const int l = LOWER ? u : NB - 1 - u;
            if (l >= nb) continue;  // uniform: nb is the same for every thread
            const int owner = l >> 3, slot = l & 7;
            T xl = __shfl_sync(0xffffffffu, x[slot], owner, 8);
            const bool live = xl != T(0);  // the reference skips zero pivots
            if (!UNIT) xl *= inv[l];
            if (q == owner && live) x[slot] = xl;
            const T* col = Ls + l * LD;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const int r = q * 8 + s;
                const bool below = LOWER ? (r > l) : (r < l);
                const T a = col[s * 8 + q];
                if (live && below) x[s] -= xl * a;
            }
        }
        if (active) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const int r = q * 8 + s;
                if (r < nb) bj[r] = x[s];
            }
        }
    }
}

// R[0:nb, :] -= tri(op(A)) X[0:nb, :] for one diagonal block (residual leaf).
template <typename T, bool LOWER, bool TRANS, bool UNIT>
__global__ void __launch_bounds__(DS_WARPS * 32)
diag_residual_kernel(int nb, i64 ncols, const T* __restrict__ A, i64 lda, const T* __restrict__ X,
                     i64 ldx, T* __restrict__ R, i64 ldr) {
    __shared__ T Ls[NB * (NB + 1)];
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        int i, l;
        if (TRANS) { l = e % nb; i = e / nb; } else { i = e % nb; l = e / nb; }
        const bool in_tri = LOWER ? (i >= l) : (i <= l);
        T v = T(0);
        if (in_tri && !(UNIT && i == l)) v = TRANS ? A[l + (i64)i * lda] : A[i + (i64)l * lda];
        if (UNIT && i == l) v = T(1);
        Ls[l * (NB + 1) + i] = v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (i64 j = (i64)blockIdx.x * DS_WARPS + warp; j < ncols; j += (i64)gridDim.x * DS_WARPS) {
        const T* xj = X + j * ldx;
        T a0 = T(0), a1 = T(0);
        for (int l = 0; l < nb; ++l) {
            const T xl = xj[l];
            a0 = fma(Ls[l * (NB + 1) + lane], xl, a0);
            if (lane + 32 < nb) a1 = fma(Ls[l * (NB + 1) + lane + 32], xl, a1);
        }
        T* rj = R + j * ldr;
        if (lane < nb) rj[lane] -= a0;
        if (lane + 32 < nb) rj[lane + 32] -= a1;
    }
}

template <typename T>
__global__ void transpose_scale_kernel(i64 rows, i64 cols, T alpha, const T* __restrict__ src,
                                       i64 lds, T* __restrict__ dst, i64 ldd) {
    __shared__ T tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const i64 i = i0 + threadIdx.x, j = j0 + r;
        if (i < rows && j < cols) tile[r][threadIdx.x] = alpha * src[i + j * lds];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const i64 j = j0 + threadIdx.x, i = i0 + r;
        if (i < rows && j < cols) dst[j + i * ldd] = tile[threadIdx.x][r];
    }
}

template <typename T>
__global__ void axpy_matrix_kernel(i64 m, i64 n, T alpha, const T* __restrict__ x, i64 ldx,
                                   T* __restrict__ y, i64 ldy) {
    for (i64 j = blockIdx.y; j < n; j += gridDim.y)
        for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x)
            y[i + j * ldy] += alpha * x[i + j * ldx];
}

template <typename T>
__global__ void copy_scale_kernel(i64 m, i64 n, T alpha, const T* __restrict__ x, i64 ldx,
                                  T* __restrict__ y, i64 ldy) {
    for (i64 j = blockIdx.y; j < n; j += gridDim.y)
        for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x)
            y[i + j * ldy] = alpha * x[i + j * ldx];
}

unsigned ds_grid(i64 ncols) {  // residual leaf: one warp per column
    return (unsigned)imax(1, imin(cdiv(ncols, DS_WARPS), 148 * 8));
}
unsigned ds_solve_grid(i64 ncols) {  // solve leaf: four columns per warp
    const i64 cap = tuning().trsm_leaf_ctas > 0 ? tuning().trsm_leaf_ctas : 148 * 8;
    return (unsigned)imax(1, imin(cdiv(ncols, DS_WARPS * 4), cap));
}

template <typename T>
int launch_diag_solve(bool lower, bool trans, bool unit, int nb, i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    ProfScope prof("trsm_diag_solve");
    const dim3 g(ds_solve_grid(n)), blk(DS_WARPS * 32);
    cudaStream_t s = stream();
#define DS(L, TR, U) diag_solve_kernel<T, L, TR, U><<<g, blk, 0, s>>>(nb, n, a, lda, b, ldb)
    if (lower) {
        if (trans) { if (unit) DS(true, true, true); else DS(true, true, false); }
        else { if (unit) DS(true, false, true); else DS(true, false, false); }
    } else {
        if (trans) { if (unit) DS(false, true, true); else DS(false, true, false); }
        else { if (unit) DS(false, false, true); else DS(false, false, false); }
    }
#undef DS
    return check_launch("trsm_diag_solve");
}

// Largest nb block_solve_kernel takes: its strip (32 columns x nb rows) and the
// two staging buffers must fit the 227 KB of shared memory a CTA may use.
template <typename T>
constexpr int bs_max_rows() { return sizeof(T) == 8 ? 512 : 1024; }

template <typename T, bool L, bool TR, bool U>
int launch_block_solve_t(int nb, i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    auto kern = block_solve_kernel<T, L, TR, U, BS_COLS>;
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bs_smem_bytes<T>(bs_max_rows<T>())));
        mark_configured(configured, dev);
    }
    const i64 strips = cdiv(n, BS_COLS);
    kern<<<(unsigned)imin(strips, 1 << 20), BS_THREADS, bs_smem_bytes<T>(nb), stream()>>>(nb, n, a, lda, b, ldb);
    return check_launch("trsm_block_solve");
}

template <typename T>
int launch_block_solve(bool lower, bool trans, bool unit, int nb, i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    if (nb > bs_max_rows<T>()) return MBG_ERR_UNSUPPORTED;
    ProfScope prof("trsm_block_solve");
#define BSV(L, TR, U) return launch_block_solve_t<T, L, TR, U>(nb, n, a, lda, b, ldb)
    if (lower) {
        if (trans) { if (unit) BSV(true, true, true); else BSV(true, true, false); }
        else { if (unit) BSV(true, false, true); else BSV(true, false, false); }
    } else {
        if (trans) { if (unit) BSV(false, true, true); else BSV(false, true, false); }
        else { if (unit) BSV(false, false, true); else BSV(false, false, false); }
    }
#undef BSV
}

// Rows of the diagonal blocks solved in one block_solve_kernel launch for n
// right-hand sides (0: leaves of NB rows and gemm updates in between).  Each
// CTA of that kernel serialises its sub-blocks, so it pays only when there are
// enough column strips to fill the GPU.
template <typename T>
inline i64 block_rows(i64 n) {
    const Tuning& t = tuning();
    if (t.trsm_block_rows <= NB || n < t.trsm_block_min_cols) return 0;
    return imin(t.trsm_block_rows, bs_max_rows<T>());
}

template <typename T>
int launch_diag_residual(bool lower, bool trans, bool unit, int nb, i64 n, const T* a, i64 lda,
                         const T* x, i64 ldx, T* r, i64 ldr) {
    ProfScope prof("trsm_diag_residual");
    const dim3 g(ds_grid(n)), blk(DS_WARPS * 32);
    cudaStream_t s = stream();
#define DR(L, TR, U) diag_residual_kernel<T, L, TR, U><<<g, blk, 0, s>>>(nb, n, a, lda, x, ldx, r, ldr)
    if (lower) {
        if (trans) { if (unit) DR(true, true, true); else DR(true, true, false); }
        else { if (unit) DR(true, false, true); else DR(true, false, false); }
    } else {
        if (trans) { if (unit) DR(false, true, true); else DR(false, true, false); }
        else { if (unit) DR(false, false, true); else DR(false, false, false); }
    }
#undef DR
    return check_launch("trsm_diag_residual");
}

// gemm in a precision mode, device operands.  Updates with a short reduction
// (k below the tuning table's trsm_tc_min_k) carry few flops and would pay the
// split/slice pre-pass for little work: they run on the plain kernel, which is
// as accurate as the split / Ozaki forms.
inline int gemm_in_mode(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, float alpha,
                        const float* a, i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    (void)slices;
    if (k < tuning().trsm_tc_min_k) mode = MBG_MODE_PLAIN;
    return sgemm_mode(mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
inline int gemm_in_mode(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
                        const double* a, i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    if (k < tuning().trsm_tc_min_k) mode = MBG_MODE_PLAIN;
    return dgemm_mode(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

inline i64 split_point(i64 m) { return cdiv(cdiv(m, 2), NB) * NB; }

// Pointer to op(A)[r, c] for a column-major A.
template <typename T>
inline const T* op_at(const T* a, i64 lda, bool trans, i64 r, i64 c) {
    return trans ? a + c + r * lda : a + r + c * lda;
}

// op(A) X = B (in place), left side, op(A) effectively lower/upper.
template <typename T>
int solve_left(int mode, int slices, bool lower, bool trans, bool unit, i64 m, i64 n, const T* a,
               i64 lda, T* b, i64 ldb) {
    if (m <= NB) return launch_diag_solve<T>(lower, trans, unit, (int)m, n, a, lda, b, ldb);
    if (m <= block_rows<T>(n)) return launch_block_solve<T>(lower, trans, unit, (int)m, n, a, lda, b, ldb);
    const i64 m1 = split_point(m), m2 = m - m1;
    const char tc = trans ? 'T' : 'N';
    const T* a11 = a;
    const T* a22 = a + m1 + m1 * lda;
    if (lower) {
        MBG_TRY(solve_left<T>(mode, slices, lower, trans, unit, m1, n, a11, lda, b, ldb));
        MBG_TRY(gemm_in_mode(mode, slices, tc, 'N', m2, n, m1, T(-1), op_at(a, lda, trans, m1, 0), lda,
                             b, ldb, T(1), b + m1, ldb));
        return solve_left<T>(mode, slices, lower, trans, unit, m2, n, a22, lda, b + m1, ldb);
    }
    MBG_TRY(solve_left<T>(mode, slices, lower, trans, unit, m2, n, a22, lda, b + m1, ldb));
    MBG_TRY(gemm_in_mode(mode, slices, tc, 'N', m1, n, m2, T(-1), op_at(a, lda, trans, 0, m1), lda,
                         b + m1, ldb, T(1), b, ldb));
    return solve_left<T>(mode, slices, lower, trans, unit, m1, n, a11, lda, b, ldb);
}

// W[0:m, 0:m] = tri(op(A)) as a dense column-major block: the effective triangle
// (unit diagonal when UNIT, a zero diagonal when ZERO_DIAG), zeros elsewhere; the
// other triangle of A is not read.
template <typename T>
__global__ void tri_dense_kernel(i64 m, const T* __restrict__ A, i64 lda, bool lower, bool trans, bool unit,
                                 bool zero_diag, T* __restrict__ W) {
    for (i64 l = blockIdx.y; l < m; l += gridDim.y)
        for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x) {
            const bool in = lower ? i > l : i < l;
            T v = T(0);
            if (i == l) v = zero_diag ? T(0) : (unit ? T(1) : A[i + i * lda]);
            else if (in) v = trans ? A[l + i * lda] : A[i + l * lda];
            W[i + l * m] = v;
        }
}

// R -= tri(op(A)) X, left side.  Diagonal blocks up to the fused solve's size
// are one plain GEMM with a dense copy of the triangle (input precision, all of
// R's rows in parallel); larger ones recurse with the accurate products between.
template <typename T>
int residual_left(int mode, int slices, bool lower, bool trans, bool unit, i64 m, i64 n, const T* a,
                  i64 lda, const T* x, i64 ldx, T* r, i64 ldr) {
    if (m > NB && m <= block_rows<T>(n)) {
        Workspace ww;
        MBG_TRY(ww.reserve(sizeof(T) * size_t(m) * size_t(m)));
        {
            ProfScope prof("trsm_tri_dense");
            dim3 g((unsigned)imin(cdiv(m, 256), 64), (unsigned)imin(m, 65535));
            tri_dense_kernel<T><<<g, 256, 0, stream()>>>(m, a, lda, lower, trans, unit, false, ww.as<T>());
            MBG_TRY(check_launch("trsm_tri_dense"));
        }
        return gemm_plain<T>('N', 'N', m, n, m, T(-1), ww.as<T>(), m, x, ldx, T(1), r, ldr);
    }
    if (m <= NB) return launch_diag_residual<T>(lower, trans, unit, (int)m, n, a, lda, x, ldx, r, ldr);
    const i64 m1 = split_point(m), m2 = m - m1;
    const char tc = trans ? 'T' : 'N';
    MBG_TRY(residual_left<T>(mode, slices, lower, trans, unit, m1, n, a, lda, x, ldx, r, ldr));
    MBG_TRY(residual_left<T>(mode, slices, lower, trans, unit, m2, n, a + m1 + m1 * lda, lda, x + m1,
                             ldx, r + m1, ldr));
    if (lower)  // R2 -= op(A)21 X1
        return gemm_in_mode(mode, slices, tc, 'N', m2, n, m1, T(-1), op_at(a, lda, trans, m1, 0), lda,
                            x, ldx, T(1), r + m1, ldr);
    // R1 -= op(A)12 X2
    return gemm_in_mode(mode, slices, tc, 'N', m1, n, m2, T(-1), op_at(a, lda, trans, 0, m1), lda,
                        x + m1, ldx, T(1), r, ldr);
}

template <typename T>
int launch_transpose(i64 rows, i64 cols, T alpha, const T* src, i64 lds, T* dst, i64 ldd) {
    ProfScope prof("transpose");
    dim3 g((unsigned)cdiv(rows, 32), (unsigned)cdiv(cols, 32)), blk(32, 8);
    if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
    transpose_scale_kernel<T><<<g, blk, 0, stream()>>>(rows, cols, alpha, src, lds, dst, ldd);
    return check_launch("transpose");
}

template <typename T>
int launch_axpy(i64 m, i64 n, T alpha, const T* x, i64 ldx, T* y, i64 ldy) {
    ProfScope prof("axpy");
    dim3 g((unsigned)imin(cdiv(m, 256), 64), (unsigned)imin(n, 65535));
    axpy_matrix_kernel<T><<<g, 256, 0, stream()>>>(m, n, alpha, x, ldx, y, ldy);
    return check_launch("axpy");
}

template <typename T>
int launch_copy(i64 m, i64 n, T alpha, const T* x, i64 ldx, T* y, i64 ldy) {
    ProfScope prof("copy");
    dim3 g((unsigned)imin(cdiv(m, 256), 64), (unsigned)imin(n, 65535));
    copy_scale_kernel<T><<<g, 256, 0, stream()>>>(m, n, alpha, x, ldx, y, ldy);
    return check_launch("copy");
}

// ---- inverted diagonal blocks (split / Ozaki modes) ---------------------------------
// The split / Ozaki solve: every diagonal block of NBI rows is inverted once in the
// input precision (fused block solves of the identity, all blocks in one launch), the
// inverses' planes are made once, and the solve recurses as solve_left does, except that
// each leaf is one product X_b = inv(op(A)_bb) B_b on the tensor cores instead of a
// substitution.  So every flop of the solve runs in split / Ozaki products: the leaves'
// pivot chains leave the critical path (MAGMA's inverted-diagonal-block trsm, with the
// products in the precision mode).  The forward error of X_b = inv(A_bb) B_b is bounded like
// the substitution's by cond(A_bb) times the working precision (triangular inverses,
// Higham, Accuracy and Stability of Numerical Algorithms, ch. 8 and 14).

// W (m x NBI, column-major, ldw) block b := inv(op(A)_bb), solved against identity columns
// made in shared memory: blockIdx.y = b, blockIdx.x = 32-column strip of the block.
template <typename T, bool LOWER, bool TRANS, bool UNIT>
__global__ void __launch_bounds__(BS_THREADS, 1)
block_invert_kernel(i64 m, int nbi, const T* __restrict__ A, i64 lda, T* __restrict__ W, i64 ldw) {
    extern __shared__ __align__(16) unsigned char bs_smem_raw[];
    const i64 r0 = i64(blockIdx.y) * nbi;
    const int nbb = int(min(i64(nbi), m - r0));
    const i64 c0 = i64(blockIdx.x) * BS_COLS;
    if (c0 >= nbb) return;
    bs::block_solve_strip<T, LOWER, TRANS, UNIT, BS_COLS, 2, true>(nbb, nbb, A + r0 + r0 * lda, lda, W + r0, ldw, c0,
                                                                   T(1), bs_smem_raw);
}

template <typename T>
i64 inv_block_rows() {  // the tuning table's 256 or 512 (<= bs_max_rows<T>() for both precisions)
    return tuning().trsm_inverse_block == 256 ? 256 : 512;
}

template <typename T, bool L, bool TR, bool U>
int launch_block_invert_t(i64 m, int nbi, const T* a, i64 lda, T* w, i64 ldw) {
    auto kern = block_invert_kernel<T, L, TR, U>;
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bs_smem_bytes<T>(bs_max_rows<T>())));
        mark_configured(configured, dev);
    }
    const dim3 g(unsigned(cdiv(nbi, BS_COLS)), unsigned(cdiv(m, nbi)));
    kern<<<g, BS_THREADS, bs_smem_bytes<T>(nbi), stream()>>>(m, nbi, a, lda, w, ldw);
    return check_launch("trsm_block_invert");
}

// W := the inverses of op(A)'s diagonal blocks of nbi rows, stacked (m x nbi, ld m).
template <typename T>
int invert_diagonal_blocks(bool lower, bool trans, bool unit, i64 m, int nbi, const T* a, i64 lda, T* w) {
    ProfScope prof("trsm_block_invert");
    // the strips solve against identity columns made in shared memory and write every column
    // of their block; a last block shorter than nbi leaves columns nbb .. nbi - 1 of its rows,
    // which the leaf products read as zeros
    const i64 r_last = (m - 1) / nbi * nbi, nb_last = m - r_last;
    if (nb_last < nbi)
        MBG_CUDA(cudaMemset2DAsync(w + r_last + nb_last * m, size_t(m) * sizeof(T), 0, size_t(nb_last) * sizeof(T),
                                   size_t(nbi - nb_last), stream()));
#define BIV(L, TR, U) return launch_block_invert_t<T, L, TR, U>(m, nbi, a, lda, w, m)
    if (lower) {
        if (trans) { if (unit) BIV(true, true, true); else BIV(true, true, false); }
        else { if (unit) BIV(true, false, true); else BIV(true, false, false); }
    } else {
        if (trans) { if (unit) BIV(false, true, true); else BIV(false, true, false); }
        else { if (unit) BIV(false, false, true); else BIV(false, false, false); }
    }
#undef BIV
}

// The inverses' planes (bf16 split terms or Ozaki slices), made once per solve.
template <typename T> struct InvPlanes;
template <> struct InvPlanes<float> {
    SplitA p;
    int make(int mode, int, i64 m, i64 nbi, float* w) {
        return split_a_planes(mode == MBG_MODE_BF16X6 ? 3 : 2, 'N', m, nbi, w, m, p);
    }
    // B[0:mb, :] := inv block (rows r0 .. r0 + mb of the stack) times B[0:mb, :]
    int leaf(i64 r0, i64 mb, i64 n, float* b, i64 ldb) const {
        return sgemm_split_tc_with_a_rows(p, r0, mb, mb, 'N', n, 1.0f, b, ldb, 0.0f, b, ldb);
    }
};
// The Ozaki leaves keep each inverse's diagonal out of the slices: an inverted block of a
// diagonally dominant triangle is dominated by its diagonal, and the slices are scaled per
// row, so with the diagonal inside them the off-diagonal entries would keep few bits.  The
// slices hold the strict triangle (exponents from its entries only) and the epilogue adds
// the diagonal term with one fused multiply-add: X_b = W_off B_b + d .* B_b, B_b read by the
// thread that overwrites it.
__global__ void split_block_diagonal_kernel(i64 m, int nbi, double* __restrict__ W, i64 ldw,
                                            double* __restrict__ d) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < m; r += (i64)gridDim.x * blockDim.x) {
        double* p = W + r + (r % nbi) * ldw;
        d[r] = *p;
        *p = 0.0;
    }
}
template <> struct InvPlanes<double> {
    OzakiA p;
    Workspace wd;
    double* d = nullptr;
    int make(int, int slices, i64 m, i64 nbi, double* w) {
        MBG_TRY(wd.reserve(sizeof(double) * size_t(m)));
        d = wd.as<double>();
        split_block_diagonal_kernel<<<unsigned(imin(cdiv(m, 256), 1024)), 256, 0, stream()>>>(m, int(nbi), w, m, d);
        MBG_TRY(check_launch("trsm_block_invert"));
        return ozaki_slice_a(slices, 'N', m, nbi, w, m, p);
    }
    int leaf(i64 r0, i64 mb, i64 n, double* b, i64 ldb) const {
        return dgemm_ozaki_tc_with_a(p, r0, mb, mb, 'N', n, 1.0, b, ldb, 0.0, b, ldb, d + r0);
    }
};

// The off-diagonal update blocks op(A)21 (op(A)12 for an upper triangle) of the recursion,
// in the order the solve uses them: (row r of the sub-problem, m1, m2).
struct UpdateBlock {
    i64 r, m1, m2;
};
inline void collect_updates(bool lower, i64 r, i64 m, i64 nbi, std::vector<UpdateBlock>& out) {
    if (m <= nbi) return;
    const i64 m1 = cdiv(cdiv(m, 2), nbi) * nbi, m2 = m - m1;
    if (lower) {
        collect_updates(lower, r, m1, nbi, out);
        out.push_back({r, m1, m2});
        collect_updates(lower, r + m1, m2, nbi, out);
    } else {
        collect_updates(lower, r + m1, m2, nbi, out);
        out.push_back({r, m1, m2});
        collect_updates(lower, r, m1, nbi, out);
    }
}

// Split and Ozaki solves: every update block's planes (bf16 split terms or int8 slices) are
// made up front on a second stream, issued before the diagonal blocks' inversion, so the
// splitting of op(A) (which depends on neither the inverses nor the solution) runs beside
// the inversion, the leaves and the updates instead of before each update; each update
// waits only for its own block.
template <typename T> struct UpdatePlanes;
template <> struct UpdatePlanes<float> { using type = SplitA; };
template <> struct UpdatePlanes<double> { using type = OzakiA; };
template <typename T>
struct PreSlicedUpdates {
    std::vector<typename UpdatePlanes<T>::type> planes;  // in use order
    std::vector<cudaEvent_t> ready;  // recorded on the second stream after each block's planes
    size_t next = 0;
    bool on = false;
    ~PreSlicedUpdates() {
        for (auto e : ready)
            if (e) cudaEventDestroy(e);
    }
};

// op(A)[r:r+m, r:r+m] X = B (in place; b points at row r of B), leaves from the inverses.
template <typename T>
int solve_left_inv_rec(const InvPlanes<T>& inv, PreSlicedUpdates<T>& pre, int mode, int slices, bool lower, bool trans,
                       i64 r, i64 m, i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    const i64 nbi = inv_block_rows<T>();
    if (m <= nbi) {
        ProfScope prof("trsm_inverse_leaf");
        return inv.leaf(r, m, n, b, ldb);
    }
    const i64 m1 = cdiv(cdiv(m, 2), nbi) * nbi, m2 = m - m1;
    const char tc = trans ? 'T' : 'N';
    const T* ar = a + r + r * lda;  // op(A)[r, r]
    // B_dst -= op(A)block B_src: rows x k
    auto update = [&](const T* ablk, i64 rows, i64 k, const T* bsrc, T* bdst) -> int {
        if (pre.on) {
            const size_t i = pre.next++;
            MBG_CUDA(cudaStreamWaitEvent(stream(), pre.ready[i], 0));
            if constexpr (sizeof(T) == 8)
                return dgemm_ozaki_tc_with_a(pre.planes[i], 0, rows, k, 'N', n, -1.0, bsrc, ldb, 1.0, bdst, ldb);
            else
                return sgemm_split_tc_with_a_rows(pre.planes[i], 0, rows, k, 'N', n, -1.0f, bsrc, ldb, 1.0f, bdst,
                                                  ldb);
        }
        return gemm_in_mode(mode, slices, tc, 'N', rows, n, k, T(-1), ablk, lda, bsrc, ldb, T(1), bdst, ldb);
    };
    if (lower) {
        MBG_TRY(solve_left_inv_rec<T>(inv, pre, mode, slices, lower, trans, r, m1, n, a, lda, b, ldb));
        MBG_TRY(update(op_at(ar, lda, trans, m1, 0), m2, m1, b, b + m1));
        return solve_left_inv_rec<T>(inv, pre, mode, slices, lower, trans, r + m1, m2, n, a, lda, b + m1, ldb);
    }
    MBG_TRY(solve_left_inv_rec<T>(inv, pre, mode, slices, lower, trans, r + m1, m2, n, a, lda, b + m1, ldb));
    MBG_TRY(update(op_at(ar, lda, trans, 0, m1), m1, m2, b + m1, b));
    return solve_left_inv_rec<T>(inv, pre, mode, slices, lower, trans, r, m1, n, a, lda, b, ldb);
}

// Planes of every update block of a split or Ozaki solve, on the second stream (see above).
template <typename T>
int pre_slice_updates(int mode, int slices, bool lower, bool trans, i64 m, const T* a, i64 lda,
                      PreSlicedUpdates<T>& pre) {
    std::vector<UpdateBlock> ub;
    collect_updates(lower, 0, m, inv_block_rows<T>(), ub);
    if (ub.empty()) return MBG_OK;
    if constexpr (sizeof(T) == 8)
        for (const auto& u : ub)
            if ((lower ? u.m1 : u.m2) > ozaki_max_k(slices)) return MBG_OK;  // longer reductions: sliced per update
    cudaStream_t s = stream(), aux = nullptr;
    MBG_TRY(aux_stream(&aux));
    cudaEvent_t start = nullptr;
    MBG_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    const cudaError_t e1 = cudaEventRecord(start, s);  // A is ready once the work before this call is
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(aux, start, 0) : e1;
    cudaEventDestroy(start);
    MBG_CUDA(e2);
    pre.planes.resize(ub.size());
    pre.ready.assign(ub.size(), nullptr);
    StreamScope on_aux(aux);
    const char tc = trans ? 'T' : 'N';
    for (size_t i = 0; i < ub.size(); ++i) {
        const UpdateBlock& u = ub[i];
        const T* ar = a + u.r + u.r * lda;
        const i64 rows = lower ? u.m2 : u.m1, k = lower ? u.m1 : u.m2;
        const T* blk = lower ? op_at(ar, lda, trans, u.m1, 0) : op_at(ar, lda, trans, 0, u.m1);
        if constexpr (sizeof(T) == 8) MBG_TRY(ozaki_slice_a(slices, tc, rows, k, blk, lda, pre.planes[i]));
        else MBG_TRY(split_a_planes(mode == MBG_MODE_BF16X6 ? 3 : 2, tc, rows, k, blk, lda, pre.planes[i]));
        MBG_CUDA(cudaEventCreateWithFlags(&pre.ready[i], cudaEventDisableTiming));
        MBG_CUDA(cudaEventRecord(pre.ready[i], aux));
    }
    pre.on = true;
    return MBG_OK;
}

// Before the pre-sliced planes go back to the second stream's workspace pool, that stream
// waits for the solve's work that reads them.
template <typename T>
int release_pre_sliced(PreSlicedUpdates<T>& pre) {
    if (!pre.on) return MBG_OK;
    cudaStream_t aux = nullptr;
    MBG_TRY(aux_stream(&aux));
    cudaEvent_t done = nullptr;
    MBG_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    const cudaError_t e1 = cudaEventRecord(done, stream());
    const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(aux, done, 0) : e1;
    cudaEventDestroy(done);
    MBG_CUDA(e2);
    return MBG_OK;
}

// Whether the inverted-block solve runs: a split / Ozaki mode, more than one diagonal block,
// and enough right-hand sides to repay the inversions (about NBI^2 / 3 multiply-adds per
// row of A, against m n / 2 for the solve itself).
template <typename T>
bool use_inverse_solve(int mode, i64 m, i64 n) {
    if (mode == MBG_MODE_PLAIN || tuning().trsm_inverse_min_cols <= 0) return false;
    return m > inv_block_rows<T>() && n >= tuning().trsm_inverse_min_cols;
}

template <typename T>
int solve_left_inv(int mode, int slices, bool lower, bool trans, bool unit, i64 m, i64 n, const T* a, i64 lda,
                   T* b, i64 ldb) {
    const int nbi = int(inv_block_rows<T>());
    Workspace ww;
    MBG_TRY(ww.reserve(sizeof(T) * size_t(m) * size_t(nbi)));
    PreSlicedUpdates<T> pre;
    if (tuning().trsm_preslice) MBG_TRY(pre_slice_updates<T>(mode, slices, lower, trans, m, a, lda, pre));
    MBG_TRY(invert_diagonal_blocks<T>(lower, trans, unit, m, nbi, a, lda, ww.as<T>()));
    InvPlanes<T> inv;
    int st = inv.make(mode, slices, m, nbi, ww.as<T>());
    if (!st) st = solve_left_inv_rec<T>(inv, pre, mode, slices, lower, trans, 0, m, n, a, lda, b, ldb);
    const int rel = release_pre_sliced(pre);
    return st ? st : rel;
}

int accurate_mode(float) { return MBG_MODE_BF16X6; }
int accurate_mode(double) { return MBG_MODE_OZAKI; }

// Left-side solve with optional refinement; B already holds alpha*B.
template <typename T>
int solve_left_any(int mode, int slices, bool lower, bool trans, bool unit, i64 m, i64 n, const T* a, i64 lda,
                   T* b, i64 ldb) {
    if (use_inverse_solve<T>(mode, m, n))
        return solve_left_inv<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb);
    return solve_left<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb);
}

template <typename T>
int solve_left_refined(int mode, int slices, int refine, bool lower, bool trans, bool unit, i64 m,
                       i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    if (refine <= 0 || mode == MBG_MODE_PLAIN)
        return solve_left_any<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb);
    Workspace w_rhs, w_res;
    MBG_TRY(w_rhs.reserve(sizeof(T) * size_t(m) * size_t(n)));
    MBG_TRY(w_res.reserve(sizeof(T) * size_t(m) * size_t(n)));
    T* rhs = w_rhs.as<T>();
    T* res = w_res.as<T>();
    MBG_TRY(launch_copy<T>(m, n, T(1), b, ldb, rhs, m));
    MBG_TRY(solve_left_any<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb));
    const int acc_mode = accurate_mode(T(0));
    for (int it = 0; it < refine; ++it) {
        MBG_TRY(launch_copy<T>(m, n, T(1), rhs, m, res, m));
        MBG_TRY(residual_left<T>(acc_mode, 8, lower, trans, unit, m, n, a, lda, b, ldb, res, m));
        MBG_TRY(solve_left_any<T>(mode, slices, lower, trans, unit, m, n, a, lda, res, m));
        MBG_TRY(launch_axpy<T>(m, n, T(1), res, m, b, ldb));
    }
    return MBG_OK;
}

// ---- triangular multiply ---------------------------------------------------
template <typename T>
int launch_tri_dense(i64 m, const T* a, i64 lda, bool lower, bool trans, bool unit, bool zero_diag, T* w) {
    ProfScope prof("trsm_tri_dense");
    dim3 g((unsigned)imin(cdiv(m, 256), 64), (unsigned)imin(m, 65535));
    tri_dense_kernel<T><<<g, 256, 0, stream()>>>(m, a, lda, lower, trans, unit, zero_diag, w);
    return check_launch("trsm_tri_dense");
}

// B += alpha diag(A) X (left) or alpha X diag(A) (right): the diagonal term of a
// triangular product in working precision, one fused multiply-add per element.
// Each thread owns rows i and walks columns j: a left-side diagonal entry is
// loaded once per row, a right-side one is the same for the whole block.
template <typename T>
__global__ void trmm_diag_kernel(i64 m, i64 n, T alpha, const T* __restrict__ A, i64 lda, bool unit, bool left,
                                 const T* __restrict__ X, i64 ldx, T* __restrict__ B, i64 ldb) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x) {
        const T arow = (left && !unit) ? alpha * A[i + i * lda] : alpha;
#pragma unroll 4
        for (i64 j = blockIdx.y; j < n; j += gridDim.y) {
            const T ad = (left || unit) ? arow : alpha * A[j + j * lda];
            B[i + j * ldb] = fma(ad, X[i + j * ldx], B[i + j * ldb]);
        }
    }
}

template <typename T>
int launch_trmm_diag(i64 m, i64 n, T alpha, const T* a, i64 lda, bool unit, bool left, const T* x, i64 ldx, T* b,
                     i64 ldb) {
    ProfScope prof("trmm_diag");
    dim3 g((unsigned)imin(cdiv(m, 256), 1024), (unsigned)imin(n, 64));
    trmm_diag_kernel<T><<<g, 256, 0, stream()>>>(m, n, alpha, a, lda, unit, left, x, ldx, b, ldb);
    return check_launch("trmm_diag");
}

// C := alpha op(A) op(B) (NN, beta = 0) with one operand a dense triangle (band
// KB_*), in a precision mode: every tile runs only the slabs its band needs.
inline int gemm_banded(int mode, int slices, int band, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda,
                       const float* b, i64 ldb, float* c, i64 ldc) {
    (void)slices;
    if (mode == MBG_MODE_PLAIN) return sgemm_f32('N', 'N', m, n, k, alpha, a, lda, b, ldb, 0.0f, c, ldc, band);
    if (mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return sgemm_split_tc(mode == MBG_MODE_BF16X6 ? 3 : 2, 'N', 'N', m, n, k, alpha, a, lda, b, ldb, 0.0f, c, ldc,
                          0, band);
}
inline int gemm_banded(int mode, int slices, int band, i64 m, i64 n, i64 k, double alpha, const double* a,
                       i64 lda, const double* b, i64 ldb, double* c, i64 ldc) {
    if (mode == MBG_MODE_PLAIN) return dgemm_dmma('N', 'N', m, n, k, alpha, a, lda, b, ldb, 0.0, c, ldc, band);
    if (mode != MBG_MODE_OZAKI) return MBG_ERR_INVALID_MODE;
    return dgemm_ozaki_tc(slices, 'N', 'N', m, n, k, alpha, a, lda, b, ldb, 0.0, c, ldc, 0, band);
}

// d[i] = alpha * A(i, i) (alpha for a unit diagonal): the epilogue's multiplier of B.
template <typename T>
__global__ void trmm_dvec_kernel(i64 n, T alpha, const T* __restrict__ A, i64 lda, bool unit, T* __restrict__ d) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        d[i] = unit ? alpha : alpha * A[i + i * lda];
}

inline int gemm_tri_operand(int mode, int slices, int band, char ta, char tb, i64 m, i64 n, i64 k, float alpha,
                            const float* a, i64 lda, const float* b, i64 ldb, float* c, i64 ldc,
                            const TriOperand* t) {
    (void)slices;
    if (mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return sgemm_split_tc(mode == MBG_MODE_BF16X6 ? 3 : 2, ta, tb, m, n, k, alpha, a, lda, b, ldb, 0.0f, c, ldc, 0,
                          band, t);
}
inline int gemm_tri_operand(int mode, int slices, int band, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
                            const double* a, i64 lda, const double* b, i64 ldb, double* c, i64 ldc,
                            const TriOperand* t) {
    if (mode != MBG_MODE_OZAKI) return MBG_ERR_INVALID_MODE;
    return dgemm_ozaki_tc(slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, 0.0, c, ldc, 0, band, t);
}

// Split / Ozaki trmm in place, with no copy of A or B: the pre-pass reads the
// strict triangle of op(A) straight from A and B into its planes, the GEMM's
// tiles run their band of the reduction, and each epilogue thread forms
// alpha * (off-diagonal sum) + alpha d_i B(i, j) from the old B(i, j) it then
// overwrites (the diagonal term in working precision, one FMA).
template <typename T>
int trmm_in_place(int mode, int slices, bool left, bool lower, bool trans, bool unit, i64 m, i64 n, T alpha,
                  const T* a, i64 lda, T* b, i64 ldb) {
    const i64 na = left ? m : n;
    Workspace wd;
    MBG_TRY(wd.reserve(sizeof(T) * size_t(na)));
    T* dv = wd.as<T>();
    {
        ProfScope prof("trmm_diag");
        trmm_dvec_kernel<T><<<(unsigned)imin(cdiv(na, 256), 1024), 256, 0, stream()>>>(na, alpha, a, lda, unit, dv);
        MBG_TRY(check_launch("trmm_diag"));
    }
    TriOperand t;
    t.dvec = dv;
    const char tc = trans ? 'T' : 'N';
    if (left) {
        t.keep_a = lower ? 1 : 2;  // op(A)(r, l) kept for l < r (lower) or l > r
        t.dvec_mode = 1;
        return gemm_tri_operand(mode, slices, lower ? KB_A_LOWER : KB_A_UPPER, tc, 'N', m, n, m, alpha, a, lda, b,
                                ldb, b, ldb, &t);
    }
    t.keep_b = lower ? 2 : 1;  // op(B)^T(r, l) = op(A)(l, r): kept for l > r (lower) or l < r
    t.dvec_mode = 2;
    return gemm_tri_operand(mode, slices, lower ? KB_B_LOWER : KB_B_UPPER, 'N', tc, m, n, n, alpha, b, ldb, a, lda,
                            b, ldb, &t);
}

}  // namespace

// B := alpha op(A) B (side 'L') or alpha B op(A) (side 'R'), A triangular.
// One GEMM out of place: W = tri(op(A)) as a dense block (zeros outside the
// triangle, unit diagonal when diag 'U'; the other triangle of A is not read),
// X = a copy of B, then B = alpha W X (or alpha X W) with the triangular band, so
// each output tile runs only the part of the reduction where W is nonzero:
// m^2 n multiply-adds plus the diagonal tiles' halves, in one launch.
// The split / Ozaki modes keep the diagonal out of the split product: its term
// alpha d_i x_ij is added with one FMA in working precision, so the product's
// accuracy does not depend on the ratio between the diagonal and the rest of a
// row (Ozaki slices are scaled per row, so a dominant diagonal would leave the
// off-diagonal entries few bits).  They run in place (trmm_in_place above); an
// Ozaki product longer than one exact launch (ozaki_max_k) takes this path with W
// holding the strictly triangular part and a separate diagonal pass.
template <typename T>
int trmm_device(int mode, int slices, char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha,
                const T* a, i64 lda, T* b, i64 ldb) {
    if (m == 0 || n == 0) return MBG_OK;
    if (alpha == T(0)) return scale_matrix<T>(m, n, T(0), b, ldb);  // trmm.mojo:94-98: zeros
    const bool trans = is_t(ta), unit = is_u(diag), left = is_l(side);
    const bool lower = (!is_u(uplo)) != trans;  // effective op(A) lower triangular
    const i64 na = left ? m : n;
    if (mode != MBG_MODE_PLAIN && !(sizeof(T) == 8 && na > ozaki_max_k(slices)))
        return trmm_in_place<T>(mode, slices, left, lower, trans, unit, m, n, alpha, a, lda, b, ldb);
    Workspace ww, wx;
    MBG_TRY(ww.reserve(sizeof(T) * size_t(na) * size_t(na)));
    MBG_TRY(wx.reserve(sizeof(T) * size_t(m) * size_t(n)));
    T* w = ww.as<T>();
    T* x = wx.as<T>();
    const bool split_diag = mode != MBG_MODE_PLAIN;
    MBG_TRY(launch_tri_dense<T>(na, a, lda, lower, trans, unit, split_diag, w));
    MBG_TRY(launch_copy<T>(m, n, T(1), b, ldb, x, m));
    if (left) MBG_TRY(gemm_banded(mode, slices, lower ? KB_A_LOWER : KB_A_UPPER, m, n, m, alpha, w, na, x, m, b, ldb));
    else MBG_TRY(gemm_banded(mode, slices, lower ? KB_B_LOWER : KB_B_UPPER, m, n, n, alpha, x, m, w, na, b, ldb));
    if (!split_diag) return MBG_OK;
    return launch_trmm_diag<T>(m, n, alpha, a, lda, unit, left, x, m, b, ldb);
}
template int trmm_device<float>(int, int, char, char, char, char, i64, i64, float, const float*, i64, float*, i64);
template int trmm_device<double>(int, int, char, char, char, char, i64, i64, double, const double*, i64, double*,
                                 i64);

template <typename T>
int trsm_device(int mode, int slices, int refine, char side, char uplo, char ta, char diag, i64 m,
                i64 n, T alpha, const T* a, i64 lda, T* b, i64 ldb) {
    if (m == 0 || n == 0) return MBG_OK;
    const bool trans = is_t(ta), unit = is_u(diag), up = is_u(uplo);
    if (is_l(side)) {
        if (alpha != T(1)) MBG_TRY(scale_matrix<T>(m, n, alpha, b, ldb));
        const bool lower = (!up) != trans;  // effective op(A) lower triangular
        return solve_left_refined<T>(mode, slices, refine, lower, trans, unit, m, n, a, lda, b, ldb);
    }
    // right side: op(A)^T X^T = alpha B^T
    Workspace wt;
    MBG_TRY(wt.reserve(sizeof(T) * size_t(m) * size_t(n)));
    T* bt = wt.as<T>();
    MBG_TRY(launch_transpose<T>(m, n, alpha, b, ldb, bt, n));   // bt is n x m, ld n
    const bool trans2 = !trans;
    const bool lower2 = (!up) != trans2;
    MBG_TRY(solve_left_refined<T>(mode, slices, refine, lower2, trans2, unit, n, m, a, lda, bt, n));
    return launch_transpose<T>(n, m, T(1), bt, n, b, ldb);
}

template int trsm_device<float>(int, int, int, char, char, char, char, i64, i64, float, const float*, i64, float*, i64);
template int trsm_device<double>(int, int, int, char, char, char, char, i64, i64, double, const double*, i64, double*, i64);

}  // namespace mbg
