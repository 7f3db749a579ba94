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
#include "mbg_internal.cuh"

namespace mbg {

namespace {

constexpr int NB = 64;        // diagonal block (leaf) size
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

template <typename T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

constexpr int BS_COLS = 32;                       // right-hand sides per CTA of block_solve_kernel
constexpr int BS_THREADS = 8 * BS_COLS;           // eight lanes per column in the substitution
constexpr int BS_TILE = NB * 72;                  // diagonal block + reciprocals (64 x 65 + 64), or a 64 x 72 tile

inline int bs_strip_ld(int nb) { return (int)(cdiv(nb, NB) * NB) + 2; }
template <typename T>
inline size_t bs_smem_bytes(int nb) { return sizeof(T) * (size_t(BS_COLS) * bs_strip_ld(nb) + 2 * BS_TILE); }

// One element copied global -> shared without a register round trip; zero-filled
// (nothing read) when !valid, in which case src only has to be some valid pointer.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? (int)sizeof(T) : 0;
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Solves op(A)[0:nb, 0:nb] X = B[0:nb, :] in place, nb up to 512 (double) or
// 1024 (float) rows, in one launch.  Each CTA owns W right-hand-side columns (a
// strip) and keeps the strip's nb rows in shared memory, column-major with
// leading dimension roundup(nb, 64) + 2 (= 2 mod 16, so that the column pairs
// one warp reads fall in different banks).  It runs the recursive solve's own
// blocked substitution over 64-row sub-blocks without leaving the SM:
//   for each sub-block b (forward for lower op(A), backward for upper):
//     - solve the 64 x 64 diagonal block exactly as diag_solve_kernel does
//       (eight lanes per column, pivot broadcast by shuffle, reciprocal
//       multiply, zero pivots skipped — src/level3/trsm.mojo:130-148);
//     - subtract op(A)[t, b] X_b from every sub-block t still to be solved,
//       one 64 x 64 tile of op(A) at a time, each thread keeping 4 rows x 4
//       columns of the product over half of the 64-long reduction in
//       registers and reading the tile and X_b as 8/16-byte pairs.
// The diagonal blocks and tiles form one sequence per strip that is staged
// with cp.async into two alternating buffers: the next item is in flight while
// the current one is computed, so the L2 latency of A (shared by every CTA)
// is hidden.  The strip is read from and written to HBM once; only
// off-diagonal blocks above the launch's size go through gemm.  Rows at or
// past nb stay zero in the strip and staged items are zero outside op(A)'s
// block, so ragged edges need no special case in the inner loops.
template <typename T, bool LOWER, bool TRANS, bool UNIT, int W>
__global__ void __launch_bounds__(8 * W, 1)
block_solve_kernel(int nb, i64 ncols, const T* __restrict__ A, i64 lda, T* __restrict__ B, i64 ldb) {
    using P2 = typename Pair<T>::type;
    static_assert(W == 32, "the tile update maps 256 threads onto 64 rows x 32 columns x 2 halves");
    constexpr int NT = 8 * W;
    constexpr int LDL = NB + 1;               // diagonal block, interleaved rows
    constexpr int LT = TRANS ? NB + 2 : NB + 8;  // update tile: [l][r] (plain) or [r][l] (transposed)
    extern __shared__ __align__(16) unsigned char bs_smem_raw[];
    const int nsub = (nb + NB - 1) / NB, nbr = nsub * NB, ldbs = nbr + 2;
    T* Bs = reinterpret_cast<T*>(bs_smem_raw);
    T* const buf0 = Bs + (size_t)W * ldbs;  // two staging buffers of BS_TILE elements
    const int tid = threadIdx.x;

    // item (step, tt): tt < 0 is the diagonal block of sub-block b(step), else its tt-th trailing tile
    auto sub_of = [&](int step) { return LOWER ? step : nsub - 1 - step; };
    auto tiles_of = [&](int b) { return LOWER ? nsub - 1 - b : b; };
    auto advance = [&](int& step, int& tt) {
        if (tt + 1 < tiles_of(sub_of(step))) ++tt; else { ++step; tt = -1; }
    };
    auto issue = [&](int step, int tt, T* buf) {
        const int b = sub_of(step), r0 = b * NB, nbb = min(NB, nb - r0);
        if (tt < 0) {
            const T* Ad = A + r0 + (i64)r0 * lda;
#pragma unroll 4
            for (int e = tid; e < NB * NB; e += NT) {
                const int fast = e & (NB - 1), slow = e >> 6;  // fast index runs along contiguous memory
                const int i = TRANS ? slow : fast, l = TRANS ? fast : slow;
                const bool v = i < nbb && l < nbb;
                cp_async_elem(buf + l * LDL + (i & 7) * 8 + (i >> 3),
                              v ? (TRANS ? Ad + l + (i64)i * lda : Ad + i + (i64)l * lda) : A, v);
            }
        } else {
            const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
#pragma unroll 4
            for (int e = tid; e < NB * NB; e += NT) {
                const int fast = e & (NB - 1), slow = e >> 6;
                // plain: buf[l][r] = A[rt0 + r, r0 + l]; transposed: buf[r][l] = A[r0 + l, rt0 + r]
                const bool v = TRANS ? (rt0 + slow < nb && fast < nbb) : (rt0 + fast < nb && slow < nbb);
                const T* src = TRANS ? A + (r0 + fast) + (i64)(rt0 + slow) * lda
                                     : A + (rt0 + fast) + (i64)(r0 + slow) * lda;
                cp_async_elem(buf + slow * LT + fast, v ? src : A, v);
            }
        }
    };

    const i64 nstrips = (ncols + W - 1) / W;
    for (i64 strip = blockIdx.x; strip < nstrips; strip += gridDim.x) {
        const i64 c0 = strip * W;
#pragma unroll 4
        for (int c = 0; c < W; ++c) {
            const bool live = c0 + c < ncols;
            const T* bc = B + (live ? c0 + c : 0) * ldb;
            for (int r = tid; r < nbr; r += NT) cp_async_elem(Bs + c * ldbs + r, live && r < nb ? bc + r : B, live && r < nb);
        }
        issue(0, -1, buf0);
        cp_async_commit();
        int step = 0, tt = -1;
        for (int it = 0; step < nsub; ++it) {
            T* cur = buf0 + (it & 1) * BS_TILE;
            cp_async_wait_all();
            __syncthreads();  // item `it` has landed everywhere; buffer (it + 1) & 1 is free
            int ns = step, nt = tt;
            advance(ns, nt);
            if (ns < nsub) issue(ns, nt, buf0 + ((it + 1) & 1) * BS_TILE);
            cp_async_commit();
            const int b = sub_of(step), r0 = b * NB, nbb = min(NB, nb - r0);
            if (tt < 0) {
                // ---- diagonal sub-block: substitution ----
                T* inv = cur + NB * LDL;
                for (int l = tid; l < nbb; l += NT) inv[l] = UNIT ? T(1) : T(1) / cur[l * LDL + (l & 7) * 8 + (l >> 3)];
                __syncthreads();
                const int q = tid & 7;
                T* bc = Bs + (tid >> 3) * ldbs + r0;
                T x[8];
#pragma unroll
                for (int s = 0; s < 8; ++s) x[s] = bc[q * 8 + s];
#pragma unroll
                for (int u = 0; u < NB; ++u) {
                    const int l = LOWER ? u : NB - 1 - u;
                    if (l >= nbb) continue;  // uniform
                    const int owner = l >> 3, slot = l & 7;
                    T xl = __shfl_sync(0xffffffffu, x[slot], owner, 8);
                    const bool live = xl != T(0);  // the reference skips zero pivots
                    if (!UNIT) xl *= inv[l];
                    if (q == owner && live) x[slot] = xl;
                    const T* col = cur + l * LDL;
#pragma unroll
                    for (int s = 0; s < 8; ++s) {
                        const int r = q * 8 + s;
                        const bool below = LOWER ? (r > l) : (r < l);
                        const T a = col[s * 8 + q];
                        if (live && below) x[s] -= xl * a;
                    }
                }
#pragma unroll
                for (int s = 0; s < 8; ++s)
                    if (q * 8 + s < nbb) bc[q * 8 + s] = x[s];
            } else {
                // ---- trailing tile: B_t -= op(A)[t, b] X_b ----
                if constexpr (sizeof(T) == 8) {
                    // FP64 tensor-core MMA (m8n8k4): warp w owns rows 16 (w % 4) .. +16
                    // and columns 16 (w / 4) .. +16 of the 64 x 32 product, 2 x 2
                    // fragments, the full 64-long reduction in registers.  Fragment
                    // loads: A[row = lane / 4][k = lane % 4], X[k = lane % 4][col =
                    // lane / 4]; with the tile's leading dimension (72 or 66) and the
                    // strip's (2 mod 16) each is two wavefronts, the minimum for 256 B.
                    const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
                    const int lane = tid & 31, w = tid >> 5;
                    const int m0 = 16 * (w & 3), n0 = 16 * (w >> 2);
                    const int lr = lane >> 2, lk = lane & 3;
                    double d[2][2][2];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int nj = 0; nj < 2; ++nj) d[mi][nj][0] = d[mi][nj][1] = 0.0;
                    const double* tile = reinterpret_cast<const double*>(cur);
                    const double* xs = reinterpret_cast<const double*>(Bs) + r0;
#pragma unroll 4
                    for (int k0 = 0; k0 < NB; k0 += 4) {
                        double af[2], bf[2];
#pragma unroll
                        for (int mi = 0; mi < 2; ++mi) {
                            const int r = m0 + 8 * mi + lr, k = k0 + lk;
                            af[mi] = TRANS ? tile[r * LT + k] : tile[k * LT + r];
                        }
#pragma unroll
                        for (int nj = 0; nj < 2; ++nj) bf[nj] = xs[(n0 + 8 * nj + lr) * ldbs + k0 + lk];
#pragma unroll
                        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                            for (int nj = 0; nj < 2; ++nj)
                                asm volatile(
                                    "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                                    : "+d"(d[mi][nj][0]), "+d"(d[mi][nj][1])
                                    : "d"(af[mi]), "d"(bf[nj]));
                    }
                    double* bs = reinterpret_cast<double*>(Bs);
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        const int r = rt0 + m0 + 8 * mi + lr;  // D fragment: row lane / 4, columns 2 (lane % 4) + {0, 1}
                        if (r < nb) {
#pragma unroll
                            for (int nj = 0; nj < 2; ++nj)
#pragma unroll
                                for (int e = 0; e < 2; ++e) bs[(n0 + 8 * nj + 2 * lk + e) * ldbs + r] -= d[mi][nj][e];
                        }
                    }
                } else {
                const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
                const int lane = tid & 31, wq = (tid >> 5) & 3, h = tid >> 7;
                const int rg = (lane >> 2) + 8 * (wq & 1), cp = (lane & 3) + 4 * (wq >> 1);
                int rows[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) rows[i] = TRANS ? rg + 16 * i : 2 * rg + (i & 1) + 32 * (i >> 1);
                const T* xb = Bs + cp * ldbs + r0;
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
#pragma unroll 4
                for (int l = 32 * h; l < 32 * h + 32; l += 2) {
                    P2 xv[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) xv[j] = *reinterpret_cast<const P2*>(xb + 8 * j * ldbs + l);
                    T a[4][2];  // a[i][dl] = op(A)[rows[i]][l + dl]
                    if (!TRANS) {
#pragma unroll
                        for (int dl = 0; dl < 2; ++dl) {
                            const P2 p0 = *reinterpret_cast<const P2*>(cur + (l + dl) * LT + 2 * rg);
                            const P2 p1 = *reinterpret_cast<const P2*>(cur + (l + dl) * LT + 2 * rg + 32);
                            a[0][dl] = p0.x; a[1][dl] = p0.y; a[2][dl] = p1.x; a[3][dl] = p1.y;
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const P2 p = *reinterpret_cast<const P2*>(cur + rows[i] * LT + l);
                            a[i][0] = p.x; a[i][1] = p.y;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            acc[i][j] = fma(a[i][0], xv[j].x, acc[i][j]);
                            acc[i][j] = fma(a[i][1], xv[j].y, acc[i][j]);
                        }
                }
                // the two halves subtract their partial products in turn
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    if (h == half) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int r = rt0 + rows[i];
                            if (r < nb) {
#pragma unroll
                                for (int j = 0; j < 4; ++j) Bs[(cp + 8 * j) * ldbs + r] -= acc[i][j];
                            }
                        }
                    }
                    if (half == 0) __syncthreads();
                }
                }
            }
            step = ns;
            tt = nt;
        }
        __syncthreads();
        for (int c = 0; c < W; ++c) {
            if (c0 + c >= ncols) break;
            T* bc = B + (c0 + c) * ldb;
            for (int r = tid; r < nb; r += NT) bc[r] = Bs[c * ldbs + r];
        }
        __syncthreads();
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
    static unsigned configured = 0;  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (dev < 32 && !(configured & (1u << dev))) {
        MBG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bs_smem_bytes<T>(bs_max_rows<T>())));
        configured |= 1u << dev;
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

// R -= tri(op(A)) X, left side.
template <typename T>
int residual_left(int mode, int slices, bool lower, bool trans, bool unit, i64 m, i64 n, const T* a,
                  i64 lda, const T* x, i64 ldx, T* r, i64 ldr) {
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

int accurate_mode(float) { return MBG_MODE_BF16X6; }
int accurate_mode(double) { return MBG_MODE_OZAKI; }

// Left-side solve with optional refinement; B already holds alpha*B.
template <typename T>
int solve_left_refined(int mode, int slices, int refine, bool lower, bool trans, bool unit, i64 m,
                       i64 n, const T* a, i64 lda, T* b, i64 ldb) {
    if (refine <= 0 || mode == MBG_MODE_PLAIN)
        return solve_left<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb);
    Workspace w_rhs, w_res;
    MBG_TRY(w_rhs.reserve(sizeof(T) * size_t(m) * size_t(n)));
    MBG_TRY(w_res.reserve(sizeof(T) * size_t(m) * size_t(n)));
    T* rhs = w_rhs.as<T>();
    T* res = w_res.as<T>();
    MBG_TRY(launch_copy<T>(m, n, T(1), b, ldb, rhs, m));
    MBG_TRY(solve_left<T>(mode, slices, lower, trans, unit, m, n, a, lda, b, ldb));
    const int acc_mode = accurate_mode(T(0));
    for (int it = 0; it < refine; ++it) {
        MBG_TRY(launch_copy<T>(m, n, T(1), rhs, m, res, m));
        MBG_TRY(residual_left<T>(acc_mode, 8, lower, trans, unit, m, n, a, lda, b, ldb, res, m));
        MBG_TRY(solve_left<T>(mode, slices, lower, trans, unit, m, n, a, lda, res, m));
        MBG_TRY(launch_axpy<T>(m, n, T(1), res, m, b, ldb));
    }
    return MBG_OK;
}

}  // namespace

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
