// Plain FP64 GEMM on the FP64 tensor pipe (mma.sync.m8n8k4.f64) — the double
// precision drop-in arithmetic for mojoBLAS gemm (src/level3/gemm.mojo:56-377,
// v3 :385, v7 :817) and, with a triangular tile schedule, dsyrk
// (src/level3/syrk.mojo:20-200).
//
// Each m8n8k4 MMA is 256 fused multiply-adds in IEEE double precision, so the
// arithmetic is the same FP64 FMA chain as the CUDA-core kernel (every element's
// sum runs over k in ascending order, four terms per MMA); it issues one
// instruction where the CUDA-core kernel needs eight and reads each operand
// element from shared memory once per warp instead of once per thread.
//
// CTA tile BM x BN with (BM / WM) x (BN / WN) warps, warp tile WM x WN made of
// (WM / 8) x (WN / 8) MMA fragments.  K advances in slabs of 32 through a
// 3-stage cp.async pipeline: every element is copied global -> shared on its
// own (8 bytes), so any transpose, leading dimension and ragged edge is served
// by the same code (elements outside the matrix are zero-filled).  Each operand
// keeps in shared memory the orientation it has in global memory, so a warp's
// copies land in consecutive words: [k][m] rows of BM + 8 doubles for an
// m-contiguous operand, [m][k] rows of 36 doubles for a k-contiguous one.  Both
// paddings make the fragment loads A[row = lane / 4][k = lane % 4] and
// B[k = lane % 4][col = lane / 4] two wavefronts each, the minimum for 256 bytes.
#include "mbg_internal.cuh"

namespace mbg {

namespace {

constexpr int DK = 32, DSTAGES = 3;
constexpr int DKP = DK + 4;  // row of a k-contiguous tile: 36 doubles = 72 words = 8 mod 32

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}
// 16 bytes (two doubles) of which the first `bytes` are read (16, 8 or 0), the rest zero-filled
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Lower (TRI == 1) or upper (TRI == 2) tile schedule: linear id -> (ti >= tj).
__device__ __forceinline__ void dmma_tri_tile(i64 t, i64& ti, i64& tj) {
    i64 r = (i64)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    ti = r;
    tj = t - r * (r + 1) / 2;
}

template <int BM, int BN, int WM, int WN>
struct DmmaCfg {
    static constexpr int WARPS = (BM / WM) * (BN / WN);
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int MI = WM / 8, NJ = WN / 8;
    // a stage holds each operand in the orientation it is contiguous in: [k][m] rows of
    // BM + 8 doubles, or [m][k] rows of DKP doubles; both sizes are reserved
    static constexpr int A_ELEMS = (DK * (BM + 8) > BM * DKP) ? DK * (BM + 8) : BM * DKP;
    static constexpr int B_ELEMS = (DK * (BN + 8) > BN * DKP) ? DK * (BN + 8) : BN * DKP;
    static constexpr size_t SMEM = sizeof(double) * size_t(DSTAGES) * (A_ELEMS + B_ELEMS);
};

// VEC = 2: both operands 16-byte aligned with even leading dimensions, so pairs
// of elements along the contiguous index are copied 16 bytes at a time.
template <class C, bool TA, bool TB, int TRI, int BM, int BN, int VEC>
__global__ void __launch_bounds__(C::THREADS, 1)
gemm_dmma_kernel(i64 m, i64 n, i64 k, double alpha, const double* __restrict__ A, i64 lda,
                 const double* __restrict__ B, i64 ldb, double beta, double* __restrict__ Cm, i64 ldc, int band) {
    extern __shared__ __align__(16) double dsm[];
    // A: TA (k contiguous in memory) -> [m][DKP], else [k][BM + 8]; B: !TB -> [n][DKP], else [k][BN + 8]
    constexpr int LA = TA ? DKP : BM + 8, LB = TB ? BN + 8 : DKP;
    double* As = dsm;
    double* Bs = dsm + size_t(DSTAGES) * C::A_ELEMS;

    i64 tm, tn;
    if (TRI == 0) {
        tm = blockIdx.x;
        tn = blockIdx.y;
        band_order(band, tm, tn);
    } else {
        i64 ti, tj;
        dmma_tri_tile(blockIdx.x, ti, tj);
        if (TRI == 1) { tm = ti; tn = tj; } else { tm = tj; tn = ti; }
    }
    const i64 m0 = tm * BM, n0 = tn * BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int WGM = BM / (C::MI * 8);  // warps along m
    const int wm0 = (warp % WGM) * C::MI * 8, wn0 = (warp / WGM) * C::NJ * 8;
    const int lr = lane >> 2, lk = lane & 3;

    auto issue = [&](i64 kt, int st) {
        const i64 k0 = kt * DK;
        double* as = As + size_t(st) * C::A_ELEMS;
        double* bs = Bs + size_t(st) * C::B_ELEMS;
#pragma unroll
        for (int e0 = tid; e0 < BM * DK / VEC; e0 += C::THREADS) {
            const int e = e0 * VEC;
            int i, l;
            if (!TA) { i = e % BM; l = e / BM; } else { l = e % DK; i = e / DK; }  // contiguous index first
            const i64 gi = m0 + i, gl = k0 + l;
            double* dst = as + (TA ? i * LA + l : l * LA + i);
            if (VEC == 1) {
                const bool v = gi < m && gl < k;
                cp_async8(dst, v ? (TA ? A + gl + gi * lda : A + gi + gl * lda) : A, v);
            } else {  // the pair runs along the contiguous index; the second may fall off the edge
                const i64 c0 = TA ? gl : gi, cend = TA ? k : m;
                const bool v = TA ? gi < m : gl < k;
                const int bytes = (!v || c0 >= cend) ? 0 : (c0 + 1 < cend ? 16 : 8);
                cp_async16(dst, bytes ? (TA ? A + gl + gi * lda : A + gi + gl * lda) : A, bytes);
            }
        }
#pragma unroll
        for (int e0 = tid; e0 < BN * DK / VEC; e0 += C::THREADS) {
            const int e = e0 * VEC;
            int j, l;
            if (!TB) { l = e % DK; j = e / DK; } else { j = e % BN; l = e / BN; }
            const i64 gj = n0 + j, gl = k0 + l;
            double* dst = bs + (TB ? l * LB + j : j * LB + l);
            if (VEC == 1) {
                const bool v = gj < n && gl < k;
                cp_async8(dst, v ? (TB ? B + gj + gl * ldb : B + gl + gj * ldb) : B, v);
            } else {
                const i64 c0 = TB ? gj : gl, cend = TB ? n : k;
                const bool v = TB ? gl < k : gj < n;
                const int bytes = (!v || c0 >= cend) ? 0 : (c0 + 1 < cend ? 16 : 8);
                cp_async16(dst, bytes ? (TB ? B + gj + gl * ldb : B + gl + gj * ldb) : B, bytes);
            }
        }
    };

    double acc[C::MI][C::NJ][2];
#pragma unroll
    for (int i = 0; i < C::MI; ++i)
#pragma unroll
        for (int j = 0; j < C::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    // slabs [kt0, kt0 + nk) of the reduction: all of them, or the tile's band
    i64 kt0 = 0, kt1 = (k + DK - 1) / DK;
    if (band != KB_NONE) band_slabs(band, m0, BM, n0, BN, 0, DK, kt1, kt0, kt1);
    const i64 nk = kt1 - kt0;
#pragma unroll
    for (int s = 0; s < DSTAGES - 1; ++s) {
        if (s < nk) issue(kt0 + s, s);
        cp_commit();
    }
    for (i64 kt = 0; kt < nk; ++kt) {
        cp_wait<DSTAGES - 2>();
        __syncthreads();  // slab kt has landed; the buffer of slab kt - 1 is free
        if (kt + DSTAGES - 1 < nk) issue(kt0 + kt + DSTAGES - 1, int((kt + DSTAGES - 1) % DSTAGES));
        cp_commit();
        const int st = int(kt % DSTAGES);
        // fragment element (row wm0 + 8i + lr, k kk + lk) and (k kk + lk, column wn0 + 8j + lr)
        const double* as = As + size_t(st) * C::A_ELEMS + (TA ? (wm0 + lr) * LA + lk : lk * LA + wm0 + lr);
        const double* bs = Bs + size_t(st) * C::B_ELEMS + (TB ? lk * LB + wn0 + lr : (wn0 + lr) * LB + lk);
#pragma unroll
        for (int kk = 0; kk < DK; kk += 4) {
            double af[C::MI], bf[C::NJ];
#pragma unroll
            for (int i = 0; i < C::MI; ++i) af[i] = TA ? as[8 * i * LA + kk] : as[kk * LA + 8 * i];
#pragma unroll
            for (int j = 0; j < C::NJ; ++j) bf[j] = TB ? bs[kk * LB + 8 * j] : bs[8 * j * LB + kk];
#pragma unroll
            for (int i = 0; i < C::MI; ++i)
#pragma unroll
                for (int j = 0; j < C::NJ; ++j) dmma(acc[i][j], af[i], bf[j]);
        }
    }
    cp_wait<0>();

    // D fragment: row lane / 4, columns 2 (lane % 4) + {0, 1}
#pragma unroll
    for (int i = 0; i < C::MI; ++i) {
        const i64 gi = m0 + wm0 + 8 * i + lr;
        if (gi >= m) continue;
        bool live[C::NJ][2];
        double cv[C::NJ][2];
#pragma unroll
        for (int j = 0; j < C::NJ; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const i64 gj = n0 + wn0 + 8 * j + 2 * lk + e;
                live[j][e] = gj < n && !(TRI == 1 && gi < gj) && !(TRI == 2 && gi > gj);
                cv[j][e] = (live[j][e] && beta != 0.0 && beta != 1.0) ? Cm[gi + gj * ldc] : 0.0;
            }
#pragma unroll
        for (int j = 0; j < C::NJ; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (!live[j][e]) continue;
                double* cp = Cm + gi + (n0 + wn0 + 8 * j + 2 * lk + e) * ldc;
                const double v = alpha * acc[i][j][e];
                if (beta == 0.0) *cp = v;
                else if (beta == 1.0) atomicAdd(cp, v);  // one add per element: c + v, as fma(1, c, v)
                else *cp = fma(beta, cv[j][e], v);
            }
    }
}

using Big = DmmaCfg<128, 128, 64, 32>;   // 8 warps
using Small = DmmaCfg<64, 64, 32, 32>;   // 4 warps

template <class C, int TRI, int BM, int BN, int VEC>
int launch_dmma_v(bool ta, bool tb, dim3 grid, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
                  const double* b, i64 ldb, double beta, double* c, i64 ldc, int band) {
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {  // all four transposes, on a device's first call
        MBG_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<C, false, false, TRI, BM, BN, VEC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<C, false, true, TRI, BM, BN, VEC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<C, true, false, TRI, BM, BN, VEC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<C, true, true, TRI, BM, BN, VEC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
        mark_configured(configured, dev);
    }
    cudaStream_t s = stream();
#define DM(TA_, TB_) \
    gemm_dmma_kernel<C, TA_, TB_, TRI, BM, BN, VEC><<<grid, C::THREADS, C::SMEM, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band)
    if (!ta && !tb) DM(false, false);
    else if (!ta && tb) DM(false, true);
    else if (ta && !tb) DM(true, false);
    else DM(true, true);
#undef DM
    return check_launch("gemm_dmma_f64");
}

template <class C, int TRI, int BM, int BN>
int launch_dmma(bool ta, bool tb, dim3 grid, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
                const double* b, i64 ldb, double beta, double* c, i64 ldc, int band = KB_NONE) {
    const bool vec = (reinterpret_cast<uintptr_t>(a) % 16 == 0) && (reinterpret_cast<uintptr_t>(b) % 16 == 0) &&
                     lda % 2 == 0 && ldb % 2 == 0;
    if (vec) return launch_dmma_v<C, TRI, BM, BN, 2>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
    return launch_dmma_v<C, TRI, BM, BN, 1>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
}

}  // namespace

// C := alpha op(A) op(B) + beta C in FP64 on the tensor pipe (alpha != 0, k > 0).
// band (KB_*): one operand is a dense triangle; each tile runs its part of k.
int dgemm_dmma(char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
               const double* b, i64 ldb, double beta, double* c, i64 ldc, int band) {
    ProfScope prof("gemm_dmma_f64");
    const i64 gm = cdiv(m, 128), gn = cdiv(n, 128);
    if (gm * gn < 2 * 148) {  // under two waves of 128 x 128 tiles: 64 x 64 tiles
        const i64 sm = cdiv(m, 64), sn = cdiv(n, 64);
        if (sn > 65535 || sm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
        return launch_dmma<Small, 0, 64, 64>(is_t(ta), is_t(tb), dim3((unsigned)sm, (unsigned)sn), m, n, k, alpha,
                                             a, lda, b, ldb, beta, c, ldc, band);
    }
    if (gn > 65535 || gm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    return launch_dmma<Big, 0, 128, 128>(is_t(ta), is_t(tb), dim3((unsigned)gm, (unsigned)gn), m, n, k, alpha, a,
                                         lda, b, ldb, beta, c, ldc, band);
}

// Lower ('L') or upper triangle of C := alpha op(A) op(B) + beta C (dsyrk).
int dgemmt_dmma(char uplo, char ta, char tb, i64 n, i64 k, double alpha, const double* a, i64 lda,
                const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    ProfScope prof("gemm_dmma_f64");
    const i64 t = cdiv(n, 128);
    const i64 tiles = t * (t + 1) / 2;
    if (tiles > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    if (is_l(uplo))
        return launch_dmma<Big, 1, 128, 128>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda, b,
                                             ldb, beta, c, ldc);
    return launch_dmma<Big, 2, 128, 128>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda, b,
                                         ldb, beta, c, ldc);
}

}  // namespace mbg
