// Plain FP32 / FP64 GEMM on the CUDA cores — the drop-in arithmetic for
// mojoBLAS gemm (src/level3/gemm.mojo:56-377, v3 :385, v7 :817, v11 :2092) and,
// with a triangular tile schedule, syrk (src/level3/syrk.mojo:20-200).
//
// One 256-thread CTA computes a 128 x 128 tile of C.  K advances in slabs of 8:
// each thread fetches 4 elements of op(A) and 4 of op(B) from global memory into
// registers (coalesced along whichever dimension is contiguous for the given
// transpose), the CTA stores them k-major into a double-buffered shared tile,
// and every thread accumulates an 8 x 8 register block (rows tx*4+{0..3} and
// 64+tx*4+{0..3}, columns likewise from ty) with one FMA per product.  Each
// element's sum runs over k in ascending order, like the reference's per-column
// axpy loops; beta is applied once in the epilogue (beta == 0 does not read C).
// Launches that would fill fewer than two waves of 128 x 128 tiles (the
// tall-skinny updates inside trsm, small problems) use 64 x 64 tiles with a
// 4 x 4 register block instead, for four times as many CTAs.
#include "mbg_internal.cuh"

namespace mbg {

namespace {

constexpr int BK = 8, NT = 256;

// Shared-tile row padding: with 8-byte elements a pad of 4 spreads the k-major
// stores of eight consecutive k rows over distinct bank pairs.
template <typename T> struct Pad;
template <> struct Pad<float> { static constexpr int v = 4; };
template <> struct Pad<double> { static constexpr int v = 4; };

// Resident CTAs per SM the register budget is sized for: the fp32 128-tile
// fits two (128 registers), the fp64 one needs 240+ registers and keeps one.
template <typename T, int TILE> struct MinBlocks { static constexpr int v = TILE == 128 ? 1 : 2; };
template <> struct MinBlocks<float, 128> { static constexpr int v = 2; };

template <typename T>
__device__ __forceinline__ void lds4(const T* p, T (&o)[4]);
template <>
__device__ __forceinline__ void lds4<float>(const float* p, float (&o)[4]) {
    float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <>
__device__ __forceinline__ void lds4<double>(const double* p, double (&o)[4]) {
    double2 v0 = *reinterpret_cast<const double2*>(p);
    double2 v1 = *reinterpret_cast<const double2*>(p + 2);
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
}

// Lower (TRI == 1) or upper (TRI == 2) tile schedule: linear id -> (ti >= tj).
__device__ __forceinline__ void tri_tile(i64 t, i64& ti, i64& tj) {
    i64 r = (i64)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    ti = r;
    tj = t - r * (r + 1) / 2;
}

// TILE = 128: 128 x 128 tile, 8 x 8 per thread (rows tx*4+{0..3} and
// 64+tx*4+{0..3}); TILE = 64: 64 x 64 tile, 4 x 4 per thread (rows tx*4+{0..3}),
// four times as many CTAs for launches that would not fill the GPU.
template <typename T, bool TA, bool TB, int TRI, int TILE>
__global__ void __launch_bounds__(NT, MinBlocks<T, TILE>::v)
gemm_simt_kernel(i64 m, i64 n, i64 k, T alpha, const T* __restrict__ A, i64 lda,
                 const T* __restrict__ B, i64 ldb, T beta, T* __restrict__ C, i64 ldc) {
    constexpr int BM = TILE, BN = TILE;
    constexpr int TM = TILE / 16;        // 8 or 4 rows (and columns) per thread
    constexpr int LPT = BM * BK / NT;    // elements of each operand a thread loads per slab
    constexpr int P = Pad<T>::v;
    __shared__ __align__(16) T As[2][BK][BM + P];
    __shared__ __align__(16) T Bs[2][BK][BN + P];

    i64 tm, tn;
    if (TRI == 0) {
        tm = blockIdx.x;
        tn = blockIdx.y;
    } else {
        i64 ti, tj;
        tri_tile(blockIdx.x, ti, tj);
        if (TRI == 1) { tm = ti; tn = tj; } else { tm = tj; tn = ti; }
    }
    const i64 m0 = tm * BM, n0 = tn * BN;  // tile origin
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;

    T ra[LPT], rb[LPT];
    auto load_global = [&](i64 k0) {
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int e = tid + r * NT;
            int i, l;
            if (!TA) { i = e % BM; l = e / BM; } else { i = e / BK; l = e % BK; }
            const i64 gi = m0 + i, gl = k0 + l;
            T v = T(0);
            if (gi < m && gl < k) v = TA ? A[gl + gi * lda] : A[gi + gl * lda];
            ra[r] = v;
        }
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int e = tid + r * NT;
            int j, l;
            if (!TB) { j = e / BK; l = e % BK; } else { j = e % BN; l = e / BN; }
            const i64 gj = n0 + j, gl = k0 + l;
            T v = T(0);
            if (gj < n && gl < k) v = TB ? B[gj + gl * ldb] : B[gl + gj * ldb];
            rb[r] = v;
        }
    };
    auto store_shared = [&](int buf) {
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int e = tid + r * NT;
            int i, l;
            if (!TA) { i = e % BM; l = e / BM; } else { i = e / BK; l = e % BK; }
            As[buf][l][i] = ra[r];
        }
#pragma unroll
        for (int r = 0; r < LPT; ++r) {
            const int e = tid + r * NT;
            int j, l;
            if (!TB) { j = e / BK; l = e % BK; } else { j = e % BN; l = e / BN; }
            Bs[buf][l][j] = rb[r];
        }
    };

    T acc[TM][TM];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM; ++j) acc[i][j] = T(0);

    const i64 nk = (k + BK - 1) / BK;
    load_global(0);
    store_shared(0);
    __syncthreads();
    for (i64 kt = 0; kt < nk; ++kt) {
        const int buf = int(kt & 1);
        if (kt + 1 < nk) load_global((kt + 1) * BK);
#pragma unroll
        for (int l = 0; l < BK; ++l) {
            T a[TM], b[TM];
            T t4[4];
            lds4<T>(&As[buf][l][tx * 4], t4);
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = t4[q];
            lds4<T>(&Bs[buf][l][ty * 4], t4);
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = t4[q];
            if (TM == 8) {
                lds4<T>(&As[buf][l][64 + tx * 4], t4);
#pragma unroll
                for (int q = 0; q < 4; ++q) a[(4 + q) % TM] = t4[q];
                lds4<T>(&Bs[buf][l][64 + ty * 4], t4);
#pragma unroll
                for (int q = 0; q < 4; ++q) b[(4 + q) % TM] = t4[q];
            }
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TM; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) store_shared(buf ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int j = 0; j < TM; ++j) {
        const i64 gj = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
        if (gj >= n) continue;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const i64 gi = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            if (gi >= m) continue;
            if (TRI == 1 && gi < gj) continue;
            if (TRI == 2 && gi > gj) continue;
            T* cp = C + gi + gj * ldc;
            const T v = alpha * acc[i][j];
            *cp = (beta == T(0)) ? v : fma(beta, *cp, v);
        }
    }
}

template <typename T, int TRI>
__global__ void scale_kernel(i64 m, i64 n, T beta, T* __restrict__ C, i64 ldc) {
    for (i64 j = blockIdx.y; j < n; j += gridDim.y) {
        i64 i0 = 0, i1 = m;
        if (TRI == 1) i0 = j;                 // lower: rows j..m-1
        if (TRI == 2) i1 = (j + 1 < m) ? j + 1 : m;  // upper: rows 0..j
        for (i64 i = i0 + blockIdx.x * (i64)blockDim.x + threadIdx.x; i < i1;
             i += (i64)gridDim.x * blockDim.x) {
            T* p = C + i + j * ldc;
            *p = (beta == T(0)) ? T(0) : beta * *p;
        }
    }
}

template <typename T, int TRI, int TILE>
int launch_gemm(bool ta, bool tb, dim3 grid, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
                const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    ProfScope prof(sizeof(T) == 4 ? "gemm_simt_f32" : "gemm_simt_f64");
    cudaStream_t s = stream();
    if (!ta && !tb) gemm_simt_kernel<T, false, false, TRI, TILE><<<grid, NT, 0, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    else if (!ta && tb) gemm_simt_kernel<T, false, true, TRI, TILE><<<grid, NT, 0, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    else if (ta && !tb) gemm_simt_kernel<T, true, false, TRI, TILE><<<grid, NT, 0, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    else gemm_simt_kernel<T, true, true, TRI, TILE><<<grid, NT, 0, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    return check_launch(sizeof(T) == 4 ? "gemm_simt_f32" : "gemm_simt_f64");
}

}  // namespace

template <typename T>
int scale_matrix(i64 m, i64 n, T beta, T* c, i64 ldc) {
    if (m <= 0 || n <= 0 || beta == T(1)) return MBG_OK;
    ProfScope prof("scale");
    dim3 grid((unsigned)imin(cdiv(m, 256), 64), (unsigned)imin(n, 65535));
    scale_kernel<T, 0><<<grid, 256, 0, stream()>>>(m, n, beta, c, ldc);
    return check_launch("scale");
}

template <typename T>
int scale_triangle(char uplo, i64 n, T beta, T* c, i64 ldc) {
    if (n <= 0 || beta == T(1)) return MBG_OK;
    ProfScope prof("scale");
    dim3 grid((unsigned)imin(cdiv(n, 256), 64), (unsigned)imin(n, 65535));
    if (is_l(uplo)) scale_kernel<T, 1><<<grid, 256, 0, stream()>>>(n, n, beta, c, ldc);
    else scale_kernel<T, 2><<<grid, 256, 0, stream()>>>(n, n, beta, c, ldc);
    return check_launch("scale");
}

template <typename T>
int gemm_plain(char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
               const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    if (m == 0 || n == 0) return MBG_OK;
    if (alpha == T(0) || k == 0) return scale_matrix<T>(m, n, beta, c, ldc);
    if constexpr (sizeof(T) == 8)
        if (!tuning().plain_fp64_simt)
            return dgemm_dmma(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    if constexpr (sizeof(T) == 4)
        if (!tuning().plain_fp32_staged) return sgemm_f32(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    const i64 gm = cdiv(m, 128), gn = cdiv(n, 128);
    if (gm * gn < 2 * 148) {  // under two waves of 128 x 128 tiles: use 64 x 64 tiles
        const i64 sm = cdiv(m, 64), sn = cdiv(n, 64);
        if (sn > 65535 || sm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
        return launch_gemm<T, 0, 64>(is_t(ta), is_t(tb), dim3((unsigned)sm, (unsigned)sn), m, n, k, alpha,
                                     a, lda, b, ldb, beta, c, ldc);
    }
    if (gn > 65535 || gm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    return launch_gemm<T, 0, 128>(is_t(ta), is_t(tb), dim3((unsigned)gm, (unsigned)gn), m, n, k, alpha,
                                  a, lda, b, ldb, beta, c, ldc);
}

template <typename T>
int gemmt_plain(char uplo, char ta, char tb, i64 n, i64 k, T alpha, const T* a, i64 lda,
                const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    if (n == 0) return MBG_OK;
    if (alpha == T(0) || k == 0) return scale_triangle<T>(uplo, n, beta, c, ldc);
    if constexpr (sizeof(T) == 8)
        if (!tuning().plain_fp64_simt)
            return dgemmt_dmma(uplo, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    if constexpr (sizeof(T) == 4)
        if (!tuning().plain_fp32_staged) return sgemmt_f32(uplo, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    const i64 t = cdiv(n, 128);
    const i64 tiles = t * (t + 1) / 2;
    if (tiles > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    if (is_l(uplo))
        return launch_gemm<T, 1, 128>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda,
                                      b, ldb, beta, c, ldc);
    return launch_gemm<T, 2, 128>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda, b,
                                  ldb, beta, c, ldc);
}

template int gemm_plain<float>(char, char, i64, i64, i64, float, const float*, i64, const float*, i64, float, float*, i64);
template int gemm_plain<double>(char, char, i64, i64, i64, double, const double*, i64, const double*, i64, double, double*, i64);
template int gemmt_plain<float>(char, char, char, i64, i64, float, const float*, i64, const float*, i64, float, float*, i64);
template int gemmt_plain<double>(char, char, char, i64, i64, double, const double*, i64, const double*, i64, double, double*, i64);
template int scale_matrix<float>(i64, i64, float, float*, i64);
template int scale_matrix<double>(i64, i64, double, double*, i64);
template int scale_triangle<float>(char, i64, float, float*, i64);
template int scale_triangle<double>(char, i64, double, double*, i64);

}  // namespace mbg
