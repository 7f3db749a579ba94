// Plain FP32 GEMM on the CUDA cores, 128 x 128 or 64 x 64 tiles — the single-precision
// drop-in arithmetic for mojoBLAS gemm (src/level3/gemm.mojo:56-377, v11
// :2092-2436) and, with a triangular tile schedule, ssyrk
// (src/level3/syrk.mojo:20-200).
//
// One CTA per 128 x 128 tile of C, or per 64 x 64 tile for launches that would
// fill fewer than two waves of 128-tiles; the tile code (cp.async pipeline,
// register blocking, epilogue) is gemm_f32_tile.cuh, shared with the grouped
// sgemm plans.
#include "mbg_internal.cuh"
#include "gemm_f32_tile.cuh"

namespace mbg {

namespace {

using namespace f32t;

template <int FT, bool TA, bool TB, int TRI, bool VA, bool VB>
__global__ void __launch_bounds__(FNT, FT == 128 ? 2 : 4)
gemm_f32_kernel(i64 m, i64 n, i64 k, float alpha, const float* __restrict__ A, i64 lda,
                const float* __restrict__ B, i64 ldb, float beta, float* __restrict__ C, i64 ldc, int band) {
    extern __shared__ __align__(16) float fsm[];
    i64 tm, tn;
    if (TRI == 0) {
        tm = blockIdx.x;
        tn = blockIdx.y;
        band_order(band, tm, tn);
    } else {
        i64 ti, tj;
        f32_tri_tile(blockIdx.x, ti, tj);
        if (TRI == 1) { tm = ti; tn = tj; } else { tm = tj; tn = ti; }
    }
    f32_tile<FT, TA, TB, TRI, VA, VB>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tm, tn, fsm, band);
}


template <int FT, int TRI, bool VA, bool VB>
int launch_f32_v(bool ta, bool tb, dim3 grid, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda,
                 const float* b, i64 ldb, float beta, float* c, i64 ldc, int band) {
    constexpr size_t SM = f32_smem<FT>();
    static std::atomic<unsigned> configured{0};  // one bit per device: more than 48 KB of shared memory needs an opt-in
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(gemm_f32_kernel<FT, false, false, TRI, VA, VB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_f32_kernel<FT, false, true, TRI, VA, VB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_f32_kernel<FT, true, false, TRI, VA, VB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM));
        MBG_CUDA(cudaFuncSetAttribute(gemm_f32_kernel<FT, true, true, TRI, VA, VB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM));
        mark_configured(configured, dev);
    }
    cudaStream_t s = stream();
#define F32(TA_, TB_) \
    gemm_f32_kernel<FT, TA_, TB_, TRI, VA, VB><<<grid, FNT, SM, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band)
    if (!ta && !tb) F32(false, false);
    else if (!ta && tb) F32(false, true);
    else if (ta && !tb) F32(true, false);
    else F32(true, true);
#undef F32
    return check_launch("gemm_f32");
}


template <int FT, int TRI>
int launch_f32(bool ta, bool tb, dim3 grid, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda,
               const float* b, i64 ldb, float beta, float* c, i64 ldc, int band = KB_NONE) {
    const bool va = f32_vec(!ta, a, lda), vb = f32_vec(tb, b, ldb);
    if (va && vb)
        return launch_f32_v<FT, TRI, true, true>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
    if (va)
        return launch_f32_v<FT, TRI, true, false>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
    if (vb)
        return launch_f32_v<FT, TRI, false, true>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
    return launch_f32_v<FT, TRI, false, false>(ta, tb, grid, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
}

// dst[j + i * ldd] = src[i + j * lds] for i < rows, j < cols (32 x 32 tiles through shared memory)
__global__ void f32_transpose_kernel(i64 rows, i64 cols, const float* __restrict__ src, i64 lds,
                                     float* __restrict__ dst, i64 ldd) {
    __shared__ float tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const i64 i = i0 + threadIdx.x, j = j0 + r;
        if (i < rows && j < cols) tile[r][threadIdx.x] = src[i + j * lds];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const i64 j = j0 + threadIdx.x, i = i0 + r;
        if (i < rows && j < cols) dst[j + i * ldd] = tile[threadIdx.x][r];
    }
}

int launch_f32_transpose(i64 rows, i64 cols, const float* src, i64 lds, float* dst, i64 ldd) {
    ProfScope prof("gemm_f32_transpose");
    dim3 g((unsigned)cdiv(rows, 32), (unsigned)cdiv(cols, 32)), blk(32, 8);
    if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
    f32_transpose_kernel<<<g, blk, 0, stream()>>>(rows, cols, src, lds, dst, ldd);
    return check_launch("gemm_f32_transpose");
}

}  // namespace

// C := alpha op(A) op(B) + beta C (alpha != 0, k > 0): 128 x 128 tiles, or 64 x 64
// tiles (4 x 4 per thread) when 128-tiles would fill fewer than two waves.
// band (KB_*): one operand is a dense triangle; each tile runs its part of k.
// The tiles copy an operand 16 bytes at a time only when it is contiguous along m
// (op(A)) or n (op(B)), as in NT.  In a large call (m n k >= 2^30) an operand that is
// contiguous along k instead (A with 'T', B with 'N') is first transposed into a
// workspace (2 x 4 bytes per element against the GEMM's 2k flops per element of C);
// every element's sum is unchanged, the NT tiles run.
int sgemm_f32(char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda, const float* b,
              i64 ldb, float beta, float* c, i64 ldc, int band) {
    if (double(m) * double(n) * double(k) >= double(1ll << 30) && (is_t(ta) || is_n(tb))) {
        Workspace wa, wb;
        if (is_t(ta)) {  // A is k x m (k contiguous): At = m x k
            const i64 ld = cdiv(m, 4) * 4;
            MBG_TRY(wa.reserve(sizeof(float) * size_t(ld) * size_t(k)));
            MBG_TRY(launch_f32_transpose(k, m, a, lda, wa.as<float>(), ld));
            a = wa.as<float>();
            lda = ld;
            ta = 'N';
        }
        if (is_n(tb)) {  // B is k x n (k contiguous): Bt = n x k, used as op(B) = Bt^T
            const i64 ld = cdiv(n, 4) * 4;
            MBG_TRY(wb.reserve(sizeof(float) * size_t(ld) * size_t(k)));
            MBG_TRY(launch_f32_transpose(k, n, b, ldb, wb.as<float>(), ld));
            b = wb.as<float>();
            ldb = ld;
            tb = 'T';
        }
        return sgemm_f32(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, band);
    }
    ProfScope prof("gemm_f32");
    const i64 gm = cdiv(m, 128), gn = cdiv(n, 128);
    if (gm * gn < 2 * 148) {
        const i64 sm = cdiv(m, 64), sn = cdiv(n, 64);
        if (sn > 65535 || sm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
        return launch_f32<64, 0>(is_t(ta), is_t(tb), dim3((unsigned)sm, (unsigned)sn), m, n, k, alpha, a, lda, b,
                                 ldb, beta, c, ldc, band);
    }
    if (gn > 65535 || gm > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    return launch_f32<128, 0>(is_t(ta), is_t(tb), dim3((unsigned)gm, (unsigned)gn), m, n, k, alpha, a, lda, b,
                              ldb, beta, c, ldc, band);
}

// Lower ('L') or upper triangle of C := alpha op(A) op(B) + beta C (ssyrk).
int sgemmt_f32(char uplo, char ta, char tb, i64 n, i64 k, float alpha, const float* a, i64 lda,
               const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    ProfScope prof("gemm_f32");
    const i64 t = cdiv(n, 128);
    const i64 tiles = t * (t + 1) / 2;
    if (tiles > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    if (is_l(uplo))
        return launch_f32<128, 1>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    return launch_f32<128, 2>(is_t(ta), is_t(tb), dim3((unsigned)tiles), n, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

}  // namespace mbg
