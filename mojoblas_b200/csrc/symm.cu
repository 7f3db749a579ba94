// symm and syr2k on device operands: the symmetric and rank-2k neighbours of
// gemm / syrk, run on the same GEMM kernels in every precision mode.
//
// symm (mojoBLAS src/level3/symm.mojo:20-241): C := alpha*A*B + beta*C (side 'L')
// or alpha*B*A + beta*C (side 'R') with A symmetric, one triangle stored.  The
// stored triangle is expanded once into a dense workspace copy of A (na^2
// elements, an HBM-bound pass that costs 2*na^2 element moves against the
// GEMM's 2*m*n*na flops), and the product runs as a plain NN GEMM (FP32 / FP64
// kernels), a BF16x3 / BF16x6 split product or an Ozaki int8 product.
//
// syr2k (src/level3/syr2k.mojo:20-190): C := alpha*(op(A) op(B)^T + op(B) op(A)^T)
// + beta*C on one triangle, op(X) = X ('N', n x k) or X^T ('T', X is k x n).  Two
// triangle-only GEMMs: the first applies beta, the second adds into C (beta = 1,
// one rounding per element, as c + v).
#include "mbg_internal.cuh"

namespace mbg {

namespace {

constexpr int SY_T = 32;

// W[0:n, 0:n] = the symmetric matrix whose `upper` / lower triangle is stored in
// A.  One CTA per 32 x 32 tile of W: the tile and its mirror are read coalesced
// into shared memory, each output element takes the stored one of the two.
template <typename T>
__global__ void symmetrize_kernel(i64 n, const T* __restrict__ A, i64 lda, bool upper, T* __restrict__ W) {
    __shared__ T direct[SY_T][SY_T + 1];
    __shared__ T mirror[SY_T][SY_T + 1];
    const i64 i0 = (i64)blockIdx.x * SY_T, j0 = (i64)blockIdx.y * SY_T;
    const int tx = threadIdx.x;
    for (int ty = threadIdx.y; ty < SY_T; ty += blockDim.y) {
        const i64 i = i0 + tx, j = j0 + ty;    // direct tile: A(i, j)
        if (i < n && j < n) direct[ty][tx] = A[i + j * lda];
        const i64 mi = j0 + tx, mj = i0 + ty;  // mirror tile: A(j0 + tx, i0 + ty)
        if (mi < n && mj < n) mirror[ty][tx] = A[mi + mj * lda];
    }
    __syncthreads();
    for (int ty = threadIdx.y; ty < SY_T; ty += blockDim.y) {
        const i64 i = i0 + tx, j = j0 + ty;
        if (i >= n || j >= n) continue;
        const bool stored = upper ? i <= j : i >= j;
        // W(i, j) = A(i, j) if stored, else A(j, i) = mirror[i - i0][j - j0]
        W[i + j * n] = stored ? direct[ty][tx] : mirror[tx][ty];
    }
}

template <typename T>
int launch_symmetrize(i64 n, const T* a, i64 lda, bool upper, T* w) {
    ProfScope prof("symmetrize");
    dim3 g((unsigned)cdiv(n, SY_T), (unsigned)cdiv(n, SY_T)), blk(SY_T, 8);
    if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
    symmetrize_kernel<T><<<g, blk, 0, stream()>>>(n, a, lda, upper, w);
    return check_launch("symmetrize");
}

inline int gemm_mode_t(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a,
                       i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    (void)slices;
    return sgemm_mode(mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
inline int gemm_mode_t(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
                       const double* a, i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    return dgemm_mode(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

// Triangle `uplo` of C := alpha*op(A)*op(B) + beta*C in a precision mode.
inline int gemmt_mode(int mode, int slices, char uplo, char ta, char tb, i64 n, i64 k, float alpha,
                      const float* a, i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    (void)slices;
    const char tri = is_l(uplo) ? 'L' : 'U';
    if (mode == MBG_MODE_PLAIN) return gemmt_plain<float>(tri, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    if (mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return sgemm_split_tc(mode == MBG_MODE_BF16X6 ? 3 : 2, ta, tb, n, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                          tri);
}
inline int gemmt_mode(int mode, int slices, char uplo, char ta, char tb, i64 n, i64 k, double alpha,
                      const double* a, i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    const char tri = is_l(uplo) ? 'L' : 'U';
    if (mode == MBG_MODE_PLAIN) return gemmt_plain<double>(tri, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    if (mode != MBG_MODE_OZAKI) return MBG_ERR_INVALID_MODE;
    return dgemm_ozaki_tc(slices, ta, tb, n, n, k, alpha, a, lda, b, ldb, beta, c, ldc, tri);
}

}  // namespace

template <typename T>
int symm_device(int mode, int slices, char side, char uplo, i64 m, i64 n, T alpha, const T* a, i64 lda,
                const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    if (m == 0 || n == 0) return MBG_OK;
    if (alpha == T(0)) return scale_matrix<T>(m, n, beta, c, ldc);
    const bool left = is_l(side);
    const i64 na = left ? m : n;
    Workspace ww;
    MBG_TRY(ww.reserve(sizeof(T) * size_t(na) * size_t(na)));
    T* w = ww.as<T>();
    MBG_TRY(launch_symmetrize<T>(na, a, lda, is_u(uplo), w));
    if (left) return gemm_mode_t(mode, slices, 'N', 'N', m, n, m, alpha, w, na, b, ldb, beta, c, ldc);
    return gemm_mode_t(mode, slices, 'N', 'N', m, n, n, alpha, b, ldb, w, na, beta, c, ldc);
}

template <typename T>
int syr2k_device(int mode, int slices, char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda,
                 const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    if (n == 0) return MBG_OK;
    if (alpha == T(0) || k == 0) return scale_triangle<T>(uplo, n, beta, c, ldc);
    // op(X) op(Y)^T: X as stored for 'N' (n x k), transposed for 'T' (k x n)
    const char ta = is_n(trans) ? 'N' : 'T';
    const char tb = is_n(trans) ? 'T' : 'N';
    MBG_TRY(gemmt_mode(mode, slices, uplo, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc));
    return gemmt_mode(mode, slices, uplo, ta, tb, n, k, alpha, b, ldb, a, lda, T(1), c, ldc);
}

template int symm_device<float>(int, int, char, char, i64, i64, float, const float*, i64, const float*, i64, float,
                                float*, i64);
template int symm_device<double>(int, int, char, char, i64, i64, double, const double*, i64, const double*, i64,
                                 double, double*, i64);
template int syr2k_device<float>(int, int, char, char, i64, i64, float, const float*, i64, const float*, i64, float,
                                 float*, i64);
template int syr2k_device<double>(int, int, char, char, i64, i64, double, const double*, i64, const double*, i64,
                                  double, double*, i64);

}  // namespace mbg
