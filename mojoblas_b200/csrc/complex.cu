// Complex GEMM (cgemm / zgemm) on the real kernels of every precision mode.
//
// mojoBLAS lists complex dtypes on its roadmap (README.md:152) and has no complex
// routine to restate; these entry points keep its gemm's argument order and
// `info` numbering (src/level3/gemm.mojo:56-78, :179-213) and add the Netlib
// meaning of trans 'C' (conjugate transpose).  Matrices are column-major with
// interleaved (re, im) elements, as Fortran / C99 complex arrays store them.
//
// Design (the real embedding, "4M": four real products per complex one).  With
// op(A) = Ar + i Ai and op(B) = Br + i Bi,
//     [Re C]   [Ar  -Ai] [Br]
//     [Im C] = [Ai   Ar] [Bi]
// is one real GEMM of 2m x n x 2k.  Interleaving its rows and reduction index,
//     A'(2i, 2l) = Re a,  A'(2i, 2l+1) = -Im a,  A'(2i+1, 2l) = Im a,  A'(2i+1, 2l+1) = Re a
//     B'(2l, j) = Re b,   B'(2l+1, j) = Im b,    C'(2i, j) = Re c,     C'(2i+1, j) = Im c
// with a = alpha op(A)(i, l), b = op(B)(l, j): C' is C itself read as a real
// matrix with leading dimension 2 ldc, and for op(B) = B so is B' (leading
// dimension 2 ldb).  So one expansion kernel writes A' (alpha folded in, as
// Netlib's cgemm folds alpha into its temporaries), op(B) = B^T / B^H is
// de-interleaved into B', beta scales C in complex arithmetic first, and the
// real product runs in the caller's precision mode (plain FP32 / FP64, BF16x3 /
// BF16x6 split, Ozaki int8 slices) with beta' = 1 (or 0), so every real output
// is one real dot product of length 2k: the accuracy of the real kernel at 2k.
#include "mbg_internal.cuh"

namespace mbg {
namespace {

inline bool is_c(char t) { return t == 'C' || t == 'c'; }

// A' (2m x 2k, ld 2m) from op(A) with alpha folded in; conj: op is the conjugate transpose.
template <typename T>
__global__ void complex_expand_a_kernel(i64 m, i64 k, T ar, T ai, const T* __restrict__ a, i64 lda, bool trans,
                                        bool conj, T* __restrict__ w) {
    const i64 ldw = 2 * m;
    for (i64 l = blockIdx.y; l < k; l += gridDim.y)
        for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x) {
            const T* p = trans ? a + 2 * (l + i * lda) : a + 2 * (i + l * lda);
            const T re = p[0], im = conj ? -p[1] : p[1];
            const T xr = ar * re - ai * im, xi = ar * im + ai * re;  // alpha * op(A)(i, l)
            T* c0 = w + 2 * i + (2 * l) * ldw;
            T* c1 = c0 + ldw;
            c0[0] = xr;
            c0[1] = xi;
            c1[0] = -xi;
            c1[1] = xr;
        }
}

// B' (2k x n, ld 2k) from op(B) = B^T or B^H.
template <typename T>
__global__ void complex_expand_b_kernel(i64 k, i64 n, const T* __restrict__ b, i64 ldb, bool conj,
                                        T* __restrict__ w) {
    for (i64 j = blockIdx.y; j < n; j += gridDim.y)
        for (i64 l = blockIdx.x * (i64)blockDim.x + threadIdx.x; l < k; l += (i64)gridDim.x * blockDim.x) {
            const T* p = b + 2 * (j + l * ldb);  // op(B)(l, j) = B(j, l) (conjugated for 'C')
            w[2 * l + j * 2 * k] = p[0];
            w[2 * l + 1 + j * 2 * k] = conj ? -p[1] : p[1];
        }
}

// C := beta C in complex arithmetic (beta = 0 stores zeros).
template <typename T>
__global__ void complex_scale_kernel(i64 m, i64 n, T br, T bi, T* __restrict__ c, i64 ldc) {
    const bool zero = br == T(0) && bi == T(0);
    for (i64 j = blockIdx.y; j < n; j += gridDim.y)
        for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < m; i += (i64)gridDim.x * blockDim.x) {
            T* p = c + 2 * (i + j * ldc);
            if (zero) {
                p[0] = T(0);
                p[1] = T(0);
            } else {
                const T re = p[0], im = p[1];
                p[0] = br * re - bi * im;
                p[1] = br * im + bi * re;
            }
        }
}

inline dim3 ew_grid(i64 rows, i64 cols) {
    return dim3((unsigned)imax(1, imin(cdiv(rows, 256), 64)), (unsigned)imax(1, imin(cols, 65535)));
}

inline int real_gemm(int mode, int slices, char tb, i64 m, i64 n, i64 k, const float* a, i64 lda, const float* b,
                     i64 ldb, float beta, float* c, i64 ldc) {
    (void)slices;
    return sgemm_mode(mode, 'N', tb, m, n, k, 1.0f, a, lda, b, ldb, beta, c, ldc);
}
inline int real_gemm(int mode, int slices, char tb, i64 m, i64 n, i64 k, const double* a, i64 lda,
                     const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    return dgemm_mode(mode, slices, 'N', tb, m, n, k, 1.0, a, lda, b, ldb, beta, c, ldc);
}

// Device operands (interleaved complex), arguments already checked, m, n > 0.
template <typename T>
int complex_gemm_device(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, const T* alpha, const T* a,
                        i64 lda, const T* b, i64 ldb, const T* beta, T* c, i64 ldc) {
    const T ar = alpha[0], ai = alpha[1], br = beta[0], bi = beta[1];
    const bool no_product = (ar == T(0) && ai == T(0)) || k == 0;
    const bool beta_one = br == T(1) && bi == T(0), beta_zero = br == T(0) && bi == T(0);
    if (!beta_one && (no_product || !beta_zero)) {
        ProfScope prof("complex_scale");
        complex_scale_kernel<T><<<ew_grid(m, n), 256, 0, stream()>>>(m, n, br, bi, c, ldc);
        MBG_TRY(check_launch("complex_scale"));
    }
    if (no_product) return MBG_OK;
    Workspace wa, wb;
    MBG_TRY(wa.reserve(sizeof(T) * size_t(4) * size_t(m) * size_t(k)));
    {
        ProfScope prof("complex_expand");
        complex_expand_a_kernel<T><<<ew_grid(m, k), 256, 0, stream()>>>(m, k, ar, ai, a, lda, is_t(ta), is_c(ta),
                                                                          wa.as<T>());
        MBG_TRY(check_launch("complex_expand"));
    }
    const T* bp = b;
    i64 bld = 2 * ldb;
    if (!is_n(tb)) {
        MBG_TRY(wb.reserve(sizeof(T) * size_t(2) * size_t(k) * size_t(n)));
        ProfScope prof("complex_expand");
        complex_expand_b_kernel<T><<<ew_grid(k, n), 256, 0, stream()>>>(k, n, b, ldb, is_c(tb), wb.as<T>());
        MBG_TRY(check_launch("complex_expand"));
        bp = wb.as<T>();
        bld = 2 * k;
    }
    // beta was applied above (or is 0 / 1): C' += A' B' (or C' = A' B' for beta = 0)
    return real_gemm(mode, slices, 'N', 2 * m, n, 2 * k, wa.as<T>(), 2 * m, bp, bld, beta_zero ? T(0) : T(1), c,
                     2 * ldc);
}

template <typename T>
int complex_gemm_entry(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, const T* alpha, const T* a,
                       i64 lda, const T* b, i64 ldb, const T* beta, T* c, i64 ldc) {
    // argument checks numbered as mojoBLAS gemm numbers them (gemm.mojo:179-213); 'C' is accepted
    if (!is_n(ta) && !is_t(ta)) return 1;
    if (!is_n(tb) && !is_t(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    if (lda < imax(1, is_n(ta) ? m : k)) return 8;
    if (ldb < imax(1, is_n(tb) ? k : n)) return 10;
    if (ldc < imax(1, m)) return 13;
    if (m == 0 || n == 0) return MBG_OK;
    if (!alpha || !beta) return MBG_ERR_INVALID_MODE;
    const bool need_ab = !((alpha[0] == T(0) && alpha[1] == T(0)) || k == 0);
    // host operands are staged as real matrices of twice the rows
    Operand A, B, Cc;
    if (need_ab) {
        MBG_TRY(A.prepare(a, 2 * (is_n(ta) ? m : k), is_n(ta) ? k : m, 2 * lda, sizeof(T), true, false));
        MBG_TRY(B.prepare(b, 2 * (is_n(tb) ? k : n), is_n(tb) ? n : k, 2 * ldb, sizeof(T), true, false));
    }
    const bool beta_zero = beta[0] == T(0) && beta[1] == T(0);
    MBG_TRY(Cc.prepare(c, 2 * m, n, 2 * ldc, sizeof(T), !beta_zero, true));
    MBG_TRY(complex_gemm_device<T>(mode, slices, ta, tb, m, n, k, alpha, (const T*)A.dev, A.dev_ld / 2,
                                   (const T*)B.dev, B.dev_ld / 2, beta, (T*)Cc.dev, Cc.dev_ld / 2));
    MBG_TRY(Cc.finish());
    return finish_call(A.staged || B.staged || Cc.staged);
}

}  // namespace
}  // namespace mbg

using namespace mbg;

extern "C" {

int mbg_cgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const float* alpha, const float* a, int64_t lda,
              const float* b, int64_t ldb, const float* beta, float* c, int64_t ldc) {
    return complex_gemm_entry<float>(MBG_MODE_PLAIN, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_zgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha, const double* a, int64_t lda,
              const double* b, int64_t ldb, const double* beta, double* c, int64_t ldc) {
    return complex_gemm_entry<double>(MBG_MODE_PLAIN, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_cgemm_ex(int mode, char ta, char tb, int64_t m, int64_t n, int64_t k, const float* alpha, const float* a,
                 int64_t lda, const float* b, int64_t ldb, const float* beta, float* c, int64_t ldc) {
    if (mode != MBG_MODE_PLAIN && mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return complex_gemm_entry<float>(mode, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_zgemm_ex(int mode, int slices, char ta, char tb, int64_t m, int64_t n, int64_t k, const double* alpha,
                 const double* a, int64_t lda, const double* b, int64_t ldb, const double* beta, double* c,
                 int64_t ldc) {
    if (mode != MBG_MODE_PLAIN && !(mode == MBG_MODE_OZAKI && slices >= 2 && slices <= 8))
        return MBG_ERR_INVALID_MODE;
    return complex_gemm_entry<double>(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

}  // extern "C"
