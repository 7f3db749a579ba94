// Adjoint (reverse-mode) kernels for gemm and trsm.  The reference has no
// derivatives; these are new entry points built on the same GEMM / trsm cores.
//
// gemm, C = alpha*op(A)*op(B):  d op(A) = alpha*G*op(B)^T,  d op(B) = alpha*op(A)^T*G,
// mapped back through the transposes so each is one GEMM call.
//
// trsm, X = alpha*op(A)^{-1}*B (left) or X = alpha*B*op(A)^{-1} (right):
//   W = op(A)^{-T} G (left) or G op(A)^{-T} (right);   dB = alpha*W  (a trsm);
//   d op(A) = -W X^T (left) or -X^T W (right), restricted to the stored
//   triangle — computed by the triangle-only GEMM (tiles of the other triangle
//   are never computed, diagonal tiles are masked) with coefficient -1/alpha
//   applied to dB; for a unit diagonal the diagonal carries no parameter and its
//   gradient is set to 0.  The other triangle of dA is not written.
#include "mbg_internal.cuh"

#include <type_traits>

namespace mbg {

namespace {

template <typename T>
__global__ void zero_diag_kernel(i64 n, T* a, i64 lda) {
    const i64 i = i64(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) a[i + i * lda] = T(0);
}

inline char flip(char t) { return is_n(t) ? 'T' : 'N'; }

int gemm_any(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a,
             i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    (void)slices;
    return sgemm_mode(mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int gemm_any(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a,
             i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    return dgemm_mode(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

// lower / upper triangle of C := alpha*op(A)*op(B) in the precision mode
int gemmt_any(int mode, int, char uplo, char ta, char tb, i64 n, i64 k, float alpha, const float* a,
              i64 lda, const float* b, i64 ldb, float* c, i64 ldc) {
    if (mode == MBG_MODE_BF16X3 || mode == MBG_MODE_BF16X6)
        return sgemm_split_tc(mode == MBG_MODE_BF16X6 ? 3 : 2, ta, tb, n, n, k, alpha, a, lda, b, ldb, 0.0f, c, ldc,
                              is_l(uplo) ? 'L' : 'U');
    return gemmt_plain<float>(uplo, ta, tb, n, k, alpha, a, lda, b, ldb, 0.0f, c, ldc);
}
int gemmt_any(int mode, int slices, char uplo, char ta, char tb, i64 n, i64 k, double alpha, const double* a,
              i64 lda, const double* b, i64 ldb, double* c, i64 ldc) {
    if (mode == MBG_MODE_OZAKI)
        return dgemm_ozaki_tc(slices, ta, tb, n, n, k, alpha, a, lda, b, ldb, 0.0, c, ldc, is_l(uplo) ? 'L' : 'U');
    return gemmt_plain<double>(uplo, ta, tb, n, k, alpha, a, lda, b, ldb, 0.0, c, ldc);
}

template <typename T>
int copy_matrix(i64 m, i64 n, const T* src, i64 lds, T* dst, i64 ldd) {
    if (m <= 0 || n <= 0) return MBG_OK;
    MBG_CUDA(cudaMemcpy2DAsync(dst, size_t(ldd) * sizeof(T), src, size_t(lds) * sizeof(T), size_t(m) * sizeof(T),
                               size_t(n), cudaMemcpyDeviceToDevice, stream()));
    return MBG_OK;
}

template <typename T>
int gemm_adjoint(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
                 const T* b, i64 ldb, const T* g, i64 ldg, T* da, i64 ldda, T* db, i64 lddb) {
    // argument checks: gemm numbering for 1..10 (src/level3/gemm.mojo:179-213), then ldg 12, ldda 14, lddb 16
    if (!is_n(ta) && !is_t(ta)) return 1;
    if (!is_n(tb) && !is_t(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    if (lda < imax(1, is_n(ta) ? m : k)) return 8;
    if (ldb < imax(1, is_n(tb) ? k : n)) return 10;
    if (ldg < imax(1, m)) return 12;
    if (da && ldda < imax(1, is_n(ta) ? m : k)) return 14;
    if (db && lddb < imax(1, is_n(tb) ? k : n)) return 16;
    Operand A, B, Gm, dA, dB;
    const bool need_a = db != nullptr, need_b = da != nullptr;
    if (need_a) MBG_TRY(A.prepare(a, is_n(ta) ? m : k, is_n(ta) ? k : m, lda, sizeof(T), true, false));
    if (need_b) MBG_TRY(B.prepare(b, is_n(tb) ? k : n, is_n(tb) ? n : k, ldb, sizeof(T), true, false));
    MBG_TRY(Gm.prepare(g, m, n, ldg, sizeof(T), true, false));
    if (da) MBG_TRY(dA.prepare(da, is_n(ta) ? m : k, is_n(ta) ? k : m, ldda, sizeof(T), false, true));
    if (db) MBG_TRY(dB.prepare(db, is_n(tb) ? k : n, is_n(tb) ? n : k, lddb, sizeof(T), false, true));
    const T* A_ = (const T*)A.dev;
    const T* B_ = (const T*)B.dev;
    const T* G_ = (const T*)Gm.dev;
    // dA and dB are independent products that each fill only part of the GPU at the
    // adjoint sizes (e.g. 96 and 64 tiles of 128 x 256 on 148 SMs): dB runs on a second
    // stream beside dA, ordered after the work before this call and before the work after it
    cudaStream_t s = stream(), aux = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    const bool overlap = da && db && mode != MBG_MODE_PLAIN;
    if constexpr (std::is_same<T, float>::value) {
        // split modes, products that together give fewer than four 128 x 256 tiles per SM:
        // both in one launch (sgemm_split_tc_dual), whose last wave is balanced across the
        // SMs; larger ones fill the GPU on their own with the wide tiles
        int dev = 0, sms = 148;
        bool small = false;
        if (overlap && (mode == MBG_MODE_BF16X3 || mode == MBG_MODE_BF16X6) && m > 0 && n > 0 && k > 0 &&
            alpha != T(0)) {
            MBG_CUDA(cudaGetDevice(&dev));
            MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const i64 wide = cdiv(m, 128) * cdiv(k, 256) + cdiv(k, 128) * cdiv(n, 256);
            small = wide < 4 * i64(sms);
        }
        if (small) {
            SplitProduct pa{}, pb{};
            T* oa = (T*)dA.dev;
            T* ob = (T*)dB.dev;
            if (is_n(ta))  // dA = alpha * G * op(B)^T   (m x k)
                pa = SplitProduct{'N', flip(tb), m, k, n, alpha, G_, Gm.dev_ld, B_, B.dev_ld, oa, dA.dev_ld};
            else           // dA = alpha * op(B) * G^T   (k x m)
                pa = SplitProduct{tb, 'T', k, m, n, alpha, B_, B.dev_ld, G_, Gm.dev_ld, oa, dA.dev_ld};
            if (is_n(tb))  // dB = alpha * op(A)^T * G   (k x n)
                pb = SplitProduct{flip(ta), 'N', k, n, m, alpha, A_, A.dev_ld, G_, Gm.dev_ld, ob, dB.dev_ld};
            else           // dB = alpha * G^T * op(A)   (n x k)
                pb = SplitProduct{'T', ta, n, k, m, alpha, G_, Gm.dev_ld, A_, A.dev_ld, ob, dB.dev_ld};
            MBG_TRY(sgemm_split_tc_dual(mode == MBG_MODE_BF16X6 ? 3 : 2, pa, pb));
            MBG_TRY(dA.finish());
            MBG_TRY(dB.finish());
            return finish_call(A.staged || B.staged || Gm.staged || dA.staged || dB.staged);
        }
    }
    if (overlap) {
        MBG_TRY(aux_stream(&aux));
        MBG_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
        MBG_CUDA(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
        MBG_CUDA(cudaEventRecord(ev_in, s));
        MBG_CUDA(cudaStreamWaitEvent(aux, ev_in, 0));
        cudaEventDestroy(ev_in);
        int st;
        {
            StreamScope on_aux(aux);
            T* o = (T*)dB.dev;
            if (is_n(tb))
                st = gemm_any(mode, slices, flip(ta), 'N', k, n, m, alpha, A_, A.dev_ld, G_, Gm.dev_ld, T(0), o,
                              dB.dev_ld);
            else
                st = gemm_any(mode, slices, 'T', ta, n, k, m, alpha, G_, Gm.dev_ld, A_, A.dev_ld, T(0), o, dB.dev_ld);
        }
        const cudaError_t e1 = cudaEventRecord(ev_out, aux);
        const cudaError_t e2 = cudaStreamWaitEvent(s, ev_out, 0);
        cudaEventDestroy(ev_out);
        if (st) return st;
        MBG_CUDA(e1);
        MBG_CUDA(e2);
    }
    if (da) {
        T* o = (T*)dA.dev;
        if (is_n(ta))  // dA = alpha * G * op(B)^T   (m x k)
            MBG_TRY(gemm_any(mode, slices, 'N', flip(tb), m, k, n, alpha, G_, Gm.dev_ld, B_, B.dev_ld, T(0), o, dA.dev_ld));
        else           // dA = alpha * op(B) * G^T   (k x m)
            MBG_TRY(gemm_any(mode, slices, tb, 'T', k, m, n, alpha, B_, B.dev_ld, G_, Gm.dev_ld, T(0), o, dA.dev_ld));
        MBG_TRY(dA.finish());
    }
    if (db && overlap) MBG_TRY(dB.finish());
    if (db && !overlap) {
        T* o = (T*)dB.dev;
        if (is_n(tb))  // dB = alpha * op(A)^T * G   (k x n)
            MBG_TRY(gemm_any(mode, slices, flip(ta), 'N', k, n, m, alpha, A_, A.dev_ld, G_, Gm.dev_ld, T(0), o, dB.dev_ld));
        else           // dB = alpha * G^T * op(A)   (n x k)
            MBG_TRY(gemm_any(mode, slices, 'T', ta, n, k, m, alpha, G_, Gm.dev_ld, A_, A.dev_ld, T(0), o, dB.dev_ld));
        MBG_TRY(dB.finish());
    }
    return finish_call(A.staged || B.staged || Gm.staged || dA.staged || dB.staged);
}

template <typename T>
int trsm_adjoint(int mode, int slices, char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha,
                 const T* a, i64 lda, const T* x, i64 ldx, const T* g, i64 ldg, T* db, i64 lddb, T* da,
                 i64 ldda) {
    // trsm numbering for 1..9 (src/level3/trsm.mojo:62-89), then ldx 11, ldg 13, lddb 15, ldda 17
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (!is_n(ta) && !is_t(ta)) return 3;
    if (!is_u(diag) && !is_n(diag)) return 4;
    if (m < 0) return 5;
    if (n < 0) return 6;
    const i64 na = is_l(side) ? m : n;
    if (lda < imax(1, na)) return 9;
    if (ldx < imax(1, m)) return 11;
    if (ldg < imax(1, m)) return 13;
    if (lddb < imax(1, m)) return 15;
    if (da && ldda < imax(1, na)) return 17;
    if (m == 0 || n == 0) return MBG_OK;
    Operand A, X, Gm, dB, dA;
    MBG_TRY(A.prepare(a, na, na, lda, sizeof(T), true, false));
    MBG_TRY(Gm.prepare(g, m, n, ldg, sizeof(T), true, false));
    MBG_TRY(dB.prepare(db, m, n, lddb, sizeof(T), false, true));
    if (da) {
        MBG_TRY(X.prepare(x, m, n, ldx, sizeof(T), true, false));
        MBG_TRY(dA.prepare(da, na, na, ldda, sizeof(T), true, true));  // other triangle preserved
    }
    T* dB_ = (T*)dB.dev;
    // dB = alpha * op(A)^{-T} G (left) or alpha * G op(A)^{-T} (right)
    MBG_TRY(copy_matrix<T>(m, n, (const T*)Gm.dev, Gm.dev_ld, dB_, dB.dev_ld));
    MBG_TRY(trsm_device<T>(mode, slices, 0, side, uplo, flip(ta), diag, m, n, alpha, (const T*)A.dev, A.dev_ld,
                           dB_, dB.dev_ld));
    if (da) {
        T* dA_ = (T*)dA.dev;
        const T* X_ = (const T*)X.dev;
        if (alpha == T(0)) {
            MBG_TRY(scale_triangle<T>(uplo, na, T(0), dA_, dA.dev_ld));  // X = 0: no gradient
        } else {
            const T c = T(-1) / alpha;  // W = dB / alpha
            if (is_l(side)) {
                if (is_n(ta))  // dA = -tri(W X^T)
                    MBG_TRY(gemmt_any(mode, slices, uplo, 'N', 'T', na, n, c, dB_, dB.dev_ld, X_, X.dev_ld, dA_, dA.dev_ld));
                else           // dA = -tri(X W^T)
                    MBG_TRY(gemmt_any(mode, slices, uplo, 'N', 'T', na, n, c, X_, X.dev_ld, dB_, dB.dev_ld, dA_, dA.dev_ld));
            } else {
                if (is_n(ta))  // dA = -tri(X^T W)
                    MBG_TRY(gemmt_any(mode, slices, uplo, 'T', 'N', na, m, c, X_, X.dev_ld, dB_, dB.dev_ld, dA_, dA.dev_ld));
                else           // dA = -tri(W^T X)
                    MBG_TRY(gemmt_any(mode, slices, uplo, 'T', 'N', na, m, c, dB_, dB.dev_ld, X_, X.dev_ld, dA_, dA.dev_ld));
            }
        }
        if (is_u(diag)) {
            zero_diag_kernel<T><<<unsigned(cdiv(na, 256)), 256, 0, stream()>>>(na, dA_, dA.dev_ld);
            MBG_TRY(check_launch("zero_diag"));
        }
        MBG_TRY(dA.finish());
    }
    MBG_TRY(dB.finish());
    return finish_call(A.staged || X.staged || Gm.staged || dB.staged || dA.staged);
}

}  // namespace
}  // namespace mbg

using namespace mbg;

extern "C" {

int mbg_sgemm_adjoint(int mode, char ta, char tb, int64_t m, int64_t n, int64_t k, float alpha, const float* a,
                      int64_t lda, const float* b, int64_t ldb, const float* g, int64_t ldg, float* da,
                      int64_t ldda, float* db, int64_t lddb) {
    if (mode != MBG_MODE_PLAIN && mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return gemm_adjoint<float>(mode, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, g, ldg, da, ldda, db, lddb);
}
int mbg_dgemm_adjoint(int mode, int slices, char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                      const double* a, int64_t lda, const double* b, int64_t ldb, const double* g, int64_t ldg,
                      double* da, int64_t ldda, double* db, int64_t lddb) {
    if (!(mode == MBG_MODE_PLAIN || (mode == MBG_MODE_OZAKI && slices >= 2 && slices <= 8))) return MBG_ERR_INVALID_MODE;
    return gemm_adjoint<double>(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, g, ldg, da, ldda, db, lddb);
}
int mbg_strsm_adjoint(int mode, char side, char uplo, char ta, char diag, int64_t m, int64_t n, float alpha,
                      const float* a, int64_t lda, const float* x, int64_t ldx, const float* g, int64_t ldg,
                      float* db, int64_t lddb, float* da, int64_t ldda) {
    if (mode != MBG_MODE_PLAIN && mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    return trsm_adjoint<float>(mode, 0, side, uplo, ta, diag, m, n, alpha, a, lda, x, ldx, g, ldg, db, lddb, da, ldda);
}
int mbg_dtrsm_adjoint(int mode, int slices, char side, char uplo, char ta, char diag, int64_t m, int64_t n,
                      double alpha, const double* a, int64_t lda, const double* x, int64_t ldx, const double* g,
                      int64_t ldg, double* db, int64_t lddb, double* da, int64_t ldda) {
    if (!(mode == MBG_MODE_PLAIN || (mode == MBG_MODE_OZAKI && slices >= 2 && slices <= 8))) return MBG_ERR_INVALID_MODE;
    return trsm_adjoint<double>(mode, slices, side, uplo, ta, diag, m, n, alpha, a, lda, x, ldx, g, ldg, db, lddb, da,
                                ldda);
}

}  // extern "C"
