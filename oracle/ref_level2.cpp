// ORACLE — test infrastructure only.
//
// A CPU restatement of the two level-2 routines of mojoBLAS that sit next to the
// level-3 hot path: gemv (y := alpha op(A) x + beta y) and trsv (op(A) x = b),
// written from the reference's algorithm so that the tests can compare the
// CUDA library's gemv / trsv with what the reference computes on the same
// inputs.  Nothing in the shipped library links, loads or calls this file.  It
// is built into the same shared object as ref_level3.cpp.
//
// Every routine cites the reference file:line it restates (paths relative to
// the mojoBLAS project root).  Vector indices follow the reference's 1-based
// kx / ky bookkeeping for negative increments (Netlib's convention: the first
// element of a vector with incx < 0 sits at x[(1 - n) * incx]).
//
// Reference behaviour kept as is: gemv accepts trans "N", "T", "C" in upper case
// only (src/level2/gemv.mojo:70-71), and lower-case letters are argument error 1.
// Reference behaviour NOT restated: trsv with uplo 'U', trans 'N' and incx != 1
// decrements its index before the first use (src/level2/trsv.mojo:113-125), so
// it pairs x[j - 1] with column j and, on the last step, reads before the start
// of x; the oracle computes Netlib's result there, under any flag.

#include <cstdint>
#include <algorithm>
#include <omp.h>

typedef int64_t i64;

namespace {

inline bool up(char t) { return t == 'U' || t == 'u'; }
inline bool lo(char t) { return t == 'L' || t == 'l'; }
inline bool tn(char t) { return t == 'N' || t == 'n'; }
inline bool tt(char t) { return t == 'T' || t == 't' || t == 'C' || t == 'c'; }

// gemv, src/level2/gemv.mojo:23-212.  Info (:69-84); quick return (:86-87);
// beta first, over y in its storage order (:107-127); alpha == 0 returns
// (:128-129).  NoTrans (:133-175): per column j with x(j) != 0, y += alpha x(j)
// A(:, j).  Trans (:176-210): per column j a dot product of A(:, j) with x,
// added as alpha * temp when temp != 0 (columns in parallel for n >= 256 when
// incx == 1).
template <typename T>
int gemv_ref(char trans, i64 m, i64 n, T alpha, const T* a, i64 lda, const T* x, i64 incx, T beta, T* y,
             i64 incy) {
    if (trans != 'N' && trans != 'T' && trans != 'C') return 1;
    if (m < 0) return 2;
    if (n < 0) return 3;
    if (lda < std::max<i64>(1, m)) return 6;
    if (incx == 0) return 8;
    if (incy == 0) return 11;
    if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return 0;
    const bool notrans = trans == 'N';
    const i64 lenx = notrans ? n : m, leny = notrans ? m : n;
    const i64 kx = incx > 0 ? 1 : 1 - (lenx - 1) * incx;  // 1-based start
    const i64 ky = incy > 0 ? 1 : 1 - (leny - 1) * incy;
    if (beta != T(1)) {
        i64 iy = ky;
        for (i64 i = 0; i < leny; ++i, iy += incy) y[iy - 1] = beta == T(0) ? T(0) : beta * y[iy - 1];
    }
    if (alpha == T(0)) return 0;
    if (notrans) {
        i64 jx = kx;
        for (i64 j = 0; j < n; ++j, jx += incx) {
            const T xj = x[jx - 1];
            if (xj == T(0)) continue;
            const T temp = alpha * xj;
            i64 iy = ky;
            for (i64 i = 0; i < m; ++i, iy += incy) y[iy - 1] = y[iy - 1] + temp * a[i + j * lda];
        }
        return 0;
    }
#pragma omp parallel for schedule(static) if (n >= 256 && incx == 1)
    for (i64 j = 0; j < n; ++j) {
        T temp = T(0);
        i64 ix = kx;
        for (i64 i = 0; i < m; ++i, ix += incx) temp = temp + a[i + j * lda] * x[ix - 1];
        if (temp != T(0)) {
            const i64 jy = ky - 1 + j * incy;
            y[jy] = y[jy] + alpha * temp;
        }
    }
    return 0;
}

// trsv, src/level2/trsv.mojo:20-214.  Info (:56-79); quick return (:81-82).
// NoTrans: column-oriented substitution, skipping zero entries of x (upper
// backwards :96-125, lower forwards :126-155).  Trans: dot-product substitution
// (upper forwards :157-183, lower backwards :184-213); x(j) /= A(j, j) unless
// diag 'U'.
template <typename T>
int trsv_ref(char uplo, char trans, char diag, i64 n, const T* a, i64 lda, T* x, i64 incx) {
    if (!up(uplo) && !lo(uplo)) return 1;
    if (!tn(trans) && !tt(trans)) return 2;
    if (!up(diag) && !(diag == 'N' || diag == 'n')) return 3;
    if (n < 0) return 4;
    if (lda < std::max<i64>(1, n)) return 6;
    if (incx == 0) return 8;
    if (n == 0) return 0;
    const bool nounit = !up(diag), upper = up(uplo);
    const i64 kx = incx > 0 ? 0 : -(n - 1) * incx;  // 0-based position of element 0
    auto X = [&](i64 j) -> T& { return x[kx + j * incx]; };
    if (tn(trans)) {
        if (upper) {
            for (i64 j = n - 1; j >= 0; --j) {
                if (X(j) == T(0)) continue;
                if (nounit) X(j) = X(j) / a[j + j * lda];
                const T temp = X(j);
                for (i64 i = j - 1; i >= 0; --i) X(i) = X(i) - temp * a[i + j * lda];
            }
        } else {
            for (i64 j = 0; j < n; ++j) {
                if (X(j) == T(0)) continue;
                if (nounit) X(j) = X(j) / a[j + j * lda];
                const T temp = X(j);
                for (i64 i = j + 1; i < n; ++i) X(i) = X(i) - temp * a[i + j * lda];
            }
        }
        return 0;
    }
    if (upper) {
        for (i64 j = 0; j < n; ++j) {
            T temp = X(j);
            for (i64 i = 0; i < j; ++i) temp = temp - a[i + j * lda] * X(i);
            if (nounit) temp = temp / a[j + j * lda];
            X(j) = temp;
        }
    } else {
        for (i64 j = n - 1; j >= 0; --j) {
            T temp = X(j);
            for (i64 i = n - 1; i > j; --i) temp = temp - a[i + j * lda] * X(i);
            if (nounit) temp = temp / a[j + j * lda];
            X(j) = temp;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int orc_sgemv(char trans, i64 m, i64 n, float alpha, const float* a, i64 lda, const float* x, i64 incx,
              float beta, float* y, i64 incy) {
    return gemv_ref<float>(trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
int orc_dgemv(char trans, i64 m, i64 n, double alpha, const double* a, i64 lda, const double* x, i64 incx,
              double beta, double* y, i64 incy) {
    return gemv_ref<double>(trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
int orc_strsv(char uplo, char trans, char diag, i64 n, const float* a, i64 lda, float* x, i64 incx) {
    return trsv_ref<float>(uplo, trans, diag, n, a, lda, x, incx);
}
int orc_dtrsv(char uplo, char trans, char diag, i64 n, const double* a, i64 lda, double* x, i64 incx) {
    return trsv_ref<double>(uplo, trans, diag, n, a, lda, x, incx);
}

}  // extern "C"
