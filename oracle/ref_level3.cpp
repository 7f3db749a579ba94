// ORACLE — test infrastructure only.
//
// A CPU restatement of mojoBLAS's level-3 routines (gemm / syrk / trsm, and the
// neighbours built on the same GEMM core: symm / syr2k / trmm), written
// from the reference's algorithm so that tests, the smoke check and the CPU
// baseline leg of the benchmark can compare the CUDA library against what the
// reference computes on the same inputs.  Nothing in the shipped library links,
// loads or calls this file.
//
// Every routine cites the reference file:line it restates (paths are relative to
// the mojoBLAS project root).  Blocking constants are the reference's
// (src/level3/_tuning.mojo) with the Apple-M2 SIMD widths that the reference was
// tuned for (float32 SIMD width 4, float64 SIMD width 2), because the row
// grouping of gemm_v3 / gemm_v7 depends on them.
//
// Behavioural quirks of the reference are reproduced only when the caller sets
// ORC_BUG_COMPAT in `flags`:
//   * gemm_v7 (float64 NN, n >= 512) never applies alpha
//     (src/level3/gemm.mojo:912-1132);
//   * trsm with side='R' ignores trans_a: the Trans branches are copies of the
//     NoTrans ones (src/level3/trsm.mojo:224-273 vs :170-222);
//   * left-side symm skips step l of column j entirely when B(l,j) == 0, which
//     also drops that step's alpha * sum_i A(i,l) B(i,j) from C(l,j)
//     (src/level3/symm.mojo:113, :131).
// Without the flag the oracle computes the Netlib-defined result with the same
// loop structure, which is what the CUDA library implements.
//
// Threading: OpenMP over the same loop the reference parallelises.

#include <cstdint>
#include <cstring>
#include <algorithm>
#include <omp.h>

typedef int64_t i64;

enum { ORC_BUG_COMPAT = 1 };

static inline bool is_n(char t) { return t == 'N' || t == 'n'; }
static inline bool is_t(char t) { return t == 'T' || t == 't' || t == 'C' || t == 'c'; }
static inline bool is_u(char t) { return t == 'U' || t == 'u'; }
static inline bool is_l(char t) { return t == 'L' || t == 'l'; }
static inline bool is_r(char t) { return t == 'R' || t == 'r'; }

// Tuning constants, src/level3/_tuning.mojo:4,13-16,51-57.
static const i64 GEMM_DISPATCH_THRESHOLD = 512;
static const i64 V3_MR = 4, V3_NR = 8, V3_TK = 256;        // gemm.mojo:380-382 (MR = f32 SIMD width on M2)
static const i64 V7_MR = 2, V7_NR = 16, V7_TK = 128, V7_MC = 256;  // _tuning.mojo:13-16 (MR = f64 SIMD width on M2)
static const i64 V11_TK = 1024, V11_ROW_PAR_THRESHOLD = 1024;      // _tuning.mojo:51-57
static const i64 PAR_THRESHOLD = 64;                                // gemm.mojo:255, syrk.mojo:112

// Netlib argument checks shared by _gemm_naive / gemm_v3 / gemm_v7,
// src/level3/gemm.mojo:179-213.
static int gemm_info(char ta, char tb, i64 m, i64 n, i64 k, i64 lda, i64 ldb, i64 ldc) {
    if (!is_n(ta) && !is_t(ta)) return 1;
    if (!is_n(tb) && !is_t(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    if (lda < std::max<i64>(1, is_n(ta) ? m : k)) return 8;
    if (ldb < std::max<i64>(1, is_n(tb) ? k : n)) return 10;
    if (ldc < std::max<i64>(1, m)) return 13;
    return 0;
}

template <typename T>
static void scale_or_zero(i64 m, i64 n, T beta, T* c, i64 ldc) {
    if (beta == T(0)) {
        for (i64 j = 0; j < n; ++j)
            for (i64 i = 0; i < m; ++i) c[i + j * ldc] = T(0);
    } else if (beta != T(1)) {
        for (i64 j = 0; j < n; ++j)
            for (i64 i = 0; i < m; ++i) c[i + j * ldc] = beta * c[i + j * ldc];
    }
}

// Threads that ran the last _gemm_naive call's column loop (1 when n is below
// the reference's parallel threshold), reported by orc_naive_threads().
static int g_naive_threads = 0;

// _gemm_naive, src/level3/gemm.mojo:127-377.  Column j of C is owned by one task
// (parallel when n >= 64, :255/:276); within it, beta first, then an axpy per l in
// ascending order, skipped when the B element is zero (:263, :299, :336, :365).
template <typename T>
static int gemm_naive(char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
                      const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    int info = gemm_info(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    if (alpha == T(0) || k == 0) {  // :220-237
        scale_or_zero(m, n, beta, c, ldc);
        return 0;
    }
    const bool nta = is_n(ta), ntb = is_n(tb);
    int used = 1;
#pragma omp parallel if (n >= PAR_THRESHOLD)
    {
#pragma omp single
        used = omp_get_num_threads();
#pragma omp for schedule(dynamic, 1)
        for (i64 j = 0; j < n; ++j) {
            T* cj = c + j * ldc;
            if (beta == T(0)) {
                for (i64 i = 0; i < m; ++i) cj[i] = T(0);
            } else if (beta != T(1)) {
                for (i64 i = 0; i < m; ++i) cj[i] = beta * cj[i];
            }
            for (i64 l = 0; l < k; ++l) {
                const T bv = ntb ? b[l + j * ldb] : b[j + l * ldb];
                if (bv == T(0)) continue;
                const T temp = alpha * bv;
                if (nta) {  // NN :262-274, NT :298-310 — vectorised column axpy
                    const T* al = a + l * lda;
                    for (i64 i = 0; i < m; ++i) cj[i] = cj[i] + temp * al[i];
                } else {    // TN :335-340, TT :364-369 — scalar strided loads
                    const T* al = a + l;
                    for (i64 i = 0; i < m; ++i) cj[i] = cj[i] + temp * al[i * lda];
                }
            }
        }
    }
    g_naive_threads = used;
    return 0;
}

// gemm_v3, src/level3/gemm.mojo:385-560 (float64 NN, n < 512).  Beta first
// (:462-477); per 8-column group and 256-deep k panel, each full MR-row block
// accumulates sum_l (alpha*a) * b in registers and adds it to C (:499-545); tail
// rows add alpha * sum_l a*b (:547-553).
template <typename T>
static int gemm_v3(i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda, const T* b, i64 ldb,
                   T beta, T* c, i64 ldc) {
    int info = gemm_info('N', 'N', m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    scale_or_zero(m, n, beta, c, ldc);
    if (alpha == T(0) || k == 0) return 0;
    const i64 groups = (n + V3_NR - 1) / V3_NR;
#pragma omp parallel for schedule(dynamic, 1) if (groups >= 8)
    for (i64 g = 0; g < groups; ++g) {
        const i64 j0 = g * V3_NR, jlen = std::min(V3_NR, n - j0);
        for (i64 k0 = 0; k0 < k; k0 += V3_TK) {
            const i64 klen = std::min(V3_TK, k - k0);
            i64 ir = 0;
            for (; ir + V3_MR <= m; ir += V3_MR) {
                T acc[V3_NR][V3_MR] = {};
                for (i64 l = 0; l < klen; ++l) {
                    T av[V3_MR];
                    for (i64 r = 0; r < V3_MR; ++r) av[r] = alpha * a[ir + r + (k0 + l) * lda];
                    for (i64 q = 0; q < V3_NR; ++q) {
                        const T bq = q < jlen ? b[(k0 + l) + (j0 + q) * ldb] : T(0);
                        for (i64 r = 0; r < V3_MR; ++r) acc[q][r] = av[r] * bq + acc[q][r];
                    }
                }
                for (i64 q = 0; q < jlen; ++q)
                    for (i64 r = 0; r < V3_MR; ++r) c[ir + r + (j0 + q) * ldc] += acc[q][r];
            }
            for (; ir < m; ++ir) {
                for (i64 q = 0; q < jlen; ++q) {
                    T s = 0;
                    for (i64 l = 0; l < klen; ++l) s += a[ir + (k0 + l) * lda] * b[(k0 + l) + (j0 + q) * ldb];
                    c[ir + (j0 + q) * ldc] += alpha * s;
                }
            }
        }
    }
    return 0;
}

// gemm_v7, src/level3/gemm.mojo:817-1132 (float64 NN, n >= 512).  Beta first
// (:895-910); for each 256-row block and 128-deep k panel, C += sum_l a*b per
// 16-column group (:912-1124).  The reference never multiplies by alpha
// (pack :927-928, kernel :972-991, tail :1117-1123); ORC_BUG_COMPAT keeps that,
// otherwise alpha scales each panel sum.
template <typename T>
static int gemm_v7(i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda, const T* b, i64 ldb,
                   T beta, T* c, i64 ldc, int flags) {
    int info = gemm_info('N', 'N', m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return 0;
    scale_or_zero(m, n, beta, c, ldc);
    if (alpha == T(0) || k == 0) return 0;
    const bool apply_alpha = !(flags & ORC_BUG_COMPAT);
    const i64 groups = (n + V7_NR - 1) / V7_NR;
    for (i64 mc0 = 0; mc0 < m; mc0 += V7_MC) {
        const i64 mc_len = std::min(V7_MC, m - mc0);
        for (i64 k0 = 0; k0 < k; k0 += V7_TK) {
            const i64 klen = std::min(V7_TK, k - k0);
#pragma omp parallel for schedule(dynamic, 1) if (groups >= 12)
            for (i64 g = 0; g < groups; ++g) {
                const i64 j0 = g * V7_NR, jlen = std::min(V7_NR, n - j0);
                i64 ir = 0;
                for (; ir + V7_MR <= mc_len; ir += V7_MR) {
                    T acc[V7_NR][V7_MR] = {};
                    for (i64 l = 0; l < klen; ++l) {
                        T av[V7_MR];
                        for (i64 r = 0; r < V7_MR; ++r) av[r] = a[mc0 + ir + r + (k0 + l) * lda];
                        for (i64 q = 0; q < V7_NR; ++q) {
                            const T bq = q < jlen ? b[(k0 + l) + (j0 + q) * ldb] : T(0);
                            for (i64 r = 0; r < V7_MR; ++r) acc[q][r] = av[r] * bq + acc[q][r];
                        }
                    }
                    for (i64 q = 0; q < jlen; ++q)
                        for (i64 r = 0; r < V7_MR; ++r) {
                            T v = acc[q][r];
                            if (apply_alpha) v = alpha * v;
                            c[mc0 + ir + r + (j0 + q) * ldc] += v;
                        }
                }
                for (; ir < mc_len; ++ir) {
                    for (i64 q = 0; q < jlen; ++q) {
                        T s = 0;
                        for (i64 l = 0; l < klen; ++l) s += a[mc0 + ir + (k0 + l) * lda] * b[(k0 + l) + (j0 + q) * ldb];
                        if (apply_alpha) s = alpha * s;
                        c[(mc0 + ir) + (j0 + q) * ldc] += s;
                    }
                }
            }
        }
    }
    return 0;
}

// gemm_v11 arithmetic, src/level3/gemm.mojo:2092-2436 (float32 NN).  The
// reference runs Apple-AMX outer products; what it computes per element is:
// no argument checks (the dispatcher calls it directly, :107-112); alpha==0 or
// k==0 scales C (:2170-2187); beta is applied first unless beta==0 and
// n <= 1024, in which case the first k panel stores instead of adds
// (:2189-2207, :2346-2349); alpha is folded into the packed A (:2256-2258); each
// 1024-deep k panel's fused-multiply-add sum is added to C (:2215, :2286-2353).
static int gemm_v11(i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda, const float* b,
                    i64 ldb, float beta, float* c, i64 ldc) {
    if (m == 0 || n == 0) return 0;
    if (alpha == 0.0f || k == 0) {
        scale_or_zero(m, n, beta, c, ldc);
        return 0;
    }
    const bool direct = (beta == 0.0f) && n <= V11_ROW_PAR_THRESHOLD;
    if (beta == 0.0f && !direct) scale_or_zero(m, n, 0.0f, c, ldc);
    else if (beta != 0.0f && beta != 1.0f) scale_or_zero(m, n, beta, c, ldc);
    for (i64 k0 = 0; k0 < k; k0 += V11_TK) {
        const i64 klen = std::min(V11_TK, k - k0);
        const bool store = direct && k0 == 0;
#pragma omp parallel for schedule(static)
        for (i64 j = 0; j < n; ++j) {
            float* cj = c + j * ldc;
            const float* bj = b + k0 + j * ldb;
            // accumulate the panel in a column buffer (one Z-tile column per lane)
            float zb[64];
            for (i64 i0 = 0; i0 < m; i0 += 64) {
                const i64 ilen = std::min<i64>(64, m - i0);
                for (i64 r = 0; r < ilen; ++r) zb[r] = 0.0f;
                for (i64 l = 0; l < klen; ++l) {
                    const float bv = bj[l];
                    const float* al = a + i0 + (k0 + l) * lda;
                    for (i64 r = 0; r < ilen; ++r) zb[r] = __builtin_fmaf(alpha * al[r], bv, zb[r]);
                }
                if (store) for (i64 r = 0; r < ilen; ++r) cj[i0 + r] = zb[r];
                else       for (i64 r = 0; r < ilen; ++r) cj[i0 + r] += zb[r];
            }
        }
    }
    return 0;
}

// gemm dispatcher, src/level3/gemm.mojo:56-124: float32 NN -> v11; float64 NN ->
// v3 (n < 512) or v7; every transposed case -> _gemm_naive.
template <typename T> struct Dispatch;
template <> struct Dispatch<float> {
    static int nn(i64 m, i64 n, i64 k, float al, const float* a, i64 lda, const float* b, i64 ldb,
                  float be, float* c, i64 ldc, int) {
        return gemm_v11(m, n, k, al, a, lda, b, ldb, be, c, ldc);
    }
};
template <> struct Dispatch<double> {
    static int nn(i64 m, i64 n, i64 k, double al, const double* a, i64 lda, const double* b, i64 ldb,
                  double be, double* c, i64 ldc, int flags) {
        if (n < GEMM_DISPATCH_THRESHOLD) return gemm_v3(m, n, k, al, a, lda, b, ldb, be, c, ldc);
        return gemm_v7(m, n, k, al, a, lda, b, ldb, be, c, ldc, flags);
    }
};

template <typename T>
static int gemm_dispatch(char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
                         const T* b, i64 ldb, T beta, T* c, i64 ldc, int flags) {
    if (is_n(ta) && is_n(tb)) return Dispatch<T>::nn(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags);
    return gemm_naive(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

// syrk, src/level3/syrk.mojo:20-200.  Info (:60-83); quick return (:85-86);
// beta on the triangle (:93-110); NoTrans: per-column axpy over the triangle,
// skipped when A(j,l)==0 (:115-166); Trans: scalar dot per (i,j) (:167-198).
template <typename T>
static int syrk_ref(char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda, T beta,
                    T* c, i64 ldc) {
    if (!is_u(uplo) && !is_l(uplo)) return 1;
    if (!is_n(trans) && !is_t(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    if (lda < std::max<i64>(1, is_n(trans) ? n : k)) return 7;
    if (ldc < std::max<i64>(1, n)) return 10;
    if (n == 0 || (alpha == T(0) && beta == T(1))) return 0;
    const bool upper = is_u(uplo);
    if (beta == T(0)) {
        for (i64 j = 0; j < n; ++j)
            for (i64 i = upper ? 0 : j; i < (upper ? j + 1 : n); ++i) c[i + j * ldc] = T(0);
    } else if (beta != T(1)) {
        for (i64 j = 0; j < n; ++j)
            for (i64 i = upper ? 0 : j; i < (upper ? j + 1 : n); ++i) c[i + j * ldc] = beta * c[i + j * ldc];
    }
    if (alpha == T(0)) return 0;
    if (is_n(trans)) {
#pragma omp parallel for schedule(dynamic, 1) if (n >= PAR_THRESHOLD)
        for (i64 j = 0; j < n; ++j) {
            T* cj = c + j * ldc;
            const i64 i0 = upper ? 0 : j, i1 = upper ? j + 1 : n;
            for (i64 l = 0; l < k; ++l) {
                const T ajl = a[j + l * lda];
                if (ajl == T(0)) continue;
                const T temp = alpha * ajl;
                const T* al = a + l * lda;
                for (i64 i = i0; i < i1; ++i) cj[i] = cj[i] + temp * al[i];
            }
        }
    } else {
#pragma omp parallel for schedule(dynamic, 1) if (n >= PAR_THRESHOLD)
        for (i64 j = 0; j < n; ++j) {
            const i64 i0 = upper ? 0 : j, i1 = upper ? j + 1 : n;
            for (i64 i = i0; i < i1; ++i) {
                T temp = 0;
                for (i64 l = 0; l < k; ++l) temp = temp + a[l + i * lda] * a[l + j * lda];
                c[i + j * ldc] = c[i + j * ldc] + alpha * temp;
            }
        }
    }
    return 0;
}

// trsm, src/level3/trsm.mojo:20-275.  Info (:62-89); quick return (:91-92);
// B *= alpha when alpha != 1 (:96-103); then unblocked substitution.  The
// reference is single-threaded; the oracle parallelises over right-hand-side
// columns for the left side (columns are independent) to keep the tests quick,
// which does not change any element's arithmetic.
template <typename T>
static int trsm_ref(char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha, const T* a,
                    i64 lda, T* b, i64 ldb, int flags) {
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (!is_n(ta) && !is_t(ta)) return 3;
    if (!is_u(diag) && !is_n(diag)) return 4;
    if (m < 0) return 5;
    if (n < 0) return 6;
    if (lda < std::max<i64>(1, is_l(side) ? m : n)) return 9;
    if (ldb < std::max<i64>(1, m)) return 11;
    if (m == 0 || n == 0) return 0;
    if (alpha != T(1))
        for (i64 j = 0; j < n; ++j)
            for (i64 i = 0; i < m; ++i) b[i + j * ldb] = alpha * b[i + j * ldb];
    const bool upper = is_u(uplo), notrans = is_n(ta), nounit = is_n(diag);
    if (is_l(side)) {
        if (notrans) {
            if (upper) {  // :111-129 backward column axpy
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
                for (i64 j = 0; j < n; ++j) {
                    T* bj = b + j * ldb;
                    for (i64 l = m - 1; l >= 0; --l) {
                        if (bj[l] == T(0)) continue;
                        if (nounit) bj[l] = bj[l] / a[l + l * lda];
                        const T piv = bj[l];
                        const T* al = a + l * lda;
                        for (i64 i = 0; i < l; ++i) bj[i] = bj[i] - piv * al[i];
                    }
                }
            } else {      // :130-148 forward column axpy
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
                for (i64 j = 0; j < n; ++j) {
                    T* bj = b + j * ldb;
                    for (i64 l = 0; l < m; ++l) {
                        if (bj[l] == T(0)) continue;
                        if (nounit) bj[l] = bj[l] / a[l + l * lda];
                        const T piv = bj[l];
                        const T* al = a + l * lda;
                        for (i64 i = l + 1; i < m; ++i) bj[i] = bj[i] - piv * al[i];
                    }
                }
            }
        } else {
            if (upper) {  // :152-160 U^T X = B, forward dots
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
                for (i64 j = 0; j < n; ++j) {
                    T* bj = b + j * ldb;
                    for (i64 i = 0; i < m; ++i) {
                        for (i64 l = 0; l < i; ++l) bj[i] = bj[i] - a[l + i * lda] * bj[l];
                        if (nounit) bj[i] = bj[i] / a[i + i * lda];
                    }
                }
            } else {      // :161-168 L^T X = B, backward dots
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
                for (i64 j = 0; j < n; ++j) {
                    T* bj = b + j * ldb;
                    for (i64 i = m - 1; i >= 0; --i) {
                        for (i64 l = i + 1; l < m; ++l) bj[i] = bj[i] - a[l + i * lda] * bj[l];
                        if (nounit) bj[i] = bj[i] / a[i + i * lda];
                    }
                }
            }
        }
        return 0;
    }
    // Right side, :169-273.  The reference's Trans branches repeat the NoTrans
    // loops (:224-273); Netlib's X*op(A)=B with op(A)=A^T walks the other way
    // and reads A(j,l) instead of A(l,j).
    const bool right_trans = !notrans && !(flags & ORC_BUG_COMPAT);
    // forward over columns when the effective op(A) is upper triangular
    const bool forward = right_trans ? !upper : upper;
    auto aval = [&](i64 l, i64 j) -> T { return right_trans ? a[j + l * lda] : a[l + j * lda]; };
    if (forward) {
        for (i64 j = 0; j < n; ++j) {
            T* bj = b + j * ldb;
            for (i64 l = 0; l < j; ++l) {
                const T alj = aval(l, j);
                const T* bl = b + l * ldb;
                for (i64 i = 0; i < m; ++i) bj[i] = bj[i] - alj * bl[i];
            }
            if (nounit) {
                const T inv = T(1) / a[j + j * lda];
                for (i64 i = 0; i < m; ++i) bj[i] = bj[i] * inv;
            }
        }
    } else {
        for (i64 j = n - 1; j >= 0; --j) {
            T* bj = b + j * ldb;
            for (i64 l = j + 1; l < n; ++l) {
                const T alj = aval(l, j);
                const T* bl = b + l * ldb;
                for (i64 i = 0; i < m; ++i) bj[i] = bj[i] - alj * bl[i];
            }
            if (nounit) {
                const T inv = T(1) / a[j + j * lda];
                for (i64 i = 0; i < m; ++i) bj[i] = bj[i] * inv;
            }
        }
    }
    return 0;
}

// symm, src/level3/symm.mojo:20-241.  Info (:69-86); quick return (:88-89);
// columns of C in parallel when n >= 64 (:152-156, :235-239).  Per column: beta
// first (:102-110, :163-171).  Left side: for each l (downwards for 'U', :112-129;
// upwards for 'L', :130-151) C(i,j) += alpha*B(l,j)*A(i,l) over the stored part of
// column l, and C(l,j) += alpha*B(l,j)*A(l,l) + alpha*sum_i A(i,l)*B(i,j).  Right
// side (:173-233): C(:,j) += alpha*A(j,j)*B(:,j), then the off-diagonal columns of
// B with A read from the stored triangle.
// The reference skips the whole step l when B(l,j) == 0 (:113, :131), which also
// drops the alpha*sum term of C(l,j); that quirk reproduces only with
// ORC_BUG_COMPAT, otherwise the sum is always added (Netlib dsymm).
template <typename T>
static int symm_ref(char side, char uplo, i64 m, i64 n, T alpha, const T* a, i64 lda, const T* b,
                    i64 ldb, T beta, T* c, i64 ldc, int flags) {
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (lda < std::max<i64>(1, is_l(side) ? m : n)) return 7;
    if (ldb < std::max<i64>(1, m)) return 9;
    if (ldc < std::max<i64>(1, m)) return 12;
    if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return 0;
    const bool left = is_l(side), upper = is_u(uplo);
    const bool skip_zero_pivot = (flags & ORC_BUG_COMPAT) != 0;
#pragma omp parallel for schedule(dynamic, 1) if (n >= PAR_THRESHOLD)
    for (i64 j = 0; j < n; ++j) {
        T* cj = c + j * ldc;
        const T* bj = b + j * ldb;
        if (beta == T(0)) {
            for (i64 i = 0; i < m; ++i) cj[i] = T(0);
        } else if (beta != T(1)) {
            for (i64 i = 0; i < m; ++i) cj[i] = beta * cj[i];
        }
        if (left) {
            for (i64 s = 0; s < m; ++s) {
                const i64 l = upper ? m - 1 - s : s;
                if (bj[l] == T(0) && skip_zero_pivot) continue;
                const T temp1 = alpha * bj[l];
                T temp2 = T(0);
                const T* al = a + l * lda;
                const i64 i0 = upper ? 0 : l + 1, i1 = upper ? l : m;
                for (i64 i = i0; i < i1; ++i) {
                    cj[i] = cj[i] + temp1 * al[i];
                    temp2 = temp2 + al[i] * bj[i];
                }
                cj[l] = cj[l] + temp1 * al[l] + alpha * temp2;
            }
        } else {
            const T td = alpha * a[j + j * lda];
            for (i64 i = 0; i < m; ++i) cj[i] = cj[i] + td * bj[i];
            for (i64 k = 0; k < n; ++k) {
                if (k == j) continue;
                // A(k,j) for k < j lives above the diagonal; for k > j below it
                const bool above = k < j;
                const T akj = (above == upper) ? a[k + j * lda] : a[j + k * lda];
                const T temp = alpha * akj;
                const T* bk = b + k * ldb;
                for (i64 i = 0; i < m; ++i) cj[i] = cj[i] + temp * bk[i];
            }
        }
    }
    return 0;
}

// syr2k, src/level3/syr2k.mojo:20-190.  Info (:69-93); quick return (:95-96);
// beta on the triangle (:101-118); alpha == 0 returns (:120-121).  NoTrans
// (:125-167): per column j and each l with A(j,l) or B(j,l) nonzero,
// C(i,j) += alpha*A(j,l)*B(i,l) + alpha*B(j,l)*A(i,l) over the triangle's rows.
// Trans (:169-188): two dot products per element, C(i,j) += alpha*(t1 + t2).
// The reference runs the columns serially; they are independent, so the oracle
// runs them in parallel, which changes no element's arithmetic.
template <typename T>
static int syr2k_ref(char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda, const T* b,
                     i64 ldb, T beta, T* c, i64 ldc) {
    if (!is_u(uplo) && !is_l(uplo)) return 1;
    if (!is_n(trans) && !is_t(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    if (lda < std::max<i64>(1, is_n(trans) ? n : k)) return 7;
    if (ldb < std::max<i64>(1, is_n(trans) ? n : k)) return 9;
    if (ldc < std::max<i64>(1, n)) return 12;
    if (n == 0 || (alpha == T(0) && beta == T(1))) return 0;
    const bool upper = is_u(uplo);
    for (i64 j = 0; j < n; ++j)
        for (i64 i = upper ? 0 : j; i < (upper ? j + 1 : n); ++i)
            c[i + j * ldc] = beta == T(0) ? T(0) : (beta == T(1) ? c[i + j * ldc] : beta * c[i + j * ldc]);
    if (alpha == T(0)) return 0;
#pragma omp parallel for schedule(dynamic, 1) if (n >= PAR_THRESHOLD)
    for (i64 j = 0; j < n; ++j) {
        T* cj = c + j * ldc;
        const i64 i0 = upper ? 0 : j, i1 = upper ? j + 1 : n;
        if (is_n(trans)) {
            for (i64 l = 0; l < k; ++l) {
                const T ajl = a[j + l * lda], bjl = b[j + l * ldb];
                if (ajl == T(0) && bjl == T(0)) continue;
                const T temp1 = alpha * ajl, temp2 = alpha * bjl;
                const T* al = a + l * lda;
                const T* bl = b + l * ldb;
                for (i64 i = i0; i < i1; ++i) cj[i] = cj[i] + temp1 * bl[i] + temp2 * al[i];
            }
        } else {
            for (i64 i = i0; i < i1; ++i) {
                T t1 = T(0), t2 = T(0);
                for (i64 l = 0; l < k; ++l) {
                    t1 = t1 + a[l + i * lda] * b[l + j * ldb];
                    t2 = t2 + b[l + i * ldb] * a[l + j * lda];
                }
                cj[i] = cj[i] + alpha * (t1 + t2);
            }
        }
    }
    return 0;
}

// trmm, src/level3/trmm.mojo:20-305.  Info (:63-89); quick return (:91-92);
// alpha == 0 sets B to zero (:94-98).  Left side: each column of B is
// independent (the reference parallelises the Trans branches, :148-185, and runs
// the NoTrans ones serially, :108-147; the oracle runs all of them in parallel,
// which changes no element's arithmetic).  Left/NoTrans/Upper walks k upwards,
// B(0:k,j) += alpha*B(k,j)*A(0:k,k), then B(k,j) = alpha*B(k,j)*A(k,k) (:109-127);
// Lower walks k downwards (:128-147); both skip B(k,j) == 0.  Left/Trans forms
// each B(i,j) as a dot product with the not yet updated entries (:150-185).
// Right/NoTrans runs columns in the order of the dependence (downwards for 'U',
// :189-218; upwards for 'L', :219-248): scale column j by alpha*A(j,j), then add
// alpha*A(k,j)*B(:,k) over the stored part, skipping A(k,j) == 0.  Right/Trans
// (:249-305) adds alpha*A(j,k)*B(:,k) into the columns j before (U) or after (L)
// k, then scales column k when alpha*A(k,k) != 1.
template <typename T>
static int trmm_ref(char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha, const T* a,
                    i64 lda, T* b, i64 ldb) {
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (!is_n(ta) && !is_t(ta)) return 3;
    if (!is_u(diag) && !is_n(diag)) return 4;
    if (m < 0) return 5;
    if (n < 0) return 6;
    if (lda < std::max<i64>(1, is_l(side) ? m : n)) return 9;
    if (ldb < std::max<i64>(1, m)) return 11;
    if (m == 0 || n == 0) return 0;
    if (alpha == T(0)) {
        for (i64 j = 0; j < n; ++j)
            for (i64 i = 0; i < m; ++i) b[i + j * ldb] = T(0);
        return 0;
    }
    const bool upper = is_u(uplo), notrans = is_n(ta), nounit = is_n(diag);
    if (is_l(side)) {
#pragma omp parallel for schedule(static) if (n >= PAR_THRESHOLD)
        for (i64 j = 0; j < n; ++j) {
            T* bj = b + j * ldb;
            if (notrans && upper) {
                for (i64 k = 0; k < m; ++k) {
                    if (bj[k] == T(0)) continue;
                    T temp = alpha * bj[k];
                    const T* ak = a + k * lda;
                    for (i64 i = 0; i < k; ++i) bj[i] = bj[i] + temp * ak[i];
                    if (nounit) temp = temp * ak[k];
                    bj[k] = temp;
                }
            } else if (notrans) {
                for (i64 k = m - 1; k >= 0; --k) {
                    if (bj[k] == T(0)) continue;
                    const T temp = alpha * bj[k];
                    const T* ak = a + k * lda;
                    bj[k] = nounit ? temp * ak[k] : temp;
                    for (i64 i = k + 1; i < m; ++i) bj[i] = bj[i] + temp * ak[i];
                }
            } else if (upper) {
                for (i64 i = m - 1; i >= 0; --i) {
                    T temp = bj[i];
                    if (nounit) temp = temp * a[i + i * lda];
                    for (i64 l = 0; l < i; ++l) temp = temp + a[l + i * lda] * bj[l];
                    bj[i] = alpha * temp;
                }
            } else {
                for (i64 i = 0; i < m; ++i) {
                    T temp = bj[i];
                    if (nounit) temp = temp * a[i + i * lda];
                    for (i64 l = i + 1; l < m; ++l) temp = temp + a[l + i * lda] * bj[l];
                    bj[i] = alpha * temp;
                }
            }
        }
        return 0;
    }
    auto axpy_col = [&](T temp, i64 src, i64 dst) {
        const T* bs = b + src * ldb;
        T* bd = b + dst * ldb;
        for (i64 i = 0; i < m; ++i) bd[i] = bd[i] + temp * bs[i];
    };
    auto scale_col = [&](T temp, i64 j) {
        T* bj = b + j * ldb;
        for (i64 i = 0; i < m; ++i) bj[i] = temp * bj[i];
    };
    if (notrans) {
        for (i64 s = 0; s < n; ++s) {
            const i64 j = upper ? n - 1 - s : s;
            scale_col(nounit ? alpha * a[j + j * lda] : alpha, j);
            const i64 k0 = upper ? 0 : j + 1, k1 = upper ? j : n;
            for (i64 k = k0; k < k1; ++k)
                if (a[k + j * lda] != T(0)) axpy_col(alpha * a[k + j * lda], k, j);
        }
        return 0;
    }
    for (i64 s = 0; s < n; ++s) {
        const i64 k = upper ? s : n - 1 - s;
        const i64 j0 = upper ? 0 : k + 1, j1 = upper ? k : n;
        for (i64 j = j0; j < j1; ++j)
            if (a[j + k * lda] != T(0)) axpy_col(alpha * a[j + k * lda], k, j);
        const T temp = nounit ? alpha * a[k + k * lda] : alpha;
        if (temp != T(1)) scale_col(temp, k);
    }
    return 0;
}

extern "C" {

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_max_threads(void) { return omp_get_max_threads(); }
int orc_naive_threads(void) { return g_naive_threads; }

// Full dispatch, as a user of the reference's gemm reaches it.
int orc_sgemm(char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda,
              const float* b, i64 ldb, float beta, float* c, i64 ldc, int flags) {
    return gemm_dispatch<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags);
}
int orc_dgemm(char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
              const double* b, i64 ldb, double beta, double* c, i64 ldc, int flags) {
    return gemm_dispatch<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags);
}
// Individual kernels, so that a bounded sample (a column slice) runs the same
// algorithm the full-size call is dispatched to.
int orc_sgemm_naive(char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda,
                    const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    return gemm_naive<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_dgemm_naive(char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
                    const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    return gemm_naive<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_sgemm_v11(i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda, const float* b,
                  i64 ldb, float beta, float* c, i64 ldc) {
    return gemm_v11(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_dgemm_v3(i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda, const double* b,
                 i64 ldb, double beta, double* c, i64 ldc) {
    return gemm_v3<double>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_dgemm_v7(i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda, const double* b,
                 i64 ldb, double beta, double* c, i64 ldc, int flags) {
    return gemm_v7<double>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags);
}
int orc_ssyrk(char uplo, char trans, i64 n, i64 k, float alpha, const float* a, i64 lda,
              float beta, float* c, i64 ldc) {
    return syrk_ref<float>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_dsyrk(char uplo, char trans, i64 n, i64 k, double alpha, const double* a, i64 lda,
              double beta, double* c, i64 ldc) {
    return syrk_ref<double>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_strsm(char side, char uplo, char ta, char diag, i64 m, i64 n, float alpha, const float* a,
              i64 lda, float* b, i64 ldb, int flags) {
    return trsm_ref<float>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, flags);
}
int orc_dtrsm(char side, char uplo, char ta, char diag, i64 m, i64 n, double alpha, const double* a,
              i64 lda, double* b, i64 ldb, int flags) {
    return trsm_ref<double>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, flags);
}
int orc_ssymm(char side, char uplo, i64 m, i64 n, float alpha, const float* a, i64 lda, const float* b,
              i64 ldb, float beta, float* c, i64 ldc, int flags) {
    return symm_ref<float>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, flags);
}
int orc_dsymm(char side, char uplo, i64 m, i64 n, double alpha, const double* a, i64 lda,
              const double* b, i64 ldb, double beta, double* c, i64 ldc, int flags) {
    return symm_ref<double>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, flags);
}
int orc_ssyr2k(char uplo, char trans, i64 n, i64 k, float alpha, const float* a, i64 lda, const float* b,
               i64 ldb, float beta, float* c, i64 ldc) {
    return syr2k_ref<float>(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_dsyr2k(char uplo, char trans, i64 n, i64 k, double alpha, const double* a, i64 lda,
               const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    return syr2k_ref<double>(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_strmm(char side, char uplo, char ta, char diag, i64 m, i64 n, float alpha, const float* a,
              i64 lda, float* b, i64 ldb) {
    return trmm_ref<float>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int orc_dtrmm(char side, char uplo, char ta, char diag, i64 m, i64 n, double alpha, const double* a,
              i64 lda, double* b, i64 ldb) {
    return trmm_ref<double>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}

}  // extern "C"
