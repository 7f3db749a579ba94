// ORACLE — test infrastructure only.
//
// A float64 checker that is more accurate than a float64 GEMM: selected rows of
// C = op(A) op(B), each element a compensated dot product ("Dot2" of Ogita,
// Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6),
// 2005, Algorithm 5.3).  Each product is split exactly into p + e with one FMA
// (e = fma(a, b, -p), exact when no underflow occurs), the running sum is
// carried with Knuth's TwoSum (s + q exactly), and the rounding errors are
// accumulated separately and added once at the end.  The result is as accurate
// as the plain dot product computed in twice the working precision: error
// <= u |result| + gamma_n^2 sum |a_l b_l| (u = 2^-53).  A float64 GEMM's own
// error (about sqrt(k) u relative at k = 4096) is therefore visible against it,
// which a float64 numpy reference cannot show.
//
// Also an element-wise fused multiply-add (x y + z with one rounding, C++'s
// std::fma), which numpy lacks, for restating epilogues that use one.
//
// Nothing in the shipped library links, loads or calls this file; it is built
// into the oracle's shared object beside the reference restatements.

#include <cmath>
#include <cstdint>
#include <vector>
#include <omp.h>

typedef int64_t i64;

namespace {

// Knuth's TwoSum: s + err == a + b exactly (round to nearest).
inline void two_sum(double a, double b, double& s, double& err) {
    s = a + b;
    const double z = s - a;
    err = (a - (s - z)) + (b - z);
}

}  // namespace

extern "C" {

// out[r + j * nrows] = sum_l op(A)[rows[r], l] * op(B)[l, j] for r < nrows, j < n,
// compensated; op(X) = X for 'N'/'n', X^T otherwise; column-major A (lda) and B (ldb).
int orc_dgemm_dot2_rows(char ta, char tb, i64 n, i64 k, const double* a, i64 lda, const double* b, i64 ldb,
                        const i64* rows, i64 nrows, double* out) {
    const bool an = ta == 'N' || ta == 'n', bn = tb == 'N' || tb == 'n';
    // the sampled rows of op(A), packed contiguously (op(A)'s rows are strided for 'N')
    std::vector<double> ar(size_t(nrows) * size_t(k));
    for (i64 r = 0; r < nrows; ++r)
        for (i64 l = 0; l < k; ++l) ar[size_t(r) * k + l] = an ? a[rows[r] + l * lda] : a[l + rows[r] * lda];
#pragma omp parallel for collapse(2) schedule(static)
    for (i64 j = 0; j < n; ++j) {
        for (i64 r = 0; r < nrows; ++r) {
            const double* xr = ar.data() + size_t(r) * k;
            double s = 0.0, c = 0.0;
            for (i64 l = 0; l < k; ++l) {
                const double x = xr[l];
                const double y = bn ? b[l + j * ldb] : b[j + l * ldb];
                const double p = x * y;
                const double pe = std::fma(x, y, -p);  // p + pe == x * y exactly
                double t, se;
                two_sum(s, p, t, se);
                s = t;
                c += se + pe;
            }
            out[r + j * nrows] = s + c;
        }
    }
    return 0;
}

// out[i] = fma(x[i], y[i], z[i]): x y + z rounded once.
int orc_fma(i64 n, const double* x, const double* y, const double* z, double* out) {
    for (i64 i = 0; i < n; ++i) out[i] = std::fma(x[i], y[i], z[i]);
    return 0;
}

}  // extern "C"
