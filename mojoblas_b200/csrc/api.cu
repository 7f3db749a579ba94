// C ABI entry points: argument checks (Netlib numbering as in the mojoBLAS
// routines), quick returns, host-operand staging and precision-mode dispatch.
#include "mbg_internal.cuh"

#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace mbg {

// ---- argument checks ----------------------------------------------------------
// src/level3/gemm.mojo:179-213
static int gemm_info(char ta, char tb, i64 m, i64 n, i64 k, i64 lda, i64 ldb, i64 ldc) {
    if (!is_n(ta) && !is_t(ta)) return 1;
    if (!is_n(tb) && !is_t(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    if (lda < imax(1, is_n(ta) ? m : k)) return 8;
    if (ldb < imax(1, is_n(tb) ? k : n)) return 10;
    if (ldc < imax(1, m)) return 13;
    return 0;
}
// src/level3/syrk.mojo:60-83
static int syrk_info(char uplo, char trans, i64 n, i64 k, i64 lda, i64 ldc) {
    if (!is_u(uplo) && !is_l(uplo)) return 1;
    if (!is_n(trans) && !is_t(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    if (lda < imax(1, is_n(trans) ? n : k)) return 7;
    if (ldc < imax(1, n)) return 10;
    return 0;
}
// src/level3/trsm.mojo:62-89
static int trsm_info(char side, char uplo, char ta, char diag, i64 m, i64 n, i64 lda, i64 ldb) {
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (!is_n(ta) && !is_t(ta)) return 3;
    if (!is_u(diag) && !is_n(diag)) return 4;
    if (m < 0) return 5;
    if (n < 0) return 6;
    if (lda < imax(1, is_l(side) ? m : n)) return 9;
    if (ldb < imax(1, m)) return 11;
    return 0;
}

// src/level3/symm.mojo:69-82
static int symm_info(char side, char uplo, i64 m, i64 n, i64 lda, i64 ldb, i64 ldc) {
    if (!is_l(side) && !is_r(side)) return 1;
    if (!is_u(uplo) && !is_l(uplo)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (lda < imax(1, is_l(side) ? m : n)) return 7;
    if (ldb < imax(1, m)) return 9;
    if (ldc < imax(1, m)) return 12;
    return 0;
}
// src/level3/syr2k.mojo:69-89
static int syr2k_info(char uplo, char trans, i64 n, i64 k, i64 lda, i64 ldb, i64 ldc) {
    if (!is_u(uplo) && !is_l(uplo)) return 1;
    if (!is_n(trans) && !is_t(trans)) return 2;
    if (n < 0) return 3;
    if (k < 0) return 4;
    if (lda < imax(1, is_n(trans) ? n : k)) return 7;
    if (ldb < imax(1, is_n(trans) ? n : k)) return 9;
    if (ldc < imax(1, n)) return 12;
    return 0;
}
// src/level3/trmm.mojo:63-85 (the same numbering as trsm)
static int trmm_info(char side, char uplo, char ta, char diag, i64 m, i64 n, i64 lda, i64 ldb) {
    return trsm_info(side, uplo, ta, diag, m, n, lda, ldb);
}

// src/level2/gemv.mojo:69-84 (trans in upper case only, as the reference checks it)
static int gemv_info(char trans, i64 m, i64 n, i64 lda, i64 incx, i64 incy) {
    if (trans != 'N' && trans != 'T' && trans != 'C') return 1;
    if (m < 0) return 2;
    if (n < 0) return 3;
    if (lda < imax(1, m)) return 6;
    if (incx == 0) return 8;
    if (incy == 0) return 11;
    return 0;
}
// src/level2/trsv.mojo:56-79
static int trsv_info(char uplo, char trans, char diag, i64 n, i64 lda, i64 incx) {
    if (!is_u(uplo) && !is_l(uplo)) return 1;
    if (!is_n(trans) && !is_t(trans)) return 2;
    if (!is_u(diag) && !is_n(diag)) return 3;
    if (n < 0) return 4;
    if (lda < imax(1, n)) return 6;
    if (incx == 0) return 8;
    return 0;
}

static bool valid_smode(int mode) {
    return mode == MBG_MODE_PLAIN || mode == MBG_MODE_BF16X3 || mode == MBG_MODE_BF16X6;
}
static bool valid_dmode(int mode, int slices) {
    if (mode == MBG_MODE_PLAIN) return true;
    return mode == MBG_MODE_OZAKI && slices >= 2 && slices <= 8;
}

// ---- precision dispatch on device operands -------------------------------------
int sgemm_mode(int mode, char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a,
               i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc) {
    if (m == 0 || n == 0) return MBG_OK;
    if (alpha == 0.0f || k == 0) return scale_matrix<float>(m, n, beta, c, ldc);
    switch (mode) {
        case MBG_MODE_PLAIN: return gemm_plain<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
        case MBG_MODE_BF16X3: return sgemm_split_tc(2, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 0);
        case MBG_MODE_BF16X6: return sgemm_split_tc(3, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 0);
        default: return MBG_ERR_INVALID_MODE;
    }
}

int dgemm_mode(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
               const double* a, i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc) {
    if (m == 0 || n == 0) return MBG_OK;
    if (alpha == 0.0 || k == 0) return scale_matrix<double>(m, n, beta, c, ldc);
    switch (mode) {
        case MBG_MODE_PLAIN: return gemm_plain<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
        case MBG_MODE_OZAKI: return dgemm_ozaki_tc(slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
        default: return MBG_ERR_INVALID_MODE;
    }
}

// ---- staged drivers ------------------------------------------------------------
template <typename T>
static int gemm_compute(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
                        const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    if (sizeof(T) == 4)
        return sgemm_mode(mode, ta, tb, m, n, k, (float)alpha, (const float*)a, lda, (const float*)b, ldb,
                          (float)beta, (float*)c, ldc);
    return dgemm_mode(mode, slices, ta, tb, m, n, k, (double)alpha, (const double*)a, lda, (const double*)b, ldb,
                      (double)beta, (double*)c, ldc);
}

// Large gemm with host operands: the host <-> device copies overlap the
// arithmetic.  C is cut into column blocks: GEMM_PIPE_BLOCKS blocks of equal
// width (multiples of 256 columns, so every tile of C is the same as in one call
// over all of C), the last of them halved down to 256 columns so that little
// arithmetic and little copying is left after op(B)'s last columns land.  A copy
// stream brings op(A) over first and then, block by block, the columns of op(B)
// (and of C when beta != 0); the library's stream computes each block as soon as
// its operands have landed (in the split modes op(A) is split once, when it has
// landed, and its planes serve every block); a second copy stream returns each
// finished block of C, so the two directions of the PCIe link run at the same
// time.  The device buffers are the same full-size copies the sequential path uses.
constexpr int GEMM_PIPE_BLOCKS = 8;

static std::vector<i64> pipeline_widths(i64 n) {
    const i64 nb = cdiv(cdiv(n, GEMM_PIPE_BLOCKS), 256) * 256;
    std::vector<i64> w;
    i64 rest = n;
    while (rest > nb) {
        w.push_back(nb);
        rest -= nb;
    }
    while (rest > 256) {  // the last block: 1/2, 1/4, ... down to 256 columns
        const i64 h = cdiv(cdiv(rest, 2), 256) * 256;
        w.push_back(h);
        rest -= h;
    }
    w.push_back(rest);
    return w;
}

template <typename T>
static bool gemm_pipeline_pays(const T* a, const T* b, const T* c, i64 m, i64 n, i64 k) {
    if (n < 4096 || double(m) * double(n) * double(k) < double(1ll << 34)) return false;
    return !is_device_pointer(a) || !is_device_pointer(b) || !is_device_pointer(c);
}

template <typename T>
static int gemm_host_pipelined(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, T alpha,
                               const T* a, i64 lda, const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    cudaStream_t s = stream(), sin = nullptr, sout = nullptr;
    MBG_TRY(copy_streams(&sin, &sout));
    const bool ha = !is_device_pointer(a), hb = !is_device_pointer(b), hc = !is_device_pointer(c);
    const i64 ar = is_n(ta) ? m : k, ac = is_n(ta) ? k : m;  // stored shape of A
    const i64 br = is_n(tb) ? k : n, bc = is_n(tb) ? n : k;  // stored shape of B
    const size_t e = sizeof(T);
    Workspace wa, wb, wc;
    const T* da = a;
    const T* db = b;
    T* dc = c;
    i64 dlda = lda, dldb = ldb, dldc = ldc;
    if (ha) { MBG_TRY(wa.reserve(e * size_t(ar) * size_t(ac))); da = wa.as<T>(); dlda = ar; }
    if (hb) { MBG_TRY(wb.reserve(e * size_t(br) * size_t(bc))); db = wb.as<T>(); dldb = br; }
    if (hc) { MBG_TRY(wc.reserve(e * size_t(m) * size_t(n))); dc = wc.as<T>(); dldc = m; }

    const std::vector<i64> widths = pipeline_widths(n);
    struct Guard {  // on every return: the copy streams' work is ordered before the library stream's
        std::vector<cudaEvent_t> v;   // next use of the workspace blocks, then the events are destroyed
        cudaStream_t s = nullptr, sin = nullptr, sout = nullptr;
        ~Guard() {
            cudaEvent_t tail[2] = {nullptr, nullptr};
            cudaStream_t from[2] = {sin, sout};
            for (int i = 0; i < 2; ++i)
                if (from[i] && cudaEventCreateWithFlags(&tail[i], cudaEventDisableTiming) == cudaSuccess) {
                    cudaEventRecord(tail[i], from[i]);
                    cudaStreamWaitEvent(s, tail[i], 0);
                    cudaEventDestroy(tail[i]);
                }
            for (auto x : v)
                if (x) cudaEventDestroy(x);
        }
    } guard;
    guard.s = s;
    guard.sin = sin;
    guard.sout = sout;
    auto& ev = guard.v;
    ev.assign(2 * widths.size() + 2, nullptr);
    for (auto& x : ev) MBG_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    cudaEvent_t ev_start = ev[0], ev_end = ev[1];
    MBG_CUDA(cudaEventRecord(ev_start, s));  // earlier work on the library stream (workspace reuse) first
    MBG_CUDA(cudaStreamWaitEvent(sin, ev_start, 0));
    MBG_CUDA(cudaStreamWaitEvent(sout, ev_start, 0));

    // C's blocks go back to the host in order as they finish.  Into pageable memory
    // that takes the host's hands (unpacking from the bounce buffers), so a helper
    // thread does it while this thread packs op(B)'s next blocks.
    std::mutex out_mu;
    std::condition_variable out_cv;
    int recorded = 0;       // blocks whose ev_done is recorded
    bool abort_out = false;
    int out_st = MBG_OK;
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    const bool c_pageable = hc && !is_pinned_host(c);
    auto copy_out_block = [&](int blk) -> int {
        i64 j0 = 0;
        for (int i = 0; i < blk; ++i) j0 += widths[size_t(i)];
        const i64 w = widths[size_t(blk)];
        return copy_d2h_2d(c + j0 * ldc, size_t(ldc) * e, dc + j0 * dldc, size_t(dldc) * e, size_t(m) * e,
                           size_t(w), sout, ev[3 + 2 * blk]);
    };
    std::thread out_thread;
    if (c_pageable) {
        out_thread = std::thread([&] {
            cudaSetDevice(dev);
            for (int blk = 0; blk < int(widths.size()); ++blk) {
                {
                    std::unique_lock<std::mutex> lk(out_mu);
                    out_cv.wait(lk, [&] { return recorded > blk || abort_out; });
                    if (recorded <= blk) return;  // aborted before this block was computed
                }
                const int r = copy_out_block(blk);
                if (r) {
                    out_st = r;
                    return;
                }
            }
        });
    }
    struct Join {  // the helper thread ends before this function's state goes away
        std::thread& t;
        std::mutex& mu;
        std::condition_variable& cv;
        bool& abort;
        ~Join() {
            if (!t.joinable()) return;
            {
                std::lock_guard<std::mutex> lk(mu);
                abort = true;
            }
            cv.notify_all();
            t.join();
        }
    } join{out_thread, out_mu, out_cv, abort_out};

    if (ha) MBG_TRY(copy_h2d_2d(const_cast<T*>(da), size_t(ar) * e, a, size_t(lda) * e, size_t(ar) * e, size_t(ac), sin));
    // split modes: op(A)'s planes once, on the library stream after op(A) has landed
    const bool split_once = sizeof(T) == 4 && (mode == MBG_MODE_BF16X3 || mode == MBG_MODE_BF16X6);
    SplitA sa;
    int st = MBG_OK;
    i64 j0 = 0;
    for (size_t blk = 0; blk < widths.size() && !st; ++blk) {
        const i64 w = widths[blk];
        cudaEvent_t ev_in = ev[2 + 2 * blk], ev_done = ev[3 + 2 * blk];
        // op(B)[:, j0 : j0 + w] is columns j0.. of B ('N') or rows j0.. of B ('T')
        if (hb) {
            if (is_n(tb))
                MBG_TRY(copy_h2d_2d(const_cast<T*>(db) + j0 * dldb, size_t(dldb) * e, b + j0 * ldb, size_t(ldb) * e,
                                    size_t(k) * e, size_t(w), sin));
            else
                MBG_TRY(copy_h2d_2d(const_cast<T*>(db) + j0, size_t(dldb) * e, b + j0, size_t(ldb) * e,
                                    size_t(w) * e, size_t(k), sin));
        }
        if (hc && beta != T(0))
            MBG_TRY(copy_h2d_2d(dc + j0 * dldc, size_t(dldc) * e, c + j0 * ldc, size_t(ldc) * e, size_t(m) * e,
                                size_t(w), sin));
        MBG_CUDA(cudaEventRecord(ev_in, sin));
        MBG_CUDA(cudaStreamWaitEvent(s, ev_in, 0));
        const T* bj = is_n(tb) ? db + j0 * dldb : db + j0;
        if (split_once) {
            if (blk == 0)
                st = split_a_planes(mode == MBG_MODE_BF16X6 ? 3 : 2, ta, m, k, (const float*)da, dlda, sa);
            if (!st)
                st = sgemm_split_tc_with_a(sa, tb, w, (float)alpha, (const float*)bj, dldb, (float)beta,
                                           (float*)(dc + j0 * dldc), dldc);
        } else {
            st = gemm_compute<T>(mode, slices, ta, tb, m, w, k, alpha, da, dlda, bj, dldb, beta, dc + j0 * dldc,
                                 dldc);
        }
        MBG_CUDA(cudaEventRecord(ev_done, s));
        if (hc && !c_pageable) MBG_TRY(copy_out_block(int(blk)));
        if (c_pageable) {
            {
                std::lock_guard<std::mutex> lk(out_mu);
                recorded = int(blk) + 1;
            }
            out_cv.notify_all();
        }
        j0 += w;
    }
    if (out_thread.joinable()) {
        if (st) {
            std::lock_guard<std::mutex> lk(out_mu);
            abort_out = true;
        }
        out_cv.notify_all();
        out_thread.join();
        if (!st) st = out_st;
    }
    MBG_CUDA(cudaEventRecord(ev_end, sout));
    MBG_CUDA(cudaStreamWaitEvent(s, ev_end, 0));  // the library stream completes after the last copy back
    const int fin = finish_call(true);
    return st ? st : fin;
}

template <typename T>
static int gemm_entry(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, T alpha,
                      const T* a, i64 lda, const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    int info = gemm_info(ta, tb, m, n, k, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0) return MBG_OK;
    const bool need_ab = !(alpha == T(0) || k == 0);
    if (need_ab && gemm_pipeline_pays<T>(a, b, c, m, n, k))
        return gemm_host_pipelined<T>(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    Operand A, B, Cc;
    if (need_ab) {
        MBG_TRY(A.prepare(a, is_n(ta) ? m : k, is_n(ta) ? k : m, lda, sizeof(T), true, false));
        MBG_TRY(B.prepare(b, is_n(tb) ? k : n, is_n(tb) ? n : k, ldb, sizeof(T), true, false));
    }
    MBG_TRY(Cc.prepare(c, m, n, ldc, sizeof(T), beta != T(0), true));
    int st;
    if (sizeof(T) == 4)
        st = sgemm_mode(mode, ta, tb, m, n, k, (float)alpha, (const float*)A.dev, A.dev_ld,
                        (const float*)B.dev, B.dev_ld, (float)beta, (float*)Cc.dev, Cc.dev_ld);
    else
        st = dgemm_mode(mode, slices, ta, tb, m, n, k, (double)alpha, (const double*)A.dev, A.dev_ld,
                        (const double*)B.dev, B.dev_ld, (double)beta, (double*)Cc.dev, Cc.dev_ld);
    if (st) return st;
    MBG_TRY(Cc.finish());
    return finish_call(A.staged || B.staged || Cc.staged);
}

template <typename T>
static int syrk_entry(int mode, char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda,
                      T beta, T* c, i64 ldc, int slices = 8) {
    int info = syrk_info(uplo, trans, n, k, lda, ldc);
    if (info) return info;
    if (n == 0 || (alpha == T(0) && beta == T(1))) return MBG_OK;  // syrk.mojo:85-86
    const bool need_a = !(alpha == T(0) || k == 0);
    Operand A, Cc;
    if (need_a) MBG_TRY(A.prepare(a, is_n(trans) ? n : k, is_n(trans) ? k : n, lda, sizeof(T), true, false));
    MBG_TRY(Cc.prepare(c, n, n, ldc, sizeof(T), true, true));  // other triangle must survive
    const T* ad = (const T*)A.dev;
    T* cd = (T*)Cc.dev;
    // C := alpha*op(A)*op(A)^T + beta*C; op(A)^T is A with the other transpose
    const char ta = is_n(trans) ? 'N' : 'T';
    const char tb = is_n(trans) ? 'T' : 'N';
    int st;
    if (!need_a) st = scale_triangle<T>(uplo, n, beta, cd, Cc.dev_ld);
    else if (mode == MBG_MODE_PLAIN)
        st = gemmt_plain<T>(uplo, ta, tb, n, k, alpha, ad, A.dev_ld, ad, A.dev_ld, beta, cd, Cc.dev_ld);
    else if (sizeof(T) == 8)  // Ozaki int8 slices, one set of slices for both operands
        st = dgemm_ozaki_tc(slices, ta, tb, n, n, k, (double)alpha, (const double*)ad, A.dev_ld,
                            (const double*)ad, A.dev_ld, (double)beta, (double*)cd, Cc.dev_ld, is_l(uplo) ? 'L' : 'U');
    else
        st = sgemm_split_tc(mode == MBG_MODE_BF16X6 ? 3 : 2, ta, tb, n, n, k, (float)alpha,
                            (const float*)ad, A.dev_ld, (const float*)ad, A.dev_ld, (float)beta,
                            (float*)cd, Cc.dev_ld, is_l(uplo) ? 'L' : 'U');
    if (st) return st;
    MBG_TRY(Cc.finish());
    return finish_call(A.staged || Cc.staged);
}

template <typename T>
static int trsm_entry(int mode, int slices, int refine, char side, char uplo, char ta, char diag,
                      i64 m, i64 n, T alpha, const T* a, i64 lda, T* b, i64 ldb) {
    int info = trsm_info(side, uplo, ta, diag, m, n, lda, ldb);
    if (info) return info;
    if (m == 0 || n == 0) return MBG_OK;  // trsm.mojo:91-92
    const i64 na = is_l(side) ? m : n;
    Operand A, B;
    MBG_TRY(A.prepare(a, na, na, lda, sizeof(T), true, false));
    MBG_TRY(B.prepare(b, m, n, ldb, sizeof(T), true, true));
    int st = trsm_device<T>(mode, slices, refine, side, uplo, ta, diag, m, n, alpha, (const T*)A.dev,
                            A.dev_ld, (T*)B.dev, B.dev_ld);
    if (st) return st;
    MBG_TRY(B.finish());
    return finish_call(A.staged || B.staged);
}

template <typename T>
static int symm_entry(int mode, int slices, char side, char uplo, i64 m, i64 n, T alpha, const T* a, i64 lda,
                      const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    int info = symm_info(side, uplo, m, n, lda, ldb, ldc);
    if (info) return info;
    if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return MBG_OK;  // symm.mojo:88-89
    const bool need_ab = alpha != T(0);
    const i64 na = is_l(side) ? m : n;
    Operand A, B, Cc;
    if (need_ab) {
        MBG_TRY(A.prepare(a, na, na, lda, sizeof(T), true, false));
        MBG_TRY(B.prepare(b, m, n, ldb, sizeof(T), true, false));
    }
    MBG_TRY(Cc.prepare(c, m, n, ldc, sizeof(T), beta != T(0), true));
    int st = symm_device<T>(mode, slices, side, uplo, m, n, alpha, (const T*)A.dev, A.dev_ld, (const T*)B.dev,
                            B.dev_ld, beta, (T*)Cc.dev, Cc.dev_ld);
    if (st) return st;
    MBG_TRY(Cc.finish());
    return finish_call(A.staged || B.staged || Cc.staged);
}

template <typename T>
static int syr2k_entry(int mode, int slices, char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda,
                       const T* b, i64 ldb, T beta, T* c, i64 ldc) {
    int info = syr2k_info(uplo, trans, n, k, lda, ldb, ldc);
    if (info) return info;
    if (n == 0 || (alpha == T(0) && beta == T(1))) return MBG_OK;  // syr2k.mojo:95-96
    const bool need_ab = !(alpha == T(0) || k == 0);
    const i64 rows = is_n(trans) ? n : k, cols = is_n(trans) ? k : n;
    Operand A, B, Cc;
    if (need_ab) {
        MBG_TRY(A.prepare(a, rows, cols, lda, sizeof(T), true, false));
        MBG_TRY(B.prepare(b, rows, cols, ldb, sizeof(T), true, false));
    }
    MBG_TRY(Cc.prepare(c, n, n, ldc, sizeof(T), true, true));  // the other triangle must survive
    int st = syr2k_device<T>(mode, slices, uplo, trans, n, k, alpha, (const T*)A.dev, A.dev_ld, (const T*)B.dev,
                             B.dev_ld, beta, (T*)Cc.dev, Cc.dev_ld);
    if (st) return st;
    MBG_TRY(Cc.finish());
    return finish_call(A.staged || B.staged || Cc.staged);
}

template <typename T>
static int trmm_entry(int mode, int slices, char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha,
                      const T* a, i64 lda, T* b, i64 ldb) {
    int info = trmm_info(side, uplo, ta, diag, m, n, lda, ldb);
    if (info) return info;
    if (m == 0 || n == 0) return MBG_OK;  // trmm.mojo:91-92
    const i64 na = is_l(side) ? m : n;
    Operand A, B;
    if (alpha != T(0)) MBG_TRY(A.prepare(a, na, na, lda, sizeof(T), true, false));
    MBG_TRY(B.prepare(b, m, n, ldb, sizeof(T), alpha != T(0), true));
    int st = trmm_device<T>(mode, slices, side, uplo, ta, diag, m, n, alpha, (const T*)A.dev, A.dev_ld,
                            (T*)B.dev, B.dev_ld);
    if (st) return st;
    MBG_TRY(B.finish());
    return finish_call(A.staged || B.staged);
}

// A strided vector of `len` elements as a 1 x len operand with leading dimension
// |inc| (storage order kept, so a negative increment stays negative); a staged
// copy is compact, increment +-1.
static int prepare_vector(Operand& v, const void* p, i64 len, i64 inc, size_t elem, bool copy_in, bool copy_out,
                          i64* dev_inc) {
    const i64 ainc = inc > 0 ? inc : -inc;
    MBG_TRY(v.prepare(p, 1, len, ainc, elem, copy_in, copy_out));
    *dev_inc = v.staged ? (inc > 0 ? 1 : -1) : inc;
    return MBG_OK;
}

template <typename T>
static int gemv_entry(char trans, i64 m, i64 n, T alpha, const T* a, i64 lda, const T* x, i64 incx, T beta, T* y,
                      i64 incy) {
    int info = gemv_info(trans, m, n, lda, incx, incy);
    if (info) return info;
    if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return MBG_OK;  // gemv.mojo:86-87
    const i64 lenx = trans == 'N' ? n : m, leny = trans == 'N' ? m : n;
    Operand A, X, Y;
    i64 dix = incx, diy = incy;
    if (alpha != T(0)) {
        MBG_TRY(A.prepare(a, m, n, lda, sizeof(T), true, false));
        MBG_TRY(prepare_vector(X, x, lenx, incx, sizeof(T), true, false, &dix));
    }
    MBG_TRY(prepare_vector(Y, y, leny, incy, sizeof(T), beta != T(0), true, &diy));
    int st = gemv_device<T>(trans, m, n, alpha, (const T*)A.dev, A.dev_ld, (const T*)X.dev, dix, beta, (T*)Y.dev,
                            diy);
    if (st) return st;
    MBG_TRY(Y.finish());
    return finish_call(A.staged || X.staged || Y.staged);
}

template <typename T>
static int trsv_entry(char uplo, char trans, char diag, i64 n, const T* a, i64 lda, T* x, i64 incx) {
    int info = trsv_info(uplo, trans, diag, n, lda, incx);
    if (info) return info;
    if (n == 0) return MBG_OK;  // trsv.mojo:81-82
    Operand A, X;
    i64 dix = incx;
    MBG_TRY(A.prepare(a, n, n, lda, sizeof(T), true, false));
    MBG_TRY(prepare_vector(X, x, n, incx, sizeof(T), true, true, &dix));
    int st = trsv_device<T>(uplo, trans, diag, n, (const T*)A.dev, A.dev_ld, (T*)X.dev, dix);
    if (st) return st;
    MBG_TRY(X.finish());
    return finish_call(A.staged || X.staged);
}

}  // namespace mbg

using namespace mbg;

extern "C" {

int mbg_sgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, float alpha, const float* a,
              int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc) {
    return gemm_entry<float>(MBG_MODE_PLAIN, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a,
              int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
    return gemm_entry<double>(MBG_MODE_PLAIN, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_sgemm_ex(int mode, char ta, char tb, int64_t m, int64_t n, int64_t k, float alpha,
                 const float* a, int64_t lda, const float* b, int64_t ldb, float beta, float* c,
                 int64_t ldc) {
    if (!valid_smode(mode)) return MBG_ERR_INVALID_MODE;
    return gemm_entry<float>(mode, 0, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dgemm_ex(int mode, int slices, char ta, char tb, int64_t m, int64_t n, int64_t k,
                 double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                 double beta, double* c, int64_t ldc) {
    if (!valid_dmode(mode, slices)) return MBG_ERR_INVALID_MODE;
    return gemm_entry<double>(mode, slices, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

int mbg_ssyrk(char uplo, char trans, int64_t n, int64_t k, float alpha, const float* a,
              int64_t lda, float beta, float* c, int64_t ldc) {
    return syrk_entry<float>(MBG_MODE_PLAIN, uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int mbg_dsyrk(char uplo, char trans, int64_t n, int64_t k, double alpha, const double* a,
              int64_t lda, double beta, double* c, int64_t ldc) {
    return syrk_entry<double>(MBG_MODE_PLAIN, uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int mbg_ssyrk_ex(int mode, char uplo, char trans, int64_t n, int64_t k, float alpha,
                 const float* a, int64_t lda, float beta, float* c, int64_t ldc) {
    if (!valid_smode(mode)) return MBG_ERR_INVALID_MODE;
    return syrk_entry<float>(mode, uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int mbg_dsyrk_ex(int mode, int slices, char uplo, char trans, int64_t n, int64_t k, double alpha,
                 const double* a, int64_t lda, double beta, double* c, int64_t ldc) {
    if (!valid_dmode(mode, slices)) return MBG_ERR_INVALID_MODE;
    return syrk_entry<double>(mode, uplo, trans, n, k, alpha, a, lda, beta, c, ldc, slices);
}

int mbg_strsm(char side, char uplo, char ta, char diag, int64_t m, int64_t n, float alpha,
              const float* a, int64_t lda, float* b, int64_t ldb) {
    return trsm_entry<float>(MBG_MODE_PLAIN, 0, 0, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_dtrsm(char side, char uplo, char ta, char diag, int64_t m, int64_t n, double alpha,
              const double* a, int64_t lda, double* b, int64_t ldb) {
    return trsm_entry<double>(MBG_MODE_PLAIN, 0, 0, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_strsm_ex(int mode, int refine, char side, char uplo, char ta, char diag, int64_t m,
                 int64_t n, float alpha, const float* a, int64_t lda, float* b, int64_t ldb) {
    if (!valid_smode(mode) || refine < 0) return MBG_ERR_INVALID_MODE;
    return trsm_entry<float>(mode, 0, refine, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_dtrsm_ex(int mode, int slices, int refine, char side, char uplo, char ta, char diag,
                 int64_t m, int64_t n, double alpha, const double* a, int64_t lda, double* b,
                 int64_t ldb) {
    if (!valid_dmode(mode, slices) || refine < 0) return MBG_ERR_INVALID_MODE;
    return trsm_entry<double>(mode, slices, refine, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}

// ---- gemv / trsv ----
int mbg_sgemv(char trans, int64_t m, int64_t n, float alpha, const float* a, int64_t lda, const float* x,
              int64_t incx, float beta, float* y, int64_t incy) {
    return gemv_entry<float>(trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
int mbg_dgemv(char trans, int64_t m, int64_t n, double alpha, const double* a, int64_t lda, const double* x,
              int64_t incx, double beta, double* y, int64_t incy) {
    return gemv_entry<double>(trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
int mbg_strsv(char uplo, char trans, char diag, int64_t n, const float* a, int64_t lda, float* x, int64_t incx) {
    return trsv_entry<float>(uplo, trans, diag, n, a, lda, x, incx);
}
int mbg_dtrsv(char uplo, char trans, char diag, int64_t n, const double* a, int64_t lda, double* x,
              int64_t incx) {
    return trsv_entry<double>(uplo, trans, diag, n, a, lda, x, incx);
}

// ---- symm / syr2k / trmm ----
int mbg_ssymm(char side, char uplo, int64_t m, int64_t n, float alpha, const float* a, int64_t lda,
              const float* b, int64_t ldb, float beta, float* c, int64_t ldc) {
    return symm_entry<float>(MBG_MODE_PLAIN, 0, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dsymm(char side, char uplo, int64_t m, int64_t n, double alpha, const double* a, int64_t lda,
              const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
    return symm_entry<double>(MBG_MODE_PLAIN, 0, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_ssymm_ex(int mode, char side, char uplo, int64_t m, int64_t n, float alpha, const float* a, int64_t lda,
                 const float* b, int64_t ldb, float beta, float* c, int64_t ldc) {
    if (!valid_smode(mode)) return MBG_ERR_INVALID_MODE;
    return symm_entry<float>(mode, 0, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dsymm_ex(int mode, int slices, char side, char uplo, int64_t m, int64_t n, double alpha, const double* a,
                 int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
    if (!valid_dmode(mode, slices)) return MBG_ERR_INVALID_MODE;
    return symm_entry<double>(mode, slices, side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}

int mbg_ssyr2k(char uplo, char trans, int64_t n, int64_t k, float alpha, const float* a, int64_t lda,
               const float* b, int64_t ldb, float beta, float* c, int64_t ldc) {
    return syr2k_entry<float>(MBG_MODE_PLAIN, 0, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dsyr2k(char uplo, char trans, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
               const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
    return syr2k_entry<double>(MBG_MODE_PLAIN, 0, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_ssyr2k_ex(int mode, char uplo, char trans, int64_t n, int64_t k, float alpha, const float* a, int64_t lda,
                  const float* b, int64_t ldb, float beta, float* c, int64_t ldc) {
    if (!valid_smode(mode)) return MBG_ERR_INVALID_MODE;
    return syr2k_entry<float>(mode, 0, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int mbg_dsyr2k_ex(int mode, int slices, char uplo, char trans, int64_t n, int64_t k, double alpha,
                  const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
                  int64_t ldc) {
    if (!valid_dmode(mode, slices)) return MBG_ERR_INVALID_MODE;
    return syr2k_entry<double>(mode, slices, uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

int mbg_strmm(char side, char uplo, char ta, char diag, int64_t m, int64_t n, float alpha, const float* a,
              int64_t lda, float* b, int64_t ldb) {
    return trmm_entry<float>(MBG_MODE_PLAIN, 0, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_dtrmm(char side, char uplo, char ta, char diag, int64_t m, int64_t n, double alpha, const double* a,
              int64_t lda, double* b, int64_t ldb) {
    return trmm_entry<double>(MBG_MODE_PLAIN, 0, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_strmm_ex(int mode, char side, char uplo, char ta, char diag, int64_t m, int64_t n, float alpha,
                 const float* a, int64_t lda, float* b, int64_t ldb) {
    if (!valid_smode(mode)) return MBG_ERR_INVALID_MODE;
    return trmm_entry<float>(mode, 0, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int mbg_dtrmm_ex(int mode, int slices, char side, char uplo, char ta, char diag, int64_t m, int64_t n,
                 double alpha, const double* a, int64_t lda, double* b, int64_t ldb) {
    if (!valid_dmode(mode, slices)) return MBG_ERR_INVALID_MODE;
    return trmm_entry<double>(mode, slices, side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}

}  // extern "C"
