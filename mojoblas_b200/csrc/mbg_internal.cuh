// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstddef>
#include <cstdio>
#include <string>

#include "../../include/mojoblas_gpu.h"

typedef int64_t i64;

namespace mbg {

// ---- character flags (Netlib spelling, either case; 'C' == 'T' for reals) ----
inline bool is_n(char t) { return t == 'N' || t == 'n'; }
inline bool is_t(char t) { return t == 'T' || t == 't' || t == 'C' || t == 'c'; }
inline bool is_u(char t) { return t == 'U' || t == 'u'; }
inline bool is_l(char t) { return t == 'L' || t == 'l'; }
inline bool is_r(char t) { return t == 'R' || t == 'r'; }
inline i64 imax(i64 a, i64 b) { return a > b ? a : b; }
inline i64 imin(i64 a, i64 b) { return a < b ? a : b; }
inline i64 cdiv(i64 a, i64 b) { return (a + b - 1) / b; }

// ---- one-time per-device setup ----------------------------------------------
// Kernel attributes (the dynamic shared-memory opt-in) belong to a device's
// context, so each kernel is configured once per device, from any host thread:
// a caller that finds its device's bit clear sets the attribute (setting it
// twice is harmless) and only then publishes the bit, so no thread launches
// before the attribute is in place.  Devices 32 and up are configured on every call.
inline bool configured_on(const std::atomic<unsigned>& mask, int dev) {
    return dev < 32 && (mask.load(std::memory_order_acquire) & (1u << dev));
}
inline void mark_configured(std::atomic<unsigned>& mask, int dev) {
    if (dev < 32) mask.fetch_or(1u << dev, std::memory_order_release);
}

// ---- runtime state ----------------------------------------------------------
cudaStream_t stream();
bool sync_mode();
void set_error(const char* what, cudaError_t e);
void set_error_msg(const std::string& msg);

// Wraps a CUDA runtime call; on failure records it and returns MBG_ERR_CUDA.
#define MBG_CUDA(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            ::mbg::set_error(#call, e_);                                       \
            return (e_ == cudaErrorNoDevice || e_ == cudaErrorInsufficientDriver) \
                       ? MBG_ERR_NO_DEVICE : MBG_ERR_CUDA;                     \
        }                                                                      \
    } while (0)

#define MBG_TRY(expr)                                                          \
    do {                                                                       \
        int s_ = (expr);                                                       \
        if (s_ != 0) return s_;                                                \
    } while (0)

// Checks the launch that was just enqueued (configuration errors only).
int check_launch(const char* name);

// A second non-blocking compute stream of the current device (created on first use,
// kept), for independent work within one call that can run beside the library stream.
int aux_stream(cudaStream_t* out);
// For its lifetime, the calling thread's library work goes to stream s (workspace
// blocks from s's pool); the previous setting comes back when it ends.
struct StreamScope {
    cudaStream_t saved;
    bool saved_on;
    explicit StreamScope(cudaStream_t s);
    ~StreamScope();
    StreamScope(const StreamScope&) = delete;
    StreamScope& operator=(const StreamScope&) = delete;
};

// Two non-blocking streams of the current device (host->device and device->host
// copies of the pipelined host path), created on first use and kept.
int copy_streams(cudaStream_t* in, cudaStream_t* out);

// ---- device workspace: a per-device, per-stream cache of blocks ---------------
// Blocks are handed out for the duration of one library call and returned to
// the pool of the stream that call ran on when it finishes enqueueing; a pool
// serves only calls on its own stream, so a block reused by a later call is
// ordered after its last use by stream order (calls from several host threads
// on their own streams never share a block in flight).
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t owner = nullptr;  // the stream whose pool the block returns to
    Workspace() = default;
    Workspace(const Workspace&) = delete;
    Workspace& operator=(const Workspace&) = delete;
    Workspace(Workspace&& o) noexcept : ptr(o.ptr), bytes(o.bytes), owner(o.owner) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    ~Workspace();
    int reserve(size_t nbytes);   // MBG_OK or MBG_ERR_ALLOC
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// ---- host/device operand staging ---------------------------------------------
// A matrix operand of `rows` x `cols` elements with leading dimension `ld`.
// If the pointer is not device-accessible, a compact device copy (ld = rows) is
// made (copy_in) and written back on finish() (copy_out).
struct Operand {
    const void* user = nullptr;
    void* dev = nullptr;
    i64 rows = 0, cols = 0, ld = 0, dev_ld = 0;
    size_t elem = 0;
    bool staged = false, copy_out = false;
    Workspace ws;
    int prepare(const void* p, i64 rows, i64 cols, i64 ld, size_t elem, bool copy_in, bool copy_out);
    int finish();  // copies back if staged && copy_out
};
bool is_device_pointer(const void* p);
bool is_pinned_host(const void* p);  // page-locked host memory (cudaHostAlloc / cudaHostRegister)
// Host <-> device 2-D copies (width bytes x height rows, pitches in bytes; staging.cu).
// Pageable host memory goes through page-locked bounce buffers, packed / unpacked by
// host threads while the DMAs of neighbouring chunks run; pinned memory is copied
// directly on s.  copy_h2d_2d: ordered after the work on s, and later work on s sees
// the data.  copy_d2h_2d: ordered after `after` (or, if null, the work on s); for
// pageable dst it returns when the data is there, for pinned dst it enqueues on s.
int copy_h2d_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                cudaStream_t s);
int copy_d2h_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                cudaStream_t s, cudaEvent_t after);

// ---- timing of library kernels (optional) ------------------------------------
struct ProfScope {
    int slot = -1;
    explicit ProfScope(const char* name);
    ~ProfScope();
};
void count_launch(int n = 1);

// Device-side error flag (bounded waits that expired set it): a mapped pinned
// int[4] — [0] error code, [1] site — or nullptr if it could not be created.
int* device_error_flag();
int read_and_clear_device_error();  // the mapped flag and the no-allocation flag
int noalloc_take_error(int* site);   // the no-allocation kernels' flag: code, cleared (tc_gemm.cu)
int finish_call(bool any_staged);  // synchronises when required, checks flag

// ---- tuning table (defaults; mbg_set_tuning / mbg_load_tuning override) ------
struct Tuning {
    i64 trsm_tc_min_k = 512;   // trsm off-diagonal updates with shorter k use the plain kernel
    i64 grouped_gemm_tile = 64;  // tile edge of grouped sgemm plans (64 or 128)
    i64 trsm_leaf_ctas = 0;      // CTA cap of the trsm diagonal-block solve (0: 8 per SM)
    i64 trsm_block_rows = 512;   // diagonal blocks solved in one fused launch (<= 64: leaves + gemm)
    i64 trsm_block_min_cols = 64;    // ... when there are at least this many right-hand sides
    i64 trsm_inverse_min_cols = 256;  // split / Ozaki trsm: inverted diagonal blocks from this many
                                      // right-hand sides (0: never; substitution leaves instead)
    i64 trsm_inverse_block = 512;     // ... of this many rows (256 or 512)
    i64 plain_fp64_simt = 0;     // 1: plain FP64 gemm/syrk on the CUDA cores instead of the FP64 tensor pipe
    i64 plain_fp32_staged = 0;   // 1: plain FP32 128-tiles staged through registers (the earlier kernel)
    i64 ozaki_fused_slicing = 1;  // K-contiguous Ozaki operands: exponents and slices in one pass
    i64 trsm_preslice = 1;        // split / Ozaki trsm: update blocks of op(A) split up front on a second stream
    i64 ozaki_cta_pair = 2;      // Ozaki products on CTA pairs (tcgen05 cta_group::2): 1 one launch of
                                 // all pair tiles, 2 persistent clusters; 0: one CTA per 128 x 128 tile
    // grouped sgemm plans, per transposes (NN, NT, TN, TT) and size class (grouped_size_class):
    // tile edge of the plain form (64 / 128) and tile width of the split form (64 / 128); 0 = default
    i64 grouped_simt_tile[4][5] = {};
    i64 grouped_tc_bn[4][5] = {};
};
Tuning& tuning();

// Size class of a grouped gemm problem by max(m, n): <= 32, <= 64, <= 128, <= 256, larger.
inline int grouped_size_class(i64 m, i64 n) {
    const i64 x = imax(m, n);
    return x <= 32 ? 0 : x <= 64 ? 1 : x <= 128 ? 2 : x <= 256 ? 3 : 4;
}
// Tile edge of the plain grouped sgemm for one problem (the class's entry, else grouped_gemm_tile).
inline int grouped_simt_tile(i64 m, i64 n, int ta, int tb) {
    const i64 v = tuning().grouped_simt_tile[ta * 2 + tb][grouped_size_class(m, n)];
    if (v == 64 || v == 128) return int(v);
    return tuning().grouped_gemm_tile == 128 ? 128 : 64;
}
// Tile width of the split grouped sgemm for one problem (the class's entry, else 64 for n <= 64).
inline int grouped_tc_tile_cols(i64 m, i64 n, i64 k, int ta, int tb) {
    (void)k;
    const i64 v = tuning().grouped_tc_bn[ta * 2 + tb][grouped_size_class(m, n)];
    if (v == 64 || v == 128) return int(v);
    return n <= 64 ? 64 : 128;
}
// The tensor-core grouped sgemm (grouped_tc.cu): device table, launch, release.
struct GroupedTcPlan {
    int terms = 3;
    void* table = nullptr;
    int count = 0, ntiles = 0, grid = 0;
    size_t tiles_off = 0;
    int* err = nullptr;  // the library's wait-error flag, created before the graph capture
};
int grouped_tc_build(int terms, int count, const mbg_sgemm_problem* probs, GroupedTcPlan& out);
int grouped_tc_enqueue(const GroupedTcPlan& p, cudaStream_t s);
void grouped_tc_free(GroupedTcPlan& p);

// ---- banded reduction: one operand triangular --------------------------------
// When op(A) (or op(B)) is a dense copy of a triangular matrix, zero outside its
// triangle, an output tile needs only part of the reduction:
//   KB_A_LOWER  op(A)(i, l) = 0 for l > i:  l < m0 + bm
//   KB_A_UPPER  op(A)(i, l) = 0 for l < i:  l >= m0
//   KB_B_LOWER  op(B)(l, j) = 0 for l < j:  l >= n0
//   KB_B_UPPER  op(B)(l, j) = 0 for l > j:  l < n0 + bn
// band_slabs gives the slabs [s0, s1) of `slab` elements (of `nslabs`; this
// launch's reduction starts at element k0 of the full one) that a tile at
// (m0, n0) of bm x bn must run; the skipped slabs multiply exact zeros.  At
// least one slab is kept, so every tile's pipeline runs (an extra slab outside
// the band adds only zero products).
enum { KB_NONE = 0, KB_A_LOWER = 1, KB_A_UPPER = 2, KB_B_LOWER = 3, KB_B_UPPER = 4 };

__host__ __device__ inline void band_slabs(int band, i64 m0, i64 bm, i64 n0, i64 bn, i64 k0, i64 slab,
                                           i64 nslabs, i64& s0, i64& s1) {
    const i64 end = nslabs * slab;
    i64 lo = 0, hi = end;
    if (band == KB_A_LOWER) hi = m0 + bm - k0;
    else if (band == KB_A_UPPER) lo = m0 - k0;
    else if (band == KB_B_LOWER) lo = n0 - k0;
    else if (band == KB_B_UPPER) hi = n0 + bn - k0;
    s0 = lo <= 0 ? 0 : lo / slab;
    s1 = hi >= end ? nslabs : (hi <= 0 ? 0 : (hi + slab - 1) / slab);
    if (s0 > nslabs - 1) s0 = nslabs - 1;
    if (s1 < s0 + 1) s1 = s0 + 1;
}

// Tile order of a banded launch on a (tiles_m, tiles_n) grid, heaviest tiles
// first so that the last wave holds the short ones: for an op(A) band the block
// index walks the n-tiles of one m-tile row before the next row (rows by
// decreasing work), for KB_B_UPPER the n-tiles are taken from the last.
__device__ inline void band_order(int band, i64& tm, i64& tn) {
    if (band == KB_A_LOWER || band == KB_A_UPPER) {
        const i64 lin = blockIdx.x + i64(blockIdx.y) * gridDim.x;
        tn = lin % gridDim.y;
        tm = lin / gridDim.y;
        if (band == KB_A_LOWER) tm = gridDim.x - 1 - tm;
    } else if (band == KB_B_UPPER) {
        tn = gridDim.y - 1 - tn;
    }
}

// ---- kernels (implemented in the other translation units) --------------------
template <typename T>
int gemm_plain(char ta, char tb, i64 m, i64 n, i64 k, T alpha, const T* a, i64 lda,
               const T* b, i64 ldb, T beta, T* c, i64 ldc);
// FP32 CUDA-core GEMM, 128 x 128 tiles, cp.async pipeline (gemm_f32.cu): alpha != 0, k > 0
int sgemm_f32(char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a, i64 lda, const float* b,
              i64 ldb, float beta, float* c, i64 ldc, int band = KB_NONE);
int sgemmt_f32(char uplo, char ta, char tb, i64 n, i64 k, float alpha, const float* a, i64 lda,
               const float* b, i64 ldb, float beta, float* c, i64 ldc);
// FP64 tensor-pipe GEMM (gemm_dmma.cu): alpha != 0, k > 0
int dgemm_dmma(char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a, i64 lda,
               const double* b, i64 ldb, double beta, double* c, i64 ldc, int band = KB_NONE);
int dgemmt_dmma(char uplo, char ta, char tb, i64 n, i64 k, double alpha, const double* a, i64 lda,
                const double* b, i64 ldb, double beta, double* c, i64 ldc);
// lower (uplo 'L') or upper triangle of C := alpha*op(A)*op(B) + beta*C
template <typename T>
int gemmt_plain(char uplo, char ta, char tb, i64 n, i64 k, T alpha, const T* a, i64 lda,
                const T* b, i64 ldb, T beta, T* c, i64 ldc);
template <typename T>
int scale_matrix(i64 m, i64 n, T beta, T* c, i64 ldc);  // C := beta*C (beta==0 stores 0)
template <typename T>
int scale_triangle(char uplo, i64 n, T beta, T* c, i64 ldc);

// precision-mode gemm (dispatch to plain / split / Ozaki), device operands
int sgemm_mode(int mode, char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a,
               i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc);
int dgemm_mode(int mode, int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
               const double* a, i64 lda, const double* b, i64 ldb, double beta, double* c,
               i64 ldc);
// tensor-core paths (tc_gemm.cu)
// A triangular operand read straight from the user's matrix (trmm): its split /
// slicing pre-pass keeps only the strict triangle of the logical operand (row r,
// reduction index l; keep 1: l < r, keep 2: l > r; the other triangle and the
// diagonal read as zero and are never loaded), and the epilogue forms
//     C = alpha op(A) op(B) + d .* C,   d per row (dvec_mode 1) or column (2),
// reading each element of C before the same thread overwrites it, so C may be
// the other operand: the GEMM reads the operands only through the pre-pass planes.
struct TriOperand {
    int keep_a = 0, keep_b = 0;   // pre-pass masks of op(A) and of op(B)^T
    const void* dvec = nullptr;   // float* or double* by the routine's precision
    int dvec_mode = 0;
};
// tri_uplo 'L' / 'U': only that triangle of C is written (syrk, triangular adjoints);
// band: one operand triangular (KB_*), each tile runs only its part of the reduction
int sgemm_split_tc(int terms, char ta, char tb, i64 m, i64 n, i64 k, float alpha,
                   const float* a, i64 lda, const float* b, i64 ldb, float beta, float* c,
                   i64 ldc, char tri_uplo, int band = KB_NONE, const TriOperand* tri_op = nullptr);
int dgemm_ozaki_tc(int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha,
                   const double* a, i64 lda, const double* b, i64 ldb, double beta,
                   double* c, i64 ldc, char tri_uplo = 0, int band = KB_NONE,
                   const TriOperand* tri_op = nullptr);
// longest reduction of one Ozaki launch (int32-exact accumulators)
i64 ozaki_max_k(int slices);
// op(A)'s bf16 split planes made once for several column blocks of op(B) (the
// pipelined host path); the workspace lives as long as the SplitA
struct SplitA {
    Workspace ws;
    int terms = 0;
    i64 m = 0, k = 0, Mp = 0, Kp = 0;
};
int split_a_planes(int terms, char ta, i64 m, i64 k, const float* a, i64 lda, SplitA& out);
int sgemm_split_tc_with_a(const SplitA& A, char tb, i64 n, float alpha, const float* b, i64 ldb, float beta,
                          float* c, i64 ldc);
// rows r0 .. r0 + mb - 1 of op(A) (r0 a multiple of 128) against a k x n op(B), k <= A.k
int sgemm_split_tc_with_a_rows(const SplitA& A, i64 r0, i64 mb, i64 k, char tb, i64 n, float alpha, const float* b,
                               i64 ldb, float beta, float* c, i64 ldc);
// One product C := alpha op(A) op(B) (beta 0) of a pair run by sgemm_split_tc_dual.
struct SplitProduct {
    char ta, tb;
    i64 m, n, k;
    float alpha;
    const float* a;
    i64 lda;
    const float* b;
    i64 ldb;
    float* c;
    i64 ldc;
};
// Two independent split products (device operands, m, n, k > 0) in one persistent launch of
// 128 x 256 tiles, the longer reduction's tiles first and a stream-K tail balanced across
// the SMs.
int sgemm_split_tc_dual(int terms, const SplitProduct& x, const SplitProduct& y);
// op(A)'s Ozaki slices and row exponents made once for several row-block products
struct OzakiA {
    Workspace ws;
    int slices = 0;
    i64 m = 0, k = 0, Mp = 0, Kp = 0;
    int8_t* planes = nullptr;
    int* e = nullptr;
};
int ozaki_slice_a(int slices, char ta, i64 m, i64 k, const double* a, i64 lda, OzakiA& out);
int dgemm_ozaki_tc_with_a(const OzakiA& A, i64 r0, i64 mb, i64 k, char tb, i64 n, double alpha, const double* b,
                          i64 ldb, double beta, double* c, i64 ldc, const double* dvec = nullptr);

// trsm and trmm on device operands (trsm.cu)
template <typename T>
int trsm_device(int mode, int slices, int refine, char side, char uplo, char ta, char diag,
                i64 m, i64 n, T alpha, const T* a, i64 lda, T* b, i64 ldb);
template <typename T>
int trmm_device(int mode, int slices, char side, char uplo, char ta, char diag, i64 m, i64 n, T alpha,
                const T* a, i64 lda, T* b, i64 ldb);

// gemv and trsv on device operands (level2.cu)
template <typename T>
int gemv_device(char trans, i64 m, i64 n, T alpha, const T* a, i64 lda, const T* x, i64 incx, T beta, T* y,
                i64 incy);
template <typename T>
int trsv_device(char uplo, char trans, char diag, i64 n, const T* a, i64 lda, T* x, i64 incx);

// symm and syr2k on device operands (symm.cu)
template <typename T>
int symm_device(int mode, int slices, char side, char uplo, i64 m, i64 n, T alpha, const T* a, i64 lda,
                const T* b, i64 ldb, T beta, T* c, i64 ldc);
template <typename T>
int syr2k_device(int mode, int slices, char uplo, char trans, i64 n, i64 k, T alpha, const T* a, i64 lda,
                 const T* b, i64 ldb, T beta, T* c, i64 ldc);

}  // namespace mbg
