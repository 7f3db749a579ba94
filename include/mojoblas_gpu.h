/*
 * mojoblas_gpu.h — C ABI of the B200 (sm_100a) level-3 BLAS library.
 *
 * Drop-in boundary for mojoBLAS's level-3 routines (the gemm / syrk / trsm hot
 * path, and symm / syr2k / trmm on the same kernels) and for the level-2
 * gemv / trsv next to them.  Every routine keeps the
 * argument order and meaning of the mojoBLAS routine it replaces (column-major
 * storage, element (i,j) of a matrix at p[i + j*ld], Netlib transpose / uplo /
 * side / diag characters), and returns:
 *     0               success
 *     > 0             Netlib `info`: the 1-based position of the first invalid
 *                     argument, numbered as the mojoBLAS routine numbers it
 *     < 0             an MBG_ERR_* code below (CUDA failure, allocation, ...)
 * Where mojoBLAS prints "<routine>: Info <n>" and returns, this library returns
 * n and prints nothing.
 *
 * Pointers may be device pointers (the fast path) or ordinary host pointers; the
 * library detects which with cudaPointerGetAttributes and, for host data, copies
 * the operands to the device and the result back, so a host caller sees the
 * same in-place semantics as the reference.  Calls are synchronous unless
 * mbg_set_sync(0) is in effect and every operand is a device pointer.
 *
 * Quick returns, argument checks and the alpha == 0 / k == 0 paths follow the
 * reference; the arithmetic follows Netlib where the reference departs from it:
 * alpha is applied in float64 NN gemm for n >= 512 (the reference's gemm_v7,
 * src/level3/gemm.mojo:817-1132, never applies it), and side 'R' with trans 'T'
 * solves X op(A)^T = alpha B (the reference's right-side transposed branches run
 * the NoTrans loops, src/level3/trsm.mojo:224-273).
 */
#ifndef MOJOBLAS_GPU_H
#define MOJOBLAS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MBG_OK                 0
#define MBG_ERR_CUDA          -1  /* a CUDA runtime call failed (mbg_last_error has it) */
#define MBG_ERR_ALLOC         -2  /* device workspace allocation failed               */
#define MBG_ERR_UNSUPPORTED   -3  /* valid arguments, combination not implemented     */
#define MBG_ERR_NO_DEVICE     -4  /* no usable CUDA device / driver                   */
#define MBG_ERR_TIMEOUT       -5  /* a kernel's bounded wait expired (error flag set)  */
#define MBG_ERR_INVALID_MODE  -6  /* unknown precision mode or slice count            */
#define MBG_ERR_SCRATCH_LIMIT -7  /* problem exceeds mbg_sgemm_ex_noalloc's fixed scratch */

/* ---- precision modes ---------------------------------------------------- */
#define MBG_MODE_PLAIN   0  /* the drop-in: FP32 FMA on the CUDA cores; FP64 on the FP64
                               tensor pipe (DMMA, mma.sync m8n8k4 f64: IEEE FP64 FMAs)   */
#define MBG_MODE_BF16X3  1  /* fp32: a = a1 + a2 in bf16, a1b1 + a1b2 + a2b1 on tcgen05  */
#define MBG_MODE_BF16X6  2  /* fp32: a = a1 + a2 + a3 in bf16, 6 products on tcgen05     */
#define MBG_MODE_OZAKI   3  /* fp64: int8 slices, exact int32 tcgen05 products, fp64 sum */

/* ---- level 3: the reference's routines ---------------------------------- */

/* C := alpha*op(A)*op(B) + beta*C.
 * Replaces mojoBLAS gemm[float32] (src/level3/gemm.mojo:56-124), which routes to
 * gemm_v11 (NN, :2092) or _gemm_naive (:127). */
int mbg_sgemm(char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
              float alpha, const float* a, int64_t lda, const float* b, int64_t ldb,
              float beta, float* c, int64_t ldc);

/* Replaces mojoBLAS gemm[float64] (src/level3/gemm.mojo:56-124: gemm_v3 :385,
 * gemm_v7 :817, _gemm_naive :127). */
int mbg_dgemm(char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
              double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
              double beta, double* c, int64_t ldc);

/* C := alpha*A*A^T + beta*C or alpha*A^T*A + beta*C on the `uplo` triangle.
 * Replaces mojoBLAS syrk (src/level3/syrk.mojo:20-200). */
int mbg_ssyrk(char uplo, char trans, int64_t n, int64_t k, float alpha,
              const float* a, int64_t lda, float beta, float* c, int64_t ldc);
int mbg_dsyrk(char uplo, char trans, int64_t n, int64_t k, double alpha,
              const double* a, int64_t lda, double beta, double* c, int64_t ldc);

/* op(A)*X = alpha*B or X*op(A) = alpha*B, X overwrites B.
 * Replaces mojoBLAS trsm (src/level3/trsm.mojo:20-275). */
int mbg_strsm(char side, char uplo, char trans_a, char diag, int64_t m, int64_t n,
              float alpha, const float* a, int64_t lda, float* b, int64_t ldb);
int mbg_dtrsm(char side, char uplo, char trans_a, char diag, int64_t m, int64_t n,
              double alpha, const double* a, int64_t lda, double* b, int64_t ldb);

/* C := alpha*A*B + beta*C (side 'L', A is m x m) or alpha*B*A + beta*C (side 'R',
 * A is n x n), A symmetric with only its `uplo` triangle read.
 * Replaces mojoBLAS symm (src/level3/symm.mojo:20-241).  Where B(l,j) == 0 the
 * reference also drops alpha * sum_i A(i,l) B(i,j) from C(l,j) (:113, :131);
 * this library computes the full product. */
int mbg_ssymm(char side, char uplo, int64_t m, int64_t n, float alpha, const float* a,
              int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc);
int mbg_dsymm(char side, char uplo, int64_t m, int64_t n, double alpha, const double* a,
              int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc);

/* C := alpha*(A*B^T + B*A^T) + beta*C (trans 'N', A and B n x k) or
 * alpha*(A^T*B + B^T*A) + beta*C (trans 'T' / 'C', A and B k x n), on the
 * `uplo` triangle of C only.  Replaces mojoBLAS syr2k (src/level3/syr2k.mojo:20-190). */
int mbg_ssyr2k(char uplo, char trans, int64_t n, int64_t k, float alpha, const float* a,
               int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc);
int mbg_dsyr2k(char uplo, char trans, int64_t n, int64_t k, double alpha, const double* a,
               int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc);

/* B := alpha*op(A)*B (side 'L') or alpha*B*op(A) (side 'R'), A triangular
 * (`uplo`, unit diagonal not read when diag 'U'), B overwritten.
 * Replaces mojoBLAS trmm (src/level3/trmm.mojo:20-305); alpha == 0 writes zeros. */
int mbg_strmm(char side, char uplo, char trans_a, char diag, int64_t m, int64_t n,
              float alpha, const float* a, int64_t lda, float* b, int64_t ldb);
int mbg_dtrmm(char side, char uplo, char trans_a, char diag, int64_t m, int64_t n,
              double alpha, const double* a, int64_t lda, double* b, int64_t ldb);

/* ---- level 2: the matrix-vector neighbours --------------------------------
 * Vectors are strided: element i of x sits at x[i * incx] for incx > 0 and at
 * x[(n - 1 - i) * |incx|] for incx < 0 (Netlib's convention); incx == 0 is an
 * argument error. */

/* y := alpha*op(A)*x + beta*y, A m x n.  Replaces mojoBLAS gemv
 * (src/level2/gemv.mojo:23-212); like the reference, trans must be 'N', 'T' or
 * 'C' in upper case (anything else is info 1). */
int mbg_sgemv(char trans, int64_t m, int64_t n, float alpha, const float* a, int64_t lda,
              const float* x, int64_t incx, float beta, float* y, int64_t incy);
int mbg_dgemv(char trans, int64_t m, int64_t n, double alpha, const double* a, int64_t lda,
              const double* x, int64_t incx, double beta, double* y, int64_t incy);

/* op(A)*x = b, A n x n triangular, the solution overwrites b in x.  Replaces
 * mojoBLAS trsv (src/level2/trsv.mojo:20-214).  With uplo 'U', trans 'N' and
 * incx != 1 the reference pairs x[j - 1] with column j and reads before the
 * start of x (:113-125); this library solves the system. */
int mbg_strsv(char uplo, char trans, char diag, int64_t n, const float* a, int64_t lda,
              float* x, int64_t incx);
int mbg_dtrsv(char uplo, char trans, char diag, int64_t n, const double* a, int64_t lda,
              double* x, int64_t incx);

/* ---- the same routines with a precision mode ----------------------------
 * mode: MBG_MODE_PLAIN, MBG_MODE_BF16X3 or MBG_MODE_BF16X6 for float;
 *       MBG_MODE_PLAIN or MBG_MODE_OZAKI for double.
 * slices: Ozaki int8 slices per operand (2..8; s slices keep 8s - 2 bits of each
 *         value relative to its row's (column's) largest); ignored
 *         by the other modes.
 * refine: trsm only — iterative-refinement steps after the solve (0 or more):
 *         R = alpha*B - op(A)*X in the accurate mode, solve, X += correction.
 * Same argument numbering for `info` as the plain routine (mode arguments are
 * not counted). */
int mbg_sgemm_ex(int mode, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
                 float alpha, const float* a, int64_t lda, const float* b, int64_t ldb,
                 float beta, float* c, int64_t ldc);
int mbg_dgemm_ex(int mode, int slices, char trans_a, char trans_b, int64_t m, int64_t n,
                 int64_t k, double alpha, const double* a, int64_t lda, const double* b,
                 int64_t ldb, double beta, double* c, int64_t ldc);
int mbg_ssyrk_ex(int mode, char uplo, char trans, int64_t n, int64_t k, float alpha,
                 const float* a, int64_t lda, float beta, float* c, int64_t ldc);
/* dsyrk in MBG_MODE_PLAIN or MBG_MODE_OZAKI (slices as for mbg_dgemm_ex; one set of
 * int8 slices serves both operands, only the uplo triangle is computed). */
int mbg_dsyrk_ex(int mode, int slices, char uplo, char trans, int64_t n, int64_t k, double alpha,
                 const double* a, int64_t lda, double beta, double* c, int64_t ldc);
int mbg_strsm_ex(int mode, int refine, char side, char uplo, char trans_a, char diag,
                 int64_t m, int64_t n, float alpha, const float* a, int64_t lda,
                 float* b, int64_t ldb);
int mbg_dtrsm_ex(int mode, int slices, int refine, char side, char uplo, char trans_a,
                 char diag, int64_t m, int64_t n, double alpha, const double* a,
                 int64_t lda, double* b, int64_t ldb);
/* symm, syr2k and trmm with a precision mode (same modes and slices as gemm). */
int mbg_ssymm_ex(int mode, char side, char uplo, int64_t m, int64_t n, float alpha,
                 const float* a, int64_t lda, const float* b, int64_t ldb, float beta,
                 float* c, int64_t ldc);
int mbg_dsymm_ex(int mode, int slices, char side, char uplo, int64_t m, int64_t n,
                 double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                 double beta, double* c, int64_t ldc);
int mbg_ssyr2k_ex(int mode, char uplo, char trans, int64_t n, int64_t k, float alpha,
                  const float* a, int64_t lda, const float* b, int64_t ldb, float beta,
                  float* c, int64_t ldc);
int mbg_dsyr2k_ex(int mode, int slices, char uplo, char trans, int64_t n, int64_t k,
                  double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                  double beta, double* c, int64_t ldc);
int mbg_strmm_ex(int mode, char side, char uplo, char trans_a, char diag, int64_t m,
                 int64_t n, float alpha, const float* a, int64_t lda, float* b, int64_t ldb);
int mbg_dtrmm_ex(int mode, int slices, char side, char uplo, char trans_a, char diag,
                 int64_t m, int64_t n, double alpha, const double* a, int64_t lda,
                 double* b, int64_t ldb);

/* ---- split-precision sgemm that allocates nothing -------------------------
 * No counterpart in the reference (mojoBLAS allocates host memory freely).
 * For callers that must not have a library allocate device memory: a host
 * framework that owns a fixed device-memory budget, a latency-critical loop
 * where cudaMalloc / cudaFree may synchronise the device, or code inside an
 * allocator's out-of-memory handling.  Same arguments, numbering and result as
 * mbg_sgemm_ex with mode MBG_MODE_BF16X3 or MBG_MODE_BF16X6, but:
 *   - a, b and c must be device pointers (host data would need staging
 *     buffers); otherwise MBG_ERR_UNSUPPORTED;
 *   - the bf16 split planes live in a fixed 32 MiB device array owned by the
 *     library (resident on every GPU that loads it, until the process exits):
 *     terms * (roundup(m,128) + roundup(n,256)) * roundup(k,32) * 2 bytes must
 *     fit (terms = 2 for BF16X3, 3 for BF16X6; e.g. m = n = k = 2048 with
 *     BF16X3), else MBG_ERR_SCRATCH_LIMIT before any device work;
 *   - the first call on a device resolves that array's device address and sets
 *     the kernels' shared-memory limit, so make it before any stream capture;
 *   - every call reuses the same array: calls that overlap on the GPU (other
 *     streams, other host threads) race and must be serialised by the caller;
 *   - an expired kernel wait is returned as MBG_ERR_TIMEOUT by the call itself
 *     in synchronous mode, else by the next mbg_synchronize() (once).
 * No cudaMalloc, cudaFree or other allocating routine is called. */
int mbg_sgemm_ex_noalloc(int mode, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
                         float alpha, const float* a, int64_t lda, const float* b, int64_t ldb,
                         float beta, float* c, int64_t ldc);

/* ---- complex gemm ---------------------------------------------------------
 * C := alpha*op(A)*op(B) + beta*C for single (c) and double (z) complex, with
 * op(X) = X ('N'), X^T ('T') or X^H ('C', conjugate transpose).  Matrices are
 * column-major arrays of interleaved (re, im) pairs (lda, ldb, ldc count
 * complex elements); alpha and beta point at one (re, im) pair each in host
 * memory.  No counterpart in the reference: complex dtypes are on mojoBLAS's
 * roadmap (README.md:152); the argument order and `info` numbering are those
 * of its gemm (src/level3/gemm.mojo:56-78, :179-213).  Computed as one real
 * product of 2m x n x 2k (the real embedding [Ar -Ai; Ai Ar] [Br; Bi], rows
 * and reduction interleaved so C is written in place) in the mode given:
 * MBG_MODE_PLAIN / BF16X3 / BF16X6 for c, MBG_MODE_PLAIN / OZAKI (slices) for z. */
int mbg_cgemm(char trans_a, char trans_b, int64_t m, int64_t n, int64_t k, const float* alpha,
              const float* a, int64_t lda, const float* b, int64_t ldb, const float* beta, float* c,
              int64_t ldc);
int mbg_zgemm(char trans_a, char trans_b, int64_t m, int64_t n, int64_t k, const double* alpha,
              const double* a, int64_t lda, const double* b, int64_t ldb, const double* beta, double* c,
              int64_t ldc);
int mbg_cgemm_ex(int mode, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k, const float* alpha,
                 const float* a, int64_t lda, const float* b, int64_t ldb, const float* beta, float* c,
                 int64_t ldc);
int mbg_zgemm_ex(int mode, int slices, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
                 const double* alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                 const double* beta, double* c, int64_t ldc);

/* ---- adjoints (reverse mode) --------------------------------------------
 * No counterpart in the reference.  Given the upstream gradient G = dL/dC of
 * C = alpha*op(A)*op(B), the gemm adjoint writes dA (shape of A, skipped if da
 * is NULL) and dB (shape of B, skipped if db is NULL):
 *     d op(A) = alpha * G * op(B)^T,   d op(B) = alpha * op(A)^T * G.
 * Given X (the trsm result) and G = dL/dX, the trsm adjoint writes
 *     dB = alpha * op(A)^{-T} G                    (side 'L'; G op(A)^{-T} for 'R')
 *     dA = -tri(W X^T)  with W = op(A)^{-T} G      (left, trans 'N'; the other
 *          cases are the corresponding transposes), only on the stored
 *          triangle of A (a triangle-only GEMM: the other triangle's tiles are
 *          not computed, nor written); zero diagonal for diag 'U'; da may be NULL.
 * `info` numbering follows the argument position (mode / slices not counted). */
int mbg_sgemm_adjoint(int mode, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k, float alpha,
                      const float* a, int64_t lda, const float* b, int64_t ldb, const float* g, int64_t ldg,
                      float* da, int64_t ldda, float* db, int64_t lddb);
int mbg_dgemm_adjoint(int mode, int slices, char trans_a, char trans_b, int64_t m, int64_t n, int64_t k,
                      double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                      const double* g, int64_t ldg, double* da, int64_t ldda, double* db, int64_t lddb);
int mbg_strsm_adjoint(int mode, char side, char uplo, char trans_a, char diag, int64_t m, int64_t n,
                      float alpha, const float* a, int64_t lda, const float* x, int64_t ldx,
                      const float* g, int64_t ldg, float* db, int64_t lddb, float* da, int64_t ldda);
int mbg_dtrsm_adjoint(int mode, int slices, char side, char uplo, char trans_a, char diag, int64_t m,
                      int64_t n, double alpha, const double* a, int64_t lda, const double* x,
                      int64_t ldx, const double* g, int64_t ldg, double* db, int64_t lddb, double* da,
                      int64_t ldda);

/* ---- batched: many independent problems in one persistent launch ----------
 * No counterpart in the reference, whose callers loop over gemm / trsm.
 * A plan validates the problems (Netlib numbering per problem; the first
 * invalid problem's info is returned and described by mbg_last_error), copies
 * the problem table to the device once and records [reset; persistent kernel]
 * into a CUDA graph; mbg_plan_execute replays it on the library stream.  All
 * matrix pointers must be device pointers and stay valid for the plan's life.
 *   sgemm, MBG_MODE_PLAIN: any transposes, any sizes; FP32 CUDA-core tiles of
 *          64 or 128 per problem (the tuning table's entry for the problem's
 *          transposes and size class, else "grouped_gemm_tile"), largest problems
 *          first, atomic tile counter (one persistent kernel per tile size).
 *   sgemm, MBG_MODE_BF16X3 / BF16X6: one persistent tcgen05 kernel; its producer
 *          warps load and split each problem's operands into bf16 terms in
 *          shared memory (no pre-pass, any leading dimension), tiles of 128 x 64
 *          or 128 x 128 per problem (tuning table), longest reduction first.
 *   strsm: side 'L' only, m <= 256 (the triangle order), any uplo/trans/diag;
 *          32-column strips solved by the fused diagonal-block routine;
 *          mode MBG_MODE_PLAIN. */
typedef struct {
    char trans_a, trans_b;
    int64_t m, n, k;
    float alpha, beta;
    const float* a; int64_t lda;
    const float* b; int64_t ldb;
    float* c; int64_t ldc;
} mbg_sgemm_problem;

typedef struct {
    char side, uplo, trans_a, diag;
    int64_t m, n;
    float alpha;
    const float* a; int64_t lda;
    float* b; int64_t ldb;
} mbg_strsm_problem;

typedef struct mbg_plan mbg_plan;

int mbg_sgemm_grouped_plan(int mode, int count, const mbg_sgemm_problem* problems, mbg_plan** plan);
int mbg_strsm_grouped_plan(int mode, int count, const mbg_strsm_problem* problems, mbg_plan** plan);
int mbg_plan_execute(mbg_plan* plan);
int mbg_plan_destroy(mbg_plan* plan);
/* one-shot forms: plan, execute, destroy */
int mbg_sgemm_grouped(int mode, int count, const mbg_sgemm_problem* problems);
int mbg_strsm_grouped(int mode, int count, const mbg_strsm_problem* problems);

/* ---- runtime ------------------------------------------------------------ */
/* Stream for subsequent calls from any thread (a cudaStream_t; NULL = legacy
 * default stream, the initial value). */
int   mbg_set_stream(void* stream);
/* on != 0: subsequent calls from the calling host thread use `stream` instead
 * of the process-wide one; on == 0: back to the process-wide stream.  Threads
 * that each set their own stream run their calls concurrently: device
 * workspace blocks are pooled per stream, so no block is shared by work in
 * flight on two streams.  (The reference's routines take no stream; a Mojo
 * caller that runs them from several threads sets one stream per thread.) */
int   mbg_set_thread_stream(int on, void* stream);
/* the stream the calling thread's calls use */
void* mbg_get_stream(void);
/* 1 (default): every call returns after its device work finished.
 * 0: calls whose operands are all device pointers return after enqueueing. */
int   mbg_set_sync(int on);
/* Synchronise the library stream and report a pending kernel error flag. */
int   mbg_synchronize(void);
const char* mbg_status_string(int status);
const char* mbg_last_error(void);
int   mbg_version(void);
/* Release cached device workspace. */
int   mbg_release_workspace(void);

/* ---- tuning table -------------------------------------------------------
 * Keys: "trsm_tc_min_k" — trsm off-diagonal updates with a shorter reduction
 * run on the plain kernel instead of the split / Ozaki forms (default 512);
 * "grouped_gemm_tile" — 64 or 128, tile edge of grouped sgemm plans (default 64);
 * "trsm_leaf_ctas" — CTA cap of the trsm 64-row diagonal-block solve (0 = 8 per SM);
 * "trsm_block_rows" — diagonal blocks up to this many rows (capped at 512 for
 * double, 1024 for float) are solved in one fused launch, sub-block updates
 * included (default 512; 64 or less: 64-row leaves with gemm updates between them);
 * "trsm_block_min_cols" — the fused launch is used only with at least this
 * many right-hand sides (default 64);
 * "trsm_inverse_min_cols" — split / Ozaki trsm with at least this many
 * right-hand sides inverts its diagonal blocks once (native precision)
 * and applies each inverse as a split / Ozaki product (default 256; 0 = never:
 * substitution in the diagonal blocks);
 * "trsm_inverse_block" — rows of those diagonal blocks, 256 or 512 (default 512);
 * "ozaki_cta_pair" — Ozaki products on CTA pairs (tcgen05 cta_group::2,
 * 256 x 128 tiles over two SMs): 1 one cluster per tile, 2 persistent clusters
 * (one per two SMs, the epilogue of a tile overlapping the next tile's products);
 * 0: one CTA per 128 x 128 tile; default 2;
 * "trsm_preslice" — 1 (default): a split or Ozaki trsm makes the planes of all
 * its off-diagonal update blocks of op(A) up front on a second stream, beside
 * the diagonal blocks' inversion (0: before each update);
 * "ozaki_fused_slicing" — 1 (default): a K-contiguous Ozaki operand's exponents
 * and slices in one pass (0: the separate exponent and slicing kernels);
 * "grouped_simt_tile_<TT>_c<d>", "grouped_tc_bn_<TT>_c<d>" — grouped sgemm
 * plans' tile table, per transposes TT (NN, NT, TN, TT) and size class d of
 * max(m, n) (0: <= 32, 1: <= 64, 2: <= 128, 3: <= 256, 4: larger): the plain
 * form's tile edge and the split form's tile width, 64 or 128 (0 = default:
 * "grouped_gemm_tile", resp. 64 for n <= 64 else 128);
 * "plain_fp64_simt" — 1: plain FP64 gemm / syrk on the CUDA cores instead of the
 * FP64 tensor pipe (default 0); "plain_fp32_staged" — 1: plain FP32 gemm / syrk
 * with the register-staged tiles instead of the cp.async pipeline (default 0).
 * mbg_load_tuning reads "key value" lines (or a flat JSON object of them) as
 * written by the autotuner (mojoblas_b200/autotune.py).
 * mbg_get_tuning returns -1 for an unknown key. */
int     mbg_set_tuning(const char* key, int64_t value);
int64_t mbg_get_tuning(const char* key);
int     mbg_load_tuning(const char* path);

/* ---- peak probes ----------------------------------------------------------
 * Measured throughput (TFLOP/s, dense, 2 ops per multiply-add) of fp32 and fp64
 * FMA loops on the CUDA cores and of back-to-back tcgen05.mma kind::f16 (bf16)
 * and kind::i8 on one CTA per SM: the roofline denominators of the plain and
 * Ozaki kernels.  Any output pointer may be NULL. */
int mbg_probe_peaks(double* fp32_tflops, double* fp64_tflops, double* bf16_tflops, double* int8_tops);

/* ---- kernel timing (CUDA events around each library kernel launch) ------ */
int mbg_prof_enable(int on);
int mbg_prof_reset(void);
/* Total device milliseconds and launch count recorded for kernels whose name
 * contains `name_substring` since the last reset (events are resolved here). */
int mbg_prof_query(const char* name_substring, double* total_ms, int64_t* launches);
/* Launches of library kernels since the last reset, counted on the host. */
int64_t mbg_launch_count(void);

/* ---- test hooks ----------------------------------------------------------- */
/* Make the n-th device allocation from now on fail (n >= 1); 0 disables. */
int mbg_debug_fail_alloc(int nth);
/* Launch one kernel whose bounded mbarrier wait can never be satisfied and
 * gives up after limit_ns (at most 5 s): returns MBG_ERR_TIMEOUT with the
 * context still usable — the failure path of every tcgen05 kernel's waits. */
int mbg_debug_wait_probe(int64_t limit_ns);
/* Store `code` in mbg_sgemm_ex_noalloc's kernel wait flag on the current device,
 * as an expired wait would; the next synchronous call or mbg_synchronize()
 * reports it once as MBG_ERR_TIMEOUT. */
int mbg_debug_set_noalloc_error(int code);

#ifdef __cplusplus
}
#endif

#endif /* MOJOBLAS_GPU_H */
