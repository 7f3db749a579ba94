// Tensor-core GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Two precision forms, each a warp-specialised kernel sharing the PTX helpers
// and the pre-pass design:
//
//  * Split-precision sgemm (BF16x3 / BF16x6).  A pre-pass splits each fp32
//    operand element x into bf16 terms x = x1 + x2 (+ x3) + residual, with
//    x1 = bf16(x), x2 = bf16(x - x1), x3 = bf16(x - x1 - x2) (each difference is
//    exact in fp32).  The kernel forms sum_{p+q<T} A_p B_q with
//    tcgen05.mma.kind::f16 (bf16 inputs, fp32 accumulation in TMEM):
//    3 products for T=2 (BF16x3), 6 for T=3 (BF16x6).
//
//  * Ozaki-scheme dgemm (int8 slices).  A pre-pass scales each row of op(A) and
//    each column of op(B) by a power of two (x = x' 2^e, |x'| < 1), truncates x'
//    to the integer F = trunc(x' 2^(8s-2)) and writes F's signed base-256 digits,
//    x' ~ sum_p d_p 2^(-8p-6), d_p in [-128, 127] (two's-complement digits, least
//    significant first; |F| < 2^(8s-2) keeps the leading one within [-65, 65]),
//    so s slices keep 8s - 2 bits.  The kernel forms, for each diagonal
//    t = p+q < s, D_t = sum_{p+q=t} A_p B_q exactly with
//    tcgen05.mma.kind::i8 (int32 accumulation, one TMEM accumulator per t, at
//    most four at a time: more than four slices run two passes over k), and
//    the epilogue sums 2^(-8t-12) D_t from the smallest term up in fp64 and
//    applies the row and column scales (Ootomo, Ozaki, Yokota, "DGEMM on integer
//    matrix multiplication unit", IJHPCA 2024; Ozaki, Ogita, Oishi, Rump, 2012).
//
// Both pre-passes also transpose as needed, so the kernel always sees
// K-contiguous ("K-major") operands: planes[term][row][k], rows padded to the
// tile, k padded to the k-slab, zero-filled.
//
// Kernel roles (one CTA per 128 x BN output tile; BN = 256 split, 128 Ozaki):
//   warp 0      allocates TMEM; lane 0 issues TMA loads (cp.async.bulk.tensor,
//               one 3-D box per operand per stage covering every term plane)
//   warp 1      lane 0 issues the tcgen05.mma instructions and commits each
//               stage back to the producer, then the accumulators to the epilogue
//   warps 2..9  epilogue, two warps per TMEM lane quarter: tcgen05.ld (warp w
//               reads lanes 32*(w%4)..), accumulate / scale, add beta*C, store
//               column-major C with coalesced warps
// Every mbarrier wait is bounded (about 2 s of globaltimer); on expiry the
// thread records an error code in the library's mapped error flag and the CTA
// proceeds to teardown (TMEM is always freed).
#include "mbg_internal.cuh"
#include "tc_ptx.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <mutex>

namespace mbg {

namespace tc {

// ---------------------------------------------------------------------------
// Kernel configuration
// ---------------------------------------------------------------------------
// TERMS planes per operand; products (p, q) with p + q < TERMS.
//   split:  every product accumulates into one fp32 accumulator.  The tensor
//           core's fp32 accumulation truncates, so its error grows linearly in
//           k; the accumulator is therefore restarted every CHUNK slabs and the
//           epilogue warps add each chunk into fp32 registers with
//           round-to-nearest ("promotion").  Two TMEM buffers alternate so the
//           MMA issuer never waits for a drain.
//   ozaki:  product (p, q) accumulates into int32 accumulator p + q (exact, so
//           one chunk covers the whole k range).
template <bool OZAKI_, int TERMS_, int BN_, int BKB_, int STAGES_, int EPI_WARPS_, int CHUNK_>
struct Cfg {
    static constexpr bool OZAKI = OZAKI_;
    static constexpr int TERMS = TERMS_;
    static constexpr int BN = BN_;
    static constexpr int BKB = BKB_;  // k-slab bytes per row (= swizzle width)
    static constexpr int STAGES = STAGES_;
    static constexpr int EPI_WARPS = EPI_WARPS_;
    static constexpr int CHUNK = CHUNK_;  // slabs per TMEM accumulation chunk (split only)
    static constexpr int THREADS = 64 + 32 * EPI_WARPS;
    static constexpr int ELEM = OZAKI ? 1 : 2;
    static constexpr int BK = BKB / ELEM;    // k elements per slab
    static constexpr int KSTEPS = BKB / 32;  // one MMA consumes 32 bytes of k
    static constexpr int NPROD = TERMS * (TERMS + 1) / 2;
    static constexpr int NACC = OZAKI ? TERMS : 2;  // ozaki: one per diagonal; split: two buffers
    static constexpr int A_PLANE = BM * BKB;
    static constexpr int B_PLANE = BN * BKB;
    static constexpr int STAGE_BYTES = TERMS * (A_PLANE + B_PLANE);
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr uint32_t LAYOUT = BKB == 128 ? 2 : (BKB == 64 ? 4 : 6);
    static constexpr uint32_t SBO = 8 * BKB;
    static constexpr int TMEM_NEED = NACC * BN;
    static constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128
                                        : TMEM_NEED <= 256 ? 256 : 512;
    static constexpr int EPI_COLS = BN / (EPI_WARPS / 4);  // columns per epilogue thread
    static constexpr int TILE_M = BM, TILE_N = BN, TILE_GROUP = 16;  // output tile; m-tiles per L2 group
    static constexpr uint32_t IDESC = instr_desc(OZAKI, BM, BN);
    static_assert(TMEM_NEED <= 512, "accumulators exceed TMEM");
    static_assert(SMEM_BYTES <= 232448, "shared memory budget");
    static_assert(A_PLANE % 1024 == 0 && B_PLANE % 1024 == 0, "plane alignment");
    static_assert(EPI_WARPS % 4 == 0 && EPI_COLS % 16 == 0, "epilogue shape");
};

using CfgBF16x3 = Cfg<false, 2, 256, 64, 4, 8, 4>;
using CfgBF16x6 = Cfg<false, 3, 256, 64, 3, 8, 4>;
// 128 x 64 tiles for products too small to give a quarter of the SMs a 128 x 256 tile (the
// trsm recursion's 512-row blocks: 8 CTAs of the wide tile against 32 of these)
using CfgBF16x3n = Cfg<false, 2, 64, 64, 8, 8, 4>;
using CfgBF16x6n = Cfg<false, 3, 64, 64, 6, 8, 4>;
// 128 x 128 tiles for products that give fewer CTAs than SMs with 128 x 256 tiles: twice the
// CTAs, so a last partial wave idles less of the GPU (the gemm adjoint's two products)
using CfgBF16x3m = Cfg<false, 2, 128, 64, 6, 8, 4>;
using CfgBF16x6m = Cfg<false, 3, 128, 64, 4, 8, 4>;

struct Params {
    i64 m, n;
    int num_kb;            // k slabs
    int tiles_m, tiles_n;  // output tiles
    int tri;               // 0 full, 1 lower, 2 upper (element mask + tile skip)
    int band;              // KB_*: one operand triangular, each tile runs its band of slabs
    i64 band_k0;           // first k element of this launch within the full reduction
    const float* dvec;     // non-null: C = alpha acc + d .* C, d per row (dvec_mode 1) or column (2)
    int dvec_mode;
    void* c;
    i64 ldc;
    double alpha, beta;
    const int* ea;  // ozaki row exponents (op(A) rows)
    const int* eb;  // ozaki column exponents (op(B) columns)
    int* err;
};

// One output row's EPI_COLS columns from cbase of a split product: C = alpha acc (+ beta C),
// the trmm form alpha acc + d .* C, triangle masks; columns past n are skipped.
template <class C>
__device__ __forceinline__ void split_store_row(const Params& P, const i64 row, const i64 cbase,
                                                const float (&acc)[C::EPI_COLS]) {
    float* Cm = static_cast<float*>(P.c);
    const float alpha = float(P.alpha), beta = float(P.beta);
    // 8 columns at a time: all loads of C are issued before the
    // first is used, so the read-modify-write of a beta != 0 call
    // waits for memory once per 8 columns, not once per column
    // beta == 1 (the trsm updates): C += v as a reduction in L2 — one
    // add per element, rounded as c + v, with no read in the thread
    if (P.dvec) {  // trmm: C = alpha acc + d C, d per row or per column
        const float drow = P.dvec_mode == 1 ? P.dvec[row] : 0.0f;
#pragma unroll
        for (int c0 = 0; c0 < C::EPI_COLS; c0 += 8) {
            float cv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const i64 col = cbase + c0 + j;
                cv[j] = col < P.n ? Cm[row + col * P.ldc] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const i64 col = cbase + c0 + j;
                if (col >= P.n) continue;
                const float d = P.dvec_mode == 1 ? drow : P.dvec[col];
                Cm[row + col * P.ldc] = fmaf(d, cv[j], alpha * acc[c0 + j]);
            }
        }
    } else if (beta == 1.0f) {
#pragma unroll
        for (int j = 0; j < C::EPI_COLS; ++j) {
            const i64 col = cbase + j;
            if (col < P.n && !(P.tri == 1 && row < col) && !(P.tri == 2 && row > col))
                atomicAdd(Cm + row + col * P.ldc, alpha * acc[j]);
        }
    } else
#pragma unroll
    for (int c0 = 0; c0 < C::EPI_COLS; c0 += 8) {
        float cv[8];
        bool live[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const i64 col = cbase + c0 + j;
            live[j] = col < P.n && !(P.tri == 1 && row < col) && !(P.tri == 2 && row > col);
            cv[j] = (live[j] && beta != 0.0f) ? Cm[row + col * P.ldc] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (!live[j]) continue;
            const float v = alpha * acc[c0 + j];
            Cm[row + (cbase + c0 + j) * P.ldc] = (beta == 0.0f) ? v : fmaf(beta, cv[j], v);
        }
    }
}

// Output tile `tile` of the product P, its operands' planes read through tmA / tmB (kernel
// parameters): one CTA's whole work in the kernels below.
template <class C>
__device__ __forceinline__ void tc_gemm_tile(const CUtensorMap& tmA, const CUtensorMap& tmB, const Params& P,
                                             const int tile) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + C::STAGES;
    uint64_t* tfull = empty + C::STAGES;  // [2]: accumulator buffer ready for the epilogue
    uint64_t* tempty = tfull + 2;         // [2]: epilogue finished reading a buffer
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);

    // tile coordinates: groups of 16 m-tiles walk the n-tiles together (L2 reuse)
    const int group = 16;
    const int per_group = group * P.tiles_n;
    const int g = tile / per_group;
    const int first_m = g * group;
    const int gsize = min(group, P.tiles_m - first_m);
    const int in_g = tile - g * per_group;
    int tm = first_m + in_g % gsize;
    int tn = in_g / gsize;
    // banded launches: heaviest tiles first (the last wave holds the short ones)
    if (P.band == KB_A_LOWER) tm = P.tiles_m - 1 - tm;
    if (P.band == KB_B_UPPER) tn = P.tiles_n - 1 - tn;
    const i64 m0 = i64(tm) * BM, n0 = i64(tn) * C::BN;
    if (P.tri == 1 && m0 + BM <= n0) return;        // tile strictly above the diagonal
    if (P.tri == 2 && m0 > n0 + C::BN - 1) return;  // tile strictly below the diagonal

    // slabs [kb0, kb0 + nkb) of the reduction: all of them, or the tile's band
    int kb0 = 0, nkb = P.num_kb;
    if (P.band != KB_NONE) {
        i64 s0, s1;
        band_slabs(P.band, m0, BM, n0, C::BN, P.band_k0, C::BK, P.num_kb, s0, s1);
        kb0 = int(s0);
        nkb = int(s1 - s0);
    }
    const int chunk_slabs = C::OZAKI ? nkb : C::CHUNK;
    const int nchunks = (nkb + chunk_slabs - 1) / chunk_slabs;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], C::EPI_WARPS);
        }
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, C::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb % C::STAGES;
                const uint32_t ph = (kb / C::STAGES) & 1;
                if (!mbar_wait(&empty[s], ph ^ 1, P.err, 1)) break;
                uint8_t* sa = smem + s * C::STAGE_BYTES;
                uint8_t* sb = sa + C::TERMS * C::A_PLANE;
                mbar_expect_tx(&full[s], C::STAGE_BYTES);
                tma_load_3d(sa, &tmA, &full[s], (kb0 + kb) * C::BK, int(m0), 0);
                tma_load_3d(sb, &tmB, &full[s], (kb0 + kb) * C::BK, int(n0), 0);
            }
            // all issued loads must land before the CTA can exit: the last
            // STAGES slabs are the only ones possibly still in flight
            for (int kb = max(0, nkb - C::STAGES); kb < nkb; ++kb)
                mbar_wait(&full[kb % C::STAGES], (kb / C::STAGES) & 1, P.err, 2);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int chunk = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                const int kin = kb % chunk_slabs;  // slab index within the chunk
                const int buf = chunk & 1;
                if (!C::OZAKI && kin == 0 && chunk >= 2) {
                    // the epilogue must have drained this buffer's previous chunk
                    if (!mbar_wait(&tempty[buf], ((chunk >> 1) - 1) & 1, P.err, 5)) break;
                    tc_fence_after();
                }
                const int s = kb % C::STAGES;
                const uint32_t ph = (kb / C::STAGES) & 1;
                if (!mbar_wait(&full[s], ph, P.err, 3)) break;
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
                const uint32_t sb = sa + C::TERMS * C::A_PLANE;
#pragma unroll
                for (int ks = 0; ks < C::KSTEPS; ++ks) {
#pragma unroll
                    for (int pi = 0; pi < C::NPROD; ++pi) {
                        int p, q, collector;
                        product<C::TERMS, C::OZAKI>(pi, p, q, collector);
                        // the first product into an accumulator in a chunk overwrites it
                        const bool first = C::OZAKI ? (p == 0) : (pi == 0);
                        const uint32_t accumulate = (kin > 0 || ks > 0 || !first) ? 1u : 0u;
                        const uint32_t col = C::OZAKI ? uint32_t((p + q) * C::BN) : uint32_t(buf * C::BN);
                        const uint64_t ad = smem_desc(sa + p * C::A_PLANE + ks * 32, C::SBO, C::LAYOUT);
                        const uint64_t bd = smem_desc(sb + q * C::B_PLANE + ks * 32, C::SBO, C::LAYOUT);
                        umma<C::OZAKI>(tmem + col, ad, bd, C::IDESC, accumulate, collector);
                    }
                }
                umma_commit(&empty[s]);  // slot s is free once these MMAs have read it
                if (kin == chunk_slabs - 1 || kb == nkb - 1) {
                    umma_commit(&tfull[buf]);  // chunk complete
                    ++chunk;
                }
            }
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int e = warp - 2;
        const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
        const int part = e >> 2;       // which EPI_COLS-wide column range
        const i64 row = m0 + quarter * 32 + lane;
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16);
        if constexpr (!C::OZAKI) {
            float acc[C::EPI_COLS];
#pragma unroll
            for (int j = 0; j < C::EPI_COLS; ++j) acc[j] = 0.0f;
            bool ok = true;
            for (int ch = 0; ch < nchunks; ++ch) {
                const int buf = ch & 1;
                if (!mbar_wait(&tfull[buf], (ch >> 1) & 1, P.err, 4)) { ok = false; break; }
                tc_fence_after();
#pragma unroll
                for (int c0 = 0; c0 < C::EPI_COLS; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(lane_base + uint32_t(buf * C::BN + part * C::EPI_COLS + c0), r);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[c0 + j] += __uint_as_float(r[j]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (ok && row < P.m) split_store_row<C>(P, row, n0 + part * C::EPI_COLS, acc);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, C::TMEM_COLS);
    }
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params P) {
    tc_gemm_tile<C>(tmA, tmB, P, int(blockIdx.x));
}

// ---------------------------------------------------------------------------
// Ozaki kernel: 128 x 128 tiles, diagonals in up to two passes over k
// ---------------------------------------------------------------------------
// An MMA of N = 128 columns reads its A tile once per 128 outputs; N = 64 left
// the int8 pipe half idle.  Four int32 accumulators of 128 columns fill TMEM, so
// with more than four slices the diagonals are split: pass 0 accumulates the
// high diagonals 4 .. S-1 (the smallest weights, needing every slice), pass 1
// the low diagonals 0 .. 3 (needing slices 0 .. 3 only).  After each pass the
// epilogue warps add w_d * D_d into fp64 registers, smallest weights first, and
// release TMEM for the next pass.
template <int S_>
struct OzCfg {
    static constexpr int S = S_;
    static constexpr int BN = 128;
    static constexpr int BKB = 32;                    // k slab: 32 int8 per row (32-byte swizzle)
    static constexpr int EPI_WARPS = 8;
    static constexpr int THREADS = 64 + 32 * EPI_WARPS;
    static constexpr int EPI_COLS = BN / (EPI_WARPS / 4);  // 64
    static constexpr int NPASS = S <= 4 ? 1 : 2;
    static constexpr int SPLIT = S <= 4 ? 0 : 4;      // pass 0: [SPLIT, S), pass 1: [0, SPLIT)
    static constexpr int PLANE = BM * BKB;            // A and B tiles are both 128 x 32 bytes
    static constexpr int STAGE_BYTES = 2 * S * PLANE;
    static constexpr int STAGES = (196608 / STAGE_BYTES) > 6 ? 6 : (196608 / STAGE_BYTES);
    static constexpr int EXP_BYTES = EPI_WARPS * EPI_COLS * 4;  // staged column exponents
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256 + EXP_BYTES;
    static constexpr uint32_t IDESC = instr_desc(true, BM, BN);
    static constexpr uint32_t SBO = 8 * BKB, LAYOUT = 6;
    static_assert(STAGES >= 2, "pipeline depth");
};

// pass -> diagonal range [lo, hi) and the slices whose tiles it loads
template <class C>
__device__ __forceinline__ void pass_range(int pass, int& lo, int& hi, int& planes) {
    if (C::NPASS == 1) { lo = 0; hi = C::S; planes = C::S; return; }
    if (pass == 0) { lo = C::SPLIT; hi = C::S; planes = C::S; }
    else { lo = 0; hi = C::SPLIT; planes = C::SPLIT; }
}

// product index within a pass -> (p, q, collector use); ordered by p so that
// consecutive products share A_p (collector buffer), q ascending
template <int S>
__device__ __forceinline__ bool oz_product(int lo, int hi, int idx, int& p, int& q, int& collector) {
    int t = 0;
    for (int pp = 0; pp < S; ++pp) {
        const int q0 = lo - pp > 0 ? lo - pp : 0;
        const int q1 = (hi - 1 - pp) < (S - 1) ? (hi - 1 - pp) : (S - 1);
        const int cnt = q1 >= q0 ? q1 - q0 + 1 : 0;
        if (idx < t + cnt) {
            p = pp;
            q = q0 + (idx - t);
            collector = cnt > 1 ? (q == q0 ? 1 : (q == q1 ? 3 : 2)) : 0;
            return true;
        }
        t += cnt;
    }
    return false;
}

// Width in bytes of k of one slab of the Ozaki planes' layout (oz_plane_offset): the
// CTA-pair kernel loads one slab per stage, 64-byte rows with the 64-byte swizzle; the
// single-CTA kernel loads half a slab, 32-byte rows with the 32-byte swizzle.
constexpr int OZ_SLAB = 64;

struct OzParams {
    i64 m, n;
    int num_kb, tiles_m, tiles_n;
    int tri;  // 0 full, 1 lower, 2 upper (element mask + tile skip)
    int band;     // KB_*: one operand triangular, each tile runs its band of slabs
    i64 band_k0;  // first k element of this launch within the full reduction
    const double* dvec;  // non-null: C = alpha acc + d .* C, d per row (dvec_mode 1) or column (2)
    int dvec_mode;
    double* c;
    i64 ldc;
    double alpha, beta;
    const int* ea;
    const int* eb;
    int* err;
};

template <int S, int PASS> struct OzPass {
    static constexpr int NP = S <= 4 ? 1 : 2;
    static constexpr int LO = (NP == 1) ? 0 : (PASS == 0 ? 4 : 0);
    static constexpr int HI = (NP == 1) ? S : (PASS == 0 ? S : 4);
};

// Issues one pass: every k slab, the products of diagonals [LO, HI), then
// commits the accumulators to the epilogue.  Returns false if a wait expired.
template <class C, int PASS>
__device__ __forceinline__ bool oz_mma_pass(const OzParams& P, int nkb, uint8_t* smem, uint64_t* full,
                                            uint64_t* empty, uint64_t* tfull, uint64_t* tempty, uint32_t tmem) {
    constexpr int LO = OzPass<C::S, PASS>::LO, HI = OzPass<C::S, PASS>::HI;
    if (PASS > 0) {  // the epilogue must have read the previous pass's accumulators
        if (!mbar_wait(tempty, (PASS - 1) & 1, P.err, 13)) return false;
        tc_fence_after();
    }
    for (int kb = 0; kb < nkb; ++kb) {
        const int it = PASS * nkb + kb;
        const int s = it % C::STAGES;
        if (!mbar_wait(&full[s], (it / C::STAGES) & 1, P.err, 14)) return false;
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
        const uint32_t sb = sa + C::S * C::PLANE;
#pragma unroll
        for (int pi = 0; pi < C::S * C::S; ++pi) {
            int p = 0, q = 0, collector = 0;
            if (!oz_product<C::S>(LO, HI, pi, p, q, collector)) break;
            // (0, d) is the first product of diagonal d in p-major order
            const uint32_t accumulate = (kb > 0 || p > 0) ? 1u : 0u;
            const uint64_t ad = smem_desc(sa + p * C::PLANE, C::SBO, C::LAYOUT);
            const uint64_t bd = smem_desc(sb + q * C::PLANE, C::SBO, C::LAYOUT);
            umma<true>(tmem + uint32_t((p + q - LO) * C::BN), ad, bd, C::IDESC, accumulate, collector);
        }
        umma_commit(&empty[s]);
    }
    umma_commit(tfull);  // this pass's accumulators are complete
    return true;
}

// The column exponents of an epilogue warp's EPI_COLS columns, staged in the warp's own
// slice of shared memory at the start of each tile (while the tile's products run), so
// the stores wait on no global load, and the row's exponent.  `fast`: the row takes the
// short store path of oz_store_row (no triangle mask, and every scale 2^(er + ec) a
// normal number).
struct OzRowExp {
    int er;
    bool fast;
};
template <class C>
__device__ __forceinline__ OzRowExp oz_stage_exponents(const OzParams& P, i64 row, i64 cbase, int* ex, int lane) {
    __syncwarp();  // every lane has finished the previous tile's stores
    int lo = 1 << 30, hi = -(1 << 30);
#pragma unroll
    for (int j = lane; j < C::EPI_COLS; j += 32) {
        const i64 col = cbase + j;
        const int v = col < P.n ? P.eb[col] : 0;
        ex[j] = v;
        if (col < P.n) {
            lo = min(lo, v);
            hi = max(hi, v);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    OzRowExp r;
    r.er = row < P.m ? P.ea[row] : 0;
    r.fast = P.tri == 0 && (lo > hi || (r.er + lo >= -1022 && r.er + hi <= 1023));
    __syncwarp();
    return r;
}

// An int32 accumulator as a double, exactly, without the int-to-fp64 conversion unit
// (a quarter-rate pipe that bounded the accumulator drains): the bits of 2^52 + 2^51 + v
// are 0x4338000000000000 + v for |v| < 2^51, and subtracting 2^52 + 2^51 is exact.
__device__ __forceinline__ double oz_i2d(uint32_t v) {
    const int hi = 0x43380000 + (static_cast<int>(v) >> 31);
    return __hiloint2double(hi, static_cast<int>(v)) - 6755399441055744.0;  // 2^52 + 2^51
}

// 2^e for -1022 <= e <= 1023 (a normal number), from its bits.
__device__ __forceinline__ double oz_pow2(int e) { return __longlong_as_double(static_cast<long long>(e + 1023) << 52); }

// Row `row` of the tile's output, columns cbase .. cbase + EPI_COLS - 1: scales the
// fp64 sums by the row exponent and the column exponents ex (staged by
// oz_stage_exponents) and applies alpha / beta (or the trmm diagonal term), as one
// epilogue thread of either Ozaki kernel owns them.  The short path (x.fast) is
// straight-line code without branches per element, its reads of C (and of the diagonal
// term) on the read-only path so that they need not wait for the stores before them
// (each element is read once, by its own thread, before that thread writes it): the
// general one, with its masks, out-of-range scalings and a global load per column, ran a
// tile's stores at a few GB/s per SM, longer than the tile's products when k is a few
// hundred.
template <class C>
__device__ __forceinline__ void oz_store_row(const OzParams& P, i64 row, i64 cbase, const double (&acc)[C::EPI_COLS],
                                             const int* ex, OzRowExp x) {
    const int er = x.er;
    if (x.fast) {
        const int nc = int(min(i64(C::EPI_COLS), P.n - cbase));  // live columns
        double* cp = P.c + row + cbase * P.ldc;
        const i64 ldc = P.ldc;
        const double alpha = P.alpha, beta = P.beta;
        if (P.dvec) {  // trmm and the inverse-based trsm leaves: C = alpha acc + d C
            const bool per_row = P.dvec_mode == 1;
            const double drow = per_row ? __ldg(P.dvec + row) : 0.0;
            const double* dcol = P.dvec + cbase;
#pragma unroll
            for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
                const int4 e4 = *reinterpret_cast<const int4*>(ex + c0);
                const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
                double cv[4], dv[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool live = c0 + j < nc;
                    cv[j] = live ? __ldg(cp + (c0 + j) * ldc) : 0.0;
                    dv[j] = per_row ? drow : (live ? __ldg(dcol + c0 + j) : 0.0);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (c0 + j < nc) cp[(c0 + j) * ldc] = fma(dv[j], cv[j], alpha * (acc[c0 + j] * oz_pow2(er + ev[j])));
            }
        } else if (beta == 1.0) {  // reductions in L2 (the trsm updates)
#pragma unroll
            for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
                const int4 e4 = *reinterpret_cast<const int4*>(ex + c0);
                const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (c0 + j < nc) atomicAdd(cp + (c0 + j) * ldc, alpha * (acc[c0 + j] * oz_pow2(er + ev[j])));
            }
        } else if (beta == 0.0) {
#pragma unroll
            for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
                const int4 e4 = *reinterpret_cast<const int4*>(ex + c0);
                const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (c0 + j < nc) cp[(c0 + j) * ldc] = alpha * (acc[c0 + j] * oz_pow2(er + ev[j]));
            }
        } else {
#pragma unroll
            for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
                const int4 e4 = *reinterpret_cast<const int4*>(ex + c0);
                const int ev[4] = {e4.x, e4.y, e4.z, e4.w};
                double cv[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) cv[j] = c0 + j < nc ? __ldg(cp + (c0 + j) * ldc) : 0.0;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (c0 + j < nc) cp[(c0 + j) * ldc] = fma(beta, cv[j], alpha * (acc[c0 + j] * oz_pow2(er + ev[j])));
            }
        }
        return;
    }
    // beta == 1: reductions in L2, as in the split kernel's epilogue; else
    // 4 columns at a time, loads first (the 64 fp64 accumulators leave
    // room for no more)
    if (P.dvec) {  // trmm: C = alpha acc + d C, d per row or per column
        const double drow = P.dvec_mode == 1 ? P.dvec[row] : 0.0;
#pragma unroll
        for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
            double cv[4];
            int ec[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const i64 col = cbase + c0 + j;
                ec[j] = ex[c0 + j];
                cv[j] = col < P.n ? P.c[row + col * P.ldc] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const i64 col = cbase + c0 + j;
                if (col >= P.n) continue;
                const double d = P.dvec_mode == 1 ? drow : P.dvec[col];
                P.c[row + col * P.ldc] = fma(d, cv[j], P.alpha * (acc[c0 + j] * pow2_exact(er + ec[j])));
            }
        }
    } else if (P.beta == 1.0) {
#pragma unroll
        for (int j = 0; j < C::EPI_COLS; ++j) {
            const i64 col = cbase + j;
            const bool live = col < P.n && !(P.tri == 1 && row < col) && !(P.tri == 2 && row > col);
            if (live) atomicAdd(P.c + row + col * P.ldc, P.alpha * (acc[j] * pow2_exact(er + ex[j])));
        }
    } else
#pragma unroll
    for (int c0 = 0; c0 < C::EPI_COLS; c0 += 4) {
        double cv[4];
        int ec[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const i64 col = cbase + c0 + j;
            const bool live = col < P.n && !(P.tri == 1 && row < col) && !(P.tri == 2 && row > col);
            ec[j] = ex[c0 + j];
            cv[j] = (live && P.beta != 0.0) ? P.c[row + col * P.ldc] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const i64 col = cbase + c0 + j;
            if (col >= P.n || (P.tri == 1 && row < col) || (P.tri == 2 && row > col)) continue;
            const double v = P.alpha * (acc[c0 + j] * pow2_exact(er + ec[j]));
            P.c[row + col * P.ldc] = (P.beta == 0.0) ? v : fma(P.beta, cv[j], v);
        }
    }
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, 1)
ozaki_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
             const __grid_constant__ CUtensorMap tmAlo, const __grid_constant__ CUtensorMap tmBlo, OzParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + C::STAGES;
    uint64_t* tfull = empty + C::STAGES;
    uint64_t* tempty = tfull + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 1);

    const int tile = blockIdx.x;
    const int group = 16;
    const int per_group = group * P.tiles_n;
    const int g = tile / per_group;
    const int first_m = g * group;
    const int gsize = min(group, P.tiles_m - first_m);
    const int in_g = tile - g * per_group;
    int tm = first_m + in_g % gsize, tn = in_g / gsize;
    // banded launches: heaviest tiles first (the last wave holds the short ones)
    if (P.band == KB_A_LOWER) tm = P.tiles_m - 1 - tm;
    if (P.band == KB_B_UPPER) tn = P.tiles_n - 1 - tn;
    const i64 m0 = i64(tm) * BM, n0 = i64(tn) * C::BN;
    if (P.tri == 1 && m0 + BM <= n0) return;        // tile strictly above the diagonal
    if (P.tri == 2 && m0 > n0 + C::BN - 1) return;  // tile strictly below the diagonal

    // slabs [kb0, kb0 + nkb) of the reduction: all of them, or the tile's band
    int kb0 = 0, nkb = P.num_kb;
    if (P.band != KB_NONE) {
        i64 s0, s1;
        band_slabs(P.band, m0, BM, n0, C::BN, P.band_k0, C::BKB, P.num_kb, s0, s1);
        kb0 = int(s0);
        nkb = int(s1 - s0);
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(tempty, C::EPI_WARPS);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int total = C::NPASS * nkb;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            for (int it = 0; it < total; ++it) {
                const int pass = it / nkb, kb = it - pass * nkb;
                int lo, hi, planes;
                pass_range<C>(pass, lo, hi, planes);
                const int s = it % C::STAGES;
                const uint32_t ph = (it / C::STAGES) & 1;
                if (!mbar_wait(&empty[s], ph ^ 1, P.err, 11)) break;
                uint8_t* sa = smem + s * C::STAGE_BYTES;
                uint8_t* sb = sa + C::S * C::PLANE;
                mbar_expect_tx(&full[s], uint32_t(2 * planes * C::PLANE));
                const bool all = planes == C::S;
                // 32-byte slab kb is half (kb % 2) of the layout's 64-byte slab kb / 2
                constexpr int HALVES = OZ_SLAB / 32;
                const int ks = kb0 + kb, x = (ks % HALVES) * 32, z = ks / HALVES;
                tma_load_4d(sa, all ? &tmA : &tmAlo, &full[s], x, int(m0), z, 0);
                tma_load_4d(sb, all ? &tmB : &tmBlo, &full[s], x, int(n0), z, 0);
            }
            for (int it = max(0, total - C::STAGES); it < total; ++it)
                mbar_wait(&full[it % C::STAGES], (it / C::STAGES) & 1, P.err, 12);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            if (oz_mma_pass<C, 0>(P, nkb, smem, full, empty, tfull, tempty, tmem) && C::NPASS > 1)
                oz_mma_pass<C, 1>(P, nkb, smem, full, empty, tfull, tempty, tmem);
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int e = warp - 2;
        const int quarter = warp & 3;
        const int part = e >> 2;
        const i64 row = m0 + quarter * 32 + lane;
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(part * C::EPI_COLS);
        int* ex = reinterpret_cast<int*>(smem + C::STAGES * C::STAGE_BYTES + 256) + e * C::EPI_COLS;
        const OzRowExp rx = oz_stage_exponents<C>(P, row, n0 + part * C::EPI_COLS, ex, lane);
        double acc[C::EPI_COLS];
#pragma unroll
        for (int j = 0; j < C::EPI_COLS; ++j) acc[j] = 0.0;
        bool ok = true;
        for (int pass = 0; pass < C::NPASS; ++pass) {
            int lo, hi, planes;
            pass_range<C>(pass, lo, hi, planes);
            if (!mbar_wait(tfull, pass & 1, P.err, 15)) { ok = false; break; }
            tc_fence_after();
#pragma unroll 1
            for (int d = hi - 1; d >= lo; --d) {  // smallest weight first
                const double w = pow2_exact(-8 * d - 12);
#pragma unroll
                for (int c0 = 0; c0 < C::EPI_COLS; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(lane_base + uint32_t((d - lo) * C::BN + c0), r);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[c0 + j] = fma(oz_i2d(r[j]), w, acc[c0 + j]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty);
        }
        if (ok && row < P.m) oz_store_row<C>(P, row, n0 + part * C::EPI_COLS, acc, ex, rx);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

// ---------------------------------------------------------------------------
// Ozaki kernel over a CTA pair: 256 x 128 tiles, tcgen05.mma.cta_group::2
// ---------------------------------------------------------------------------
// The single-CTA kernel above is bound by shared-memory bandwidth: every
// 128 x 128 x 32 int8 MMA (64 tensor-core cycles) reads a 4 KB B tile, and the
// TMA writes of the planes come on top, about 130 B/clk per SM against the 128
// the shared memory delivers.  Here two CTAs of a cluster (one per SM) share one
// 256 x 128 output tile: each stages its own 128 rows of op(A) and its own half
// (64 rows) of op(B)^T, and the leader CTA (rank 0) issues M = 256 MMAs that read
// A from each CTA's own shared memory and each half of B from the CTA holding it,
// so every B byte serves both SMs' tensor cores.  Per SM and k slab the planes
// written fall from 88 KB to 66 KB and the MMA operand reads from about 130 KB
// to 100 KB: about 93 B/clk at the full int8 rate.  Each CTA's TMEM holds the
// accumulators of its own 128 rows (the same four diagonals, two passes for
// more than four slices, as above).
//   both CTAs   warp 0 lane 0 loads this CTA's planes (plain TMA, no multicast);
//               the loads complete on the leader's mbarrier, which expects the
//               bytes of both CTAs; warp 0 allocates TMEM for the pair
//   leader      warp 1 lane 0 issues the MMAs; each stage's completion is
//               committed to the stage's "empty" barrier in both CTAs, each
//               pass's to the "accumulators ready" barrier in both CTAs
//   both CTAs   warps 2..9 drain their own TMEM and signal the leader's
//               "accumulators read" barrier (16 arrivals: 8 per CTA)
// All waits are bounded as in the other kernels; a cluster barrier before
// teardown keeps each CTA's barriers and TMEM alive until its peer is done.
template <int S_>
struct Oz2Cfg {
    static constexpr int S = S_;
    static constexpr int BN = 128;                    // output columns of the pair's tile
    static constexpr int BNH = BN / 2;                // op(B)^T rows staged by each CTA
    // k slab: 64 int8 per row (two 32-deep MMA steps), 64-byte swizzle; the planes are
    // stored slab-major (all rows' 64-byte pieces of a slab contiguous), so one TMA box is
    // a few contiguous kilobytes per plane, in 64-byte rows (with 32-byte rows the loads
    // were bound by the SM's L1-to-L2 request rate, not by bytes)
    static constexpr int BKB = OZ_SLAB;
    static constexpr int KSTEPS = BKB / 32;
    static constexpr int EPI_WARPS = 8;
    static constexpr int THREADS = 64 + 32 * EPI_WARPS;
    static constexpr int EPI_COLS = BN / (EPI_WARPS / 4);  // 64
    static constexpr int NPASS = S <= 4 ? 1 : 2;
    static constexpr int SPLIT = S <= 4 ? 0 : 4;
    static constexpr int A_PLANE = BM * BKB;          // 8 KB
    static constexpr int B_PLANE = BNH * BKB;         // 4 KB
    static constexpr int STAGE_BYTES = S * (A_PLANE + B_PLANE);
    static constexpr int STAGES = (196608 / STAGE_BYTES) > 8 ? 8 : (196608 / STAGE_BYTES);
    // at least 120 KB, so one CTA per SM: two pairs interleaved on the same two SMs could
    // each hold one SM's TMEM while waiting for the other's (the pair allocates together)
    static constexpr int EXP_BYTES = EPI_WARPS * EPI_COLS * 4;  // staged column exponents
    static constexpr int SMEM_USED = STAGES * STAGE_BYTES + 1024 + 256 + EXP_BYTES;
    static constexpr int SMEM_BYTES = SMEM_USED > 122880 ? SMEM_USED : 122880;
    static constexpr uint32_t IDESC = instr_desc(true, 2 * BM, BN);  // M = 256 over the pair
    static constexpr uint32_t SBO = 8 * BKB, LAYOUT = BKB == 64 ? 4 : 6;
    static_assert(STAGES >= 2, "pipeline depth");
    static_assert(A_PLANE % (8 * BKB) == 0 && B_PLANE % (8 * BKB) == 0, "swizzle atoms stay aligned");
};

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// shared::cluster address of the same variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t peer_addr(const void* p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_bar) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_bar) : "memory");
}
// TMA load into this CTA's shared memory whose completion is counted on an
// mbarrier of either CTA of the pair (the leader's); no multicast.
__device__ __forceinline__ void tma_load_4d_pair(void* dst, const CUtensorMap* map, uint32_t cluster_bar, int c0,
                                                 int c1, int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(cluster_bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void tmem_alloc_pair(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// Completion of the MMAs issued so far, arriving once on the barrier at this
// address in both CTAs of the pair.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"((unsigned short)3)
        : "memory");
}
#define MBG_UMMA2(COL)                                                                   \
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"                      \
                 "tcgen05.mma.cta_group::2.kind::i8" COL " [%0], %1, %2, %3, p;\n\t}"    \
                 ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)     \
                 : "memory")
__device__ __forceinline__ void umma_i8_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate, int collector) {
    if (collector == 1) MBG_UMMA2(".collector::a::fill");
    else if (collector == 2) MBG_UMMA2(".collector::a::use");
    else if (collector == 3) MBG_UMMA2(".collector::a::lastuse");
    else MBG_UMMA2("");
}
#undef MBG_UMMA2

// One pass of one tile: every k slab, the products of diagonals [LO, HI), then the
// accumulators committed to both CTAs' epilogues.  `it` counts stage uses across
// passes and tiles; `gp` is the pass's index across tiles (the epilogue must have
// read the previous pass's accumulators before this one overwrites them).
template <class C, int PASS>
__device__ __forceinline__ bool oz2_mma_pass(const OzParams& P, int nkb, int& it, int gp, uint8_t* smem,
                                             uint64_t* full, uint64_t* empty, uint64_t* tfull, uint64_t* tempty,
                                             uint32_t tmem) {
    constexpr int LO = OzPass<C::S, PASS>::LO, HI = OzPass<C::S, PASS>::HI;
    if (gp > 0) {
        if (!mbar_wait(tempty, (gp - 1) & 1, P.err, 23)) return false;
        tc_fence_after();
    }
    for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int s = it % C::STAGES;
        if (!mbar_wait(&full[s], (it / C::STAGES) & 1, P.err, 24)) return false;
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
        const uint32_t sb = sa + C::S * C::A_PLANE;
#pragma unroll
        for (int ks = 0; ks < C::KSTEPS; ++ks) {
#pragma unroll
            for (int pi = 0; pi < C::S * C::S; ++pi) {
                int p = 0, q = 0, collector = 0;
                if (!oz_product<C::S>(LO, HI, pi, p, q, collector)) break;
                const uint32_t accumulate = (kb > 0 || ks > 0 || p > 0) ? 1u : 0u;
                const uint64_t ad = smem_desc(sa + p * C::A_PLANE + ks * 32, C::SBO, C::LAYOUT);
                const uint64_t bd = smem_desc(sb + q * C::B_PLANE + ks * 32, C::SBO, C::LAYOUT);
                umma_i8_pair(tmem + uint32_t((p + q - LO) * C::BN), ad, bd, C::IDESC, accumulate, collector);
            }
        }
        umma_commit_pair(&empty[s]);  // stage s is free in both CTAs once these MMAs have read it
    }
    umma_commit_pair(tfull);  // this pass's accumulators are complete in both CTAs
    return true;
}

// Pair tile t of a launch: its rows (pm0), columns (n0) and slabs; false when the
// triangle mask skips it.  Every role of both CTAs evaluates the same tiles.
struct OzTile {
    i64 pm0, n0;
    int kb0, nkb;
};
template <class C>
__device__ __forceinline__ bool oz2_tile(const OzParams& P, int t, OzTile& T) {
    // pair tiles of 256 x 128, groups of 8 pair rows walk the n-tiles together (L2 reuse)
    const int tiles_m2 = (P.tiles_m + 1) >> 1;
    const int group = 8;
    const int per_group = group * P.tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gsize = min(group, tiles_m2 - first_m);
    const int in_g = t - g * per_group;
    int tm = first_m + in_g % gsize, tn = in_g / gsize;
    if (P.band == KB_A_LOWER) tm = tiles_m2 - 1 - tm;
    if (P.band == KB_B_UPPER) tn = P.tiles_n - 1 - tn;
    T.pm0 = i64(tm) * 2 * BM;
    T.n0 = i64(tn) * C::BN;
    if (P.tri == 1 && T.pm0 + 2 * BM <= T.n0) return false;
    if (P.tri == 2 && T.pm0 > T.n0 + C::BN - 1) return false;
    T.kb0 = 0;
    T.nkb = P.num_kb;
    if (P.band != KB_NONE) {
        i64 s0, s1;
        band_slabs(P.band, T.pm0, 2 * BM, T.n0, C::BN, P.band_k0, C::BKB, P.num_kb, s0, s1);
        T.kb0 = int(s0);
        T.nkb = int(s1 - s0);
    }
    return true;
}

// Persistent over pair tiles: cluster c takes tiles c, c + clusters, ... (a launch
// with one cluster per tile is the plain form).  Between two tiles the epilogue
// stores the finished tile from registers while the next tile's first pass is
// already loading and multiplying: it only has to read the accumulators out first.
template <class C>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(C::THREADS, 1)
ozaki_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                  const __grid_constant__ CUtensorMap tmAlo, const __grid_constant__ CUtensorMap tmBlo, OzParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + C::STAGES;
    uint64_t* tfull = empty + C::STAGES;
    uint64_t* tempty = tfull + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 1);

    const uint32_t rank = cluster_rank();  // 0: leader (issues the MMAs), 1: peer
    const int ntiles = ((P.tiles_m + 1) >> 1) * P.tiles_n;
    const int first = blockIdx.x >> 1, stride = gridDim.x >> 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(tempty, 2 * C::EPI_WARPS);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc_pair(tmem_slot, 512);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync_all();  // barriers of both CTAs initialised, TMEM of the pair allocated
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t leader_tempty = peer_addr(tempty, 0);

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs) ----------------
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            bool ok = true;
            int it = 0;
            for (int t = first; t < ntiles && ok; t += stride) {
                OzTile T;
                if (!oz2_tile<C>(P, t, T)) continue;
                const i64 m0 = T.pm0 + i64(rank) * BM;
                for (int pass = 0; pass < C::NPASS && ok; ++pass) {
                    int lo, hi, planes;
                    pass_range<C>(pass, lo, hi, planes);
                    const bool all = planes == C::S;
                    for (int kb = 0; kb < T.nkb; ++kb, ++it) {
                        const int s = it % C::STAGES;
                        if (!mbar_wait(&empty[s], ((it / C::STAGES) & 1) ^ 1, P.err, 21)) { ok = false; break; }
                        uint8_t* sa = smem + s * C::STAGE_BYTES;
                        uint8_t* sb = sa + C::S * C::A_PLANE;
                        if (rank == 0) mbar_expect_tx(&full[s], uint32_t(2 * planes * (C::A_PLANE + C::B_PLANE)));
                        const uint32_t bar = peer_addr(&full[s], 0);
                        tma_load_4d_pair(sa, all ? &tmA : &tmAlo, bar, 0, int(m0), T.kb0 + kb, 0);
                        tma_load_4d_pair(sb, all ? &tmB : &tmBlo, bar, 0, int(T.n0 + rank * C::BNH), T.kb0 + kb,
                                         0);
                    }
                }
            }
            // the loads of the last stages land before the CTA may exit: the leader's MMAs
            // release every stage to both CTAs only after reading it
            if (ok)
                for (int i = max(0, it - C::STAGES); i < it; ++i)
                    mbar_wait(&empty[i % C::STAGES], (i / C::STAGES) & 1, P.err, 22);
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            // ---------------- MMA issuer (leader) ----------------
            int it = 0, gp = 0;
            bool ok = true;
            for (int t = first; t < ntiles && ok; t += stride) {
                OzTile T;
                if (!oz2_tile<C>(P, t, T)) continue;
                ok = oz2_mma_pass<C, 0>(P, T.nkb, it, gp++, smem, full, empty, tfull, tempty, tmem);
                if (ok && C::NPASS > 1)
                    ok = oz2_mma_pass<C, 1>(P, T.nkb, it, gp++, smem, full, empty, tfull, tempty, tmem);
            }
        }
    } else {
        // ---------------- epilogue warps (both CTAs, own rows) ----------------
        const int e = warp - 2;
        const int quarter = warp & 3;
        const int part = e >> 2;
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(part * C::EPI_COLS);
        int* ex = reinterpret_cast<int*>(smem + C::STAGES * C::STAGE_BYTES + 256) + e * C::EPI_COLS;
        int gp = 0;
        bool ok = true;
        for (int t = first; t < ntiles && ok; t += stride) {
            OzTile T;
            if (!oz2_tile<C>(P, t, T)) continue;
            const i64 row = T.pm0 + i64(rank) * BM + quarter * 32 + lane;
            const OzRowExp rx = oz_stage_exponents<C>(P, row, T.n0 + part * C::EPI_COLS, ex, lane);
            double acc[C::EPI_COLS];
#pragma unroll
            for (int j = 0; j < C::EPI_COLS; ++j) acc[j] = 0.0;
            for (int pass = 0; pass < C::NPASS; ++pass, ++gp) {
                int lo, hi, planes;
                pass_range<C>(pass, lo, hi, planes);
                if (!mbar_wait(tfull, gp & 1, P.err, 25)) { ok = false; break; }
                tc_fence_after();
#pragma unroll 1
                for (int d = hi - 1; d >= lo; --d) {  // smallest weight first
                    const double w = pow2_exact(-8 * d - 12);
#pragma unroll
                    for (int c0 = 0; c0 < C::EPI_COLS; c0 += 16) {
                        uint32_t r[16];
                        tmem_ld16(lane_base + uint32_t((d - lo) * C::BN + c0), r);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 16; ++j) acc[c0 + j] = fma(oz_i2d(r[j]), w, acc[c0 + j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_remote(leader_tempty);
            }
            if (ok && row < P.m) oz_store_row<C>(P, row, T.n0 + part * C::EPI_COLS, acc, ex, rx);
        }
    }
    tc_fence_before();
    __syncwarp();
    cluster_sync_all();  // the peer's epilogue and loads are done; no more remote barrier traffic
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc_pair(tmem, 512);
    }
}

// Work of one persistent split launch (split_sk_kernel): one or two products (the second:
// the gemm adjoint's other gradient).  Tiles are numbered product 0's first, then product 1's.
//   whole tiles:  the first dp_tiles tiles, worker (CTA) c taking tiles c, c + G, ...
//                 (G workers); the triangle mask may skip tiles; C is stored
//                 with beta.
//   stream-K:     the slabs of the remaining tiles, [sk_begin, total) in slab positions
//                 over all tiles, cut into G equal contiguous ranges, one per worker, so
//                 the last wave leaves no SM idle.  A range runs on across tile boundaries
//                 without draining the pipeline.  Whole tiles are stored; a tile two ranges
//                 share is zeroed first (sk_zero_kernel) and both add their partial sums
//                 (beta = 0 only).  Every range is at least one tile long, so no tile gets
//                 more than two partial sums, and their fp32 sum does not depend on the
//                 order they arrive in.
struct SkWork {
    int tiles0, tiles1;   // tiles of each product (tiles1 = 0: one product)
    int nkb0, nkb1;       // k slabs of each product's tiles
    int dp_tiles;         // leading tiles taken whole
    i64 sk_begin, total;  // stream-K slab positions (sk_begin == total: none)
};
struct SkSeg {
    int prod, tile, kb0, kb1;  // slabs [kb0, kb1) of tile `tile` of product `prod`
    i64 m0, n0;                // the tile's first row and column
};
struct SkCursor {
    int u, u_end, step;  // whole tiles: next tile, end, stride
    i64 pos, end;        // stream-K: the worker's slab range
};

// Tile t of P (C::TILE_M x C::TILE_N; P.tiles_m counts 128-row tiles, P.tiles_n
// TILE_N-column tiles): groups of TILE_GROUP tile rows walk the n-tiles together (L2 reuse).
template <class C>
__device__ __forceinline__ void sk_tile_origin(const Params& P, int t, i64& m0, i64& n0) {
    constexpr int R = C::TILE_M / BM;
    const int tiles_m = (P.tiles_m + R - 1) / R;
    const int per_group = C::TILE_GROUP * P.tiles_n;
    const int g = t / per_group;
    const int first_m = g * C::TILE_GROUP;
    const int gsize = min(C::TILE_GROUP, tiles_m - first_m);
    const int in_g = t - g * per_group;
    m0 = i64(first_m + in_g % gsize) * C::TILE_M;
    n0 = i64(in_g / gsize) * C::TILE_N;
}

// Stream-K slab position -> the tile holding it and the slab within it.
__device__ __forceinline__ void sk_locate(const SkWork& W, i64 pos, int& prod, int& tile, int& kb, i64& base,
                                          int& nkb) {
    const i64 w0 = i64(W.tiles0) * W.nkb0;
    prod = pos >= w0 ? 1 : 0;
    base = prod ? w0 : 0;
    nkb = prod ? W.nkb1 : W.nkb0;
    const i64 rel = pos - base;
    tile = int(rel / nkb);
    kb = int(rel - i64(tile) * nkb);
}

__device__ __forceinline__ SkCursor sk_cursor(const SkWork& W, i64 worker, i64 workers) {
    const i64 n = W.total - W.sk_begin;
    SkCursor c;
    c.u = int(worker);
    c.u_end = W.dp_tiles;
    c.step = int(workers);
    c.pos = W.sk_begin + worker * n / workers;
    c.end = W.sk_begin + (worker + 1) * n / workers;
    return c;
}

// The worker's next segment; every role of the worker's CTAs walks the same sequence.
template <class C>
__device__ __forceinline__ bool sk_next(const SkWork& W, const Params& P0, const Params& P1, SkCursor& cur,
                                        SkSeg& sg) {
    while (cur.u < cur.u_end) {
        const int u = cur.u;
        cur.u += cur.step;
        sg.prod = u >= W.tiles0 ? 1 : 0;
        const Params& P = sg.prod ? P1 : P0;
        sg.tile = sg.prod ? u - W.tiles0 : u;
        sk_tile_origin<C>(P, sg.tile, sg.m0, sg.n0);
        if (P.tri == 1 && sg.m0 + C::TILE_M <= sg.n0) continue;  // strictly above the diagonal
        if (P.tri == 2 && sg.m0 > sg.n0 + C::TILE_N - 1) continue;  // strictly below the diagonal
        sg.kb0 = 0;
        sg.kb1 = sg.prod ? W.nkb1 : W.nkb0;
        return true;
    }
    if (cur.pos >= cur.end) return false;
    i64 base;
    int nkb;
    sk_locate(W, cur.pos, sg.prod, sg.tile, sg.kb0, base, nkb);
    const i64 stop = min(cur.end, base + i64(sg.tile + 1) * nkb);
    sg.kb1 = sg.kb0 + int(stop - cur.pos);
    cur.pos = stop;
    sk_tile_origin<C>(sg.prod ? P1 : P0, sg.tile, sg.m0, sg.n0);
    return true;
}

// Zeroes the tiles two stream-K ranges share, ahead of their partial sums: block b takes
// the boundary between ranges b and b + 1 (a boundary inside a tile; ranges are at least
// a tile long, so each such tile holds one boundary).
template <class C>
__global__ void __launch_bounds__(256) sk_zero_kernel(Params P0, Params P1, SkWork W, int workers) {
    const i64 n = W.total - W.sk_begin;
    const i64 pos = W.sk_begin + (i64(blockIdx.x) + 1) * n / workers;
    int prod, tile, kb, nkb;
    i64 base;
    sk_locate(W, pos, prod, tile, kb, base, nkb);
    if (kb == 0) return;  // the boundary is a tile's start: nothing shared
    const Params& P = prod ? P1 : P0;
    i64 m0, n0;
    sk_tile_origin<C>(P, tile, m0, n0);
    float* Cm = static_cast<float*>(P.c);
    for (int j = threadIdx.x; j < C::TILE_M * C::TILE_N; j += blockDim.x) {
        const i64 r = m0 + (j % C::TILE_M), col = n0 + j / C::TILE_M;
        if (r < P.m && col < P.n) Cm[r + col * P.ldc] = 0.0f;
    }
}

// A partial tile's row: C += alpha acc (one reduction in L2 per element).
template <class C>
__device__ __forceinline__ void split_add_row(const Params& P, const i64 row, const i64 cbase,
                                              const float (&acc)[C::EPI_COLS]) {
    float* Cm = static_cast<float*>(P.c);
    const float alpha = float(P.alpha);
#pragma unroll
    for (int j = 0; j < C::EPI_COLS; ++j) {
        const i64 col = cbase + j;
        if (col < P.n) atomicAdd(Cm + row + col * P.ldc, alpha * acc[j]);
    }
}

// The split product on single CTAs, persistent over the CTA's segments (SkWork): the
// 128 x 256 tile of tc_gemm_tile, whose operand bytes per flop suit the shared memory
// best, with the stream-K schedule in place of a partly empty last wave.  Stage, chunk
// and buffer counters run on across segments, so the producer loads the next segment's
// slabs while the MMAs finish this one, and the epilogue stores a finished segment while
// the next one's first chunk accumulates in the other TMEM buffer.
template <class C>
__global__ void __launch_bounds__(C::THREADS, 1)
split_sk_kernel(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmB0,
                const __grid_constant__ Params P0, const __grid_constant__ CUtensorMap tmA1,
                const __grid_constant__ CUtensorMap tmB1, const __grid_constant__ Params P1, SkWork W) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t* empty = full + C::STAGES;
    uint64_t* tfull = empty + C::STAGES;  // [2]: accumulator buffer ready for the epilogue
    uint64_t* tempty = tfull + 2;         // [2]: epilogue finished reading a buffer
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    int* const err = P0.err;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], C::EPI_WARPS);
        }
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, C::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            prefetch_tmap(&tmA0);
            prefetch_tmap(&tmB0);
            if (W.tiles1) {
                prefetch_tmap(&tmA1);
                prefetch_tmap(&tmB1);
            }
            SkCursor cur = sk_cursor(W, blockIdx.x, gridDim.x);
            SkSeg sg;
            bool ok = true;
            int it = 0;
            while (ok && sk_next<C>(W, P0, P1, cur, sg)) {
                const CUtensorMap* ma = sg.prod ? &tmA1 : &tmA0;
                const CUtensorMap* mb = sg.prod ? &tmB1 : &tmB0;
                for (int kb = sg.kb0; kb < sg.kb1; ++kb, ++it) {
                    const int s = it % C::STAGES;
                    if (!mbar_wait(&empty[s], ((it / C::STAGES) & 1) ^ 1, err, 51)) { ok = false; break; }
                    uint8_t* sa = smem + s * C::STAGE_BYTES;
                    uint8_t* sb = sa + C::TERMS * C::A_PLANE;
                    mbar_expect_tx(&full[s], C::STAGE_BYTES);
                    tma_load_3d(sa, ma, &full[s], kb * C::BK, int(sg.m0), 0);
                    tma_load_3d(sb, mb, &full[s], kb * C::BK, int(sg.n0), 0);
                }
            }
            // all issued loads land before the CTA may exit: the MMAs release every stage
            // only after reading it
            if (ok)
                for (int i = max(0, it - C::STAGES); i < it; ++i)
                    mbar_wait(&empty[i % C::STAGES], (i / C::STAGES) & 1, err, 52);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            SkCursor cur = sk_cursor(W, blockIdx.x, gridDim.x);
            SkSeg sg;
            bool ok = true;
            int it = 0, chunk = 0;
            while (ok && sk_next<C>(W, P0, P1, cur, sg)) {
                for (int kb = sg.kb0; kb < sg.kb1; ++kb, ++it) {
                    const int kin = (kb - sg.kb0) % C::CHUNK;  // slab index within the chunk
                    const int buf = chunk & 1;
                    if (kin == 0 && chunk >= 2) {
                        // the epilogue must have drained this buffer's previous chunk
                        if (!mbar_wait(&tempty[buf], ((chunk >> 1) - 1) & 1, err, 55)) { ok = false; break; }
                        tc_fence_after();
                    }
                    const int s = it % C::STAGES;
                    if (!mbar_wait(&full[s], (it / C::STAGES) & 1, err, 53)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
                    const uint32_t sb = sa + C::TERMS * C::A_PLANE;
#pragma unroll
                    for (int ks = 0; ks < C::KSTEPS; ++ks) {
#pragma unroll
                        for (int pi = 0; pi < C::NPROD; ++pi) {
                            int p, q, collector;
                            product<C::TERMS, false>(pi, p, q, collector);
                            // the first product of a chunk overwrites the buffer
                            const uint32_t accumulate = (kin > 0 || ks > 0 || pi > 0) ? 1u : 0u;
                            const uint64_t ad = smem_desc(sa + p * C::A_PLANE + ks * 32, C::SBO, C::LAYOUT);
                            const uint64_t bd = smem_desc(sb + q * C::B_PLANE + ks * 32, C::SBO, C::LAYOUT);
                            umma<false>(tmem + uint32_t(buf * C::BN), ad, bd, C::IDESC, accumulate);
                        }
                    }
                    umma_commit(&empty[s]);  // slot s is free once these MMAs have read it
                    if (kin == C::CHUNK - 1 || kb == sg.kb1 - 1) {
                        umma_commit(&tfull[buf]);  // chunk complete
                        ++chunk;
                    }
                }
            }
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int e = warp - 2;
        const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
        const int part = e >> 2;       // which EPI_COLS-wide column range
        const uint32_t lane_base = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(part * C::EPI_COLS);
        SkCursor cur = sk_cursor(W, blockIdx.x, gridDim.x);
        SkSeg sg;
        bool ok = true;
        int chunk = 0;
        while (ok && sk_next<C>(W, P0, P1, cur, sg)) {
            const Params& P = sg.prod ? P1 : P0;
            const int nchunks = (sg.kb1 - sg.kb0 + C::CHUNK - 1) / C::CHUNK;
            float acc[C::EPI_COLS];
#pragma unroll
            for (int j = 0; j < C::EPI_COLS; ++j) acc[j] = 0.0f;
            for (int ch = 0; ch < nchunks; ++ch, ++chunk) {
                const int buf = chunk & 1;
                if (!mbar_wait(&tfull[buf], (chunk >> 1) & 1, err, 54)) { ok = false; break; }
                tc_fence_after();
#pragma unroll
                for (int c0 = 0; c0 < C::EPI_COLS; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(lane_base + uint32_t(buf * C::BN + c0), r);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[c0 + j] += __uint_as_float(r[j]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            const i64 row = sg.m0 + quarter * 32 + lane;
            if (!ok || row >= P.m) continue;
            const i64 cbase = sg.n0 + part * C::EPI_COLS;
            if (sg.kb0 == 0 && sg.kb1 == (sg.prod ? W.nkb1 : W.nkb0)) split_store_row<C>(P, row, cbase, acc);
            else split_add_row<C>(P, row, cbase, acc);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, C::TMEM_COLS);
    }
}


// ---------------------------------------------------------------------------
// Pre-pass kernels
// ---------------------------------------------------------------------------
constexpr int PT_R = 64, PT_K = 32;  // pre-pass tile: 64 rows x 32 k

// value(r, l) of the logical rows x K operand: K-major source src[l + r*ld],
// otherwise src[r + l*ld]; outside rows x K it is zero (padding).  keep (a
// triangular operand read from the user's matrix): 0 every element, 1 only
// l < r, 2 only l > r; the rest (the other triangle and the diagonal) is zero
// and never read.
__device__ __forceinline__ bool kept(int keep, i64 r, i64 l) {
    return keep == 0 || (keep == 1 ? l < r : l > r);
}

template <typename T, bool KMAJOR>
__device__ __forceinline__ void load_tile(const T* __restrict__ src, i64 ld, i64 rows, i64 K, i64 r0,
                                          i64 l0, int keep, T (&tile)[PT_R][PT_K + 1]) {
    for (int e = threadIdx.x; e < PT_R * PT_K; e += blockDim.x) {
        int rr, ll;
        if (KMAJOR) { rr = e / PT_K; ll = e % PT_K; } else { rr = e % PT_R; ll = e / PT_R; }
        const i64 r = r0 + rr, l = l0 + ll;
        T v = T(0);
        if (r < rows && l < K && kept(keep, r, l)) v = KMAJOR ? src[l + r * ld] : src[r + l * ld];
        tile[rr][ll] = v;
    }
}

// Split pre-pass: planes[t][r][l] = term t of value(r, l), TERMS bf16 terms per fp32 value
// (a1 = bf16(v), a2 = bf16(v - a1), a3 = bf16(v - a1 - a2); each subtraction is exact),
// zeros outside rows x K up to Rp x Kp.  One 256-thread CTA per 64 x 64 tile; each thread
// turns four consecutive k of one row into one 8-byte store per plane.  A k-contiguous
// source is read four values at a time (16-byte loads when aligned); a row-contiguous one
// is read four rows at a time along m and transposed through shared memory.
constexpr int SP_R = 64, SP_K = 64;

inline dim3 split_grid(i64 Rp, i64 Kp) { return dim3(unsigned((Kp + SP_K - 1) / SP_K), unsigned(Rp / SP_R)); }

template <int TERMS>
__device__ __forceinline__ void split_store4(float4 v, __nv_bfloat16* out, size_t plane) {
    float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int t = 0; t < TERMS; ++t) {
        __nv_bfloat16 h[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            h[u] = __float2bfloat16_rn(x[u]);
            x[u] -= __bfloat162float(h[u]);  // exact: x and h agree in their leading bits
        }
        const __nv_bfloat162 lo = __halves2bfloat162(h[0], h[1]), hi = __halves2bfloat162(h[2], h[3]);
        uint2 w;
        w.x = *reinterpret_cast<const unsigned*>(&lo);
        w.y = *reinterpret_cast<const unsigned*>(&hi);
        *reinterpret_cast<uint2*>(out + plane * t) = w;
    }
}

template <int TERMS, bool KMAJOR>
__global__ void __launch_bounds__(256)
split_bf16_kernel(const float* __restrict__ src, i64 ld, i64 rows, i64 K, i64 Rp, i64 Kp,
                  __nv_bfloat16* __restrict__ planes, int keep = 0) {
    const i64 r0 = i64(blockIdx.y) * SP_R, l0 = i64(blockIdx.x) * SP_K;
    const size_t plane = size_t(Rp) * size_t(Kp);
    const bool vec = reinterpret_cast<uintptr_t>(src) % 16 == 0 && ld % 4 == 0 && keep == 0;
    if (KMAJOR) {  // value(r, l) = src[l + r * ld]
        for (int q = threadIdx.x; q < SP_R * (SP_K / 4); q += 256) {
            const int rr = q / (SP_K / 4), lq = (q % (SP_K / 4)) * 4;
            const i64 r = r0 + rr, l = l0 + lq;
            if (l >= Kp) continue;
            float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (r < rows) {
                if (vec && l + 3 < K) {
                    const float4 v = *reinterpret_cast<const float4*>(src + l + r * ld);
                    t[0] = v.x; t[1] = v.y; t[2] = v.z; t[3] = v.w;
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (l + u < K && kept(keep, r, l + u)) t[u] = src[l + u + r * ld];
                }
            }
            split_store4<TERMS>(make_float4(t[0], t[1], t[2], t[3]), planes + size_t(r) * Kp + l, plane);
        }
    } else {  // value(r, l) = src[r + l * ld]
        __shared__ float tile[SP_K][SP_R + 1];
        for (int q = threadIdx.x; q < SP_K * (SP_R / 4); q += 256) {
            const int lk = q / (SP_R / 4), rq = (q % (SP_R / 4)) * 4;
            const i64 r = r0 + rq, l = l0 + lk;
            float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (l < K) {
                if (vec && r + 3 < rows) {
                    const float4 v = *reinterpret_cast<const float4*>(src + r + l * ld);
                    t[0] = v.x; t[1] = v.y; t[2] = v.z; t[3] = v.w;
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (r + u < rows && kept(keep, r + u, l)) t[u] = src[r + u + l * ld];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) tile[lk][rq + u] = t[u];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < SP_R * (SP_K / 4); q += 256) {
            const int rr = q / (SP_K / 4), lq = (q % (SP_K / 4)) * 4;
            const i64 l = l0 + lq;
            if (l >= Kp) continue;
            const float4 v = make_float4(tile[lq][rr], tile[lq + 1][rr], tile[lq + 2][rr], tile[lq + 3][rr]);
            split_store4<TERMS>(v, planes + size_t(r0 + rr) * Kp + l, plane);
        }
    }
}

// Both plane layouts of one column-major matrix G (gm x gn) from one read of it: planes R
// with G's rows as plane rows (value(r, l) = G[r + l * ld], RpR x KpR) and planes C with its
// columns as plane rows (value(r, l) = G[l + r * ld], RpC x KpC): what split_bf16_kernel
// writes for the two orientations, bit for bit (the gemm adjoint splits G once for dA = G
// op(B)^T and once for dB = op(A)^T G).  One 64 x 64 tile of G per block, staged in shared
// memory; padding rows and columns are written as zeros.
template <int TERMS>
__global__ void __launch_bounds__(256)
split_bf16_both_kernel(const float* __restrict__ src, i64 ld, i64 gm, i64 gn, __nv_bfloat16* __restrict__ pr,
                       i64 RpR, i64 KpR, __nv_bfloat16* __restrict__ pc, i64 RpC, i64 KpC) {
    const i64 i0 = i64(blockIdx.y) * SP_R, j0 = i64(blockIdx.x) * SP_K;  // rows i of G, columns j
    const bool vec = reinterpret_cast<uintptr_t>(src) % 16 == 0 && ld % 4 == 0;
    __shared__ float tile[SP_K][SP_R + 1];  // tile[j][i]
    for (int q = threadIdx.x; q < SP_K * (SP_R / 4); q += 256) {
        const int jj = q / (SP_R / 4), iq = (q % (SP_R / 4)) * 4;
        const i64 i = i0 + iq, j = j0 + jj;
        float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (j < gn) {
            if (vec && i + 3 < gm) {
                const float4 v = *reinterpret_cast<const float4*>(src + i + j * ld);
                t[0] = v.x; t[1] = v.y; t[2] = v.z; t[3] = v.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (i + u < gm) t[u] = src[i + u + j * ld];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) tile[jj][iq + u] = t[u];
    }
    __syncthreads();
    const size_t plane_r = size_t(RpR) * size_t(KpR), plane_c = size_t(RpC) * size_t(KpC);
    for (int q = threadIdx.x; q < SP_R * (SP_K / 4); q += 256) {
        // planes R: row i, k = j .. j + 3
        const int ii = q / (SP_K / 4), jq = (q % (SP_K / 4)) * 4;
        const i64 i = i0 + ii, j = j0 + jq;
        if (i < RpR && j < KpR) {
            const float4 v = make_float4(tile[jq][ii], tile[jq + 1][ii], tile[jq + 2][ii], tile[jq + 3][ii]);
            split_store4<TERMS>(v, pr + size_t(i) * KpR + j, plane_r);
        }
        // planes C: row j, k = i .. i + 3
        const int jc = q / (SP_R / 4), iq = (q % (SP_R / 4)) * 4;
        const i64 jr = j0 + jc, ik = i0 + iq;
        if (jr < RpC && ik < KpC) {
            const float4 v = make_float4(tile[jc][iq], tile[jc][iq + 1], tile[jc][iq + 2], tile[jc][iq + 3]);
            split_store4<TERMS>(v, pc + size_t(jr) * KpC + ik, plane_c);
        }
    }
}

// Row exponents for the Ozaki scaling: e(r) with max_l |value(r,l)| < 2^e(r).
// Partial maxima over k chunks are combined with atomicMax on the exponent
// (initialised by the host to 0x80808080, below any double exponent); an
// all-zero row keeps that value, which the slicing kernel maps to 0.
constexpr int OZ_EXP_KCHUNK = 64;    // k columns per CTA row block, rows contiguous in memory
constexpr int OZ_EXP_KWARP = 1024;   // k per warp, k contiguous in memory

__device__ __forceinline__ void oz_exponent_max(int* e, i64 r, double mx) {
    if (mx > 0.0) {
        int ex;
        frexp(mx, &ex);
        atomicMax(e + r, ex);
    }
}

template <bool KMAJOR>
__global__ void __launch_bounds__(256)
row_exponent_kernel(const double* __restrict__ src, i64 ld, i64 rows, i64 K, int* __restrict__ e, int keep) {
    if (KMAJOR) {  // warp per row and k chunk, lanes along k (coalesced)
        const i64 r = i64(blockIdx.x) * 8 + (threadIdx.x >> 5);
        if (r >= rows) return;
        i64 l0 = i64(blockIdx.y) * OZ_EXP_KWARP, l1 = min(K, l0 + OZ_EXP_KWARP);
        if (keep == 1) l1 = min(l1, r);       // only l < r
        if (keep == 2) l0 = max(l0, r + 1);   // only l > r
        const double* row = src + r * ld;
        double mx = 0.0;
#pragma unroll 8
        for (i64 l = l0 + (threadIdx.x & 31); l < l1; l += 32) mx = fmax(mx, fabs(row[l]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) oz_exponent_max(e, r, mx);
    } else {  // 32 rows (lanes, coalesced) x 8 k lanes per CTA, OZ_EXP_KCHUNK columns per CTA
        __shared__ double part[8][33];
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
        const i64 r = i64(blockIdx.x) * 32 + tx;
        const i64 l0 = i64(blockIdx.y) * OZ_EXP_KCHUNK;
        double mx = 0.0;
        if (r < rows) {
#pragma unroll
            for (int j = 0; j < OZ_EXP_KCHUNK / 8; ++j) {
                const i64 l = l0 + ty + 8 * j;
                if (l < K && kept(keep, r, l)) mx = fmax(mx, fabs(src[r + l * ld]));
            }
        }
        part[ty][tx] = mx;
        __syncthreads();
        if (ty == 0 && r < rows) {
#pragma unroll
            for (int y = 1; y < 8; ++y) mx = fmax(mx, part[y][tx]);
            oz_exponent_max(e, r, mx);
        }
    }
}

// trunc(v / 2^er * 2^B) from the bits of v, with v's sign: |v| = M 2^(max(E,1) - 1075)
// with the 53-bit significand M; |v| < 2^er and B <= 62 keep the magnitude below 2^B.
// Integer shifts keep the FP64 pipe free.
__device__ __forceinline__ long long oz_fixed(double v, int er, int B) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
    const int E = int((b >> 52) & 0x7ff);
    const unsigned long long M = (b & 0xfffffffffffffULL) | (E ? (1ULL << 52) : 0ULL);
    const int sh = (E ? E : 1) - 1075 - er + B;
    unsigned long long F;
    if (sh >= 0) F = sh < 64 ? M << sh : 0ULL;
    else F = sh > -64 ? M >> -sh : 0ULL;
    return (b >> 63) ? -static_cast<long long>(F) : static_cast<long long>(F);
}

// oz_fixed(v, er, B) for a row whose scale 2^(B - er) is a normal double: one product
// (exact: a power-of-two scaling of a value below 2^er stays below 2^B, and a product
// small enough to round is below 1, whose truncation is 0 either way) and one truncating
// conversion, instead of the integer shifts.
__device__ __forceinline__ bool oz_scale_ok(int er, int B) { return B - er >= -1022 && B - er <= 1023; }
__device__ __forceinline__ long long oz_fixed_scaled(double v, double scale) { return __double2ll_rz(v * scale); }

// 4 x 4 byte transpose: o[b] holds byte b of w0, w1, w2, w3 in its bytes 0, 1, 2, 3
// (eight byte permutes instead of a shift, mask and merge per byte).
__device__ __forceinline__ void byte_transpose4(unsigned w0, unsigned w1, unsigned w2, unsigned w3, unsigned* o) {
    const unsigned t0 = __byte_perm(w0, w1, 0x5140), t1 = __byte_perm(w0, w1, 0x7362);  // w0.b0 w1.b0 w0.b1 w1.b1
    const unsigned t2 = __byte_perm(w2, w3, 0x5140), t3 = __byte_perm(w2, w3, 0x7362);  // (t1, t3: bytes 2, 3)
    o[0] = __byte_perm(t0, t2, 0x5410);
    o[1] = __byte_perm(t0, t2, 0x7632);
    o[2] = __byte_perm(t1, t3, 0x5410);
    o[3] = __byte_perm(t1, t3, 0x7632);
}

// Ozaki planes are stored slab-major: plane p holds, for each OZ_SLAB-deep k slab in turn,
// the OZ_SLAB-byte pieces of all Rp rows back to back, so element (r, l) of a plane sits at
//     (l / OZ_SLAB) (Rp OZ_SLAB) + r OZ_SLAB + l % OZ_SLAB.
// One TMA box (a slab of k, a block of rows, every plane) is then a contiguous run per plane.
// Kp (the padded k) is a multiple of OZ_SLAB.
__host__ __device__ __forceinline__ size_t oz_plane_offset(i64 Rp, i64 r, i64 l) {
    return size_t(l) / OZ_SLAB * size_t(Rp) * OZ_SLAB + size_t(r) * OZ_SLAB + size_t(l) % OZ_SLAB;
}

template <bool KMAJOR>
__global__ void __launch_bounds__(256)
slice_i8_kernel(const double* __restrict__ src, i64 ld, i64 rows, i64 K, i64 Rp, i64 Kp, int slices,
                int* __restrict__ e, int8_t* __restrict__ planes, int keep) {
    __shared__ double tile[PT_R][PT_K + 1];
    const i64 r0 = i64(blockIdx.y) * PT_R, l0 = i64(blockIdx.x) * PT_K;
    load_tile<double, KMAJOR>(src, ld, rows, K, r0, l0, keep, tile);
    __syncthreads();
    const size_t plane = size_t(Rp) * size_t(Kp);
    for (int q = threadIdx.x; q < PT_R * (PT_K / 4); q += blockDim.x) {
        const int rr = q / (PT_K / 4), lq = (q % (PT_K / 4)) * 4;
        const i64 r = r0 + rr;
        int er = (r < rows) ? e[r] : 0;
        if (er < -4096) {  // all-zero row: exponent 0; the k-chunk-0 CTA stores it for the gemm kernel
            er = 0;
            if (blockIdx.x == 0 && lq == 0) e[r] = 0;
        }
        // signed base-256 digits of G = trunc(v 2^(8s-2-er)) (d in [-128, 127], G = sum_j d_j 256^j):
        // with H = G + 0x80...80 (s bytes of 0x80, modulo 2^64), byte j of H is d_j + 128, since
        // adding 128 to each byte turns the digits' borrows into plain carries.  Slice p holds the
        // digit of weight 256^(s-1-p) (weight 2^(er - 8p - 6) of v), so one add per value and a
        // byte gather per slice write it; XOR 0x80 makes each byte the signed digit.
        const int B = 8 * slices - 2;
        const unsigned long long bias = 0x8080808080808080ULL >> (64 - 8 * slices);
        unsigned long long H[4];
        const bool fast = oz_scale_ok(er, B);
        const double scale = fast ? oz_pow2(B - er) : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            H[u] = static_cast<unsigned long long>(fast ? oz_fixed_scaled(tile[rr][lq + u], scale)
                                                        : oz_fixed(tile[rr][lq + u], er, B)) + bias;
        unsigned* out = reinterpret_cast<unsigned*>(planes + oz_plane_offset(Rp, r, l0 + lq));
        unsigned w[8];  // w[b]: byte b of H[0..3]
        byte_transpose4(unsigned(H[0]), unsigned(H[1]), unsigned(H[2]), unsigned(H[3]), w);
        byte_transpose4(unsigned(H[0] >> 32), unsigned(H[1] >> 32), unsigned(H[2] >> 32), unsigned(H[3] >> 32), w + 4);
#pragma unroll
        for (int b = 0; b < 8; ++b)  // byte b is the digit of slice slices - 1 - b
            if (b < slices) out[(plane / 4) * (slices - 1 - b)] = w[b] ^ 0x80808080u;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// 3-D map over planes[term][row][k]; box = {bkb/elem, box_rows, terms}.  The map covers
// Rp rows of each plane starting at `base`; consecutive planes are plane_rows rows apart
// (default Rp: a map over whole planes; more when it covers a row block of taller planes).
int make_map(CUtensorMap* map, const void* base, bool int8, i64 Kp, i64 Rp, int terms, int bkb,
             int box_rows, i64 plane_rows = 0) {
    auto fn = encode_fn();
    if (!fn) {
        set_error_msg("cuTensorMapEncodeTiled is unavailable from the driver");
        return MBG_ERR_CUDA;
    }
    const int elem = int8 ? 1 : 2;
    cuuint64_t dims[3] = {cuuint64_t(Kp), cuuint64_t(Rp), cuuint64_t(terms)};
    if (plane_rows <= 0) plane_rows = Rp;
    cuuint64_t strides[2] = {cuuint64_t(Kp) * elem, cuuint64_t(Kp) * cuuint64_t(plane_rows) * elem};
    cuuint32_t box[3] = {cuuint32_t(bkb / elem), cuuint32_t(box_rows), cuuint32_t(terms)};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapSwizzle sw = bkb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                 : bkb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    CUresult r = fn(map, int8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                    const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error_msg("cuTensorMapEncodeTiled failed (code " + std::to_string(int(r)) + ")");
        return MBG_ERR_CUDA;
    }
    return MBG_OK;
}

// 4-D map over slab-major Ozaki planes (oz_plane_offset): dims {OZ_SLAB bytes of k, rows,
// slabs, planes}, the rows of each slab plane_rows * OZ_SLAB bytes apart, planes
// plane_rows * Kp bytes apart; the map covers `rows` rows from `base` (a row block of
// taller planes when rows < plane_rows); box = {box_k, box_rows, 1, planes} with box_k 32
// or 64 bytes: in shared memory the planes' tiles follow each other, rows box_k bytes
// apart (the K-major layout with the box_k-byte swizzle).
int make_slab_map(CUtensorMap* map, const void* base, i64 Kp, i64 rows, i64 plane_rows, int planes, int box_rows,
                  int box_k) {
    auto fn = encode_fn();
    if (!fn) {
        set_error_msg("cuTensorMapEncodeTiled is unavailable from the driver");
        return MBG_ERR_CUDA;
    }
    cuuint64_t dims[4] = {OZ_SLAB, cuuint64_t(rows), cuuint64_t(Kp / OZ_SLAB), cuuint64_t(planes)};
    cuuint64_t strides[3] = {OZ_SLAB, cuuint64_t(plane_rows) * OZ_SLAB, cuuint64_t(plane_rows) * cuuint64_t(Kp)};
    cuuint32_t box[4] = {cuuint32_t(box_k), cuuint32_t(box_rows), 1, cuuint32_t(planes)};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, box_k == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error_msg("cuTensorMapEncodeTiled (slab-major planes) failed (code " + std::to_string(int(r)) + ")");
        return MBG_ERR_CUDA;
    }
    return MBG_OK;
}

template <class C>
int launch_tc(const CUtensorMap& ma, const CUtensorMap& mb, Params& P, const char* name) {
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      C::SMEM_BYTES));
        mark_configured(configured, dev);
    }
    P.err = device_error_flag();
    const i64 tiles = i64(P.tiles_m) * P.tiles_n;
    if (tiles > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    ProfScope prof(name);
    tc_gemm_kernel<C><<<unsigned(tiles), C::THREADS, C::SMEM_BYTES, stream()>>>(ma, mb, P);
    return check_launch(name);
}

// CTAs of split_sk_kernel that can be resident at once on this device (one per SM),
// cached per device.
template <class C>
int sk_workers(int dev, int sms, i64& out) {
    static std::atomic<int> cache[64];
    if (dev >= 0 && dev < 64 && cache[dev].load() > 0) {
        out = cache[dev].load();
        return MBG_OK;
    }
    int n = 0;
    MBG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, split_sk_kernel<C>, C::THREADS, C::SMEM_BYTES));
    out = imax(1, imin(i64(n) * sms, sms));
    if (dev >= 0 && dev < 64) cache[dev].store(int(out));
    return MBG_OK;
}

// Schedule of a persistent split launch over up to G workers (SkWork): whole tiles; when
// the tiles leave a last wave partly empty (and stream_k allows), stream-K ranges over the
// last (tiles mod g) + g tiles, with g <= G workers chosen so that every range is at least
// as long as the longest tile, and only where the busiest worker then finishes clearly
// sooner than with whole tiles.  G returns the number of workers to launch.
inline SkWork sk_plan(i64 t0, int n0, i64 t1, int n1, i64& G, bool stream_k) {
    SkWork W{};
    W.tiles0 = int(t0);
    W.tiles1 = int(t1);
    W.nkb0 = n0;
    W.nkb1 = t1 ? n1 : n0;
    const i64 T = t0 + t1;
    W.dp_tiles = int(T);
    G = imin(G, T);
    if (!stream_k || G <= 0 || T % G == 0) return W;
    auto slab_pos = [&](i64 u) { return u <= t0 ? u * n0 : t0 * n0 + (u - t0) * n1; };
    const i64 longest = t1 ? imax(n0, n1) : n0;
    // all tiles in ranges of at least `longest` slabs: as many workers as that allows
    const i64 total = slab_pos(T);
    i64 g = imin(G, total / longest);
    const i64 dp = T > 2 * g ? T - (T % g) - g : 0;
    const i64 begin = slab_pos(dp);
    if (g <= 0 || (total - begin) / g < longest) return W;
    // worth it when the balanced ranges end before whole tiles would: whole tiles take
    // ceil(T / G) tile times on the busiest worker, the ranges (total - begin) / g slabs
    // after dp / g whole tiles
    const double whole = double((T + G - 1) / G) * double(longest);
    const double ranged = double(dp / g) * double(longest) + double(total - begin) / double(g);
    // the persistent kernel ran a slab about 5 % slower than tc_gemm_kernel (8192^3 NT, whole
    // tiles plus a stream-K tail: 4.43 against 4.26 ms): demand a tenth
    if (1.1 * ranged >= whole) return W;
    W.dp_tiles = int(dp);
    W.sk_begin = begin;
    W.total = total;
    G = g;
    return W;
}

// Persistent launch (split_sk_kernel, config C) of one or two split products; the shared
// tiles of a stream-K schedule are zeroed first.  declined (non-null): launch nothing and
// set it when the schedule has no stream-K part (tc_gemm_kernel does whole tiles faster).
template <class C>
int launch_sk(const CUtensorMap* ma, const CUtensorMap* mb, Params* P, int nprod, bool stream_k, const char* name,
              bool* declined = nullptr) {
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0, sms = 148;
    MBG_CUDA(cudaGetDevice(&dev));
    MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(split_sk_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      C::SMEM_BYTES));
        mark_configured(configured, dev);
    }
    i64 G = 0;
    MBG_TRY(sk_workers<C>(dev, sms, G));
    if (nprod == 1) P[1] = P[0];
    constexpr int R = C::TILE_M / BM;  // 128-row tiles per output tile
    i64 tiles[2] = {0, 0};
    for (int i = 0; i < nprod; ++i) {
        P[i].err = device_error_flag();
        tiles[i] = i64((P[i].tiles_m + R - 1) / R) * P[i].tiles_n;
        if (P[i].num_kb <= 0) return MBG_ERR_UNSUPPORTED;
        if (P[i].beta != 0.0 || P[i].tri || P[i].band != KB_NONE || P[i].dvec) stream_k = false;
    }
    P[1].err = P[0].err;
    if (tiles[0] + tiles[1] > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    const SkWork W = sk_plan(tiles[0], P[0].num_kb, tiles[1], P[1].num_kb, G, stream_k);
    if (declined) {
        *declined = W.total == W.sk_begin;
        if (*declined) return MBG_OK;
    }
    if (G <= 0) return MBG_OK;
    ProfScope prof(name);
    if (W.total > W.sk_begin && G > 1) {
        sk_zero_kernel<C><<<unsigned(G - 1), 256, 0, stream()>>>(P[0], P[1], W, int(G));
        MBG_TRY(check_launch("sk_zero"));
    }
    split_sk_kernel<C><<<unsigned(G), C::THREADS, C::SMEM_BYTES, stream()>>>(ma[0], mb[0], P[0], ma[1], mb[1], P[1],
                                                                            W);
    return check_launch(name);
}

// The split product on planes pa (op(A), a_rows rows from pa, planes a_plane_rows apart)
// and pb (op(B)^T, b_rows rows): 128 x 256 tiles (a 128 x 128 tile's MMAs read a third
// more operand bytes per flop from shared memory, so the wide tile wins wherever it fills
// more than half of the SMs); 128 x 128 when the wide ones would fill at most half, 128 x 64
// at most a quarter (counting, under a triangle mask, only the tiles it keeps).  More wide tiles than SMs with a last wave mostly empty (beta = 0, no
// band, mask or d-vector): split_sk_kernel with a stream-K tail.  Sets the B map and
// P.tiles_n.
int launch_split_product(int terms, const __nv_bfloat16* pa, i64 a_rows, i64 a_plane_rows, const __nv_bfloat16* pb,
                         i64 b_rows, i64 Kp, Params& P) {
    int dev = 0, sms = 148;
    MBG_CUDA(cudaGetDevice(&dev));
    MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    i64 wide_tiles = i64(P.tiles_m) * cdiv(P.n, 256);
    if (P.tri) {  // only the tiles the triangle mask keeps do work
        i64 live = 0;
        for (i64 tm = 0; tm < P.tiles_m; ++tm)
            for (i64 tn = 0; tn < cdiv(P.n, 256); ++tn) {
                const i64 m0 = tm * BM, n0 = tn * 256;
                if (P.tri == 1 && m0 + BM <= n0) continue;
                if (P.tri == 2 && m0 > n0 + 255) continue;
                ++live;
            }
        wide_tiles = live;
    }
    const int bn = 4 * wide_tiles <= sms ? 64 : (2 * wide_tiles <= sms ? 128 : 256);
    CUtensorMap ma, mb;
    MBG_TRY(make_map(&ma, pa, false, Kp, a_rows, terms, 64, BM, a_plane_rows));
    if (bn == 256 && wide_tiles > sms && P.beta == 0.0 && !P.tri && P.band == KB_NONE && !P.dvec) {
        // more wide tiles than SMs and a last wave mostly empty: persistent, stream-K tail
        MBG_TRY(make_map(&mb, pb, false, Kp, b_rows, terms, 64, 256));
        P.tiles_n = int(cdiv(P.n, 256));
        const CUtensorMap mas[2] = {ma, ma}, mbs[2] = {mb, mb};
        Params Ps[2] = {P, P};
        bool declined = false;
        const int st = terms == 2 ? launch_sk<CfgBF16x3>(mas, mbs, Ps, 1, true, "tc_gemm_bf16x3", &declined)
                                  : launch_sk<CfgBF16x6>(mas, mbs, Ps, 1, true, "tc_gemm_bf16x6", &declined);
        if (st || !declined) return st;
    }
    MBG_TRY(make_map(&mb, pb, false, Kp, b_rows, terms, 64, bn));
    P.tiles_n = int(cdiv(P.n, bn));
    if (terms == 2) {
        if (bn == 64) return launch_tc<CfgBF16x3n>(ma, mb, P, "tc_gemm_bf16x3");
        if (bn == 128) return launch_tc<CfgBF16x3m>(ma, mb, P, "tc_gemm_bf16x3");
        return launch_tc<CfgBF16x3>(ma, mb, P, "tc_gemm_bf16x3");
    }
    if (bn == 64) return launch_tc<CfgBF16x6n>(ma, mb, P, "tc_gemm_bf16x6");
    if (bn == 128) return launch_tc<CfgBF16x6m>(ma, mb, P, "tc_gemm_bf16x6");
    return launch_tc<CfgBF16x6>(ma, mb, P, "tc_gemm_bf16x6");
}

template <int TERMS>
int launch_split(const float* src, i64 ld, bool kmajor, i64 rows, i64 K, i64 Rp, i64 Kp, __nv_bfloat16* planes,
                 int keep = 0) {
    ProfScope prof("split_bf16");
    const dim3 g = split_grid(Rp, Kp);
    if (Rp / SP_R > 65535) return MBG_ERR_UNSUPPORTED;
    if (kmajor) split_bf16_kernel<TERMS, true><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, planes, keep);
    else split_bf16_kernel<TERMS, false><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, planes, keep);
    return check_launch("split_bf16");
}

// Exponents and slices of a K-contiguous operand in one pass over its rows: a warp per
// row reads the row once for its largest magnitude (the exponent, 0 for an all-zero
// row) and again, mostly from cache, to write its digits; padding rows (rows .. Rp)
// and columns (K .. Kp) are written as zeros.  The digits and exponents are those of
// row_exponent_kernel + slice_i8_kernel, bit for bit; this saves the second read of
// the operand from DRAM and one launch.  SCALE: each value v(r, l) read for slicing is
// then overwritten in place by dscale[l] v (the inverse-based trsm leaf: the operand is
// also the output, whose diagonal term d .* C is applied here instead of being read
// back in the product's epilogue).
template <bool SCALE>
__global__ void __launch_bounds__(256)
slice_rows_kmajor_kernel(const double* src, i64 ld, i64 rows, i64 K, i64 Rp, i64 Kp, int slices,
                         int* __restrict__ e, int8_t* __restrict__ planes, int keep, const double* __restrict__ dscale) {
    const i64 r = i64(blockIdx.x) * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= Rp) return;
    const size_t plane = size_t(Rp) * size_t(Kp);
    const double* row = src + r * ld;
    const bool live = r < rows;
    // 16-byte loads when the row starts 16-byte aligned and no triangle mask applies
    const bool vec = keep == 0 && (reinterpret_cast<uintptr_t>(row) & 15) == 0;
    double mx = 0.0;
    if (live) {
        if (vec) {
            i64 l = 2 * i64(lane);
#pragma unroll 4
            for (; l + 1 < K; l += 64) {
                const double2 v = *reinterpret_cast<const double2*>(row + l);
                mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
            }
            if (l < K) mx = fmax(mx, fabs(row[l]));
        } else {
#pragma unroll 8
            for (i64 l = lane; l < K; l += 32)
                if (kept(keep, r, l)) mx = fmax(mx, fabs(row[l]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int er = 0;
    if (mx > 0.0) frexp(mx, &er);
    if (live && lane == 0) e[r] = er;
    const int B = 8 * slices - 2;
    const unsigned long long bias = 0x8080808080808080ULL >> (64 - 8 * slices);
    const bool fast = oz_scale_ok(er, B);
    const double scale = fast ? oz_pow2(B - er) : 0.0;
    // eight consecutive k per lane and iteration (Kp is a multiple of 32, so all eight are inside Kp)
    for (i64 l0 = i64(lane) * 8; l0 < Kp; l0 += 256) {
        double x[8];
        if (live && vec && l0 + 8 <= K) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 v = *reinterpret_cast<const double2*>(row + l0 + 2 * q);
                x[2 * q] = v.x;
                x[2 * q + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const i64 l = l0 + u;
                x[u] = (live && l < K && kept(keep, r, l)) ? row[l] : 0.0;
            }
        }
        if (SCALE && live) {
            double* w = const_cast<double*>(row);
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (l0 + u < K) w[l0 + u] = dscale[l0 + u] * x[u];
        }
        unsigned long long H[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            H[u] = static_cast<unsigned long long>(fast ? oz_fixed_scaled(x[u], scale) : oz_fixed(x[u], er, B)) + bias;
        uint2* out = reinterpret_cast<uint2*>(planes + oz_plane_offset(Rp, r, l0));
        unsigned wa[8], wb[8];  // byte b of H[0..3] and of H[4..7]
        byte_transpose4(unsigned(H[0]), unsigned(H[1]), unsigned(H[2]), unsigned(H[3]), wa);
        byte_transpose4(unsigned(H[0] >> 32), unsigned(H[1] >> 32), unsigned(H[2] >> 32), unsigned(H[3] >> 32), wa + 4);
        byte_transpose4(unsigned(H[4]), unsigned(H[5]), unsigned(H[6]), unsigned(H[7]), wb);
        byte_transpose4(unsigned(H[4] >> 32), unsigned(H[5] >> 32), unsigned(H[6] >> 32), unsigned(H[7] >> 32), wb + 4);
#pragma unroll
        for (int b = 0; b < 8; ++b)  // byte b is the digit of slice slices - 1 - b
            if (b < slices)
                out[(plane / 8) * (slices - 1 - b)] = make_uint2(wa[b] ^ 0x80808080u, wb[b] ^ 0x80808080u);
    }
}

// dscale (K-major fused slicing only, keep 0): src is overwritten in place by dscale[l] v(r, l).
int launch_slices(const double* src, i64 ld, bool kmajor, i64 rows, i64 K, i64 Rp, i64 Kp, int slices,
                  int* e, int8_t* planes, int keep = 0, const double* dscale = nullptr) {
    if (dscale && (!kmajor || !tuning().ozaki_fused_slicing || keep)) return MBG_ERR_UNSUPPORTED;
    if (kmajor && tuning().ozaki_fused_slicing) {
        ProfScope prof("ozaki_slice");
        const unsigned g = unsigned(cdiv(Rp, 8));
        if (dscale)
            slice_rows_kmajor_kernel<true><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, slices, e, planes, keep,
                                                                  dscale);
        else
            slice_rows_kmajor_kernel<false><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, slices, e, planes,
                                                                   keep, nullptr);
        return check_launch("ozaki_slice");
    }
    {
        ProfScope prof("ozaki_exponent");
        MBG_CUDA(cudaMemsetAsync(e, 0x80, sizeof(int) * size_t(rows), stream()));  // 0x80808080 < any exponent
        if (kmajor) {
            dim3 g(unsigned(cdiv(rows, 8)), unsigned(cdiv(K, OZ_EXP_KWARP)));
            if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
            row_exponent_kernel<true><<<g, 256, 0, stream()>>>(src, ld, rows, K, e, keep);
        } else {
            dim3 g(unsigned(cdiv(rows, 32)), unsigned(cdiv(K, OZ_EXP_KCHUNK)));
            if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
            row_exponent_kernel<false><<<g, 256, 0, stream()>>>(src, ld, rows, K, e, keep);
        }
        MBG_TRY(check_launch("ozaki_exponent"));
    }
    ProfScope prof("ozaki_slice");
    dim3 g(unsigned(Kp / PT_K), unsigned(Rp / PT_R));
    if (g.y > 65535) return MBG_ERR_UNSUPPORTED;
    if (kmajor) slice_i8_kernel<true><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, slices, e, planes, keep);
    else slice_i8_kernel<false><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, slices, e, planes, keep);
    return check_launch("ozaki_slice");
}

inline i64 roundup(i64 x, i64 m) { return cdiv(x, m) * m; }

}  // namespace tc

// ---- split-precision sgemm ------------------------------------------------------
int sgemm_split_tc(int terms, char ta, char tb, i64 m, i64 n, i64 k, float alpha, const float* a,
                   i64 lda, const float* b, i64 ldb, float beta, float* c, i64 ldc, char tri_uplo, int band,
                   const TriOperand* tri_op) {
    const int keep_a = tri_op ? tri_op->keep_a : 0, keep_b = tri_op ? tri_op->keep_b : 0;
    using namespace tc;
    if (m == 0 || n == 0) return MBG_OK;
    if (terms != 2 && terms != 3) return MBG_ERR_INVALID_MODE;
    const int BN = 256;
    const i64 Kp = roundup(k, 32);
    const bool tri = tri_uplo != 0;
    // syrk shares one set of planes for both operands (rows padded to BN)
    const bool shared_planes = tri && a == b && lda == ldb && (is_n(ta) != is_n(tb));
    const i64 Mp = shared_planes ? roundup(m, BN) : roundup(m, BM);
    const i64 Np = roundup(n, BN);
    if (Kp > 0x7fffffff || Mp > 0x7fffffff || Np > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    const size_t a_bytes = size_t(terms) * Mp * Kp * 2, b_bytes = shared_planes ? 0 : size_t(terms) * Np * Kp * 2;
    Workspace ws;
    MBG_TRY(ws.reserve(a_bytes + b_bytes));
    __nv_bfloat16* pa = ws.as<__nv_bfloat16>();
    __nv_bfloat16* pb = shared_planes ? pa : reinterpret_cast<__nv_bfloat16*>(ws.as<uint8_t>() + a_bytes);
    // op(A) rows are K-contiguous when A is transposed; op(B)^T rows when B is not
    if (terms == 2) {
        MBG_TRY(launch_split<2>(a, lda, is_t(ta), m, k, Mp, Kp, pa, keep_a));
        if (!shared_planes) MBG_TRY(launch_split<2>(b, ldb, is_n(tb), n, k, Np, Kp, pb, keep_b));
    } else {
        MBG_TRY(launch_split<3>(a, lda, is_t(ta), m, k, Mp, Kp, pa, keep_a));
        if (!shared_planes) MBG_TRY(launch_split<3>(b, ldb, is_n(tb), n, k, Np, Kp, pb, keep_b));
    }
    Params P{};
    P.m = m; P.n = n; P.num_kb = int(Kp / 32);
    P.tiles_m = int(cdiv(m, BM));
    P.tri = tri ? (is_l(tri_uplo) ? 1 : 2) : 0;
    P.band = band; P.band_k0 = 0;
    if (tri_op && tri_op->dvec_mode) {
        P.dvec = static_cast<const float*>(tri_op->dvec);
        P.dvec_mode = tri_op->dvec_mode;
    }
    P.c = c; P.ldc = ldc; P.alpha = alpha; P.beta = beta;
    return launch_split_product(terms, pa, Mp, Mp, pb, shared_planes ? Mp : Np, Kp, P);
}

// op(A)'s split planes made once and used for several products with column blocks of
// op(B): the pipelined host path computes C block by block as op(B) arrives.
int split_a_planes(int terms, char ta, i64 m, i64 k, const float* a, i64 lda, SplitA& out) {
    using namespace tc;
    if (terms != 2 && terms != 3) return MBG_ERR_INVALID_MODE;
    out.terms = terms;
    out.m = m;
    out.k = k;
    out.Mp = roundup(m, BM);
    out.Kp = roundup(k, 32);
    if (out.Kp > 0x7fffffff || out.Mp > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    MBG_TRY(out.ws.reserve(size_t(terms) * out.Mp * out.Kp * 2));
    __nv_bfloat16* pa = out.ws.as<__nv_bfloat16>();
    if (terms == 2) return launch_split<2>(a, lda, is_t(ta), m, k, out.Mp, out.Kp, pa);
    return launch_split<3>(a, lda, is_t(ta), m, k, out.Mp, out.Kp, pa);
}

// C[:, 0:n] := alpha op(A) op(B) + beta C with op(A)'s planes from split_a_planes (alpha != 0, k > 0).
int sgemm_split_tc_with_a(const SplitA& A, char tb, i64 n, float alpha, const float* b, i64 ldb, float beta,
                          float* c, i64 ldc) {
    return sgemm_split_tc_with_a_rows(A, 0, A.m, A.k, tb, n, alpha, b, ldb, beta, c, ldc);
}

// Rows r0 .. r0 + mb - 1 of op(A) (r0 a multiple of 128) times op(B) (k x n, k <= A.k; op(B)'s
// rows k .. A.k - 1 are taken as zero): C[0:mb, 0:n] := alpha op(A)[r0:r0+mb, :] op(B) + beta C.
int sgemm_split_tc_with_a_rows(const SplitA& A, i64 r0, i64 mb, i64 k, char tb, i64 n, float alpha, const float* b,
                               i64 ldb, float beta, float* c, i64 ldc) {
    using namespace tc;
    if (mb == 0 || n == 0) return MBG_OK;
    if (r0 % BM || r0 + mb > A.m || k > A.k) return MBG_ERR_UNSUPPORTED;
    const int BN = 256;
    const i64 Np = roundup(n, BN);
    if (Np > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    Workspace ws;
    MBG_TRY(ws.reserve(size_t(A.terms) * Np * A.Kp * 2));
    __nv_bfloat16* pb = ws.as<__nv_bfloat16>();
    if (A.terms == 2) MBG_TRY(launch_split<2>(b, ldb, is_n(tb), n, k, Np, A.Kp, pb));
    else MBG_TRY(launch_split<3>(b, ldb, is_n(tb), n, k, Np, A.Kp, pb));
    const i64 rows = imin(roundup(mb, BM), A.Mp - r0);
    Params P{};
    P.m = mb; P.n = n; P.num_kb = int(A.Kp / 32);
    P.tiles_m = int(cdiv(mb, BM));
    P.c = c; P.ldc = ldc; P.alpha = alpha; P.beta = beta;
    return launch_split_product(A.terms, A.ws.as<__nv_bfloat16>() + size_t(r0) * A.Kp, rows, A.Mp, pb, Np, A.Kp, P);
}

int sgemm_split_tc_dual(int terms, const SplitProduct& x, const SplitProduct& y) {
    using namespace tc;
    if (terms != 2 && terms != 3) return MBG_ERR_INVALID_MODE;
    const SplitProduct* q[2] = {&x, &y};
    if (y.k > x.k) std::swap(q[0], q[1]);  // the longer reduction's tiles take the first blocks
    constexpr int BN = 256;
    i64 Mp[2], Np[2], Kp[2];
    size_t off[2][2], total = 0;
    for (int i = 0; i < 2; ++i) {
        const SplitProduct& p = *q[i];
        if (p.m <= 0 || p.n <= 0 || p.k <= 0) return MBG_ERR_UNSUPPORTED;
        Mp[i] = roundup(p.m, BM);
        Np[i] = roundup(p.n, BN);
        Kp[i] = roundup(p.k, 32);
        if (Kp[i] > 0x7fffffff || Mp[i] > 0x7fffffff || Np[i] > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
        off[i][0] = total;
        total += (size_t(terms) * Mp[i] * Kp[i] * 2 + 1023) / 1024 * 1024;
        off[i][1] = total;
        total += (size_t(terms) * Np[i] * Kp[i] * 2 + 1023) / 1024 * 1024;
    }
    Workspace ws;
    MBG_TRY(ws.reserve(total));
    // the four operands' planes; op(A) rows are K-contiguous when A is transposed, op(B)^T
    // rows when B is not
    struct Operand {
        const float* src;
        i64 ld;
        bool kmajor;
        i64 rows, K, Rp, Kp;
        __nv_bfloat16* planes;
        bool done;
    } op[4];
    for (int i = 0; i < 2; ++i) {
        const SplitProduct& p = *q[i];
        op[2 * i] = {p.a, p.lda, is_t(p.ta), p.m, p.k, Mp[i], Kp[i],
                     reinterpret_cast<__nv_bfloat16*>(ws.as<uint8_t>() + off[i][0]), false};
        op[2 * i + 1] = {p.b, p.ldb, is_n(p.tb), p.n, p.k, Np[i], Kp[i],
                         reinterpret_cast<__nv_bfloat16*>(ws.as<uint8_t>() + off[i][1]), false};
    }
    // one matrix in both orientations, one in each product (the adjoint's G): one read of it
    for (int u = 0; u < 2; ++u)
        for (int v = 2; v < 4; ++v) {
            Operand& a = op[u];
            Operand& b = op[v];
            if (a.done || b.done || a.src != b.src || a.ld != b.ld || a.kmajor == b.kmajor) continue;
            Operand& r = a.kmajor ? b : a;  // G's rows as plane rows
            Operand& c = a.kmajor ? a : b;  // G's columns as plane rows
            if (r.rows != c.K || r.K != c.rows) continue;
            const i64 gi = imax(r.Rp, roundup(c.Kp, SP_R)), gj = imax(c.Rp, roundup(r.Kp, SP_K));
            if (gi / SP_R > 65535) continue;
            const dim3 g(unsigned(gj / SP_K), unsigned(gi / SP_R));
            ProfScope prof("split_bf16");
            if (terms == 2)
                split_bf16_both_kernel<2><<<g, 256, 0, stream()>>>(r.src, r.ld, r.rows, r.K, r.planes, r.Rp, r.Kp,
                                                                   c.planes, c.Rp, c.Kp);
            else
                split_bf16_both_kernel<3><<<g, 256, 0, stream()>>>(r.src, r.ld, r.rows, r.K, r.planes, r.Rp, r.Kp,
                                                                   c.planes, c.Rp, c.Kp);
            MBG_TRY(check_launch("split_bf16"));
            a.done = b.done = true;
        }
    for (auto& o : op) {
        if (o.done) continue;
        if (terms == 2) MBG_TRY(launch_split<2>(o.src, o.ld, o.kmajor, o.rows, o.K, o.Rp, o.Kp, o.planes));
        else MBG_TRY(launch_split<3>(o.src, o.ld, o.kmajor, o.rows, o.K, o.Rp, o.Kp, o.planes));
    }
    CUtensorMap ma[2], mb[2];
    Params P[2] = {};
    for (int i = 0; i < 2; ++i) {
        const SplitProduct& p = *q[i];
        const __nv_bfloat16* pa = op[2 * i].planes;
        const __nv_bfloat16* pb = op[2 * i + 1].planes;
        MBG_TRY(make_map(&ma[i], pa, false, Kp[i], Mp[i], terms, 64, BM));
        MBG_TRY(make_map(&mb[i], pb, false, Kp[i], Np[i], terms, 64, BN));
        P[i].m = p.m;
        P[i].n = p.n;
        P[i].num_kb = int(Kp[i] / 32);
        P[i].tiles_m = int(cdiv(p.m, BM));
        P[i].tiles_n = int(cdiv(p.n, BN));
        P[i].c = p.c;
        P[i].ldc = p.ldc;
        P[i].alpha = p.alpha;
        P[i].beta = 0.0;
        P[i].err = device_error_flag();
    }
    if (terms == 2) return launch_sk<CfgBF16x3>(ma, mb, P, 2, true, "tc_gemm_bf16x3");
    return launch_sk<CfgBF16x6>(ma, mb, P, 2, true, "tc_gemm_bf16x6");
}

// ---- Ozaki dgemm ----------------------------------------------------------------
namespace tc {
template <class C>
int launch_ozaki(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mal, const CUtensorMap& mbl,
                 OzParams& P) {
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(ozaki_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM_BYTES));
        mark_configured(configured, dev);
    }
    P.err = device_error_flag();
    const i64 tiles = i64(P.tiles_m) * P.tiles_n;
    if (tiles > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    ProfScope prof("tc_gemm_ozaki");
    ozaki_kernel<C><<<unsigned(tiles), C::THREADS, C::SMEM_BYTES, stream()>>>(ma, mb, mal, mbl, P);
    return check_launch("tc_gemm_ozaki");
}

template <class C>
int launch_ozaki_pair(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& mal, const CUtensorMap& mbl,
                      OzParams& P) {
    static std::atomic<unsigned> configured{0};  // one bit per device
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(ozaki_pair_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      C::SMEM_BYTES));
        mark_configured(configured, dev);
    }
    P.err = device_error_flag();
    i64 ctas = 2 * i64((P.tiles_m + 1) / 2) * P.tiles_n;
    if (ctas > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    if (tuning().ozaki_cta_pair == 2) {  // persistent: one cluster per pair of SMs
        int sms = 148;
        MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        ctas = imin(ctas, i64(sms / 2) * 2);
    }
    ProfScope prof("tc_gemm_ozaki");
    ozaki_pair_kernel<C><<<unsigned(ctas), C::THREADS, C::SMEM_BYTES, stream()>>>(ma, mb, mal, mbl, P);
    return check_launch("tc_gemm_ozaki");
}

// Tensor maps over the slices of op(A) (a_rows rows from pa, planes a_plane_rows
// rows apart) and of op(B)^T (Np rows, Kp bytes of k each), then the Ozaki
// launch: the CTA-pair kernel unless the tuning table selects the single-CTA one.
int run_ozaki(int slices, const int8_t* pa, i64 a_rows, i64 a_plane_rows, const int8_t* pb, i64 Np, i64 Kp,
              OzParams& P) {
    const bool pair = tuning().ozaki_cta_pair != 0;
    const int lo = slices <= 4 ? slices : 4;
    const int bbox = pair ? 64 : 128;
    const int bk = pair ? OZ_SLAB : 32;  // bytes of k per stage
    if (Kp % OZ_SLAB) return MBG_ERR_UNSUPPORTED;
    P.num_kb = int(Kp / bk);
    CUtensorMap ma, mb, mal, mbl;
    MBG_TRY(make_slab_map(&ma, pa, Kp, a_rows, a_plane_rows, slices, BM, bk));
    MBG_TRY(make_slab_map(&mal, pa, Kp, a_rows, a_plane_rows, lo, BM, bk));
    MBG_TRY(make_slab_map(&mb, pb, Kp, Np, Np, slices, bbox, bk));
    MBG_TRY(make_slab_map(&mbl, pb, Kp, Np, Np, lo, bbox, bk));
#define OZ_CASE(S_)                                                                    \
    case S_:                                                                           \
        return pair ? launch_ozaki_pair<Oz2Cfg<S_>>(ma, mb, mal, mbl, P)               \
                    : launch_ozaki<OzCfg<S_>>(ma, mb, mal, mbl, P);
    switch (slices) {
        OZ_CASE(2) OZ_CASE(3) OZ_CASE(4) OZ_CASE(5) OZ_CASE(6) OZ_CASE(7)
        default: OZ_CASE(8)
    }
#undef OZ_CASE
}
}  // namespace tc

// Longest reduction one Ozaki launch takes: its int32 accumulators hold at most
// `slices` products of K terms of at most 128^2 each; longer k runs in several launches.
i64 ozaki_max_k(int slices) { return (i64(0x7fffffff) / (i64(slices) * 128 * 128)) / 32 * 32; }

// op(A)'s Ozaki slices and row exponents made once, for several products with
// row blocks of op(A) (the trsm's inverted diagonal blocks).  k must fit one launch.
int ozaki_slice_a(int slices, char ta, i64 m, i64 k, const double* a, i64 lda, OzakiA& out) {
    using namespace tc;
    if (slices < 2 || slices > 8) return MBG_ERR_INVALID_MODE;
    if (k > ozaki_max_k(slices) || k <= 0 || m <= 0) return MBG_ERR_UNSUPPORTED;
    out.slices = slices;
    out.m = m;
    out.k = k;
    out.Mp = roundup(m, BM);
    out.Kp = roundup(k, OZ_SLAB);
    const size_t pbytes = size_t(slices) * out.Mp * out.Kp;
    MBG_TRY(out.ws.reserve(pbytes + sizeof(int) * size_t(out.Mp) + 1024));
    out.planes = out.ws.as<int8_t>();
    out.e = reinterpret_cast<int*>(out.planes + (pbytes + 1023) / 1024 * 1024);
    return launch_slices(a, lda, is_t(ta), m, k, out.Mp, out.Kp, slices, out.e, out.planes);
}

// Rows r0 .. r0 + mb - 1 of op(A) from ozaki_slice_a (r0 a multiple of 128) times op(B) (k x n,
// k <= A.k; op(B)'s rows k .. A.k - 1 taken as zero): C[0:mb, 0:n] := alpha op(A)[r0:r0+mb, :] op(B)
// + beta C, or with dvec (mb values) C := alpha op(A)[r0:r0+mb, :] op(B) + dvec .* C (each
// element of C read by the thread that then overwrites it).  C may be op(B) itself: the kernel
// reads op(B) only through its slices.
int dgemm_ozaki_tc_with_a(const OzakiA& A, i64 r0, i64 mb, i64 k, char tb, i64 n, double alpha, const double* b,
                          i64 ldb, double beta, double* c, i64 ldc, const double* dvec) {
    using namespace tc;
    if (mb == 0 || n == 0) return MBG_OK;
    if (r0 % BM || r0 + mb > A.m || k > A.k || k <= 0) return MBG_ERR_UNSUPPORTED;
    const int slices = A.slices, BN = 128;
    const i64 Np = roundup(n, BN);
    const size_t b_bytes = size_t(slices) * Np * A.Kp;
    Workspace ws;
    MBG_TRY(ws.reserve(b_bytes + sizeof(int) * size_t(Np) + 1024));
    int8_t* pb = ws.as<int8_t>();
    int* eb = reinterpret_cast<int*>(pb + (b_bytes + 1023) / 1024 * 1024);
    // the trsm leaf (C is op(B) itself, k = mb): the slicer writes d .* C back as it reads op(B),
    // and the product is added to it in L2, instead of the epilogue reading C (one round trip
    // per few columns, longer than the leaf's products)
    const bool prescale = dvec && c == b && ldc == ldb && k == mb && is_n(tb) && tuning().ozaki_fused_slicing;
    MBG_TRY(launch_slices(b, ldb, is_n(tb), n, k, Np, A.Kp, slices, eb, pb, 0, prescale ? dvec : nullptr));
    const i64 rows = imin(roundup(mb, BM), A.Mp - r0);
    const int8_t* pa = A.planes + size_t(r0) * OZ_SLAB;  // row r0 of every slab (slab-major planes)
    OzParams P{};
    P.m = mb; P.n = n;
    P.tiles_m = int(cdiv(mb, BM)); P.tiles_n = int(cdiv(n, BN));
    P.c = c; P.ldc = ldc; P.alpha = alpha; P.beta = beta;
    P.ea = A.e + r0; P.eb = eb;
    if (prescale) {
        P.beta = 1.0;
    } else if (dvec) {  // C = alpha acc + d .* C, d per row (C read before it is overwritten)
        P.dvec = dvec;
        P.dvec_mode = 1;
    }
    return run_ozaki(slices, pa, rows, A.Mp, pb, Np, A.Kp, P);
}

int dgemm_ozaki_tc(int slices, char ta, char tb, i64 m, i64 n, i64 k, double alpha, const double* a,
                   i64 lda, const double* b, i64 ldb, double beta, double* c, i64 ldc, char tri_uplo, int band,
                   const TriOperand* tri_op) {
    using namespace tc;
    if (m == 0 || n == 0) return MBG_OK;
    if (slices < 2 || slices > 8) return MBG_ERR_INVALID_MODE;
    const int BN = 128;
    const i64 kchunk_max = ozaki_max_k(slices);
    // a masked triangular operand and the in-place epilogue need the whole k in one launch
    if (tri_op && k > kchunk_max) return MBG_ERR_UNSUPPORTED;
    const int keep_a = tri_op ? tri_op->keep_a : 0, keep_b = tri_op ? tri_op->keep_b : 0;
    const bool tri = tri_uplo != 0;
    // syrk shares one set of slices and exponents for both operands (op(B)^T = op(A))
    const bool shared_planes = tri && a == b && lda == ldb && (is_n(ta) != is_n(tb)) && m == n;
    const i64 Mp = roundup(m, BM), Np = roundup(n, BN);
    const i64 kc = imin(k, kchunk_max);
    const i64 Kp = roundup(kc, OZ_SLAB);
    const size_t a_bytes = size_t(slices) * Mp * Kp, b_bytes = shared_planes ? 0 : size_t(slices) * Np * Kp;
    Workspace ws;
    MBG_TRY(ws.reserve(a_bytes + b_bytes + sizeof(int) * size_t(Mp + Np) + 1024));
    int8_t* pa = ws.as<int8_t>();
    int8_t* pb = shared_planes ? pa : pa + a_bytes;
    int* ea = reinterpret_cast<int*>(pa + a_bytes + b_bytes + (1024 - ((a_bytes + b_bytes) & 1023)) % 1024);
    int* eb = shared_planes ? ea : ea + Mp;
    for (i64 k0 = 0; k0 < k; k0 += kc) {
        const i64 klen = imin(kc, k - k0);
        const i64 Kpc = roundup(klen, OZ_SLAB);
        // op(A)[:, k0:k0+klen] and op(B)[k0:k0+klen, :]
        const double* ak = is_n(ta) ? a + k0 * lda : a + k0;
        const double* bk = is_n(tb) ? b + k0 : b + k0 * ldb;
        MBG_TRY(launch_slices(ak, lda, is_t(ta), m, klen, Mp, Kpc, slices, ea, pa, keep_a));
        if (!shared_planes) MBG_TRY(launch_slices(bk, ldb, is_n(tb), n, klen, Np, Kpc, slices, eb, pb, keep_b));
        OzParams P{};
        P.m = m; P.n = n;
        P.tiles_m = int(cdiv(m, BM)); P.tiles_n = int(cdiv(n, BN));
        P.tri = tri ? (is_l(tri_uplo) ? 1 : 2) : 0;
        P.band = band; P.band_k0 = k0;
        if (tri_op && tri_op->dvec_mode) {
            P.dvec = static_cast<const double*>(tri_op->dvec);
            P.dvec_mode = tri_op->dvec_mode;
        }
        P.c = c; P.ldc = ldc; P.alpha = alpha;
        P.beta = (k0 == 0) ? beta : 1.0;
        P.ea = ea; P.eb = eb;
        MBG_TRY(run_ozaki(slices, pa, Mp, Mp, pb, Np, Kpc, P));
    }
    return MBG_OK;
}

}  // namespace mbg

// ---- split-precision sgemm without device allocation ---------------------------
// Some callers cannot let a library allocate device memory: a host framework
// that owns a fixed device-memory budget and forbids plugins from calling
// cudaMalloc themselves, a latency-critical loop where cudaMalloc / cudaFree
// may synchronise the whole device, or code running inside an allocator's
// out-of-memory handling, where a further allocation would fail or recurse.
// mbg_sgemm_ex_noalloc serves them: the bf16 split planes that
// sgemm_split_tc takes from the workspace cache live instead in the fixed
// array below, which the CUDA runtime creates when it loads this module on a
// device and which stays resident there until the process exits.
namespace mbg {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;  // 32 MiB per device
constexpr int NOALLOC_MAX_DEVICES = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
__device__ int g_noalloc_err[4];  // bounded-wait error flag for this entry point

struct NoallocDevice {
    bool ready = false;
    void* scratch = nullptr;  // device address of g_noalloc_scratch
    int* err = nullptr;       // device address of g_noalloc_err
};
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;

// Once per device, with that device current: resolve the device addresses of
// the static arrays (host code cannot use the array names as addresses) and
// raise the kernels' shared-memory limit.
int noalloc_setup(NoallocDevice** out) {
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return MBG_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        MBG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        void* e = nullptr;
        MBG_CUDA(cudaGetSymbolAddress(&e, g_noalloc_err));
        MBG_CUDA(cudaFuncSetAttribute(tc::tc_gemm_kernel<tc::CfgBF16x3>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tc::CfgBF16x3::SMEM_BYTES));
        MBG_CUDA(cudaFuncSetAttribute(tc::tc_gemm_kernel<tc::CfgBF16x6>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, tc::CfgBF16x6::SMEM_BYTES));
        d.scratch = p;
        d.err = static_cast<int*>(e);
        d.ready = true;
    }
    *out = &d;
    return MBG_OK;
}

template <int TERMS>
void noalloc_split(const float* src, i64 ld, bool kmajor, i64 rows, i64 K, i64 Rp, i64 Kp,
                   __nv_bfloat16* planes) {
    const dim3 g = tc::split_grid(Rp, Kp);
    if (kmajor) tc::split_bf16_kernel<TERMS, true><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, planes);
    else tc::split_bf16_kernel<TERMS, false><<<g, 256, 0, stream()>>>(src, ld, rows, K, Rp, Kp, planes);
}

}  // namespace

}  // namespace mbg

extern "C" int mbg_sgemm_ex_noalloc(int mode, char ta, char tb, int64_t m, int64_t n, int64_t k,
                                    float alpha, const float* a, int64_t lda, const float* b,
                                    int64_t ldb, float beta, float* c, int64_t ldc) {
    using namespace mbg;
    using namespace mbg::tc;
    if (mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    // argument checks as mojoBLAS gemm numbers them (src/level3/gemm.mojo:179-213)
    if (!is_n(ta) && !is_t(ta)) return 1;
    if (!is_n(tb) && !is_t(tb)) return 2;
    if (m < 0) return 3;
    if (n < 0) return 4;
    if (k < 0) return 5;
    if (lda < imax(1, is_n(ta) ? m : k)) return 8;
    if (ldb < imax(1, is_n(tb) ? k : n)) return 10;
    if (ldc < imax(1, m)) return 13;
    if (m == 0 || n == 0) return MBG_OK;
    const int terms = mode == MBG_MODE_BF16X6 ? 3 : 2;
    // any dimension this large cannot fit; checked first so the padded sizes below cannot wrap
    if (m > i64(NOALLOC_SCRATCH_BYTES) || n > i64(NOALLOC_SCRATCH_BYTES) || k > i64(NOALLOC_SCRATCH_BYTES)) {
        set_error_msg("mbg_sgemm_ex_noalloc: a dimension exceeds the scratch limit of " +
                      std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes");
        return MBG_ERR_SCRATCH_LIMIT;
    }
    const i64 Mp = roundup(m, BM), Np = roundup(n, 256), Kp = roundup(imax(k, 1), 32);
    const size_t need = size_t(terms) * size_t(Mp + Np) * size_t(Kp) * 2;
    if (need > NOALLOC_SCRATCH_BYTES) {
        set_error_msg("mbg_sgemm_ex_noalloc: needs " + std::to_string(need) + " bytes of scratch, limit " +
                      std::to_string(NOALLOC_SCRATCH_BYTES) +
                      " (terms * (roundup(m,128) + roundup(n,256)) * roundup(k,32) * 2)");
        return MBG_ERR_SCRATCH_LIMIT;
    }
    const bool need_ab = !(alpha == 0.0f || k == 0);
    if ((need_ab && (!is_device_pointer(a) || !is_device_pointer(b))) || !is_device_pointer(c)) {
        set_error_msg("mbg_sgemm_ex_noalloc: operands must be device pointers (host data would need staging)");
        return MBG_ERR_UNSUPPORTED;
    }
    NoallocDevice* d = nullptr;
    MBG_TRY(noalloc_setup(&d));
    if (!need_ab) {
        MBG_TRY(scale_matrix<float>(m, n, beta, c, ldc));
    } else {
        // planes for op(A) then op(B)^T; the split kernels write every element,
        // zero padding included, so nothing left by an earlier call is read
        __nv_bfloat16* pa = static_cast<__nv_bfloat16*>(d->scratch);
        __nv_bfloat16* pb = pa + size_t(terms) * Mp * Kp;
        if (terms == 2) {
            noalloc_split<2>(a, lda, is_t(ta), m, k, Mp, Kp, pa);
            noalloc_split<2>(b, ldb, is_n(tb), n, k, Np, Kp, pb);
        } else {
            noalloc_split<3>(a, lda, is_t(ta), m, k, Mp, Kp, pa);
            noalloc_split<3>(b, ldb, is_n(tb), n, k, Np, Kp, pb);
        }
        MBG_TRY(check_launch("split_bf16"));
        CUtensorMap ma, mb;
        MBG_TRY(make_map(&ma, pa, false, Kp, Mp, terms, 64, BM));
        MBG_TRY(make_map(&mb, pb, false, Kp, Np, terms, 64, 256));
        Params P{};
        P.m = m; P.n = n; P.num_kb = int(Kp / 32);
        P.tiles_m = int(cdiv(m, BM)); P.tiles_n = int(cdiv(n, 256));
        P.tri = 0; P.c = c; P.ldc = ldc; P.alpha = alpha; P.beta = beta;
        P.err = d->err;
        const unsigned tiles = unsigned(i64(P.tiles_m) * P.tiles_n);
        if (terms == 2)
            tc_gemm_kernel<CfgBF16x3><<<tiles, CfgBF16x3::THREADS, CfgBF16x3::SMEM_BYTES, stream()>>>(ma, mb, P);
        else
            tc_gemm_kernel<CfgBF16x6><<<tiles, CfgBF16x6::THREADS, CfgBF16x6::SMEM_BYTES, stream()>>>(ma, mb, P);
        MBG_TRY(check_launch(terms == 2 ? "tc_gemm_bf16x3" : "tc_gemm_bf16x6"));
    }
    // synchronous mode: wait, then report an expired wait (this entry point's flag is read
    // and cleared by read_and_clear_device_error, as mbg_synchronize does in asynchronous mode)
    return finish_call(false);
}

// The no-allocation kernels' bounded-wait flag on the current device: returns its code
// (0 when no wait expired) and clears it.  Called by read_and_clear_device_error, so
// the synchronous return and mbg_synchronize() both surface it exactly once.  The flag
// lives in device memory: the caller has synchronised the library stream first.
int mbg::noalloc_take_error(int* site) {
    using namespace mbg;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_dev[dev].ready) return 0;  // never used on this device
    int flag[4] = {0, 0, 0, 0};
    if (cudaMemcpy(flag, g_noalloc_dev[dev].err, sizeof(flag), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (!flag[0]) return 0;
    const int zero[4] = {0, 0, 0, 0};
    if (cudaMemcpy(g_noalloc_dev[dev].err, zero, sizeof(zero), cudaMemcpyHostToDevice) != cudaSuccess)
        cudaGetLastError();
    if (site) *site = flag[1];
    return flag[0];
}

// Test hook: stores an error code in the no-allocation kernels' wait flag on the
// current device, as an expired wait would, so the reporting path can be checked
// without making any kernel wait.
extern "C" int mbg_debug_set_noalloc_error(int code) {
    using namespace mbg;
    NoallocDevice* d = nullptr;
    MBG_TRY(noalloc_setup(&d));
    const int v[4] = {code, 77, 0, 0};
    MBG_CUDA(cudaMemcpy(d->err, v, sizeof(v), cudaMemcpyHostToDevice));
    return MBG_OK;
}

// ---- bounded-wait probe ---------------------------------------------------------
// Exercises the failure path of the kernels' bounded waits without faulting the
// GPU: one thread waits on an mbarrier phase that nothing completes, gives up
// after limit_ns, records the error code and returns.
namespace mbg {
namespace tc {
__global__ void wait_probe_kernel(int* err, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        mbar_wait(&bar, 0, err, 99, limit_ns);  // no arrival ever comes
    }
}
}  // namespace tc
}  // namespace mbg

extern "C" int mbg_debug_wait_probe(int64_t limit_ns) {
    using namespace mbg;
    if (limit_ns <= 0 || limit_ns > 5000000000LL) return MBG_ERR_INVALID_MODE;
    int* err = device_error_flag();
    if (!err) return MBG_ERR_CUDA;
    tc::wait_probe_kernel<<<1, 32, 0, stream()>>>(err, (unsigned long long)limit_ns);
    MBG_TRY(check_launch("wait_probe"));
    MBG_CUDA(cudaStreamSynchronize(stream()));
    return read_and_clear_device_error() ? MBG_ERR_TIMEOUT : MBG_OK;
}

// ---- peak probes ------------------------------------------------------------------
// Throughput probes for the roofline denominators that are not in the driver's
// measured peaks: fp32 and fp64 FMA on the CUDA cores, and back-to-back
// tcgen05.mma (kind::f16 bf16 and kind::i8) on fixed shared-memory operands.
// Operand values are irrelevant: the probes time instruction throughput.
namespace mbg {
namespace tc {

template <typename T>
__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, T seed, T* out) {
    T a0 = seed + T(threadIdx.x), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
    const T m = T(0.999), c = T(1e-3);
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == T(-12345)) out[threadIdx.x] = s;  // keeps the chains alive
}

// One CTA per SM: lane 0 of warp 1 issues `iters` MMAs of 128 x 256 x (32 bytes of k)
// into one TMEM accumulator, commits, and waits (bounded) for them to complete.
template <bool INT8>
__global__ void __launch_bounds__(128, 1) mma_probe_kernel(int iters, int* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* done = reinterpret_cast<uint64_t*>(smem + 3 * 16384);
    uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(slot, 256);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    if (threadIdx.x == 32) {
        const uint32_t sa = smem_u32(smem), sb = sa + 16384;  // A: 128 rows x 128 B, B: 256 rows x 128 B
        const uint64_t ad = smem_desc(sa, 1024, 2), bd = smem_desc(sb, 1024, 2);
        const uint32_t idesc = instr_desc(INT8, 128, 256);
#pragma unroll 1
        for (int i = 0; i < iters; ++i) umma<INT8>(tmem, ad, bd, idesc, i > 0 ? 1u : 0u);
        umma_commit(done);
        mbar_wait(done, 0, err, 98);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 256);
    }
}

}  // namespace tc
}  // namespace mbg

// Measured throughputs in TFLOP/s (tensor probes: dense ops, 2 per multiply-add).
extern "C" int mbg_probe_peaks(double* fp32_tflops, double* fp64_tflops, double* bf16_tflops, double* int8_tops) {
    using namespace mbg;
    using namespace mbg::tc;
    int dev = 0, sms = 148;
    MBG_CUDA(cudaGetDevice(&dev));
    MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = stream();
    cudaEvent_t e0, e1;
    MBG_CUDA(cudaEventCreate(&e0));
    MBG_CUDA(cudaEventCreate(&e1));
    float* f32 = nullptr;
    double* f64 = nullptr;
    Workspace ws;
    MBG_TRY(ws.reserve(4096));
    f32 = ws.as<float>();
    f64 = ws.as<double>();
    auto time_ms = [&](auto launch) -> float {
        launch();  // warm-up
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    const int blocks = sms * 8, iters = 4096;
    const double fma_flops = 2.0 * blocks * 256.0 * iters * 64.0;
    if (fp32_tflops) {
        const float ms = time_ms([&] { fma_probe_kernel<float><<<blocks, 256, 0, s>>>(iters, 1.0f, f32); });
        *fp32_tflops = fma_flops / (ms * 1e-3) / 1e12;
    }
    if (fp64_tflops) {
        const float ms = time_ms([&] { fma_probe_kernel<double><<<blocks, 256, 0, s>>>(iters / 4, 1.0, f64); });
        *fp64_tflops = fma_flops / 4 / (ms * 1e-3) / 1e12;
    }
    int* err = device_error_flag();
    const int smem = 3 * 16384 + 1024 + 64;
    const int mma_iters = 8192;
    if (bf16_tflops) {
        MBG_CUDA(cudaFuncSetAttribute(mma_probe_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        const float ms = time_ms([&] { mma_probe_kernel<false><<<sms, 128, smem, s>>>(mma_iters, err); });
        *bf16_tflops = 2.0 * sms * double(mma_iters) * 128 * 256 * 16 / (ms * 1e-3) / 1e12;
    }
    if (int8_tops) {
        MBG_CUDA(cudaFuncSetAttribute(mma_probe_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        const float ms = time_ms([&] { mma_probe_kernel<true><<<sms, 128, smem, s>>>(mma_iters, err); });
        *int8_tops = 2.0 * sms * double(mma_iters) * 128 * 256 * 32 / (ms * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MBG_TRY(check_launch("peak_probes"));
    MBG_CUDA(cudaStreamSynchronize(s));
    return read_and_clear_device_error() ? MBG_ERR_TIMEOUT : MBG_OK;
}
