// Grouped split-precision sgemm (BF16x3 / BF16x6) on the tensor cores: thousands of
// independent problems of uneven sizes in one persistent tcgen05 launch.
//
// The reference has no batched interface (a mojoBLAS caller loops over gemm,
// src/level3/gemm.mojo:56).  The single-call split kernel (tc_gemm.cu) runs a
// pre-pass that writes bf16 planes and then TMA-loads them; for problems of 16 to
// 512 rows that pre-pass would cost more than the products, and TMA needs
// 16-byte-aligned leading dimensions that batched callers rarely have.  Here the
// split is fused into the kernel's producer warps:
//   warps 0..3   op(A) producers, warps 4..7 op(B)^T producers: thread r of a group
//                owns row r of its operand's tile.  Each warp copies the raw fp32
//                values of its 32 rows for a 32-deep k slab into shared memory with
//                cp.async, one slab ahead of the one it splits, coalesced along
//                whichever dimension the operand stores contiguously (along k for a
//                k-contiguous operand, along the rows otherwise; 16-byte copies when
//                the leading dimension allows); then each thread splits its own row
//                into TERMS bf16 terms (x1 = bf16(x), x2 = bf16(x - x1),
//                x3 = bf16(x - x1 - x2); each difference is exact) and stores them in
//                the tcgen05 K-major layout with the 64-byte swizzle.  Rows past the
//                problem's edge are stored as zeros without being copied or split.
//                Then a proxy fence and an arrival on the stage's "full" barrier;
//   warp 8       lane 0 issues the TERMS (TERMS + 1) / 2 products per 16-deep k
//                step into a TMEM accumulator of 128 x BN fp32 (BN = 64 or 128
//                per problem), restarted every 128 k (the tensor core's fp32
//                accumulation truncates) into the other of two buffers;
//   warps 9..16  epilogue: add each 128-k chunk into fp32 registers with
//                round-to-nearest, then alpha / beta and the column-major store;
//                the other TMEM buffer lets the next tile's products run meanwhile.
// Tiles (problem, 128-row block, BN-column block) are ordered by reduction length,
// longest first, and dealt round robin to one persistent CTA per SM.  All waits are
// bounded (2 s) and report through the library's error flag.
#include "mbg_internal.cuh"
#include "tc_ptx.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

namespace mbg {
namespace gtc {

using namespace tc;

constexpr int GBN = 128;       // widest tile (TMEM buffer stride)
constexpr int GBKB = 64;       // k slab: 32 bf16 per row, 64-byte swizzle
constexpr int GBK = 32;
constexpr int GCHUNK = 4;      // slabs per TMEM accumulation chunk
constexpr int GPROD_WARPS = 8;  // 4 for op(A), 4 for op(B)^T
constexpr int GMMA_WARP = 8;
constexpr int GEPI_WARPS = 8;
constexpr int GEPI_WARP0 = GMMA_WARP + 1;
constexpr int GTHREADS = 32 * (GPROD_WARPS + 1 + GEPI_WARPS);
// Raw fp32 staging ring of GRAW_STAGES slabs.  Per slab and operand each producer warp
// owns a region of GRAW_WARP floats holding its 32 rows, either as 32 rows of 36 floats
// (k-contiguous source: row-major, 16-byte aligned rows whose 16-byte reads by 8
// consecutive threads hit distinct banks) or as 32 k of 32 rows (row-contiguous source:
// a thread reads its row at stride 32, conflict-free across the warp).  The regions are
// disjoint whatever the layout, so only the warp itself ever reads or overwrites its
// region (consecutive uses of a slot may have different layouts).
// Two slots: with three the loads ran no faster (they are bound by the SM's outstanding
// 4-byte copy requests, not by latency) and the larger shared-memory carve-out left L1,
// which allocates those requests' lines, a third smaller.
constexpr int GRAW_STAGES = 2;
constexpr int GRAW_LD = 36;
constexpr int GRAW_WARP = 32 * GRAW_LD;   // floats per warp per operand per slab (>= 32 x 32)
constexpr int GRAW_OP = 4 * GRAW_WARP;    // floats per operand per slab
constexpr int GRAW_BYTES = 2 * GRAW_OP * 4;

template <int TERMS>
struct GCfg {
    static constexpr int A_PLANE = BM * GBKB;   // 8 KB
    static constexpr int B_PLANE = GBN * GBKB;  // 8 KB
    static constexpr int STAGE_BYTES = TERMS * (A_PLANE + B_PLANE);
    static constexpr int STAGES = TERMS == 3 ? 2 : 3;  // split planes in flight to the MMA warp
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + GRAW_STAGES * GRAW_BYTES + 1024 + 256;
    static constexpr int NPROD = TERMS * (TERMS + 1) / 2;
    static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

struct TcDesc {
    i64 m, n, k, lda, ldb, ldc;
    const float* a;
    const float* b;
    float* c;
    float alpha, beta;
    int ta, tb;  // op(A) = A^T, op(B) = B^T
    int bn;      // tile columns: 64 or 128
    int pad_;
};
struct TcTile {
    int prob, tm, tn, nkb;  // nkb: k slabs (0 when alpha == 0 or k == 0: C := beta C only)
};

// One producer group's view of a tile: row i of its operand tile, k index l, sits at
// p0[i * ld + l] (kcontig) or p0[i + l * ld]; rows >= live are padding (zero).
struct ProdOp {
    const float* p0;
    i64 ld, K;
    int live;     // rows of the tile inside the problem
    int used;     // rows the MMA reads (128 for op(A), the tile width for op(B)^T)
    int kcontig;  // k is the contiguous dimension
    int vec;      // 16-byte copies: ld a multiple of 4 floats and p0 16-byte aligned
};

__device__ __forceinline__ ProdOp prod_op(const TcDesc& d, const TcTile& tl, bool isA) {
    ProdOp o;
    if (isA) {  // op(A)(i, l): A^T -> a[l + i lda] (k contiguous), else a[i + l lda]
        const i64 r0 = i64(tl.tm) * BM;
        o.kcontig = d.ta;
        o.ld = d.lda;
        o.p0 = d.a + (d.ta ? r0 * d.lda : r0);
        o.live = int(min(i64(BM), d.m - r0));
        o.used = BM;
    } else {  // op(B)^T(j, l) = op(B)(l, j): B^T -> b[j + l ldb], else b[l + j ldb] (k contiguous)
        const i64 r0 = i64(tl.tn) * d.bn;
        o.kcontig = !d.tb;
        o.ld = d.ldb;
        o.p0 = d.b + (d.tb ? r0 : r0 * d.ldb);
        o.live = int(min(i64(d.bn), d.n - r0));
        o.used = d.bn;
    }
    o.K = d.k;
    o.vec = (o.ld % 4 == 0) && (reinterpret_cast<uintptr_t>(o.p0) % 16 == 0);
    return o;
}

__device__ __forceinline__ void cp_async4(unsigned dst, const float* src, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(unsigned dst, const float* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// The warp's share of one slab copy: rows rw0 .. rw0 + 31 of the tile, k = k0 .. k0 + 31,
// into the warp's region wr of a ring slot: row rw0 + i, k0 + l at wr[i * GRAW_LD + l]
// (kcontig) or wr[l * 32 + i].  Rows at or past o.live are not copied (their split is a
// zero store); k past K is zero-filled.
__device__ __forceinline__ void copy_slab(float* wr, const ProdOp& o, int rw0, int lane, i64 k0) {
    const unsigned base = static_cast<unsigned>(__cvta_generic_to_shared(wr));
    if (rw0 >= o.live) return;
    if (o.kcontig) {
        if (o.vec && k0 + GBK <= o.K) {
            // lanes 8 q .. 8 q + 7: the eight 16-byte pieces of one row; four rows per copy
            const int ch = lane & 7;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int row = rw0 + 4 * j + (lane >> 3);
                if (row < o.live)
                    cp_async16(base + unsigned((row - rw0) * GRAW_LD + 4 * ch) * 4, o.p0 + i64(row) * o.ld + k0 + 4 * ch,
                               16);
            }
        } else {
            // lane = k: one row per copy, 128 contiguous bytes across the warp
            const bool kv = k0 + lane < o.K;
            const float* q = o.p0 + i64(rw0) * o.ld + (kv ? k0 + lane : 0);
            const int n = min(32, o.live - rw0);
#pragma unroll 8
            for (int i = 0; i < n; ++i, q += o.ld)
                cp_async4(base + unsigned(i * GRAW_LD + lane) * 4, kv ? q : o.p0, kv ? 4 : 0);
        }
    } else {
        if (o.vec) {
            // lanes 8 q .. 8 q + 7: 32 consecutive rows of one k (four per 16-byte copy);
            // four k per copy; partial row groups and k past K are zero-filled
            const int rr = rw0 + 4 * (lane & 7);
            const int nv = min(4, o.live - rr);
            if (nv > 0) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int l = 4 * j + (lane >> 3);
                    const bool kv = k0 + l < o.K;
                    cp_async16(base + unsigned(l * 32 + rr - rw0) * 4, kv ? o.p0 + rr + (k0 + l) * o.ld : o.p0,
                               kv ? 4 * nv : 0);
                }
            }
        } else {
            // lane = row: one k per copy, 128 contiguous bytes across the warp
            const int r = rw0 + lane;
            if (r < o.live) {
                const float* q = o.p0 + r + k0 * o.ld;
#pragma unroll 8
                for (int l = 0; l < GBK; ++l, q += o.ld) {
                    const bool kv = k0 + l < o.K;
                    cp_async4(base + unsigned(l * 32 + lane) * 4, kv ? q : o.p0, kv ? 4 : 0);
                }
            }
        }
    }
}

// Split of 16 consecutive k values into TERMS bf16 terms, written as two 16-byte chunks
// per plane at their 64-byte-swizzled positions of row r.  Pairs are rounded together
// (one bf16x2 conversion) and each term's value recovered from its bits.
template <int TERMS>
__device__ __forceinline__ void split_store16(const float (&v)[16], uint8_t* plane0, int plane_bytes, int r,
                                              int chunk0) {
    float x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = v[i];
#pragma unroll
    for (int t = 0; t < TERMS; ++t) {
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const __nv_bfloat162 pr = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);  // .x low half, .y high
            w[i] = *reinterpret_cast<const uint32_t*>(&pr);
            if (t + 1 < TERMS) {
                x[2 * i] -= __uint_as_float(w[i] << 16);  // exact: x and its bf16 agree in their leading bits
                x[2 * i + 1] -= __uint_as_float(w[i] & 0xffff0000u);
            }
        }
        uint8_t* rowp = plane0 + t * plane_bytes + r * GBKB;
        const int sw = (r >> 1) & 3;  // 64-byte swizzle: 16-byte chunk c of row r sits at c ^ ((r / 2) % 4)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = (chunk0 + h) ^ sw;
            *reinterpret_cast<uint4*>(rowp + c * 16) = make_uint4(w[4 * h], w[4 * h + 1], w[4 * h + 2], w[4 * h + 3]);
        }
    }
}

template <int TERMS>
__global__ void __launch_bounds__(GTHREADS, 1)
grouped_tc_kernel(const TcDesc* __restrict__ probs, const TcTile* __restrict__ tiles, int ntiles, int* err) {
    using C = GCfg<TERMS>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    float* raw = reinterpret_cast<float*>(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES + GRAW_STAGES * GRAW_BYTES);
    uint64_t* empty = full + C::STAGES;
    uint64_t* tfull = empty + C::STAGES;  // [2]
    uint64_t* tempty = tfull + 2;       // [2]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full[s], 32 * GPROD_WARPS);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], GEPI_WARPS);
        }
        fence_barrier_init();
    }
    if (warp == GMMA_WARP) {
        tmem_alloc(tmem_slot, 2 * GBN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < GPROD_WARPS) {
        // ---------------- producers: copy (cp.async), split, store ----------------
        const bool isA = warp < GPROD_WARPS / 2;
        const int r = isA ? threadIdx.x : threadIdx.x - BM;  // tile row 0..127 of this group's operand
        const int rw0 = r & ~31;                              // the warp's first row
        const int plane_bytes = isA ? C::A_PLANE : C::B_PLANE;
        float* const ring = raw + (isA ? 0 : GRAW_OP) + (rw0 / 32) * GRAW_WARP;  // this warp's region of slot 0
        // the slabs of this CTA's tiles form one sequence; the look-ahead cursor (tile
        // `at`, slab `akb`, operand view `ao`) walks it GRAW_STAGES - 1 slabs in front of
        // the slab being split
        int at = blockIdx.x, akb = 0, anb = 0;
        ProdOp ao{};
        if (at < ntiles) {
            const TcTile tl = tiles[at];
            anb = tl.nkb;
            ao = prod_op(probs[tl.prob], tl, isA);
        }
        auto issue_next = [&](int slot) {
            while (at < ntiles && akb >= anb) {
                at += gridDim.x;
                akb = 0;
                if (at < ntiles) {
                    const TcTile tl = tiles[at];
                    anb = tl.nkb;
                    ao = prod_op(probs[tl.prob], tl, isA);
                }
            }
            if (at < ntiles) {
                copy_slab(ring + slot * (GRAW_BYTES / 4), ao, rw0, lane, i64(akb) * GBK);
                ++akb;
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");  // one group per slab, empty at the end
        };
        for (int i = 0; i < GRAW_STAGES - 1; ++i) issue_next(i);
        int it = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const TcTile tl = tiles[t];
            const ProdOp o = prod_op(probs[tl.prob], tl, isA);
            for (int kb = 0; kb < tl.nkb; ++kb, ++it) {
                __syncwarp();  // every lane has read the warp's region that the next copy overwrites
                issue_next((it + GRAW_STAGES - 1) % GRAW_STAGES);
                asm volatile("cp.async.wait_group %0;\n" ::"n"(GRAW_STAGES - 1) : "memory");  // slab `it` landed
                __syncwarp();  // ... including the pieces of this warp's rows copied by other lanes
                const int s = it % C::STAGES;
                if (!mbar_wait(&empty[s], ((it / C::STAGES) & 1) ^ 1, err, 31)) { ok = false; break; }
                uint8_t* plane0 = smem + s * C::STAGE_BYTES + (isA ? 0 : TERMS * C::A_PLANE);
                if (r < o.live) {
                    const float* rr = ring + (it % GRAW_STAGES) * (GRAW_BYTES / 4);
                    float v[16];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (o.kcontig) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float4 f = reinterpret_cast<const float4*>(rr + lane * GRAW_LD + 16 * h)[q];
                                v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
                            }
                        } else {
#pragma unroll
                            for (int i = 0; i < 16; ++i) v[i] = rr[(16 * h + i) * 32 + lane];
                        }
                        split_store16<TERMS>(v, plane0, plane_bytes, r, 2 * h);
                    }
                } else if (r < o.used) {  // padding row: zero terms
#pragma unroll
                    for (int tt = 0; tt < TERMS; ++tt)
#pragma unroll
                        for (int c = 0; c < 4; ++c)
                            *reinterpret_cast<uint4*>(plane0 + tt * plane_bytes + r * GBKB + c * 16) =
                                make_uint4(0u, 0u, 0u, 0u);
                }
                // generic-proxy stores must be visible to the tensor core's (async proxy) reads
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(&full[s]);
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy lands after the CTA exits
    } else if (warp == GMMA_WARP) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            int it = 0, ch = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const TcTile tl = tiles[t];
                const uint32_t idesc = instr_desc(false, BM, probs[tl.prob].bn);
                for (int kb = 0; kb < tl.nkb; ++kb, ++it) {
                    const int kin = kb % GCHUNK, buf = ch & 1;
                    if (kin == 0 && ch >= 2) {  // the epilogue has drained this buffer's previous chunk
                        if (!mbar_wait(&tempty[buf], ((ch >> 1) - 1) & 1, err, 32)) { ok = false; break; }
                        tc_fence_after();
                    }
                    const int s = it % C::STAGES;
                    if (!mbar_wait(&full[s], (it / C::STAGES) & 1, err, 33)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
                    const uint32_t sb = sa + TERMS * C::A_PLANE;
#pragma unroll
                    for (int ks = 0; ks < GBKB / 32; ++ks) {
#pragma unroll
                        for (int pi = 0; pi < C::NPROD; ++pi) {
                            int p, q, collector;
                            product<TERMS, false>(pi, p, q, collector);
                            const uint32_t accumulate = (kin > 0 || ks > 0 || pi > 0) ? 1u : 0u;
                            const uint64_t ad = smem_desc(sa + p * C::A_PLANE + ks * 32, 8 * GBKB, 4);
                            const uint64_t bd = smem_desc(sb + q * C::B_PLANE + ks * 32, 8 * GBKB, 4);
                            umma<false>(tmem + uint32_t(buf * GBN), ad, bd, idesc, accumulate);
                        }
                    }
                    umma_commit(&empty[s]);
                    if (kin == GCHUNK - 1 || kb == tl.nkb - 1) {
                        umma_commit(&tfull[buf]);
                        ++ch;
                    }
                }
            }
        }
    } else {
        // ---------------- epilogue ----------------
        const int e = warp - GEPI_WARP0;
        const int quarter = warp & 3;  // the TMEM lanes this warp may read
        const int part = e >> 2;
        int ch = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const TcTile tl = tiles[t];
            const TcDesc d = probs[tl.prob];
            const int epi_cols = d.bn / 2;
            const i64 row = i64(tl.tm) * BM + quarter * 32 + lane;
            const i64 cbase = i64(tl.tn) * d.bn + part * epi_cols;
            float acc[GBN / 2];
#pragma unroll
            for (int j = 0; j < GBN / 2; ++j) acc[j] = 0.0f;
            const int nchunks = (tl.nkb + GCHUNK - 1) / GCHUNK;
            for (int c = 0; c < nchunks && ok; ++c, ++ch) {
                const int buf = ch & 1;
                if (!mbar_wait(&tfull[buf], (ch >> 1) & 1, err, 34)) { ok = false; break; }
                tc_fence_after();
                const uint32_t base = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(buf * GBN + part * epi_cols);
#pragma unroll
                for (int c0 = 0; c0 < GBN / 2; c0 += 16) {
                    if (c0 < epi_cols) {  // warp-uniform
                        uint32_t rr[16];
                        tmem_ld16(base + uint32_t(c0), rr);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 16; ++j) acc[c0 + j] += __uint_as_float(rr[j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (!ok) break;
            if (row < d.m) {
                // straight-line stores of the live columns; with beta != 0 eight loads of C
                // are issued before their stores (a store may alias any later load, so a
                // load per store would wait one round trip each)
                const int nc = int(min(i64(epi_cols), d.n - cbase));
                float* cp = d.c + row + cbase * d.ldc;
                const i64 ldc = d.ldc;
                if (d.beta == 0.0f) {
#pragma unroll
                    for (int j = 0; j < GBN / 2; ++j)
                        if (j < nc) cp[j * ldc] = d.alpha * acc[j];
                } else {
#pragma unroll
                    for (int j0 = 0; j0 < GBN / 2; j0 += 8) {
                        float cv[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) cv[j] = j0 + j < nc ? cp[(j0 + j) * ldc] : 0.0f;
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            if (j0 + j < nc) cp[(j0 + j) * ldc] = fmaf(d.beta, cv[j], d.alpha * acc[j0 + j]);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == GMMA_WARP) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 2 * GBN);
    }
}

}  // namespace gtc

// ---- plans (called by grouped.cu) -------------------------------------------------
// The device table holds TcDesc[count], then (256-byte aligned) TcTile[ntiles].

// Builds the device table of a grouped split sgemm: per problem its tile width (from
// the tuning table's size class), its tiles ordered by reduction length, longest first.
int grouped_tc_build(int terms, int count, const mbg_sgemm_problem* probs, GroupedTcPlan& out) {
    using namespace gtc;
    std::vector<TcDesc> v;
    std::vector<TcTile> t;
    v.reserve(size_t(count));
    for (int i = 0; i < count; ++i) {
        const mbg_sgemm_problem& q = probs[i];
        if (q.m == 0 || q.n == 0) continue;
        TcDesc d{};
        d.m = q.m; d.n = q.n; d.k = q.k; d.lda = q.lda; d.ldb = q.ldb; d.ldc = q.ldc;
        d.a = q.a; d.b = q.b; d.c = q.c; d.alpha = q.alpha; d.beta = q.beta;
        d.ta = is_t(q.trans_a); d.tb = is_t(q.trans_b);
        d.bn = grouped_tc_tile_cols(q.m, q.n, q.k, d.ta, d.tb);
        const int pi = int(v.size());
        v.push_back(d);
        const int nkb = (q.alpha == 0.0f || q.k == 0) ? 0 : int(cdiv(q.k, GBK));
        for (int tn = 0; tn < int(cdiv(q.n, d.bn)); ++tn)
            for (int tm = 0; tm < int(cdiv(q.m, BM)); ++tm) t.push_back(TcTile{pi, tm, tn, nkb});
    }
    std::stable_sort(t.begin(), t.end(), [](const TcTile& x, const TcTile& y) { return x.nkb > y.nkb; });
    out.terms = terms;
    out.count = int(v.size());
    out.ntiles = int(t.size());
    if (out.ntiles == 0) return MBG_OK;
    out.tiles_off = (sizeof(TcDesc) * v.size() + 255) / 256 * 256;
    const size_t bytes = out.tiles_off + sizeof(TcTile) * t.size();
    MBG_CUDA(cudaMalloc(&out.table, bytes));
    MBG_CUDA(cudaMemcpy(out.table, v.data(), sizeof(TcDesc) * v.size(), cudaMemcpyHostToDevice));
    MBG_CUDA(cudaMemcpy(static_cast<char*>(out.table) + out.tiles_off, t.data(), sizeof(TcTile) * t.size(),
                        cudaMemcpyHostToDevice));
    int dev = 0, sms = 148;
    MBG_CUDA(cudaGetDevice(&dev));
    MBG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    out.grid = int(imin(out.ntiles, sms));
    // the wait-error flag is created now: its first use must not fall inside the plan's graph capture
    out.err = device_error_flag();
    const int smem = terms == 3 ? GCfg<3>::SMEM_BYTES : GCfg<2>::SMEM_BYTES;
    if (terms == 3)
        MBG_CUDA(cudaFuncSetAttribute(grouped_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    else
        MBG_CUDA(cudaFuncSetAttribute(grouped_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return MBG_OK;
}

int grouped_tc_enqueue(const GroupedTcPlan& p, cudaStream_t s) {
    using namespace gtc;
    if (p.ntiles == 0) return MBG_OK;
    const TcDesc* d = static_cast<const TcDesc*>(p.table);
    const TcTile* t = reinterpret_cast<const TcTile*>(static_cast<const char*>(p.table) + p.tiles_off);
    if (p.terms == 3)
        grouped_tc_kernel<3><<<p.grid, GTHREADS, GCfg<3>::SMEM_BYTES, s>>>(d, t, p.ntiles, p.err);
    else
        grouped_tc_kernel<2><<<p.grid, GTHREADS, GCfg<2>::SMEM_BYTES, s>>>(d, t, p.ntiles, p.err);
    return check_launch("grouped_sgemm_tc");
}

void grouped_tc_free(GroupedTcPlan& p) {
    if (p.table) cudaFree(p.table);
    p.table = nullptr;
}

}  // namespace mbg
