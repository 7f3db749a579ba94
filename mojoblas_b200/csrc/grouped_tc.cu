// Grouped split-precision sgemm (BF16x3 / BF16x6) on the tensor cores: thousands of
// independent problems of uneven sizes in one persistent tcgen05 launch.
//
// The reference has no batched interface (a mojoBLAS caller loops over gemm,
// src/level3/gemm.mojo:56).  The single-call split kernel (tc_gemm.cu) runs a
// pre-pass that writes bf16 planes and then TMA-loads them; for problems of 16 to
// 512 rows that pre-pass would cost more than the products, and TMA needs
// 16-byte-aligned leading dimensions that batched callers rarely have.  Here the
// split is fused into the kernel's producer warps:
//   warps 0..3   producers: thread r owns row r of the tile's op(A) slab and row r
//                of its op(B)^T slab (32 k each), loads them from global memory
//                (coalesced across the warp when rows are contiguous, 16-byte
//                loads along k when k is contiguous and aligned), splits each
//                value into TERMS bf16 terms (x1 = bf16(x), x2 = bf16(x - x1),
//                x3 = bf16(x - x1 - x2); each difference is exact) and stores them
//                in the tcgen05 K-major layout with the 64-byte swizzle; then a
//                proxy fence and an arrival on the stage's "full" barrier;
//   warp 4       lane 0 issues the TERMS (TERMS + 1) / 2 products per 16-deep k
//                step into a TMEM accumulator of 128 x BN fp32 (BN = 64 or 128
//                per problem), restarted every 128 k (the tensor core's fp32
//                accumulation truncates) into the other of two buffers;
//   warps 5..12  epilogue: add each 128-k chunk into fp32 registers with
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
constexpr int GPROD_WARPS = 4;
constexpr int GMMA_WARP = 4;
constexpr int GEPI_WARPS = 8;
constexpr int GTHREADS = 32 * (GPROD_WARPS + 1 + GEPI_WARPS);
// Raw fp32 staging: each producer thread copies its own row's 32 values of op(A) and of
// op(B)^T for a slab into shared memory with cp.async, RAW_STAGES - 1 slabs ahead of the
// one it splits, so the global-memory latency overlaps the splitting of earlier slabs
// (a thread reads back only what it copied itself: no barrier is needed).  Row stride
// 36 floats: 16-byte aligned, and the 16-byte reads of 32 rows spread over all banks.
constexpr int GRAW_STAGES = 3;
constexpr int GRAW_LD = 36;
constexpr int GRAW_BYTES = 2 * BM * GRAW_LD * 4;  // op(A) rows then op(B)^T rows

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

// split of 16 consecutive k values into TERMS bf16 terms, written as two 16-byte chunks
// per plane at their 64-byte-swizzled positions of row r
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
            const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]), h1 = __float2bfloat16_rn(x[2 * i + 1]);
            x[2 * i] -= __bfloat162float(h0);  // exact: x and h agree in their leading bits
            x[2 * i + 1] -= __bfloat162float(h1);
            const __nv_bfloat162 pr = __halves2bfloat162(h0, h1);
            w[i] = *reinterpret_cast<const uint32_t*>(&pr);
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

// Copies the 32 values of logical row `row` (of `rows`), k = k0 .. k0 + 31 (of K), into
// dst[0 .. 31] with cp.async: element (row, l) at src[row * rs + l * ks]; zero outside.
// vec4: k contiguous (ks == 1) and 16-byte aligned rows (16-byte copies).
__device__ __forceinline__ void copy_row32(float* dst, const float* __restrict__ src, i64 rs, i64 ks, i64 rows,
                                           i64 K, i64 row, i64 k0, bool vec4) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    if (row < rows && vec4 && k0 + 32 <= K) {
        const float* p = src + row * rs + k0;
#pragma unroll
        for (int q = 0; q < 8; ++q)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d + 16 * q), "l"(p + 4 * q) : "memory");
        return;
    }
    const bool live = row < rows;
    const float* p = src + (live ? row * rs + k0 * ks : 0);
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        const bool v = live && k0 + l < K;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d + 4 * l), "l"(v ? p + l * ks : src),
                     "r"(v ? 4 : 0)
                     : "memory");
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
        const int r = threadIdx.x;  // tile row 0..127
        // the slabs of this CTA's tiles form one sequence; `ahead` walks it RAW_STAGES - 1
        // slabs in front of the one being split
        int at = blockIdx.x, akb = 0;  // look-ahead cursor: tile and slab
        auto issue_next = [&](int slot) {
            while (at < ntiles && akb >= tiles[at].nkb) {
                at += gridDim.x;
                akb = 0;
            }
            if (at < ntiles) {
                const TcTile tl = tiles[at];
                const TcDesc d = probs[tl.prob];
                const i64 m0 = i64(tl.tm) * BM, n0 = i64(tl.tn) * d.bn, k0 = i64(akb) * GBK;
                float* ra = raw + slot * (GRAW_BYTES / 4) + r * GRAW_LD;
                float* rb = ra + BM * GRAW_LD;
                // op(A)(i, l): A^T -> a[l + i lda] (k contiguous), else a[i + l lda]
                copy_row32(ra, d.a, d.ta ? d.lda : 1, d.ta ? 1 : d.lda, d.m, d.k, m0 + r, k0,
                           d.ta && d.lda % 4 == 0 && reinterpret_cast<uintptr_t>(d.a) % 16 == 0);
                // op(B)^T(j, l) = op(B)(l, j): B^T -> b[j + l ldb], else b[l + j ldb] (k contiguous)
                if (r < d.bn)
                    copy_row32(rb, d.b, d.tb ? 1 : d.ldb, d.tb ? d.ldb : 1, d.n, d.k, n0 + r, k0,
                               !d.tb && d.ldb % 4 == 0 && reinterpret_cast<uintptr_t>(d.b) % 16 == 0);
                ++akb;
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");  // one group per slab, empty at the end
        };
        for (int i = 0; i < GRAW_STAGES - 1; ++i) issue_next(i);
        int it = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const int nkb = tiles[t].nkb;
            const bool brow = r < probs[tiles[t].prob].bn;
            for (int kb = 0; kb < nkb; ++kb, ++it) {
                issue_next((it + GRAW_STAGES - 1) % GRAW_STAGES);
                asm volatile("cp.async.wait_group %0;\n" ::"n"(GRAW_STAGES - 1) : "memory");  // slab `it` landed
                const float* ra = raw + (it % GRAW_STAGES) * (GRAW_BYTES / 4) + r * GRAW_LD;
                const float* rb = ra + BM * GRAW_LD;
                const int s = it % C::STAGES;
                if (!mbar_wait(&empty[s], ((it / C::STAGES) & 1) ^ 1, err, 31)) { ok = false; break; }
                uint8_t* sa = smem + s * C::STAGE_BYTES;
                uint8_t* sb = sa + TERMS * C::A_PLANE;
                float v[16];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 f = reinterpret_cast<const float4*>(ra + 16 * h)[q];
                        v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
                    }
                    split_store16<TERMS>(v, sa, C::A_PLANE, r, 2 * h);
                }
                if (brow) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float4 f = reinterpret_cast<const float4*>(rb + 16 * h)[q];
                            v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
                        }
                        split_store16<TERMS>(v, sb, C::B_PLANE, r, 2 * h);
                    }
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
        const int e = warp - (GPROD_WARPS + 1);
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
#pragma unroll
                for (int j = 0; j < GBN / 2; ++j) {
                    const i64 col = cbase + j;
                    if (j < epi_cols && col < d.n) {
                        float* cp = d.c + row + col * d.ldc;
                        const float v = d.alpha * acc[j];
                        *cp = (d.beta == 0.0f) ? v : fmaf(d.beta, *cp, v);
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
