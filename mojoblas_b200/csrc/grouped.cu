// Grouped (batched) gemm and trsm: thousands of independent problems of uneven
// sizes in one persistent launch per problem type.
//
// The reference has no batched interface; a mojoBLAS caller loops over its
// gemm (src/level3/gemm.mojo:56) / trsm (src/level3/trsm.mojo:20) calls.  Here
// a host-side plan uploads a problem table once, and each execution is a CUDA
// graph of [reset the tile counter; one persistent kernel]:
//
//  * sgemm: problems are ordered by k * m * n descending and cut into square
//    tiles (64 or 128, from the tuning table); persistent CTAs take tiles from
//    an atomic counter (largest first, so the tail is short), locate the problem
//    by binary search over the tile prefix sums, and run the pipelined FP32
//    tile code of gemm_f32_tile.cuh with that problem's transposes, alpha and
//    beta (16-byte copies where that problem's operands allow them).
//  * strsm (left side, any uplo / trans / diag, n <= 256): problems are cut
//    into strips of 32 right-hand sides, ordered largest problem first;
//    persistent CTAs take strips from an atomic counter and solve each with
//    the blocked trsm's fused diagonal-block routine (block_solve.cuh): the
//    strip in shared memory, the reference's column substitution
//    (src/level3/trsm.mojo:111-168) on 64-row sub-blocks with the pivot
//    broadcast by a shuffle and multiplied by a precomputed reciprocal, and the
//    updates between sub-blocks from cp.async-staged tiles of op(A).
#include "mbg_internal.cuh"
#include "block_solve.cuh"
#include "gemm_f32_tile.cuh"

#include <algorithm>
#include <numeric>
#include <vector>

namespace mbg {

namespace {

struct GemmDesc {  // device copy of one problem
    i64 m, n, k, lda, ldb, ldc;
    const float* a;
    const float* b;
    float* c;
    float alpha, beta;
    int ta, tb;
    i64 tile0;   // first tile index of this problem
    int tiles_m;  // tiles along m
};

constexpr int GT_NT = f32t::FNT;

// Runs one tile of problem d with the pipelined FP32 tile code; the 16-byte copy
// path is chosen per problem (operand contiguity, alignment and leading dimension).
template <int TILE, bool TA, bool TB>
__device__ __forceinline__ void grouped_tile(const GemmDesc& d, i64 tm, i64 tn, float* gsm) {
    const bool va = f32t::f32_vec(!TA, d.a, d.lda), vb = f32t::f32_vec(TB, d.b, d.ldb);
#define GT(VA, VB) \
    f32t::f32_tile<TILE, TA, TB, 0, VA, VB>(d.m, d.n, d.k, d.alpha, d.a, d.lda, d.b, d.ldb, d.beta, d.c, d.ldc, tm, tn, gsm)
    if (va && vb) GT(true, true);
    else if (va) GT(true, false);
    else if (vb) GT(false, true);
    else GT(false, false);
#undef GT
}

template <int TILE>
__global__ void __launch_bounds__(GT_NT, TILE == 128 ? 1 : 3)
grouped_sgemm_kernel(const GemmDesc* __restrict__ probs, int count, i64 total_tiles,
                     unsigned long long* __restrict__ counter) {
    extern __shared__ __align__(16) float gsm[];  // f32t::f32_smem<TILE>() bytes
    __shared__ long long s_tile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const i64 t = s_tile;
        __syncthreads();  // every thread has read s_tile before it is overwritten
        if (t >= total_tiles) return;
        // problem owning tile t: the last with tile0 <= t
        int lo = 0, hi = count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (probs[mid].tile0 <= t) lo = mid; else hi = mid - 1;
        }
        const GemmDesc d = probs[lo];  // registers
        const i64 local = t - d.tile0;
        const i64 tm = local % d.tiles_m, tn = local / d.tiles_m;
        if (d.k == 0 || d.alpha == 0.0f) {  // C := beta*C on this tile
            for (int e = threadIdx.x; e < TILE * TILE; e += GT_NT) {
                const i64 gi = tm * TILE + e % TILE, gj = tn * TILE + e / TILE;
                if (gi < d.m && gj < d.n) {
                    float* cp = d.c + gi + gj * d.ldc;
                    *cp = (d.beta == 0.0f) ? 0.0f : d.beta * *cp;
                }
            }
        } else if (!d.ta && !d.tb) grouped_tile<TILE, false, false>(d, tm, tn, gsm);
        else if (!d.ta && d.tb) grouped_tile<TILE, false, true>(d, tm, tn, gsm);
        else if (d.ta && !d.tb) grouped_tile<TILE, true, false>(d, tm, tn, gsm);
        else grouped_tile<TILE, true, true>(d, tm, tn, gsm);
        __syncthreads();  // shared tiles are reused by the next tile
    }
}

struct TrsmDesc {
    i64 n, nrhs, lda, ldb;
    const float* a;
    float* b;
    float alpha;
    int lower, trans, unit;  // lower: effective op(A) lower triangular
    i64 col0;                // first global column index of this problem
};

constexpr int TR_MAXN = 256;  // largest problem order a grouped strsm plan takes
constexpr int GS_NBUF = 3;    // staging buffers per strip of the fused block solve

// One unit of grouped-strsm work: a strip of up to bs::BS_COLS right-hand sides of one problem.
struct TrsmItem {
    int prob;
    int pad_;
    i64 c0;
};

// Persistent grouped strsm: each CTA takes (problem, strip) items from an atomic
// counter — the plan orders them largest problem first, so the long solves start
// early and the small ones fill in behind them — and solves each with the fused
// diagonal-block routine of the blocked trsm: the strip in shared memory, 64-row
// substitution sub-blocks, cp.async-staged tiles of op(A), alpha applied to the
// strip as it lands.
__global__ void __launch_bounds__(bs::BS_THREADS, 2)
grouped_block_strsm_kernel(const TrsmDesc* __restrict__ probs, const TrsmItem* __restrict__ items, int nitems,
                           unsigned long long* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char gs_smem[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = int(atomicAdd(counter, 1ULL));
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has read s_item before thread 0 writes the next one
        if (it >= nitems) break;
        const TrsmItem w = items[it];
        const TrsmDesc d = probs[w.prob];
        const int nb = int(d.n);
#define GS(L, TR, U)                                                                                  \
    bs::block_solve_strip<float, L, TR, U, bs::BS_COLS, GS_NBUF>(nb, d.nrhs, d.a, d.lda, d.b, d.ldb, w.c0, d.alpha, gs_smem)
        switch ((d.lower ? 4 : 0) | (d.trans ? 2 : 0) | (d.unit ? 1 : 0)) {
            case 0: GS(false, false, false); break;
            case 1: GS(false, false, true); break;
            case 2: GS(false, true, false); break;
            case 3: GS(false, true, true); break;
            case 4: GS(true, false, false); break;
            case 5: GS(true, false, true); break;
            case 6: GS(true, true, false); break;
            default: GS(true, true, true); break;
        }
#undef GS
    }
}

// SMs of the current device (queried per plan: plans are built once, off the hot path)
int num_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        sms = 148;
    }
    return sms;
}

}  // namespace

}  // namespace mbg

// ---- plans ------------------------------------------------------------------------
struct mbg_plan {
    int kind = 0;  // 1 sgemm, 2 strsm
    void* table = nullptr;                 // device problem table
    unsigned long long* counter = nullptr;  // device tile counter
    int count = 0;
    i64 total = 0;       // tiles (sgemm) or columns (strsm)
    int tile = 64;
    int grid = 0;
    // sgemm, plain form: the problems whose size class takes 128-tiles (the 64-tile ones are above)
    void* table128 = nullptr;
    unsigned long long* counter128 = nullptr;
    int count128 = 0;
    i64 total128 = 0;
    int grid128 = 0;
    // sgemm, split forms (BF16x3 / BF16x6): the tensor-core grouped kernel
    bool tc = false;
    mbg::GroupedTcPlan tcp;
    void* items = nullptr;  // strsm: (problem, strip) work items, inside the table allocation
    int nitems = 0;
    size_t smem = 0;        // strsm: dynamic shared memory per CTA
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;  // stream the graph was captured on
};

namespace mbg {
namespace {

// Enqueues the plan's work on stream s (the capture stream: the library stream that
// other host threads may be using is never touched).
int enqueue_plan(mbg_plan* p, cudaStream_t s) {
    if (p->kind == 1 && p->tc) return grouped_tc_enqueue(p->tcp, s);
    if (p->kind == 1) {
        // the 128-tile problems (the larger size classes) first, the 64-tile ones behind them
        if (p->count128 > 0) {
            MBG_CUDA(cudaMemsetAsync(p->counter128, 0, sizeof(unsigned long long), s));
            grouped_sgemm_kernel<128><<<p->grid128, GT_NT, f32t::f32_smem<128>(), s>>>(
                static_cast<const GemmDesc*>(p->table128), p->count128, p->total128, p->counter128);
            MBG_TRY(check_launch("grouped_sgemm"));
        }
        if (p->count > 0) {
            MBG_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), s));
            grouped_sgemm_kernel<64><<<p->grid, GT_NT, f32t::f32_smem<64>(), s>>>(
                static_cast<const GemmDesc*>(p->table), p->count, p->total, p->counter);
            MBG_TRY(check_launch("grouped_sgemm"));
        }
        return MBG_OK;
    }
    MBG_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), s));
    grouped_block_strsm_kernel<<<p->grid, bs::BS_THREADS, p->smem, s>>>(
        static_cast<const TrsmDesc*>(p->table), static_cast<const TrsmItem*>(p->items), p->nitems, p->counter);
    return check_launch("grouped_strsm");
}

// Records the plan's work into a CUDA graph on a private capture stream.  The
// library's stream setting is left alone, so calls that other host threads make
// meanwhile stay on their stream and out of this graph.
int capture_plan(mbg_plan* p) {
    cudaStream_t cap = nullptr;
    MBG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    int st = MBG_OK;
    if (e == cudaSuccess) {
        st = enqueue_plan(p, cap);
        e = cudaStreamEndCapture(cap, &p->graph);
    }
    cudaStreamDestroy(cap);
    if (e != cudaSuccess) {
        set_error("graph capture of a grouped plan", e);
        return MBG_ERR_CUDA;
    }
    if (st) return st;
    MBG_CUDA(cudaGraphInstantiate(&p->exec, p->graph, 0));
    return MBG_OK;
}

template <typename D>
int upload(mbg_plan* p, const std::vector<D>& v) {
    MBG_CUDA(cudaMalloc(&p->table, sizeof(D) * v.size()));
    MBG_CUDA(cudaMemcpy(p->table, v.data(), sizeof(D) * v.size(), cudaMemcpyHostToDevice));
    return MBG_OK;
}

}  // namespace
}  // namespace mbg

using namespace mbg;

extern "C" {

int mbg_sgemm_grouped_plan(int mode, int count, const mbg_sgemm_problem* probs, mbg_plan** out) {
    if (!out) return MBG_ERR_INVALID_MODE;
    *out = nullptr;
    if (mode != MBG_MODE_PLAIN && mode != MBG_MODE_BF16X3 && mode != MBG_MODE_BF16X6) return MBG_ERR_INVALID_MODE;
    if (count < 0 || (count > 0 && !probs)) return MBG_ERR_INVALID_MODE;
    for (int i = 0; i < count; ++i) {  // argument checks per problem, numbered as gemm numbers them
        const mbg_sgemm_problem& q = probs[i];
        const char ta = q.trans_a, tb = q.trans_b;
        int info = 0;
        if (!is_n(ta) && !is_t(ta)) info = 1;
        else if (!is_n(tb) && !is_t(tb)) info = 2;
        else if (q.m < 0) info = 3;
        else if (q.n < 0) info = 4;
        else if (q.k < 0) info = 5;
        else if (q.lda < imax(1, is_n(ta) ? q.m : q.k)) info = 8;
        else if (q.ldb < imax(1, is_n(tb) ? q.k : q.n)) info = 10;
        else if (q.ldc < imax(1, q.m)) info = 13;
        if (info) {
            set_error_msg("grouped sgemm: problem " + std::to_string(i) + " has invalid argument " +
                          std::to_string(info));
            return info;
        }
        if (q.m > 0 && q.n > 0 && (!is_device_pointer(q.c) ||
                                    (q.k > 0 && (!is_device_pointer(q.a) || !is_device_pointer(q.b))))) {
            set_error_msg("grouped sgemm: problem " + std::to_string(i) + " has a host pointer (device only)");
            return MBG_ERR_UNSUPPORTED;
        }
    }
    if (mode != MBG_MODE_PLAIN) {  // split forms: one tensor-core kernel over every problem
        mbg_plan* p = new mbg_plan();
        p->kind = 1;
        p->tc = true;
        int st = grouped_tc_build(mode == MBG_MODE_BF16X6 ? 3 : 2, count, probs, p->tcp);
        p->count = p->tcp.count;
        if (!st && p->tcp.ntiles > 0) st = capture_plan(p);
        if (st) {
            mbg_plan_destroy(p);
            return st;
        }
        *out = p;
        return MBG_OK;
    }
    // plain form: each problem's tile edge from its size class in the tuning table, the
    // largest problems first within each tile size (the tail of the schedule is short tiles)
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const double cx = double(probs[x].m) * probs[x].n * imax(probs[x].k, 1);
        const double cy = double(probs[y].m) * probs[y].n * imax(probs[y].k, 1);
        return cx > cy;
    });
    std::vector<GemmDesc> v[2];  // [0]: 64-tiles, [1]: 128-tiles
    i64 tiles[2] = {0, 0};
    for (int idx : order) {
        const mbg_sgemm_problem& q = probs[idx];
        if (q.m == 0 || q.n == 0) continue;
        const int tile = grouped_simt_tile(q.m, q.n, is_t(q.trans_a), is_t(q.trans_b));
        const int w = tile == 128 ? 1 : 0;
        GemmDesc d{};
        d.m = q.m; d.n = q.n; d.k = q.k; d.lda = q.lda; d.ldb = q.ldb; d.ldc = q.ldc;
        d.a = q.a; d.b = q.b; d.c = q.c; d.alpha = q.alpha; d.beta = q.beta;
        d.ta = is_t(q.trans_a); d.tb = is_t(q.trans_b);
        d.tiles_m = int(cdiv(q.m, tile));
        d.tile0 = tiles[w];
        tiles[w] += i64(d.tiles_m) * cdiv(q.n, tile);
        v[w].push_back(d);
    }
    mbg_plan* p = new mbg_plan();
    p->kind = 1;
    p->count = int(v[0].size());
    p->total = tiles[0];
    p->count128 = int(v[1].size());
    p->total128 = tiles[1];
    int per_sm64 = 1, per_sm128 = 1;
    // dynamic shared memory above 48 KB needs the opt-in before the occupancy query and the launch
    cudaFuncSetAttribute(grouped_sgemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(f32t::f32_smem<128>()));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm128, grouped_sgemm_kernel<128>, GT_NT,
                                                  f32t::f32_smem<128>());
    cudaFuncSetAttribute(grouped_sgemm_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(f32t::f32_smem<64>()));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm64, grouped_sgemm_kernel<64>, GT_NT, f32t::f32_smem<64>());
    cudaGetLastError();
    p->grid = int(imax(1, imin(tiles[0], i64(num_sms()) * imax(per_sm64, 1))));
    p->grid128 = int(imax(1, imin(tiles[1], i64(num_sms()) * imax(per_sm128, 1))));
    int st = MBG_OK;
    auto upload_part = [&](const std::vector<GemmDesc>& vv, void** table, unsigned long long** counter) -> int {
        if (vv.empty()) return MBG_OK;
        MBG_CUDA(cudaMalloc(table, sizeof(GemmDesc) * vv.size()));
        MBG_CUDA(cudaMemcpy(*table, vv.data(), sizeof(GemmDesc) * vv.size(), cudaMemcpyHostToDevice));
        MBG_CUDA(cudaMalloc(reinterpret_cast<void**>(counter), sizeof(unsigned long long)));
        return MBG_OK;
    };
    st = upload_part(v[0], &p->table, &p->counter);
    if (!st) st = upload_part(v[1], &p->table128, &p->counter128);
    if (!st && (p->count + p->count128) > 0) st = capture_plan(p);
    if (st) {
        mbg_plan_destroy(p);
        return st;
    }
    p->count += p->count128;
    *out = p;
    return MBG_OK;
}

int mbg_strsm_grouped_plan(int mode, int count, const mbg_strsm_problem* probs, mbg_plan** out) {
    if (!out) return MBG_ERR_INVALID_MODE;
    *out = nullptr;
    if (mode != MBG_MODE_PLAIN) {
        set_error_msg("grouped strsm: only MBG_MODE_PLAIN is implemented");
        return MBG_ERR_UNSUPPORTED;
    }
    if (count < 0 || (count > 0 && !probs)) return MBG_ERR_INVALID_MODE;
    std::vector<TrsmDesc> v;
    v.reserve(count);
    i64 cols = 0;
    for (int i = 0; i < count; ++i) {
        const mbg_strsm_problem& q = probs[i];
        int info = 0;  // numbered as trsm numbers them (src/level3/trsm.mojo:62-89)
        if (!is_l(q.side) && !is_r(q.side)) info = 1;
        else if (!is_u(q.uplo) && !is_l(q.uplo)) info = 2;
        else if (!is_n(q.trans_a) && !is_t(q.trans_a)) info = 3;
        else if (!is_u(q.diag) && !is_n(q.diag)) info = 4;
        else if (q.m < 0) info = 5;
        else if (q.n < 0) info = 6;
        else if (q.lda < imax(1, is_l(q.side) ? q.m : q.n)) info = 9;
        else if (q.ldb < imax(1, q.m)) info = 11;
        if (info) {
            set_error_msg("grouped strsm: problem " + std::to_string(i) + " has invalid argument " +
                          std::to_string(info));
            return info;
        }
        if (q.m > 0 && q.n > 0 && (!is_device_pointer(q.a) || !is_device_pointer(q.b))) {
            set_error_msg("grouped strsm: problem " + std::to_string(i) + " has a host pointer (device only)");
            return MBG_ERR_UNSUPPORTED;
        }
        if (is_r(q.side) || q.m > TR_MAXN) {
            set_error_msg("grouped strsm: left side with m <= 256 only (problem " + std::to_string(i) + ")");
            return MBG_ERR_UNSUPPORTED;
        }
        if (q.m == 0 || q.n == 0) continue;
        TrsmDesc d{};
        d.n = q.m; d.nrhs = q.n; d.lda = q.lda; d.ldb = q.ldb; d.a = q.a; d.b = q.b; d.alpha = q.alpha;
        d.trans = is_t(q.trans_a);
        d.lower = (!is_u(q.uplo)) != (d.trans != 0);
        d.unit = is_u(q.diag);
        d.col0 = cols;
        cols += q.n;
        v.push_back(d);
    }
    // work items: 32-column strips, largest problem first (ties keep the caller's order)
    std::vector<TrsmItem> items;
    for (int i = 0; i < int(v.size()); ++i)
        for (i64 c0 = 0; c0 < v[size_t(i)].nrhs; c0 += bs::BS_COLS) items.push_back(TrsmItem{i, 0, c0});
    std::stable_sort(items.begin(), items.end(),
                     [&](const TrsmItem& x, const TrsmItem& y) { return v[size_t(x.prob)].n > v[size_t(y.prob)].n; });
    mbg_plan* p = new mbg_plan();
    p->kind = 2;
    p->count = int(v.size());
    p->total = cols;
    p->nitems = int(items.size());
    p->smem = bs::bs_smem_bytes<float>(TR_MAXN, GS_NBUF);
    int st = MBG_OK;
    if (p->count > 0) {
        int per_sm = 0;
        cudaError_t e = cudaFuncSetAttribute(grouped_block_strsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(p->smem));
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_block_strsm_kernel, bs::BS_THREADS,
                                                              p->smem);
        if (e != cudaSuccess) {
            set_error("grouped strsm kernel set-up", e);
            st = MBG_ERR_CUDA;
        } else {
            p->grid = int(imax(1, imin(i64(items.size()), i64(num_sms()) * imax(per_sm, 1))));
            const size_t dbytes = (sizeof(TrsmDesc) * v.size() + 255) / 256 * 256;
            const size_t ibytes = sizeof(TrsmItem) * items.size();
            e = cudaMalloc(&p->table, dbytes + ibytes);
            if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->counter), sizeof(unsigned long long));
            if (e == cudaSuccess) {
                p->items = static_cast<char*>(p->table) + dbytes;
                e = cudaMemcpy(p->table, v.data(), sizeof(TrsmDesc) * v.size(), cudaMemcpyHostToDevice);
            }
            if (e == cudaSuccess) e = cudaMemcpy(p->items, items.data(), ibytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                set_error("grouped strsm plan upload", e);
                st = MBG_ERR_CUDA;
            }
        }
        if (!st) st = capture_plan(p);
    }
    if (st) {
        mbg_plan_destroy(p);
        return st;
    }
    *out = p;
    return MBG_OK;
}

int mbg_plan_execute(mbg_plan* p) {
    if (!p) return MBG_ERR_INVALID_MODE;
    if (p->count == 0) return MBG_OK;
    ProfScope prof(p->kind == 1 ? (p->tc ? "grouped_sgemm_tc" : "grouped_sgemm") : "grouped_strsm");
    MBG_CUDA(cudaGraphLaunch(p->exec, stream()));
    count_launch(1);
    return finish_call(false);
}

int mbg_plan_destroy(mbg_plan* p) {
    if (!p) return MBG_OK;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->table) cudaFree(p->table);
    if (p->counter) cudaFree(p->counter);
    if (p->table128) cudaFree(p->table128);
    if (p->counter128) cudaFree(p->counter128);
    grouped_tc_free(p->tcp);
    delete p;
    return MBG_OK;
}

int mbg_sgemm_grouped(int mode, int count, const mbg_sgemm_problem* probs) {
    mbg_plan* p = nullptr;
    MBG_TRY(mbg_sgemm_grouped_plan(mode, count, probs, &p));
    int st = mbg_plan_execute(p);
    if (!st) st = finish_call(true);  // the plan's table is freed below
    mbg_plan_destroy(p);
    return st;
}

int mbg_strsm_grouped(int mode, int count, const mbg_strsm_problem* probs) {
    mbg_plan* p = nullptr;
    MBG_TRY(mbg_strsm_grouped_plan(mode, count, probs, &p));
    int st = mbg_plan_execute(p);
    if (!st) st = finish_call(true);
    mbg_plan_destroy(p);
    return st;
}

}  // extern "C"
