// PTX helpers for the tcgen05 / TMA kernels (tc_gemm.cu, grouped_tc.cu): mbarriers
// with bounded waits, TMA loads, TMEM allocation, tcgen05.mma / commit / ld, and
// the shared-memory matrix and instruction descriptors.
#pragma once

#include "mbg_internal.cuh"

#include <cuda.h>

namespace mbg {
namespace tc {

constexpr int BM = 128;
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int site,
                                          uint64_t limit_ns = WAIT_LIMIT_NS) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (true) {
#pragma unroll 1
        for (int i = 0; i < 256; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer() - t0 > limit_ns) {
            if (err) {
                atomicExch(err, 1);
                atomicExch(err + 1, site);
            }
            return false;
        }
    }
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0,
                                            int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// COLLECTOR: 0 = read A from shared memory only, 1 = fill the tensor core's A
// collector buffer, 2 = reuse it, 3 = reuse it for the last time.  Consecutive
// MMAs with the same A tile (Ozaki products A_p B_q for one p) read A once.
#define MBG_UMMA(KIND, COL)                                                        \
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"                \
                 "tcgen05.mma.cta_group::1.kind::" KIND COL " [%0], %1, %2, %3, p;\n\t}" \
                 ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)  \
                 : "memory")
template <bool INT8>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                     uint32_t accumulate, int collector = 0) {
    if (INT8) {
        if (collector == 1) MBG_UMMA("i8", ".collector::a::fill");
        else if (collector == 2) MBG_UMMA("i8", ".collector::a::use");
        else if (collector == 3) MBG_UMMA("i8", ".collector::a::lastuse");
        else MBG_UMMA("i8", "");
    } else {
        MBG_UMMA("f16", "");
    }
}
#undef MBG_UMMA
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor (tcgen05), K-major operand with swizzle:
// start address and stride-dimension byte offset (between 8-row groups) in
// 16-byte units, descriptor version 1 (bits 46-47), layout type in bits 61-63
// (2 = 128-byte swizzle, 4 = 64-byte, 6 = 32-byte).  Tiles are 1024-byte
// aligned so the base-offset field stays 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t sbo_bytes, uint32_t layout) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t(1) << 16;  // leading byte offset: unused for swizzled K-major tiles
    d |= uint64_t((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    d |= uint64_t(layout & 7u) << 61;
    return d;
}

// Instruction descriptor: D format (bits 4-5: 1 = f32, 2 = s32), A/B formats
// (bits 7-9 / 10-12: bf16 = 1 for kind::f16, signed = 1 for kind::i8), both
// operands K-major (bits 15/16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t instr_desc(bool int8, int M, int N) {
    return (uint32_t(int8 ? 2 : 1) << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) |
           (uint32_t(M >> 4) << 24);
}

// 2^e as a double: built from the exponent bits in the normal range (exact, no
// libm call), ldexp outside it.
__device__ __forceinline__ double pow2_exact(int e) {
    if (e >= -1022 && e <= 1023) return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
    return ldexp(1.0, e);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Product table, index -> (p, q) and collector use.
//   split: ordered by descending p+q so small contributions enter the fp32
//          accumulator first;
//   ozaki: ordered by p (A slice), q ascending, so the products that share A_p
//          run back to back and reuse it from the collector buffer; the first
//          product into diagonal d is then (0, d).
template <int TERMS, bool OZAKI>
__device__ __forceinline__ void product(int idx, int& p, int& q, int& collector) {
    collector = 0;
    if (OZAKI) {
        int t = 0;
        for (int pp = 0; pp < TERMS; ++pp) {
            const int cnt = TERMS - pp;  // q = 0 .. TERMS-1-pp
            if (idx < t + cnt) {
                p = pp;
                q = idx - t;
                if (cnt > 1) collector = (q == 0) ? 1 : (q == cnt - 1 ? 3 : 2);
                return;
            }
            t += cnt;
        }
        p = q = 0;
        return;
    }
    int t = 0;
    for (int d = TERMS - 1; d >= 0; --d) {
        for (int pp = 0; pp <= d; ++pp) {
            if (t == idx) { p = pp; q = d - pp; return; }
            ++t;
        }
    }
    p = q = 0;
}

}  // namespace tc
}  // namespace mbg
