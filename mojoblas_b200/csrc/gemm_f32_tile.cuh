// Pipelined FP32 GEMM tile (CUDA cores), shared by the plain FP32 kernel
// (gemm_f32.cu) and the grouped sgemm plans (grouped.cu).
//
// One 256-thread CTA computes an FT x FT tile of C (FT = 128: 8 x 8 register
// block per thread, rows tx*4+{0..3} and 64+tx*4+{0..3}, columns likewise from
// ty; FT = 64: 4 x 4), one FMA per product (two products per fma.rn.f32x2
// instruction), each element's sum running over k in ascending order as in the
// reference's column loops.  K advances in slabs of 16
// through a 3-stage cp.async pipeline straight into shared memory: an operand
// contiguous along m (n), 16-byte aligned with ld % 4 == 0, is copied 16 bytes
// at a time, any other operand element by element into the same k-major tiles
// (rows padded to FT + 4 floats).  beta == 0 writes C without reading it,
// beta == 1 adds with an L2 reduction (one add per element, the same rounding
// as fma(1, c, v)).
#pragma once

#include "mbg_internal.cuh"

namespace mbg {
namespace f32t {

constexpr int FK = 16, FSTAGES = 3, FNT = 256;
template <int FT> struct FTile {
    static constexpr int LD = FT + 4;     // tile row (floats)
    static constexpr int TM = FT / 16;    // rows (and columns) per thread: 8 or 4
};

__device__ __forceinline__ void cpa4(void* dst, const void* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
// 16 bytes of which the first `bytes` are read, the rest zero-filled
__device__ __forceinline__ void cpa16(void* dst, const void* src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Two fp32 values in one 64-bit register, and the packed FMA of sm_100 (fma.rn.f32x2:
// two independent IEEE fused multiply-adds, so every element's arithmetic is that of fmaf).
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void f2_fma(unsigned long long& acc, unsigned long long a, unsigned long long b) {
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void f32_tri_tile(i64 t, i64& ti, i64& tj) {
    i64 r = (i64)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    ti = r;
    tj = t - r * (r + 1) / 2;
}

// Copies one FK-deep slab of an operand into a [k][FLD] tile.  MAJ: the operand
// is contiguous along the tile's row index (m or n) in memory; else along k.
// VEC: 16-byte copies along the contiguous index.
template <int FT, bool MAJ, bool VEC>
__device__ __forceinline__ void f32_stage(float* tile, const float* __restrict__ P, i64 ld, i64 r0, i64 rows,
                                          i64 k0, i64 k, int tid) {
    constexpr int FLD = FTile<FT>::LD;
    if (MAJ && VEC) {  // 4 consecutive rows of one k per copy
#pragma unroll
        for (int e0 = tid; e0 < FT * FK / 4; e0 += FNT) {
            const int e = e0 * 4, i = e % FT, l = e / FT;
            const i64 gi = r0 + i, gl = k0 + l;
            const i64 left = (gl < k) ? rows - gi : 0;
            const int bytes = left >= 4 ? 16 : (left > 0 ? int(left) * 4 : 0);
            cpa16(tile + l * FLD + i, bytes ? P + gi + gl * ld : P, bytes);
        }
    } else {
#pragma unroll
        for (int e = tid; e < FT * FK; e += FNT) {
            int i, l;
            if (MAJ) { i = e % FT; l = e / FT; } else { l = e % FK; i = e / FK; }  // contiguous index first
            const i64 gi = r0 + i, gl = k0 + l;
            const bool v = gi < rows && gl < k;
            cpa4(tile + l * FLD + i, v ? (MAJ ? P + gi + gl * ld : P + gl + gi * ld) : P, v);
        }
    }
}

// One FT x FT tile (tm, tn) of C := alpha op(A) op(B) + beta C by the whole CTA,
// staging through `fsm` (f32_smem<FT>() bytes); every copy it issued has landed
// when it returns.  band (KB_*): one operand triangular, only the tile's slabs run.
template <int FT, bool TA, bool TB, int TRI, bool VA, bool VB>
__device__ __forceinline__ void f32_tile(i64 m, i64 n, i64 k, float alpha, const float* __restrict__ A, i64 lda,
                                         const float* __restrict__ B, i64 ldb, float beta, float* __restrict__ C,
                                         i64 ldc, i64 tm, i64 tn, float* fsm, int band = KB_NONE) {
    constexpr int FLD = FTile<FT>::LD, TM = FTile<FT>::TM;
    float* As = fsm;                               // [stage][k][FLD]
    float* Bs = fsm + size_t(FSTAGES) * FK * FLD;  // [stage][k][FLD]
    const i64 m0 = tm * FT, n0 = tn * FT;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

    // op(A) is m-contiguous when A is not transposed; op(B) is n-contiguous when B is
    auto issue = [&](i64 kt, int st) {
        f32_stage<FT, !TA, VA>(As + size_t(st) * FK * FLD, A, lda, m0, m, kt * FK, k, tid);
        f32_stage<FT, TB, VB>(Bs + size_t(st) * FK * FLD, B, ldb, n0, n, kt * FK, k, tid);
    };

    // accumulators in pairs of adjacent columns: accp[i][jp] = (acc[i][2 jp], acc[i][2 jp + 1])
    unsigned long long accp[TM][TM / 2];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM / 2; ++j) accp[i][j] = 0ull;

    // slabs [kt0, kt0 + nk) of the reduction: all of them, or the tile's band
    i64 kt0 = 0, kt1 = (k + FK - 1) / FK;
    if (band != KB_NONE) band_slabs(band, m0, FT, n0, FT, 0, FK, kt1, kt0, kt1);
    const i64 nk = kt1 - kt0;
#pragma unroll
    for (int s = 0; s < FSTAGES - 1; ++s) {
        if (s < nk) issue(kt0 + s, s);
        cpa_commit();
    }
    for (i64 kt = 0; kt < nk; ++kt) {
        cpa_wait<FSTAGES - 2>();
        __syncthreads();  // slab kt has landed; the buffer of slab kt - 1 is free
        if (kt + FSTAGES - 1 < nk) issue(kt0 + kt + FSTAGES - 1, int((kt + FSTAGES - 1) % FSTAGES));
        cpa_commit();
        const float* as = As + size_t(kt % FSTAGES) * FK * FLD;
        const float* bs = Bs + size_t(kt % FSTAGES) * FK * FLD;
#pragma unroll
        for (int l = 0; l < FK; ++l) {
            // b in pairs of adjacent columns straight from the 16-byte loads; each a duplicated
            // into both halves, so one packed FMA updates two columns of a row
            float a[TM];
            unsigned long long bp[TM / 2];
            const float4 a0 = *reinterpret_cast<const float4*>(as + l * FLD + tx * 4);
            const ulonglong2 b0 = *reinterpret_cast<const ulonglong2*>(bs + l * FLD + ty * 4);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
            bp[0] = b0.x; bp[1] = b0.y;
            if constexpr (TM == 8) {
                const float4 a1 = *reinterpret_cast<const float4*>(as + l * FLD + 64 + tx * 4);
                const ulonglong2 b1 = *reinterpret_cast<const ulonglong2*>(bs + l * FLD + 64 + ty * 4);
                a[TM - 4] = a1.x; a[TM - 3] = a1.y; a[TM - 2] = a1.z; a[TM - 1] = a1.w;
                bp[2] = b1.x; bp[3] = b1.y;
            }
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                const unsigned long long ai = f2_pack(a[i], a[i]);
#pragma unroll
                for (int j = 0; j < TM / 2; ++j) f2_fma(accp[i][j], ai, bp[j]);
            }
        }
    }
    cpa_wait<0>();

    float acc[TM][TM];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM / 2; ++j) f2_unpack(accp[i][j], acc[i][2 * j], acc[i][2 * j + 1]);

#pragma unroll
    for (int j = 0; j < TM; ++j) {
        const i64 gj = n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
        if (gj >= n) continue;
        float cv[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const i64 gi = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            cv[i] = (gi < m && beta != 0.0f && beta != 1.0f) ? C[gi + gj * ldc] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const i64 gi = m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
            if (gi >= m) continue;
            if (TRI == 1 && gi < gj) continue;
            if (TRI == 2 && gi > gj) continue;
            float* cp = C + gi + gj * ldc;
            const float v = alpha * acc[i][j];
            if (beta == 0.0f) *cp = v;
            else if (beta == 1.0f) atomicAdd(cp, v);
            else *cp = fmaf(beta, cv[i], v);
        }
    }
}

template <int FT>
constexpr size_t f32_smem() { return sizeof(float) * size_t(FSTAGES) * FK * FTile<FT>::LD * 2; }

// 16-byte copies need the operand contiguous along m (n), a 16-byte aligned base and ld % 4 == 0
__host__ __device__ inline bool f32_vec(bool contiguous_rows, const float* p, i64 ld) {
    return contiguous_rows && reinterpret_cast<uintptr_t>(p) % 16 == 0 && ld % 4 == 0;
}

}  // namespace f32t
}  // namespace mbg
