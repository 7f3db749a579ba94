// Fused diagonal-block triangular solve, shared by the blocked trsm (trsm.cu)
// and the grouped strsm plans (grouped.cu).  Included by both translation units.
#pragma once

#include "mbg_internal.cuh"

namespace mbg {
namespace bs {

constexpr int NB = 64;  // substitution sub-block

template <typename T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

constexpr int BS_COLS = 32;                       // right-hand sides per CTA of block_solve_kernel
constexpr int BS_THREADS = 8 * BS_COLS;           // eight lanes per column in the substitution
constexpr int BS_TILE = NB * 72;                  // diagonal block + reciprocals (64 x 65 + 64), or a 64 x 72 tile

inline int bs_strip_ld(int nb) { return (int)(cdiv(nb, NB) * NB) + 2; }
// nbuf: staging buffers per strip (items staged nbuf - 1 ahead of the one being computed)
template <typename T>
inline size_t bs_smem_bytes(int nb, int nbuf = 2) {
    return sizeof(T) * (size_t(BS_COLS) * bs_strip_ld(nb) + size_t(nbuf) * BS_TILE);
}

// One element copied global -> shared without a register round trip; zero-filled
// (nothing read) when !valid, in which case src only has to be some valid pointer.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? (int)sizeof(T) : 0;
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Solves op(A)[0:nb, 0:nb] X = B[0:nb, :] in place, nb up to 512 (double) or
// 1024 (float) rows, in one launch.  Each CTA owns W right-hand-side columns (a
// strip) and keeps the strip's nb rows in shared memory, column-major with
// leading dimension roundup(nb, 64) + 2 (= 2 mod 16, so that the column pairs
// one warp reads fall in different banks).  It runs the recursive solve's own
// blocked substitution over 64-row sub-blocks without leaving the SM:
//   for each sub-block b (forward for lower op(A), backward for upper):
//     - solve the 64 x 64 diagonal block exactly as diag_solve_kernel does
//       (eight lanes per column, pivot broadcast by shuffle, reciprocal
//       multiply, zero pivots skipped — src/level3/trsm.mojo:130-148);
//     - subtract op(A)[t, b] X_b from every sub-block t still to be solved,
//       one 64 x 64 tile of op(A) at a time: on the FP64 tensor pipe for
//       double (mma.sync m8n8k4, each warp a 16 x 16 part of the 64 x 32
//       product), on the CUDA cores for float (each thread 4 rows x 4 columns
//       over half of the 64-long reduction, tile and X_b read as 8-byte pairs).
// The diagonal blocks and tiles form one sequence per strip that is staged
// with cp.async into NBUF rotating buffers: the next NBUF - 1 items are in flight
// while the current one is computed, so the L2 latency of A (shared by every
// CTA) is hidden.  Two for the blocked trsm (a third measured slower there); three
// for the grouped plans' small problems (measured 9 % faster).  The strip is read from and written to HBM once; only
// off-diagonal blocks above the launch's size go through gemm.  Rows at or
// past nb stay zero in the strip and staged items are zero outside op(A)'s
// block, so ragged edges need no special case in the inner loops.
// IDENT: the right-hand side is the identity (columns c0 .. of the nb x nb block inverse),
// generated in shared memory instead of read from B; B is only written.
template <typename T, bool LOWER, bool TRANS, bool UNIT, int W, int NBUF = 2, bool IDENT = false>
__device__ __forceinline__ void block_solve_strip(int nb, i64 ncols, const T* __restrict__ A, i64 lda,
                                                  T* __restrict__ B, i64 ldb, i64 c0, T alpha,
                                                  unsigned char* bs_smem_raw) {
    using P2 = typename Pair<T>::type;
    static_assert(W == 32, "the tile update maps 256 threads onto 64 rows x 32 columns x 2 halves");
    constexpr int NT = 8 * W;
    constexpr int LDL = NB + 1;               // diagonal block, interleaved rows
    constexpr int LT = TRANS ? NB + 2 : NB + 8;  // update tile: [l][r] (plain) or [r][l] (transposed)
    const int nsub = (nb + NB - 1) / NB, nbr = nsub * NB, ldbs = nbr + 2;
    T* Bs = reinterpret_cast<T*>(bs_smem_raw);
    static_assert(NBUF >= 2, "staging depth");
    T* const buf0 = Bs + (size_t)W * ldbs;  // NBUF staging buffers of BS_TILE elements
    const int tid = threadIdx.x;

    // item (step, tt): tt < 0 is the diagonal block of sub-block b(step), else its tt-th trailing tile
    auto sub_of = [&](int step) { return LOWER ? step : nsub - 1 - step; };
    auto tiles_of = [&](int b) { return LOWER ? nsub - 1 - b : b; };
    auto advance = [&](int& step, int& tt) {
        if (tt + 1 < tiles_of(sub_of(step))) ++tt; else { ++step; tt = -1; }
    };
    auto issue = [&](int step, int tt, T* buf) {
        const int b = sub_of(step), r0 = b * NB, nbb = min(NB, nb - r0);
        if (tt < 0) {
            const T* Ad = A + r0 + (i64)r0 * lda;
#pragma unroll 4
            for (int e = tid; e < NB * NB; e += NT) {
                const int fast = e & (NB - 1), slow = e >> 6;  // fast index runs along contiguous memory
                const int i = TRANS ? slow : fast, l = TRANS ? fast : slow;
                const bool v = i < nbb && l < nbb;
                cp_async_elem(buf + l * LDL + (i & 7) * 8 + (i >> 3),
                              v ? (TRANS ? Ad + l + (i64)i * lda : Ad + i + (i64)l * lda) : A, v);
            }
        } else {
            const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
#pragma unroll 4
            for (int e = tid; e < NB * NB; e += NT) {
                const int fast = e & (NB - 1), slow = e >> 6;
                // plain: buf[l][r] = A[rt0 + r, r0 + l]; transposed: buf[r][l] = A[r0 + l, rt0 + r]
                const bool v = TRANS ? (rt0 + slow < nb && fast < nbb) : (rt0 + fast < nb && slow < nbb);
                const T* src = TRANS ? A + (r0 + fast) + (i64)(rt0 + slow) * lda
                                     : A + (rt0 + fast) + (i64)(r0 + slow) * lda;
                cp_async_elem(buf + slow * LT + fast, v ? src : A, v);
            }
        }
    };

    {
#pragma unroll 4
        for (int c = 0; c < W; ++c) {
            const bool live = c0 + c < ncols;
            if constexpr (IDENT) {
                for (int r = tid; r < nbr; r += NT) Bs[c * ldbs + r] = (live && r == c0 + c) ? T(1) : T(0);
            } else {
                const T* bc = B + (live ? c0 + c : 0) * ldb;
                for (int r = tid; r < nbr; r += NT)
                    cp_async_elem(Bs + c * ldbs + r, live && r < nb ? bc + r : B, live && r < nb);
            }
        }
        issue(0, -1, buf0);
        cp_async_commit();  // group 0: the strip and item 0; group g: item g (empty past the last)
        int is = 0, itt = -1;  // the last item issued
        for (int j = 1; j < NBUF - 1; ++j) {
            advance(is, itt);
            if (is < nsub) issue(is, itt, buf0 + j * BS_TILE);
            cp_async_commit();
        }
        int step = 0, tt = -1;
        for (int it = 0; step < nsub; ++it) {
            T* cur = buf0 + (it % NBUF) * BS_TILE;
            cp_async_wait_group<NBUF - 2>();
            __syncthreads();  // item `it` has landed everywhere; item it - 1's buffer is free
            if (it == 0 && alpha != T(1)) {  // the strip has landed: B := alpha B
                for (int e = tid; e < W * ldbs; e += NT) Bs[e] *= alpha;
                __syncthreads();
            }
            advance(is, itt);
            if (is < nsub) issue(is, itt, buf0 + ((it + NBUF - 1) % NBUF) * BS_TILE);
            cp_async_commit();
            int ns = step, nt = tt;
            advance(ns, nt);
            const int b = sub_of(step), r0 = b * NB, nbb = min(NB, nb - r0);
            if (tt < 0) {
                // ---- diagonal sub-block: substitution ----
                T* inv = cur + NB * LDL;
                for (int l = tid; l < nbb; l += NT) inv[l] = UNIT ? T(1) : T(1) / cur[l * LDL + (l & 7) * 8 + (l >> 3)];
                __syncthreads();
                const int q = tid & 7;
                T* bc = Bs + (tid >> 3) * ldbs + r0;
                T x[8];
#pragma unroll
                for (int s = 0; s < 8; ++s) x[s] = bc[q * 8 + s];
#pragma unroll
                for (int u = 0; u < NB; ++u) {
                    const int l = LOWER ? u : NB - 1 - u;
                    if (l >= nbb) continue;  // uniform
                    const int owner = l >> 3, slot = l & 7;
                    T xl = __shfl_sync(0xffffffffu, x[slot], owner, 8);
                    const bool live = xl != T(0);  // the reference skips zero pivots
                    if (!UNIT) xl *= inv[l];
                    if (q == owner && live) x[slot] = xl;
                    const T* col = cur + l * LDL;
#pragma unroll
                    for (int s = 0; s < 8; ++s) {
                        const int r = q * 8 + s;
                        const bool below = LOWER ? (r > l) : (r < l);
                        const T a = col[s * 8 + q];
                        if (live && below) x[s] -= xl * a;
                    }
                }
#pragma unroll
                for (int s = 0; s < 8; ++s)
                    if (q * 8 + s < nbb) bc[q * 8 + s] = x[s];
            } else {
                // ---- trailing tile: B_t -= op(A)[t, b] X_b ----
                if constexpr (sizeof(T) == 8) {
                    // FP64 tensor-core MMA (m8n8k4): warp w owns rows 16 (w % 4) .. +16
                    // and columns 16 (w / 4) .. +16 of the 64 x 32 product, 2 x 2
                    // fragments, the full 64-long reduction in registers.  Fragment
                    // loads: A[row = lane / 4][k = lane % 4], X[k = lane % 4][col =
                    // lane / 4]; with the tile's leading dimension (72 or 66) and the
                    // strip's (2 mod 16) each is two wavefronts, the minimum for 256 B.
                    const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
                    const int lane = tid & 31, w = tid >> 5;
                    const int m0 = 16 * (w & 3), n0 = 16 * (w >> 2);
                    const int lr = lane >> 2, lk = lane & 3;
                    double d[2][2][2];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int nj = 0; nj < 2; ++nj) d[mi][nj][0] = d[mi][nj][1] = 0.0;
                    const double* tile = reinterpret_cast<const double*>(cur);
                    const double* xs = reinterpret_cast<const double*>(Bs) + r0;
#pragma unroll 4
                    for (int k0 = 0; k0 < NB; k0 += 4) {
                        double af[2], bf[2];
#pragma unroll
                        for (int mi = 0; mi < 2; ++mi) {
                            const int r = m0 + 8 * mi + lr, k = k0 + lk;
                            af[mi] = TRANS ? tile[r * LT + k] : tile[k * LT + r];
                        }
#pragma unroll
                        for (int nj = 0; nj < 2; ++nj) bf[nj] = xs[(n0 + 8 * nj + lr) * ldbs + k0 + lk];
#pragma unroll
                        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                            for (int nj = 0; nj < 2; ++nj)
                                asm volatile(
                                    "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                                    : "+d"(d[mi][nj][0]), "+d"(d[mi][nj][1])
                                    : "d"(af[mi]), "d"(bf[nj]));
                    }
                    double* bs = reinterpret_cast<double*>(Bs);
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        const int r = rt0 + m0 + 8 * mi + lr;  // D fragment: row lane / 4, columns 2 (lane % 4) + {0, 1}
                        if (r < nb) {
#pragma unroll
                            for (int nj = 0; nj < 2; ++nj)
#pragma unroll
                                for (int e = 0; e < 2; ++e) bs[(n0 + 8 * nj + 2 * lk + e) * ldbs + r] -= d[mi][nj][e];
                        }
                    }
                } else {
                const int rt0 = (LOWER ? b + 1 + tt : tt) * NB;
                const int lane = tid & 31, wq = (tid >> 5) & 3, h = tid >> 7;
                const int rg = (lane >> 2) + 8 * (wq & 1), cp = (lane & 3) + 4 * (wq >> 1);
                int rows[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) rows[i] = TRANS ? rg + 16 * i : 2 * rg + (i & 1) + 32 * (i >> 1);
                const T* xb = Bs + cp * ldbs + r0;
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
#pragma unroll 4
                for (int l = 32 * h; l < 32 * h + 32; l += 2) {
                    P2 xv[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) xv[j] = *reinterpret_cast<const P2*>(xb + 8 * j * ldbs + l);
                    T a[4][2];  // a[i][dl] = op(A)[rows[i]][l + dl]
                    if (!TRANS) {
#pragma unroll
                        for (int dl = 0; dl < 2; ++dl) {
                            const P2 p0 = *reinterpret_cast<const P2*>(cur + (l + dl) * LT + 2 * rg);
                            const P2 p1 = *reinterpret_cast<const P2*>(cur + (l + dl) * LT + 2 * rg + 32);
                            a[0][dl] = p0.x; a[1][dl] = p0.y; a[2][dl] = p1.x; a[3][dl] = p1.y;
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const P2 p = *reinterpret_cast<const P2*>(cur + rows[i] * LT + l);
                            a[i][0] = p.x; a[i][1] = p.y;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            acc[i][j] = fma(a[i][0], xv[j].x, acc[i][j]);
                            acc[i][j] = fma(a[i][1], xv[j].y, acc[i][j]);
                        }
                }
                // the two halves subtract their partial products in turn
#pragma unroll
                for (int half = 0; half < 2; ++half) {
                    if (h == half) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int r = rt0 + rows[i];
                            if (r < nb) {
#pragma unroll
                                for (int j = 0; j < 4; ++j) Bs[(cp + 8 * j) * ldbs + r] -= acc[i][j];
                            }
                        }
                    }
                    if (half == 0) __syncthreads();
                }
                }
            }
            step = ns;
            tt = nt;
        }
        __syncthreads();
        for (int c = 0; c < W; ++c) {
            if (c0 + c >= ncols) break;
            T* bc = B + (c0 + c) * ldb;
            for (int r = tid; r < nb; r += NT) bc[r] = Bs[c * ldbs + r];
        }
        __syncthreads();
    }
}

// One launch over all strips of one problem (B already scaled by alpha).
template <typename T, bool LOWER, bool TRANS, bool UNIT, int W>
__global__ void __launch_bounds__(8 * W, 1)
block_solve_kernel(int nb, i64 ncols, const T* __restrict__ A, i64 lda, T* __restrict__ B, i64 ldb) {
    extern __shared__ __align__(16) unsigned char bs_smem_raw[];
    const i64 nstrips = (ncols + W - 1) / W;
    for (i64 strip = blockIdx.x; strip < nstrips; strip += gridDim.x)
        block_solve_strip<T, LOWER, TRANS, UNIT, W>(nb, ncols, A, lda, B, ldb, strip * W, T(1), bs_smem_raw);
}


}  // namespace bs
}  // namespace mbg
