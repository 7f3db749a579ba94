// Level-2 gemv and trsv — the matrix-vector neighbours of the level-3 path
// (mojoBLAS src/level2/gemv.mojo:23-212, src/level2/trsv.mojo:20-214).
//
// gemv streams A once from HBM, which bounds it: m n elements read, no reuse.
//   NoTrans (y = alpha A x + beta y): each thread owns one row and walks a
//     range of columns, eight independent loads in flight; a warp reads 32
//     consecutive rows of a column (one coalesced segment); sixteen for float32.  The columns are cut
//     into S ranges so that the grid fills the GPU, and a second pass adds the S
//     partial sums in a fixed order (no atomics: the result does not depend on
//     scheduling) and applies alpha and beta.
//   Trans (y = alpha A^T x + beta y): one warp per column, lanes along the
//     column (contiguous), eight (float32: sixteen) loads per lane in flight, a shuffle reduction
//     in a fixed order; long columns are cut into R row ranges the same way.
//   As in the reference, beta scales y first (beta == 0 stores zeros), and a
//   zero product sum leaves beta y unchanged; zero entries of x skip their
//   column (NoTrans).  Any increments, negative ones included, are indexed in
//   place.
//
// trsv (op(A) x = b, x overwrites b) is a dependency chain: the row block b of
// the solution needs every earlier block in solve order.  One persistent launch
// does all of it.  Each 256-thread CTA takes a ticket from an atomic counter and
// solves row block `ticket` in solve order (forward for an effectively lower
// op(A), backward otherwise), so a CTA only ever waits for CTAs that started
// before it.  Waits are on per-block flags (acquire; bounded by %globaltimer,
// with an abort flag so that one expired wait ends the others at once), and the
// published x values are read from L2.  The two blocks solved just before b
// enter through precomputed 64 x 64 matrices (L^-1 op(A)_b,p, see trsv_kernel),
// so the chain of blocks carries only a matrix-vector product per block; every
// earlier block is accumulated tile by tile as it arrives, its tile of op(A)
// loaded before the wait, and one warp solves the 64 x 64 diagonal block by
// substitution (pivot broadcast by a shuffle, multiply by the reciprocal of the
// diagonal).  The reference skips zero entries of x in the NoTrans
// substitution; so does this one.
#include "mbg_internal.cuh"

namespace mbg {

namespace {

constexpr int GV_THREADS = 256;
// loads in flight per thread: 64 bytes of A (eight doubles, sixteen floats)
template <typename T> constexpr int gv_unroll() { return sizeof(T) == 4 ? 16 : 8; }

// NoTrans: P[s * m + i] = sum over columns [s * cps, (s + 1) * cps) of A(i, j) x(j),
// or, with a single range (direct), y(i) itself.
template <typename T>
__global__ void __launch_bounds__(GV_THREADS)
gemv_n_kernel(i64 m, i64 n, const T* __restrict__ A, i64 lda, const T* __restrict__ x, i64 incx, i64 kx,
              i64 cps, T* __restrict__ P, bool direct, T alpha, T beta, T* __restrict__ y, i64 incy, i64 ky) {
    const i64 i = blockIdx.x * (i64)GV_THREADS + threadIdx.x;
    if (i >= m) return;
    const i64 j0 = blockIdx.y * cps, j1 = min(n, j0 + cps);
    constexpr int U = gv_unroll<T>();
    const T* a = A + i;
    T acc = T(0);
    i64 j = j0;
    for (; j + U <= j1; j += U) {
        T av[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            xv[u] = x[kx + (j + u) * incx];
            av[u] = a[(j + u) * lda];
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (xv[u] != T(0)) acc = fma(av[u], xv[u], acc);
    }
    for (; j < j1; ++j) {
        const T xj = x[kx + j * incx];
        if (xj != T(0)) acc = fma(a[j * lda], xj, acc);
    }
    if (direct) {
        T& yi = y[ky + i * incy];
        T v = beta == T(0) ? T(0) : (beta == T(1) ? yi : beta * yi);
        if (acc != T(0)) v = v + alpha * acc;
        yi = v;
    } else {
        P[blockIdx.y * m + i] = acc;
    }
}

// Trans: one warp per column j and row range r: P[r * n + j] = sum_i A(i, j) x(i)
// (or y(j) itself with a single range).
template <typename T>
__global__ void __launch_bounds__(GV_THREADS)
gemv_t_kernel(i64 m, i64 n, const T* __restrict__ A, i64 lda, const T* __restrict__ x, i64 incx, i64 kx,
              i64 rpr, T* __restrict__ P, bool direct, T alpha, T beta, T* __restrict__ y, i64 incy, i64 ky) {
    const int lane = threadIdx.x & 31;
    const i64 j = blockIdx.x * (i64)(GV_THREADS / 32) + (threadIdx.x >> 5);
    if (j >= n) return;
    const i64 i0 = blockIdx.y * rpr, i1 = min(m, i0 + rpr);
    constexpr int U = gv_unroll<T>();
    const T* a = A + j * lda;
    T acc = T(0);
    i64 i = i0 + lane;
    for (; i + 32 * (U - 1) < i1; i += 32 * U) {
        T av[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            av[u] = a[i + 32 * u];
            xv[u] = x[kx + (i + 32 * u) * incx];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) acc = fma(av[u], xv[u], acc);
    }
    for (; i < i1; i += 32) acc = fma(a[i], x[kx + i * incx], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane != 0) return;
    if (direct) {
        T& yj = y[ky + j * incy];
        T v = beta == T(0) ? T(0) : (beta == T(1) ? yj : beta * yj);
        if (acc != T(0)) v = v + alpha * acc;
        yj = v;
    } else {
        P[blockIdx.y * n + j] = acc;
    }
}

// float32 with A 16-byte aligned and lda % 4 == 0: each thread owns four consecutive rows
// and reads them with one 16-byte load per column (a warp moves 512 bytes per load
// instruction instead of 128); the last partial group of rows is read element-wise.
__global__ void __launch_bounds__(GV_THREADS)
sgemv_n4_kernel(i64 m, i64 n, const float* __restrict__ A, i64 lda, const float* __restrict__ x, i64 incx, i64 kx,
                i64 cps, float* __restrict__ P, bool direct, float alpha, float beta, float* __restrict__ y,
                i64 incy, i64 ky) {
    constexpr int U = 8;
    const i64 i0 = 4 * (blockIdx.x * (i64)GV_THREADS + threadIdx.x);
    if (i0 >= m) return;
    const i64 j0 = blockIdx.y * cps, j1 = min(n, j0 + cps);
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (i0 + 4 <= m) {
        i64 j = j0;
        for (; j + U <= j1; j += U) {
            float4 av[U];
            float xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                xv[u] = x[kx + (j + u) * incx];
                av[u] = *reinterpret_cast<const float4*>(A + i0 + (j + u) * lda);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (xv[u] == 0.0f) continue;
                acc[0] = fmaf(av[u].x, xv[u], acc[0]);
                acc[1] = fmaf(av[u].y, xv[u], acc[1]);
                acc[2] = fmaf(av[u].z, xv[u], acc[2]);
                acc[3] = fmaf(av[u].w, xv[u], acc[3]);
            }
        }
        for (; j < j1; ++j) {
            const float xj = x[kx + j * incx];
            if (xj == 0.0f) continue;
            const float4 a4 = *reinterpret_cast<const float4*>(A + i0 + j * lda);
            acc[0] = fmaf(a4.x, xj, acc[0]);
            acc[1] = fmaf(a4.y, xj, acc[1]);
            acc[2] = fmaf(a4.z, xj, acc[2]);
            acc[3] = fmaf(a4.w, xj, acc[3]);
        }
    } else {
        for (i64 j = j0; j < j1; ++j) {
            const float xj = x[kx + j * incx];
            if (xj == 0.0f) continue;
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (i0 + r < m) acc[r] = fmaf(A[i0 + r + j * lda], xj, acc[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const i64 i = i0 + r;
        if (i >= m) break;
        if (direct) {
            float& yi = y[ky + i * incy];
            float v = beta == 0.0f ? 0.0f : (beta == 1.0f ? yi : beta * yi);
            if (acc[r] != 0.0f) v = v + alpha * acc[r];
            yi = v;
        } else {
            P[blockIdx.y * m + i] = acc[r];
        }
    }
}

// float32 Trans with A 16-byte aligned and lda % 4 == 0: lanes read four consecutive
// elements of the column with one 16-byte load (x likewise when incx == 1 and x is
// aligned); a warp-uniform loop over 512-element steps, then the ragged rest element-wise.
// Row ranges (rpr) are multiples of 512.
__global__ void __launch_bounds__(GV_THREADS)
sgemv_t4_kernel(i64 m, i64 n, const float* __restrict__ A, i64 lda, const float* __restrict__ x, i64 incx, i64 kx,
                bool x4, i64 rpr, float* __restrict__ P, bool direct, float alpha, float beta,
                float* __restrict__ y, i64 incy, i64 ky) {
    constexpr int U = 4;  // 16-byte loads per lane per step: a step covers 32 x 4 x U = 512 rows
    const int lane = threadIdx.x & 31;
    const i64 j = blockIdx.x * (i64)(GV_THREADS / 32) + (threadIdx.x >> 5);
    if (j >= n) return;
    const i64 i0 = blockIdx.y * rpr, i1 = min(m, i0 + rpr);
    const float* a = A + j * lda;
    float acc = 0.0f;
    i64 base = i0;
    for (; base + 128 * U <= i1; base += 128 * U) {
        float4 av[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const i64 i = base + 128 * u + 4 * lane;
            av[u] = *reinterpret_cast<const float4*>(a + i);
            if (x4) xv[u] = *reinterpret_cast<const float4*>(x + i);
            else xv[u] = make_float4(x[kx + i * incx], x[kx + (i + 1) * incx], x[kx + (i + 2) * incx],
                                     x[kx + (i + 3) * incx]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            acc = fmaf(av[u].x, xv[u].x, acc);
            acc = fmaf(av[u].y, xv[u].y, acc);
            acc = fmaf(av[u].z, xv[u].z, acc);
            acc = fmaf(av[u].w, xv[u].w, acc);
        }
    }
    for (i64 i = base + lane; i < i1; i += 32) acc = fmaf(a[i], x[kx + i * incx], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane != 0) return;
    if (direct) {
        float& yj = y[ky + j * incy];
        float v = beta == 0.0f ? 0.0f : (beta == 1.0f ? yj : beta * yj);
        if (acc != 0.0f) v = v + alpha * acc;
        yj = v;
    } else {
        P[blockIdx.y * n + j] = acc;
    }
}

// y(i) = beta y(i) + alpha sum_s P[s * len + i] (partial sums in a fixed order)
template <typename T>
__global__ void gemv_finish_kernel(i64 len, i64 parts, const T* __restrict__ P, T alpha, T beta,
                                   T* __restrict__ y, i64 incy, i64 ky) {
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (i >= len) return;
    T s = T(0);
    for (i64 p = 0; p < parts; ++p) s += P[p * len + i];
    T& yi = y[ky + i * incy];
    T v = beta == T(0) ? T(0) : (beta == T(1) ? yi : beta * yi);
    if (s != T(0)) v = v + alpha * s;
    yi = v;
}

template <typename T>
__global__ void scale_vector_kernel(i64 len, T beta, T* __restrict__ y, i64 incy, i64 ky) {
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (i >= len) return;
    T& yi = y[ky + i * incy];
    yi = beta == T(0) ? T(0) : beta * yi;
}

// ---- trsv ----------------------------------------------------------------------
constexpr int TV_NB = 64, TV_THREADS = 256, TV_GROUPS = TV_THREADS / TV_NB, TV_PER = TV_NB / TV_GROUPS;
constexpr unsigned long long TV_WAIT_NS = 2000000000ull;

__device__ __forceinline__ unsigned long long tv_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int tv_load_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void tv_store_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct TrsvSync {
    int* flags;   // per row block: 1 once its part of x is published
    int* ticket;  // solve-order counter
    int* abort;   // set by an expired wait: every other wait gives up at once
    int* err;     // library error flag (code, site)
};

// Thread 0 only: wait (bounded) for `flag`; false if the launch is aborting.
__device__ bool tv_wait(const int* flag, const TrsvSync& s) {
    if (tv_load_acquire(flag)) return true;
    const unsigned long long t0 = tv_clock();
    while (true) {
#pragma unroll 1
        for (int k = 0; k < 64; ++k)
            if (tv_load_acquire(flag)) return true;
        if (*(volatile int*)s.abort) return false;
        if (tv_clock() - t0 > TV_WAIT_NS) {
            atomicExch(s.abort, 1);
            if (s.err) {
                atomicExch(s.err, 1);
                atomicExch(s.err + 1, 40);
            }
            return false;
        }
    }
}

// op(A)[i, l] for a column-major A
template <typename T, bool TRANS>
__device__ __forceinline__ T opa(const T* __restrict__ A, i64 lda, i64 i, i64 l) {
    return TRANS ? A[l + i * lda] : A[i + l * lda];
}

inline i64 vec_start(i64 len, i64 inc) { return inc > 0 ? 0 : -(len - 1) * inc; }

constexpr int TV_LD = TV_NB + 1;  // shared-memory row of a 64 x 64 block

template <typename T>
constexpr size_t trsv_smem_bytes() {
    return sizeof(T) * (size_t(3) * TV_NB * TV_LD + 2 * TV_GROUPS * TV_NB + 2 * TV_NB) + 4 * sizeof(int);
}

// Block b of the solution, with p1 and p2 the blocks solved one and two steps
// before it (b - 1, b - 2 forward; b + 1, b + 2 backward) and L the diagonal
// block of op(A):
//     x_b = L^-1 (b_b - sum_{j before p2} op(A)_bj x_j) - M2 x_p2 - M1 x_p1,
//     M1 = L^-1 op(A)_b,p1,  M2 = L^-1 op(A)_b,p2.
// M1 and M2 do not depend on x, y = L^-1 (...) needs every block before p2, and
// M2 x_p2 is applied as soon as p2 is published: once x_p1 arrives, only the
// 64 x 64 product M1 x_p1 remains on the chain of blocks, and y's 64-step
// substitution has two block steps to finish.  M1's and M2's 128 columns are
// solved by the 8 warps, 16 each (lanes own rows lane and lane + 32; pivot by
// shuffle, scaled by the reciprocal of the diagonal); y by warp 0 the same way.
// The reference's zero skip (NoTrans) is kept: a zero pivot updates nothing, and
// a zero entry of x_p1 / x_p2 skips its column of M1 / M2.
template <typename T, bool TRANS>
__global__ void __launch_bounds__(TV_THREADS)
trsv_kernel(i64 n, const T* __restrict__ A, i64 lda, T* __restrict__ x, i64 incx, i64 kx, bool lower, bool unit,
            TrsvSync s) {
    extern __shared__ __align__(16) unsigned char tv_smem[];
    T* diag = reinterpret_cast<T*>(tv_smem);      // [64][TV_LD] op(A) diagonal block, the triangle only
    T* M1 = diag + TV_NB * TV_LD;                  // [64][TV_LD] op(A)_b,p1, then L^-1 op(A)_b,p1
    T* M2 = M1 + TV_NB * TV_LD;                    // [64][TV_LD] op(A)_b,p2, then L^-1 op(A)_b,p2
    T* red = M2 + TV_NB * TV_LD;                   // [2 * TV_GROUPS][64] partial sums
    T* invs = red + 2 * TV_GROUPS * TV_NB;         // [64] reciprocals of the diagonal (1 for unit)
    T* ys = invs + TV_NB;                          // [64] y
    int* sint = reinterpret_cast<int*>(ys + TV_NB);  // [0] ticket, [1], [2] wait results
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const i64 nb = (n + TV_NB - 1) / TV_NB;
    if (tid == 0) sint[0] = atomicAdd(s.ticket, 1);
    __syncthreads();
    const i64 t = sint[0];
    const i64 b = lower ? t : nb - 1 - t;
    const i64 r0 = b * TV_NB;
    const int rows = int(min(i64(TV_NB), n - r0));
    const bool has_p1 = t >= 1, has_p2 = t >= 2;
    const i64 bp1 = lower ? b - 1 : b + 1, bp2 = lower ? b - 2 : b + 2;  // solved one / two steps before
    const i64 c10 = bp1 * TV_NB, c20 = bp2 * TV_NB;
    const int cols1 = has_p1 ? int(min(i64(TV_NB), n - c10)) : 0;
    const int cols2 = has_p2 ? int(min(i64(TV_NB), n - c20)) : 0;
    const int dp = lower ? 1 : -1;

    // the diagonal block and the tile op(A)(rows of b, columns of p); f runs along A's contiguous index
    for (int e = tid; e < TV_NB * TV_NB; e += TV_THREADS) {
        const int f = e % TV_NB, g = e / TV_NB;
        const int i = TRANS ? g : f, l = TRANS ? f : g;
        const bool in = lower ? (l < i) : (l > i);
        T v = T(0);
        if (i < rows && l < rows && (in || (l == i && !unit))) v = opa<T, TRANS>(A, lda, r0 + i, r0 + l);
        diag[i * TV_LD + l] = v;
        T w1 = T(0), w2 = T(0);
        if (i < rows && l < cols1) w1 = opa<T, TRANS>(A, lda, r0 + i, c10 + l);
        if (i < rows && l < cols2) w2 = opa<T, TRANS>(A, lda, r0 + i, c20 + l);
        M1[i * TV_LD + l] = w1;
        M2[i * TV_LD + l] = w2;
    }
    __syncthreads();
    if (tid < TV_NB) invs[tid] = (tid < rows && !unit) ? T(1) / diag[tid * TV_LD + tid] : T(1);
    T rhs0 = T(0), rhs1 = T(0);
    if (warp == 0) {
        if (lane < rows) rhs0 = x[kx + (r0 + lane) * incx];
        if (lane + 32 < rows) rhs1 = x[kx + (r0 + lane + 32) * incx];
    }
    __syncthreads();  // invs complete

    // M1 := L^-1 op(A)_b,p1 and M2 := L^-1 op(A)_b,p2: warp w solves columns w * 8 .. w * 8 + 7 of both
    if (has_p1) {
        constexpr int NC = 16;  // columns per warp: 8 of M1, then 8 of M2
        T m0[NC], m1[NC];
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
            const T* Mc = cc < 8 ? M1 : M2;
            m0[cc] = Mc[lane * TV_LD + warp * 8 + (cc & 7)];
            m1[cc] = Mc[(lane + 32) * TV_LD + warp * 8 + (cc & 7)];
        }
        int p = lower ? 0 : rows - 1;
        for (int st = 0; st < rows; ++st, p += dp) {
            const int owner = p & 31;
            const bool hi = p >= 32;
            const T ip = invs[p];
            const T d0 = diag[lane * TV_LD + p], d1 = diag[(lane + 32) * TV_LD + p];
            const bool up0 = lower ? lane > p : lane < p, up1 = lower ? lane + 32 > p : lane + 32 < p;
#pragma unroll
            for (int cc = 0; cc < NC; ++cc) {
                T mine = hi ? m1[cc] : m0[cc];
                if (!unit && (TRANS || mine != T(0))) mine = mine * ip;
                const T xp = __shfl_sync(0xffffffffu, mine, owner);
                if (lane == owner) {
                    if (hi) m1[cc] = xp;
                    else m0[cc] = xp;
                }
                if (TRANS || xp != T(0)) {
                    if (up0) m0[cc] = fma(-d0, xp, m0[cc]);
                    if (up1) m1[cc] = fma(-d1, xp, m1[cc]);
                }
            }
        }
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
            T* Mc = cc < 8 ? M1 : M2;
            Mc[lane * TV_LD + warp * 8 + (cc & 7)] = m0[cc];
            Mc[(lane + 32) * TV_LD + warp * 8 + (cc & 7)] = m1[cc];
        }
    }

    // contributions of the blocks solved before p2
    // NoTrans: thread (row r = tid % 64, columns g * 16 .. g * 16 + 15 of each tile), one sum
    // Trans:   thread (column l = tid % 64, rows g * 16 .. g * 16 + 15), sixteen sums
    const int f = tid % TV_NB, g = tid / TV_NB;
    T acc[TV_PER];
#pragma unroll
    for (int u = 0; u < TV_PER; ++u) acc[u] = T(0);
    for (i64 q = 0; q + 2 < t; ++q) {
        const i64 jb = lower ? q : nb - 1 - q;
        const i64 c0 = jb * TV_NB;
        const int cols = int(min(i64(TV_NB), n - c0));  // the last block of a backward solve may be short
        // the tile of op(A) is loaded before the wait: it does not depend on x
        T av[TV_PER];
#pragma unroll
        for (int u = 0; u < TV_PER; ++u) {
            const int i = TRANS ? g * TV_PER + u : f, l = TRANS ? f : g * TV_PER + u;
            av[u] = (i < rows && l < cols) ? opa<T, TRANS>(A, lda, r0 + i, c0 + l) : T(0);
        }
        if (tid == 0) sint[1 + (q & 1)] = tv_wait(s.flags + jb, s) ? 1 : 0;
        __syncthreads();
        if (!sint[1 + (q & 1)]) return;
        if (TRANS) {
            const T xl = f < cols ? __ldcg(x + kx + (c0 + f) * incx) : T(0);
#pragma unroll
            for (int u = 0; u < TV_PER; ++u) acc[u] = fma(av[u], xl, acc[u]);
        } else {
#pragma unroll
            for (int u = 0; u < TV_PER; ++u) {
                const int l = g * TV_PER + u;
                const T xl = l < cols ? __ldcg(x + kx + (c0 + l) * incx) : T(0);
                if (xl != T(0)) acc[0] = fma(av[u], xl, acc[0]);  // the reference's zero skip
            }
        }
    }

    // reduce: red[.][i] partial sums of row i
    if (TRANS) {
#pragma unroll
        for (int u = 0; u < TV_PER; ++u) {
            T v = acc[u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[(warp & 1) * TV_NB + g * TV_PER + u] = v;  // two warps per group of columns
        }
    } else {
        red[g * TV_NB + f] = acc[0];
    }
    __syncthreads();

    // warp 0: y = L^-1 (right-hand side minus the contributions), one pivot per step (the
    // owner scales its own value, one shuffle broadcasts it, every lane updates its rows
    // after the pivot; the next pivot's column is loaded one step ahead)
    if (warp == 0) {
        T v0, v1;
        if (TRANS) {
            v0 = rhs0 - (red[lane] + red[TV_NB + lane]);
            v1 = rhs1 - (red[lane + 32] + red[TV_NB + lane + 32]);
        } else {
            v0 = rhs0 - ((red[lane] + red[TV_NB + lane]) + (red[2 * TV_NB + lane] + red[3 * TV_NB + lane]));
            v1 = rhs1 - ((red[lane + 32] + red[TV_NB + lane + 32]) +
                         (red[2 * TV_NB + lane + 32] + red[3 * TV_NB + lane + 32]));
        }
        if (lane >= rows) v0 = T(0);
        if (lane + 32 >= rows) v1 = T(0);
        const T inv0 = invs[lane], inv1 = invs[lane + 32];
        int p = lower ? 0 : rows - 1;
        T d0 = diag[lane * TV_LD + p], d1 = diag[(lane + 32) * TV_LD + p];
        for (int st = 0; st < rows; ++st, p += dp) {
            const int owner = p & 31;
            const bool hi = p >= 32;
            T mine = hi ? v1 : v0;
            const T mi = hi ? inv1 : inv0;
            if (!unit && (TRANS || mine != T(0))) mine = mine * mi;  // the reference skips zeros (NoTrans)
            const T xp = __shfl_sync(0xffffffffu, mine, owner);
            const int pn = (st + 1 < rows) ? p + dp : p;
            const T d0n = diag[lane * TV_LD + pn], d1n = diag[(lane + 32) * TV_LD + pn];
            if (lane == owner) {
                if (hi) v1 = xp;
                else v0 = xp;
            }
            if (TRANS || xp != T(0)) {
                if (lower ? lane > p : lane < p) v0 = fma(-d0, xp, v0);
                if (lower ? lane + 32 > p : lane + 32 < p) v1 = fma(-d1, xp, v1);
            }
            d0 = d0n;
            d1 = d1n;
        }
        ys[lane] = v0;
        ys[lane + 32] = v1;
    }

    // y -= M2 x_p2 once block p2 is published, then x_b = y - M1 x_p1 once p1 is: each a 64 x 64
    // product by all threads, partial sums over four column groups added by warp 0
    for (int step = 0; step < 2; ++step) {
        const bool live = step == 0 ? has_p2 : has_p1;
        if (!live) continue;  // uniform across the CTA
        const T* Mm = step == 0 ? M2 : M1;
        const i64 cb = step == 0 ? c20 : c10;
        const int cn = step == 0 ? cols2 : cols1;
        if (tid == 0) sint[1] = tv_wait(s.flags + (step == 0 ? bp2 : bp1), s) ? 1 : 0;
        __syncthreads();  // also orders warp 0's earlier reads of red before the writes below
        if (!sint[1]) return;
        T part = T(0);
#pragma unroll
        for (int u = 0; u < TV_PER; ++u) {
            const int c = g * TV_PER + u;
            const T xc = c < cn ? __ldcg(x + kx + (cb + c) * incx) : T(0);
            if (TRANS || xc != T(0)) part = fma(Mm[f * TV_LD + c], xc, part);
        }
        red[g * TV_NB + f] = part;
        __syncthreads();
        if (warp == 0) {
            ys[lane] -= (red[lane] + red[TV_NB + lane]) + (red[2 * TV_NB + lane] + red[3 * TV_NB + lane]);
            ys[lane + 32] -= (red[lane + 32] + red[TV_NB + lane + 32]) +
                             (red[2 * TV_NB + lane + 32] + red[3 * TV_NB + lane + 32]);
        }
    }
    if (warp != 0) return;
    __syncwarp();
    if (lane < rows) x[kx + (r0 + lane) * incx] = ys[lane];
    if (lane + 32 < rows) x[kx + (r0 + lane + 32) * incx] = ys[lane + 32];
    __threadfence();
    __syncwarp();
    if (lane == 0) tv_store_release(s.flags + b, 1);
}

template <typename T, bool TRANS>
int launch_trsv_t(i64 n, const T* a, i64 lda, T* x, i64 incx, bool lower, bool unit, const TrsvSync& sync,
                  i64 nb) {
    constexpr size_t SM = trsv_smem_bytes<T>();
    static std::atomic<unsigned> configured{0};  // one bit per device: more than 48 KB of shared memory needs an opt-in
    int dev = 0;
    MBG_CUDA(cudaGetDevice(&dev));
    if (!configured_on(configured, dev)) {
        MBG_CUDA(cudaFuncSetAttribute(trsv_kernel<T, TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM));
        mark_configured(configured, dev);
    }
    trsv_kernel<T, TRANS><<<(unsigned)nb, TV_THREADS, SM, stream()>>>(n, a, lda, x, incx, vec_start(n, incx), lower,
                                                                       unit, sync);
    return check_launch("trsv");
}

}  // namespace

template <typename T>
int gemv_device(char trans, i64 m, i64 n, T alpha, const T* a, i64 lda, const T* x, i64 incx, T beta, T* y,
                i64 incy) {
    const bool notrans = trans == 'N';
    const i64 lenx = notrans ? n : m, leny = notrans ? m : n;
    const i64 kx = vec_start(lenx, incx), ky = vec_start(leny, incy);
    cudaStream_t s = stream();
    if (alpha == T(0)) {  // gemv.mojo:107-129: y = beta y, then return
        ProfScope prof("gemv");
        scale_vector_kernel<T><<<(unsigned)cdiv(leny, 256), 256, 0, s>>>(leny, beta, y, incy, ky);
        return check_launch("gemv");
    }
    const i64 target = 8 * 148;  // CTAs for a full GPU
    Workspace wp;
    // float32 with a 16-byte aligned A and lda % 4 == 0: the 16-byte load kernels
    const bool v4 = sizeof(T) == 4 && reinterpret_cast<uintptr_t>(a) % 16 == 0 && lda % 4 == 0;
    if (notrans && v4) {
        const i64 rb = cdiv(m, 4 * GV_THREADS);
        const i64 splits = imax(1, imin(cdiv(target, rb), cdiv(n, 64)));
        const i64 cps = cdiv(n, splits), parts = cdiv(n, cps);
        if (rb > 0x7fffffff || parts > 65535) return MBG_ERR_UNSUPPORTED;
        float* P = nullptr;
        if (parts > 1) {
            MBG_TRY(wp.reserve(sizeof(float) * size_t(parts) * size_t(m)));
            P = wp.as<float>();
        }
        {
            ProfScope prof("gemv");
            sgemv_n4_kernel<<<dim3((unsigned)rb, (unsigned)parts), GV_THREADS, 0, s>>>(
                m, n, (const float*)a, lda, (const float*)x, incx, kx, cps, P, parts == 1, (float)alpha,
                (float)beta, (float*)y, incy, ky);
            MBG_TRY(check_launch("gemv"));
        }
        if (parts == 1) return MBG_OK;
        ProfScope prof("gemv_finish");
        gemv_finish_kernel<float><<<(unsigned)cdiv(m, 256), 256, 0, s>>>(m, parts, P, (float)alpha, (float)beta,
                                                                         (float*)y, incy, ky);
        return check_launch("gemv_finish");
    }
    if (!notrans && v4) {
        const i64 cb = cdiv(n, GV_THREADS / 32);
        const i64 splits = imax(1, imin(cdiv(target, cb), cdiv(m, 2048)));
        const i64 rpr = cdiv(cdiv(m, splits), 512) * 512, parts = cdiv(m, rpr);
        if (cb > 0x7fffffff || parts > 65535) return MBG_ERR_UNSUPPORTED;
        const bool x4 = incx == 1 && reinterpret_cast<uintptr_t>(x) % 16 == 0;
        float* P = nullptr;
        if (parts > 1) {
            MBG_TRY(wp.reserve(sizeof(float) * size_t(parts) * size_t(n)));
            P = wp.as<float>();
        }
        {
            ProfScope prof("gemv");
            sgemv_t4_kernel<<<dim3((unsigned)cb, (unsigned)parts), GV_THREADS, 0, s>>>(
                m, n, (const float*)a, lda, (const float*)x, incx, kx, x4, rpr, P, parts == 1, (float)alpha,
                (float)beta, (float*)y, incy, ky);
            MBG_TRY(check_launch("gemv"));
        }
        if (parts == 1) return MBG_OK;
        ProfScope prof("gemv_finish");
        gemv_finish_kernel<float><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(n, parts, P, (float)alpha, (float)beta,
                                                                         (float*)y, incy, ky);
        return check_launch("gemv_finish");
    }
    if (notrans) {
        const i64 rb = cdiv(m, GV_THREADS);
        const i64 splits = imax(1, imin(cdiv(target, rb), cdiv(n, 64)));
        const i64 cps = cdiv(n, splits), parts = cdiv(n, cps);
        if (rb > 0x7fffffff || parts > 65535) return MBG_ERR_UNSUPPORTED;
        T* P = nullptr;
        if (parts > 1) {
            MBG_TRY(wp.reserve(sizeof(T) * size_t(parts) * size_t(m)));
            P = wp.as<T>();
        }
        {
            ProfScope prof("gemv");
            gemv_n_kernel<T><<<dim3((unsigned)rb, (unsigned)parts), GV_THREADS, 0, s>>>(
                m, n, a, lda, x, incx, kx, cps, P, parts == 1, alpha, beta, y, incy, ky);
            MBG_TRY(check_launch("gemv"));
        }
        if (parts == 1) return MBG_OK;
        ProfScope prof("gemv_finish");
        gemv_finish_kernel<T><<<(unsigned)cdiv(m, 256), 256, 0, s>>>(m, parts, P, alpha, beta, y, incy, ky);
        return check_launch("gemv_finish");
    }
    const i64 cb = cdiv(n, GV_THREADS / 32);
    const i64 splits = imax(1, imin(cdiv(target, cb), cdiv(m, 32 * gv_unroll<T>() * 4)));
    const i64 rpr = cdiv(m, splits), parts = cdiv(m, rpr);
    if (cb > 0x7fffffff || parts > 65535) return MBG_ERR_UNSUPPORTED;
    T* P = nullptr;
    if (parts > 1) {
        MBG_TRY(wp.reserve(sizeof(T) * size_t(parts) * size_t(n)));
        P = wp.as<T>();
    }
    {
        ProfScope prof("gemv");
        gemv_t_kernel<T><<<dim3((unsigned)cb, (unsigned)parts), GV_THREADS, 0, s>>>(
            m, n, a, lda, x, incx, kx, rpr, P, parts == 1, alpha, beta, y, incy, ky);
        MBG_TRY(check_launch("gemv"));
    }
    if (parts == 1) return MBG_OK;
    ProfScope prof("gemv_finish");
    gemv_finish_kernel<T><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(n, parts, P, alpha, beta, y, incy, ky);
    return check_launch("gemv_finish");
}

template <typename T>
int trsv_device(char uplo, char trans, char diag, i64 n, const T* a, i64 lda, T* x, i64 incx) {
    const bool tr = is_t(trans), unit = is_u(diag);
    const bool lower = (!is_u(uplo)) != tr;  // effective op(A) lower: forward substitution
    const i64 nb = cdiv(n, TV_NB);
    if (nb > 0x7fffffff) return MBG_ERR_UNSUPPORTED;
    Workspace ws;
    MBG_TRY(ws.reserve(sizeof(int) * size_t(nb + 2)));
    int* flags = ws.as<int>();
    cudaStream_t s = stream();
    MBG_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * size_t(nb + 2), s));
    TrsvSync sync{flags, flags + nb, flags + nb + 1, device_error_flag()};
    ProfScope prof("trsv");
    if (tr) return launch_trsv_t<T, true>(n, a, lda, x, incx, lower, unit, sync, nb);
    return launch_trsv_t<T, false>(n, a, lda, x, incx, lower, unit, sync, nb);
}

template int gemv_device<float>(char, i64, i64, float, const float*, i64, const float*, i64, float, float*, i64);
template int gemv_device<double>(char, i64, i64, double, const double*, i64, const double*, i64, double, double*,
                                 i64);
template int trsv_device<float>(char, char, char, i64, const float*, i64, float*, i64);
template int trsv_device<double>(char, char, char, i64, const double*, i64, double*, i64);

}  // namespace mbg
