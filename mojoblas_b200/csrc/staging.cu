// Host <-> device copies of matrices in pageable host memory.
//
// mojoBLAS's callers pass plain host allocations (BLASPtr, src/type_aliases.mojo:15;
// its tests allocate them with alloc, tests/test_level3.mojo:15-41).  A DMA engine
// reads and writes only page-locked memory, so a copy from pageable memory is
// staged somewhere; the driver's own staging is serial and blocks the host for the
// whole copy.  Here each direction runs through a ring of page-locked bounce
// buffers per device:
//   host -> device  the host threads pack chunk c + 1 of the source (whole columns,
//                   up to one buffer) into a free bounce buffer while the copy
//                   stream's DMA moves chunk c to the device;
//   device -> host  the DMAs of the first chunks into the ring are queued at once;
//                   the host threads unpack chunk c into the destination while the
//                   DMAs of the next chunks run, and each unpacked buffer takes the
//                   next chunk's DMA.
// Packing and unpacking are split over a small pool of host threads, so the host
// copies keep up with the PCIe link.  Pinned host memory (cudaHostAlloc /
// cudaHostRegister) needs no bounce: it is copied directly on the given stream.
#include "mbg_internal.cuh"

#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace mbg {

namespace {

constexpr size_t STAGE_BUF = size_t(32) << 20;  // bytes per bounce buffer
constexpr int STAGE_NBUF = 4;

// dst[0 .. n) = src[0 .. n) with non-temporal 16-byte stores where the host has them: the
// destination (a bounce buffer the DMA engine reads next, or the caller's matrix) is not
// read back by this thread soon, and plain stores first read each destination line, a
// third of the host-memory traffic of a copy that competes with the DMAs for it (measured
// on a B200 host: 8 threads copy into page-locked memory at 62 GB/s with memcpy, 77-89
// GB/s with streaming stores).
// Rows of at least 1 KiB stream; `fence` orders the streaming stores before what follows
// (one fence after the last row of a strided copy).
void stream_copy(void* dst, const void* src, size_t n, bool fence = true) {
#if defined(__x86_64__)
    if (n >= 1024) {
        char* d = static_cast<char*>(dst);
        const char* s = static_cast<const char*>(src);
        const size_t head = (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15;
        std::memcpy(d, s, head);
        d += head;
        s += head;
        n -= head;
        const size_t body = n & ~size_t(63);
        for (size_t i = 0; i < body; i += 64) {
            const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i));
            const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 16));
            const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 32));
            const __m128i e = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 48));
            _mm_stream_si128(reinterpret_cast<__m128i*>(d + i), a);
            _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 16), b);
            _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 32), c);
            _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 48), e);
        }
        if (fence) _mm_sfence();  // the stores are globally visible before the DMA or the caller reads them
        std::memcpy(d + body, s + body, n - body);
        return;
    }
#endif
    std::memcpy(dst, src, n);
}

// A pool of host threads running memcpy pieces; calls from several host threads
// share it (their pieces interleave), each waiting only for its own pieces.
class CopyPool {
public:
    static CopyPool& get() {
        // never destroyed: its worker threads wait on its condition variable until the
        // process exits, and destroying a condition variable with waiters blocks exit
        static CopyPool* pool = new CopyPool();
        return *pool;
    }
    // dst[r * dpitch .. + width] = src[r * spitch .. + width] for rows r in [0, height)
    void copy_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height) {
        const size_t bytes = width * height;
        const int parts = int(std::min<size_t>(size_t(nthreads_) + 1, std::max<size_t>(1, bytes >> 20)));
        if (parts <= 1 || height < 2) {
            rows(dst, dpitch, src, spitch, width, 0, height);
            return;
        }
        struct Sync {
            std::mutex m;
            std::condition_variable cv;
            int left;
        } sync;
        sync.left = parts - 1;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int p = 1; p < parts; ++p) {
                const size_t r0 = height * size_t(p) / size_t(parts), r1 = height * size_t(p + 1) / size_t(parts);
                jobs_.push_back([=, &sync] {
                    rows(dst, dpitch, src, spitch, width, r0, r1);
                    std::lock_guard<std::mutex> l(sync.m);
                    if (--sync.left == 0) sync.cv.notify_all();
                });
            }
        }
        cv_.notify_all();
        rows(dst, dpitch, src, spitch, width, 0, height / size_t(parts));  // the caller's share
        std::unique_lock<std::mutex> l(sync.m);
        sync.cv.wait(l, [&] { return sync.left == 0; });
    }

private:
    CopyPool() {
        unsigned hw = std::thread::hardware_concurrency();
        // the caller is one more; past 8 copying threads a B200 host's copies into page-locked
        // memory ran no faster (host-memory bound) and took cores from the callers
        nthreads_ = int(std::max(1u, std::min(7u, hw > 1 ? hw - 1 : 1u)));
        if (const char* e = std::getenv("MBG_COPY_THREADS")) nthreads_ = std::max(0, std::min(64, std::atoi(e)));
        for (int i = 0; i < nthreads_; ++i) {
            std::thread t([this] { work(); });
            t.detach();  // the pool lives until the process exits
        }
    }
    static void rows(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t r0, size_t r1) {
        if (dpitch == width && spitch == width) {
            stream_copy(static_cast<char*>(dst) + r0 * width, static_cast<const char*>(src) + r0 * width,
                        (r1 - r0) * width);
            return;
        }
        for (size_t r = r0; r < r1; ++r)
            stream_copy(static_cast<char*>(dst) + r * dpitch, static_cast<const char*>(src) + r * spitch, width, false);
#if defined(__x86_64__)
        _mm_sfence();
#endif
    }
    void work() {
        for (;;) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return !jobs_.empty(); });
                job = std::move(jobs_.front());
                jobs_.pop_front();
            }
            job();
        }
    }
    int nthreads_ = 1;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> jobs_;
};

// Bounce buffers and copy streams of one device (kept until the process exits).
// One staged copy per direction runs at a time, so a host-to-device copy and a
// device-to-host copy (two host threads of the pipelined gemm) proceed together.
struct Stager {
    struct Ring {
        std::mutex mu;
        void* buf[STAGE_NBUF] = {};
        cudaEvent_t ev[STAGE_NBUF] = {};  // last DMA that used the buffer
        cudaEvent_t dep = nullptr, done = nullptr;
        cudaStream_t cs = nullptr;
        bool ready = false;
        int setup() {
            if (ready) return MBG_OK;
            MBG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            for (int i = 0; i < STAGE_NBUF; ++i) {
                MBG_CUDA(cudaHostAlloc(&buf[i], STAGE_BUF, cudaHostAllocPortable));
                MBG_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
            }
            MBG_CUDA(cudaEventCreateWithFlags(&dep, cudaEventDisableTiming));
            MBG_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
            ready = true;
            return MBG_OK;
        }
    } in, out;
};

std::mutex g_stage_mu;
std::map<int, Stager*> g_stagers;

Stager* stager() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_stage_mu);
    Stager*& s = g_stagers[dev];
    if (!s) s = new Stager();
    return s;
}

// How pageable host memory is moved: 0 (default) through the bounce buffers, 1 the driver's
// own staged copy, 2 the region page-locked for the duration of the copy (cudaHostRegister).
// Read once from MBG_PAGEABLE_MODE; the alternatives are kept for measurements on new hosts.
int pageable_mode() {
    static const int mode = [] {
        const char* e = std::getenv("MBG_PAGEABLE_MODE");
        const int v = e ? std::atoi(e) : 0;
        return (v >= 0 && v <= 2) ? v : 0;
    }();
    return mode;
}

// Page-locks the pages under [p, p + bytes) for one copy; false if the driver refuses
// (e.g. part of the range is registered already), in which case nothing was locked.
bool register_range(const void* p, size_t bytes, void** base) {
    const uintptr_t page = 4096, a = reinterpret_cast<uintptr_t>(p) & ~(page - 1);
    const uintptr_t b = (reinterpret_cast<uintptr_t>(p) + bytes + page - 1) & ~(page - 1);
    if (cudaHostRegister(reinterpret_cast<void*>(a), b - a, cudaHostRegisterDefault) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    *base = reinterpret_cast<void*>(a);
    return true;
}

}  // namespace

bool is_pinned_host(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeHost;
}

int copy_h2d_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                cudaStream_t s) {
    if (width == 0 || height == 0) return MBG_OK;
    if (is_pinned_host(src) || width > STAGE_BUF || pageable_mode() == 1) {
        MBG_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyHostToDevice, s));
        return MBG_OK;
    }
    void* reg = nullptr;
    if (pageable_mode() == 2 && register_range(src, (height - 1) * spitch + width, &reg)) {
        const cudaError_t e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyHostToDevice, s);
        const cudaError_t w = e == cudaSuccess ? cudaStreamSynchronize(s) : e;
        cudaHostUnregister(reg);
        MBG_CUDA(e);
        MBG_CUDA(w);
        return MBG_OK;
    }
    Stager* st = stager();
    if (!st) return MBG_ERR_NO_DEVICE;
    auto& R = st->in;
    std::lock_guard<std::mutex> lk(R.mu);
    MBG_TRY(R.setup());
    MBG_CUDA(cudaEventRecord(R.dep, s));  // dst may still be read by earlier work on s
    MBG_CUDA(cudaStreamWaitEvent(R.cs, R.dep, 0));
    const size_t per = std::max<size_t>(1, STAGE_BUF / width);
    int slot = 0;
    for (size_t r0 = 0; r0 < height; r0 += per, slot = (slot + 1) % STAGE_NBUF) {
        const size_t nr = std::min(per, height - r0);
        MBG_CUDA(cudaEventSynchronize(R.ev[slot]));  // the buffer's previous DMA has finished
        CopyPool::get().copy_2d(R.buf[slot], width, static_cast<const char*>(src) + r0 * spitch, spitch, width, nr);
        MBG_CUDA(cudaMemcpy2DAsync(static_cast<char*>(dst) + r0 * dpitch, dpitch, R.buf[slot], width, width, nr,
                                   cudaMemcpyHostToDevice, R.cs));
        MBG_CUDA(cudaEventRecord(R.ev[slot], R.cs));
    }
    MBG_CUDA(cudaEventRecord(R.done, R.cs));
    MBG_CUDA(cudaStreamWaitEvent(s, R.done, 0));  // later work on s sees the data
    return MBG_OK;
}

int copy_d2h_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t height,
                cudaStream_t s, cudaEvent_t after) {
    if (width == 0 || height == 0) return MBG_OK;
    if (is_pinned_host(dst) || width > STAGE_BUF || pageable_mode() == 1) {
        if (after) MBG_CUDA(cudaStreamWaitEvent(s, after, 0));
        MBG_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost, s));
        return MBG_OK;
    }
    void* reg = nullptr;
    if (pageable_mode() == 2 && register_range(dst, (height - 1) * dpitch + width, &reg)) {
        cudaError_t e = after ? cudaStreamWaitEvent(s, after, 0) : cudaSuccess;
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost, s);
        const cudaError_t w = e == cudaSuccess ? cudaStreamSynchronize(s) : e;
        cudaHostUnregister(reg);
        MBG_CUDA(e);
        MBG_CUDA(w);
        return MBG_OK;
    }
    Stager* st = stager();
    if (!st) return MBG_ERR_NO_DEVICE;
    auto& R = st->out;
    std::lock_guard<std::mutex> lk(R.mu);
    MBG_TRY(R.setup());
    if (after) {
        MBG_CUDA(cudaStreamWaitEvent(R.cs, after, 0));
    } else {
        MBG_CUDA(cudaEventRecord(R.dep, s));  // src is produced by the work already on s
        MBG_CUDA(cudaStreamWaitEvent(R.cs, R.dep, 0));
    }
    const size_t per = std::max<size_t>(1, STAGE_BUF / width);
    const size_t nchunks = (height + per - 1) / per;
    auto issue = [&](size_t c) -> int {
        const int b = int(c % STAGE_NBUF);
        const size_t r0 = c * per, nr = std::min(per, height - r0);
        MBG_CUDA(cudaMemcpy2DAsync(R.buf[b], width, static_cast<const char*>(src) + r0 * spitch, spitch, width, nr,
                                   cudaMemcpyDeviceToHost, R.cs));
        MBG_CUDA(cudaEventRecord(R.ev[b], R.cs));
        return MBG_OK;
    };
    for (size_t c = 0; c < std::min<size_t>(nchunks, STAGE_NBUF); ++c) {
        MBG_CUDA(cudaEventSynchronize(R.ev[c % STAGE_NBUF]));  // a previous call's DMA into it
        MBG_TRY(issue(c));
    }
    for (size_t c = 0; c < nchunks; ++c) {
        const int b = int(c % STAGE_NBUF);
        const size_t r0 = c * per, nr = std::min(per, height - r0);
        MBG_CUDA(cudaEventSynchronize(R.ev[b]));
        CopyPool::get().copy_2d(static_cast<char*>(dst) + r0 * dpitch, dpitch, R.buf[b], width, width, nr);
        if (c + STAGE_NBUF < nchunks) MBG_TRY(issue(c + STAGE_NBUF));
    }
    // src may be reused by later work on s only after the DMAs have read it (they all have)
    return MBG_OK;
}

}  // namespace mbg
