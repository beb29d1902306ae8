// Host-side CUDA plumbing shared by every source of the library: error
// translation, stream-ordered device buffers, small utilities. No device code,
// so plain C++ translation units can include it.
#pragma once

#include <cuda_runtime.h>

#include "qg_error.h"

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace qg {

[[noreturn]] inline void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
    std::string msg = std::string("CUDA error in ") + what + " (" + file + ":" + std::to_string(line) +
                      "): " + cudaGetErrorString(e);
    throw Error(e == cudaErrorMemoryAllocation ? kOutOfMemory : kCudaError, msg);
}

#define QG_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t qg_e_ = (call);                                          \
        if (qg_e_ != cudaSuccess) ::qg::throw_cuda(qg_e_, #call, __FILE__, __LINE__); \
    } while (0)

// ---------------------------------------------------------------------------
// Profiling: a count of this library's kernel launches, and (when enabled)
// CUDA-event timings of named kernels recorded on the stream they run on.
// ---------------------------------------------------------------------------
struct Profiler {
    std::atomic<bool> on{false};
    std::atomic<int64_t> launches{0};
    std::mutex mu;
    struct Pending {
        std::string name;
        cudaEvent_t start, stop;
    };
    std::vector<Pending> pending;
    std::map<std::string, std::pair<double, int64_t>> totals;   // name -> (ms, launches)

    void settle() {   // folds finished event pairs into the totals (caller holds mu)
        for (auto& p : pending) {
            float ms = 0.0f;
            if (cudaEventSynchronize(p.stop) == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
                auto& t = totals[p.name];
                t.first += ms;
                t.second += 1;
            }
            cudaEventDestroy(p.start);
            cudaEventDestroy(p.stop);
        }
        pending.clear();
    }
};

inline Profiler& profiler() {
    static Profiler p;
    return p;
}

// Brackets one kernel launch with events on its stream when profiling is on.
class KernelTimer {
public:
    KernelTimer(const char* name, cudaStream_t st) : st_(st) {
        if (!profiler().on.load(std::memory_order_relaxed)) return;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;   // no timers inside a graph capture
        if (cudaStreamIsCapturing(st_, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
        name_ = name;
        if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) return;
        cudaEventRecord(a_, st_);
        armed_ = true;
    }
    ~KernelTimer() { stop(); }
    // ends the bracket early (a section of several launches)
    void stop() {
        if (!armed_) return;
        armed_ = false;
        cudaEventRecord(b_, st_);
        std::lock_guard<std::mutex> g(profiler().mu);
        profiler().pending.push_back({name_, a_, b_});
    }
    KernelTimer(const KernelTimer&) = delete;
    KernelTimer& operator=(const KernelTimer&) = delete;

private:
    cudaStream_t st_;
    std::string name_;
    cudaEvent_t a_{}, b_{};
    bool armed_ = false;
};

#define QG_LAUNCH_CHECK()                                                       \
    do {                                                                        \
        ::qg::profiler().launches.fetch_add(1, std::memory_order_relaxed);      \
        QG_CUDA(cudaGetLastError());                                            \
    } while (0)

// ---------------------------------------------------------------------------
inline size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

// Number of SMs of the current device (cached per device by the caller).
inline int sm_count() {
    int dev = 0, n = 0;
    QG_CUDA(cudaGetDevice(&dev));
    QG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

// Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync on one stream).
// Lets a kernel take the device's opt-in maximum of dynamic shared memory.
// Set once per kernel and never lowered: the attribute is process-wide, so a
// per-launch value set by one thread could undercut another thread's launch.
template <auto Kernel>
void allow_large_smem() {
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0, optin = 0;
        QG_CUDA(cudaGetDevice(&dev));
        QG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa{};
        QG_CUDA(cudaFuncGetAttributes(&fa, Kernel));   // dynamic + static must fit the opt-in limit
        QG_CUDA(cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     optin - static_cast<int>(fa.sharedSizeBytes)));
    });
}

template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaStream_t stream = nullptr;

    DevBuf() = default;
    DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream) { o.ptr = nullptr; o.count = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr; count = o.count; stream = o.stream;
            o.ptr = nullptr; o.count = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }

    void alloc(size_t n, cudaStream_t s) {
        release();
        stream = s;
        count = n;
        if (n) QG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ptr), n * sizeof(T), s));
    }
    void release() noexcept {
        // a failed free must not surface later as some launch's error
        if (ptr && cudaFreeAsync(ptr, stream) != cudaSuccess) (void)cudaGetLastError();
        ptr = nullptr;
        count = 0;
    }
    T* get() const { return ptr; }
    size_t bytes() const { return count * sizeof(T); }
};

} // namespace qg
