// Host-side CUDA plumbing shared by every source of the library: error
// translation, stream-ordered device buffers, small utilities. No device code,
// so plain C++ translation units can include it.
#pragma once

#include <cuda_runtime.h>

#include "qg_error.h"

#include <cstddef>
#include <cstdint>
#include <string>

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

#define QG_LAUNCH_CHECK() QG_CUDA(cudaGetLastError())

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
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        count = 0;
    }
    T* get() const { return ptr; }
    size_t bytes() const { return count * sizeof(T); }
};

} // namespace qg
