// qg_fast_scan_noalloc_dev: the fast-scan block sums of qg_fast_scan_dev for
// callers that must not allocate device memory.
//
// Who needs it: code that owns all of the GPU's memory through its own pool
// (a serving process that reserves the device up front, or a host framework
// whose allocator is the only one allowed to call cudaMalloc) and code on a
// latency-critical path where an allocation is not acceptable, since
// cudaMalloc can synchronise the device and can fail when memory is full.
// qg_fast_scan_dev takes its working memory (the codes repacked into
// superblocks) from the stream-ordered allocator; this variant instead uses
// one statically sized device array compiled into the library.
//
// The array, kNoAllocScratchBytes = 32 MiB, is a file-scope __device__
// variable, so every GPU that loads the library holds it until the process
// exits. It bounds the input: the repacked codes of ceil(n / 64) superblocks
// (64 * m_pad / 2 bytes each, m_pad = m rounded up to a multiple of 4) plus a
// 4-byte list entry per superblock and a 256-byte header must fit, about
// 1 million vectors at m = 64. Larger inputs are refused with
// QG_INVALID_ARGUMENT before any GPU work.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (host code may not use the symbol itself: on the host
// it names a stand-in, not device memory); make that first call before any
// stream capture. All calls share the one array and it keeps the last call's
// contents: each call rewrites every part it reads, and calls that overlap on
// the GPU (on different streams, or from different host threads) race on it.
//
// Every LUT index lut_of[sb] is checked against nluts on the device; the call
// waits for its work (as qg_fast_scan_dev does) and returns
// QG_INVALID_ARGUMENT naming the first superblock whose index is out of
// range. Inputs are refused before any product of their sizes can wrap.
#include "../../include/qann_gpu.h"

#include "qg_device.cuh"
#include "qg_ops.h"

#include <algorithm>
#include <mutex>
#include <string>

namespace qg {

void set_last_error(const std::string& msg);   // qg_capi.cu

namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;
constexpr size_t kHeaderBytes = 256;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
unsigned char* scratch_on_current_device() {
    static std::mutex mu;
    static unsigned char* ptrs[64] = {};
    int dev = 0;
    QG_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, "device ordinal out of range");
    std::lock_guard<std::mutex> g(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        QG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        ptrs[dev] = static_cast<unsigned char*>(p);
    }
    return ptrs[dev];
}

inline size_t round256(size_t b) { return (b + 255) & ~size_t{255}; }

// one list of n vectors: offsets {0, n}, superblock offsets {0, nsb}, size n;
// word 5 receives the first superblock whose LUT index is out of range
__global__ void k_noalloc_header(uint32_t* meta, uint32_t n, uint32_t nsb) {
    meta[0] = 0;
    meta[1] = n;
    meta[2] = 0;
    meta[3] = nsb;
    meta[4] = n;
    meta[5] = 0xFFFFFFFFu;
}

// octet per superblock, the LUT rows of lut_of[sb] copied to shared memory
// with zero rows up to m_pad; an index of nluts or more is not followed (the
// superblock's sums stay unwritten and the lowest such superblock goes to *bad)
__global__ void k_noalloc_sums(const uint4* __restrict__ codes, size_t nsb, const uint4* __restrict__ luts, int m,
                               int m_pad, const uint32_t* __restrict__ lut_of, size_t nluts, size_t n,
                               uint16_t* __restrict__ sums, uint32_t* bad) {
    extern __shared__ uint4 lut_sm[];
    const int oct = threadIdx.x >> 3, r = threadIdx.x & 7;
    const size_t sb = static_cast<size_t>(blockIdx.x) * (blockDim.x >> 3) + oct;
    uint4* L = lut_sm + static_cast<size_t>(oct) * m_pad;
    bool skip = sb >= nsb;
    if (!skip) {
        const uint32_t li = lut_of[sb];   // the same for the octet's 8 lanes
        if (li >= nluts) {
            if (r == 0) atomicMin(bad, static_cast<uint32_t>(sb));
            skip = true;
        } else {
            const uint4* src = luts + static_cast<size_t>(li) * m;
            for (int row = r; row < m_pad; row += 8) L[row] = row < m ? src[row] : make_uint4(0, 0, 0, 0);
        }
    }
    __syncwarp();
    if (skip) return;
    uint32_t s[8];
    octet_sums(codes + sb * static_cast<size_t>(2 * m_pad), L, m_pad, r, s);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const size_t v = sb * kSuperBlock + 8 * r + i;
        if (v < n) sums[v] = static_cast<uint16_t>(s[i]);
    }
}

} // namespace
} // namespace qg

using namespace qg;

extern "C" int qg_fast_scan_noalloc_dev(const uint8_t* lut_dev, size_t nluts, size_t m, const uint8_t* codes_dev,
                                        const uint32_t* lut_of_dev, size_t n, uint16_t* sums_dev, void* stream) {
    try {
        require(m >= 1 && m <= kFsMaxSubspaces, "m must be in [1, 1024]");
        require(nluts >= 1, "need at least one LUT");
        require(reinterpret_cast<uintptr_t>(lut_dev) % 16 == 0, "the LUT buffer must be 16-byte aligned");
        if (n > kNoAllocScratchBytes)   // at least a byte of scratch per vector; also keeps n in 32 bits
            throw Error(kInvalidArgument, "qg_fast_scan_noalloc_dev: " + std::to_string(n) +
                                              " vectors exceed the static scratch (use qg_fast_scan_dev)");
        const int mi = static_cast<int>(m), m_pad = (mi + 3) & ~3;
        const size_t nsb = ceil_div(n, kSuperBlock);
        // bound the superblock count before any product, so that no size
        // wraps around: each superblock takes 32 * m_pad bytes of the scratch
        const size_t max_sb = kNoAllocScratchBytes / (32 * static_cast<size_t>(m_pad));
        const size_t need = nsb > max_sb ? 0
                                         : kHeaderBytes + round256(nsb * sizeof(uint32_t)) +
                                               nsb * 32 * static_cast<size_t>(m_pad);
        if (nsb > max_sb || need > kNoAllocScratchBytes)
            throw Error(kInvalidArgument, "qg_fast_scan_noalloc_dev: " + std::to_string(n) + " vectors of m = " +
                                              std::to_string(m) + " need more than the " +
                                              std::to_string(kNoAllocScratchBytes) +
                                              " bytes of the static scratch (use qg_fast_scan_dev)");
        if (n == 0) return QG_OK;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        unsigned char* base = scratch_on_current_device();
        uint32_t* meta = reinterpret_cast<uint32_t*>(base);
        uint32_t* sb_list = reinterpret_cast<uint32_t*>(base + kHeaderBytes);
        uint4* packed = reinterpret_cast<uint4*>(base + kHeaderBytes + round256(nsb * sizeof(uint32_t)));
        k_noalloc_header<<<1, 1, 0, st>>>(meta, static_cast<uint32_t>(n), static_cast<uint32_t>(nsb));
        QG_LAUNCH_CHECK();
        QG_CUDA(cudaMemsetAsync(sb_list, 0, nsb * sizeof(uint32_t), st));   // every superblock is in list 0
        pack_superblocks(codes_dev, nullptr, meta, meta + 2, meta + 4, sb_list, nsb, mi, m_pad, packed, nullptr, st);
        const int opb = static_cast<int>(
            std::max<size_t>(1, std::min<size_t>(16, (96 * 1024) / (static_cast<size_t>(m_pad) * 16))));
        const size_t smem = static_cast<size_t>(opb) * m_pad * 16;
        if (smem > 48 * 1024)
            allow_large_smem<k_noalloc_sums>();
        k_noalloc_sums<<<static_cast<unsigned>(ceil_div(nsb, opb)), 8 * opb, smem, st>>>(
            packed, nsb, reinterpret_cast<const uint4*>(lut_dev), mi, m_pad, lut_of_dev, nluts, n, sums_dev,
            meta + 5);
        QG_LAUNCH_CHECK();
        // the index check's verdict, copied to a host word (no allocation)
        uint32_t bad = 0;
        QG_CUDA(cudaMemcpyAsync(&bad, meta + 5, sizeof(bad), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        require(bad == 0xFFFFFFFFu,
                "lut_of[" + std::to_string(bad) + "] is not below nluts = " + std::to_string(nluts));
        return QG_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return QG_RUNTIME_ERROR;
    }
}
