// Kernel-level entry points on device memory: the LUT rounding and the code
// scan exposed on their own so parity tests can compare them with the
// reference's quantize_lut / build_quantize_lut / fast_scan_block directly.
#include "qg_device.cuh"
#include "qg_ops.h"

namespace qg {

// One warp per table: table i = B_i (+ C_i, + A_i on row 0), rounded to
// m rows of 16 bytes.
__global__ void k_quantize_luts(const float* __restrict__ B, const float* __restrict__ C, const float* __restrict__ A,
                                size_t n, int m, uint4* __restrict__ lut, float* __restrict__ scale,
                                float* __restrict__ offset) {
    extern __shared__ float rmin_all[];
    const int warp = threadIdx.x >> 5;
    const size_t i = static_cast<size_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
    if (i >= n) return;
    float* rmin = rmin_all + static_cast<size_t>(warp) * m;
    const float* b = B + i * static_cast<size_t>(m) * 16;
    const float* c = C ? C + i * static_cast<size_t>(m) * 16 : nullptr;
    const float a = A ? A[i] : 0.0f;
    float s, o;
    warp_quantize_lut(
        [&](int r, float* out) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float t = b[r * 16 + j];
                if (c) {
                    t = __fadd_rn(t, c[r * 16 + j]);
                    if (A && r == 0) t = __fadd_rn(t, a);
                }
                out[j] = t;
            }
        },
        m, m, rmin, lut + i * m, s, o);
    if ((threadIdx.x & 31) == 0) {
        scale[i] = s;
        offset[i] = o;
    }
}

void quantize_luts(const float* B, const float* C, const float* A, size_t n, size_t m, uint8_t* lut, float* scale,
                   float* offset, cudaStream_t st) {
    require(m >= 1 && m <= kFsMaxSubspaces, "m must be in [1, 1024]");
    require(reinterpret_cast<uintptr_t>(lut) % 16 == 0, "the LUT buffer must be 16-byte aligned");
    if (n == 0) return;
    constexpr int WPB = 4;
    const size_t smem = static_cast<size_t>(WPB) * m * sizeof(float);
    k_quantize_luts<<<static_cast<unsigned>(ceil_div(n, WPB)), 32 * WPB, smem, st>>>(
        B, C, A, n, static_cast<int>(m), reinterpret_cast<uint4*>(lut), scale, offset);
    QG_LAUNCH_CHECK();
}

// Sums of superblocks: octet per superblock, its LUT (by lut_of[sb]) copied
// to shared memory with zero rows up to m_pad. A LUT index of nluts or more
// is not followed: the superblock's sums are left unwritten and the lowest
// such superblock is recorded in *bad (which starts at 0xFFFFFFFF).
__global__ void k_scan_sums(const uint4* __restrict__ codes, size_t nsb, const uint4* __restrict__ luts, int m,
                            int m_pad, const uint32_t* __restrict__ lut_of, size_t nluts, size_t n,
                            uint16_t* __restrict__ sums, uint32_t* bad) {
    extern __shared__ uint4 lut_sm[];   // one LUT per octet of the block
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

void fast_scan_sums(const uint8_t* lut, size_t nluts, size_t m, const uint8_t* codes, const uint32_t* lut_of, size_t n,
                    uint16_t* sums, cudaStream_t st) {
    require(m >= 1 && m <= kFsMaxSubspaces, "m must be in [1, 1024]");
    require(nluts >= 1, "need at least one LUT");
    require(reinterpret_cast<uintptr_t>(lut) % 16 == 0, "the LUT buffer must be 16-byte aligned");
    require(n <= 0xFFFFFFFFu, "n must fit in 32 bits");
    if (n == 0) return;
    const int mi = static_cast<int>(m), m_pad = (mi + 3) & ~3;
    const size_t nsb = ceil_div(n, kSuperBlock);
    // one list holding all n vectors; word 5 receives the first superblock
    // whose LUT index is out of range
    const uint32_t h_meta[6] = {0, static_cast<uint32_t>(n), 0, static_cast<uint32_t>(nsb), static_cast<uint32_t>(n),
                                0xFFFFFFFFu};
    DevBuf<uint32_t> meta(6, st), sbl(nsb, st);
    QG_CUDA(cudaMemcpyAsync(meta.get(), h_meta, sizeof(h_meta), cudaMemcpyHostToDevice, st));
    QG_CUDA(cudaMemsetAsync(sbl.get(), 0, nsb * 4, st));
    DevBuf<uint4> packed(nsb * 2 * m_pad, st);
    pack_superblocks(codes, nullptr, meta.get(), meta.get() + 2, meta.get() + 4, sbl.get(), nsb, mi, m_pad, packed.get(),
                     nullptr, st);
    // octets per block: as many LUT copies as fit in 96 KB of shared memory
    const int OPB = static_cast<int>(std::max<size_t>(1, std::min<size_t>(16, (96 * 1024) / (static_cast<size_t>(m_pad) * 16))));
    const size_t smem = static_cast<size_t>(OPB) * m_pad * 16;
    if (smem > 48 * 1024)
        allow_large_smem<k_scan_sums>();
    k_scan_sums<<<static_cast<unsigned>(ceil_div(nsb, OPB)), 8 * OPB, smem, st>>>(
        packed.get(), nsb, reinterpret_cast<const uint4*>(lut), mi, m_pad, lut_of, nluts, n, sums, meta.get() + 5);
    QG_LAUNCH_CHECK();
    uint32_t bad = 0;
    QG_CUDA(cudaMemcpyAsync(&bad, meta.get() + 5, 4, cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    require(bad == 0xFFFFFFFFu, "lut_of[" + std::to_string(bad) + "] is not below nluts = " + std::to_string(nluts));
}

} // namespace qg
