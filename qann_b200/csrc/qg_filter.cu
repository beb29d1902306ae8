// Filtered IVF probing (reference src/ivf_index.cpp:501-521, with coarse_all
// :358-376): a query with an allowed-set filter ranks every list by its exact
// coarse score, probes at least max(nprobe, min_probes) lists, and keeps going,
// nearest first, until it has seen `wanted` allowed vectors. The reference
// stops on its TopK's size, which before the first trim (at 2k pushes) counts
// exactly the allowed vectors scanned; so the probe count of each query is the
// first p >= min_probes whose lists hold >= wanted allowed vectors.
#include "qg_device.cuh"
#include "qg_search.h"

#include <algorithm>
#include <vector>

namespace qg {

// one block per query: every list sorted by (score, list) (float order, -0 == +0)
__global__ void __launch_bounds__(256) k_rank_lists(const float* __restrict__ scores, int nlist, int npow,
                                                    uint32_t* __restrict__ out_list, float* __restrict__ out_score) {
    extern __shared__ uint64_t keys[];
    const float* row = scores + static_cast<size_t>(blockIdx.x) * nlist;
    for (int i = threadIdx.x; i < npow; i += blockDim.x)
        keys[i] = i < nlist ? (static_cast<uint64_t>(float_key_eq0(row[i])) << 32) | static_cast<uint32_t>(i) : ~0ull;
    bitonic_sort_keys(keys, npow);
    for (int i = threadIdx.x; i < nlist; i += blockDim.x) {
        const uint32_t l = static_cast<uint32_t>(keys[i]);
        out_list[static_cast<size_t>(blockIdx.x) * nlist + i] = l;
        out_score[static_cast<size_t>(blockIdx.x) * nlist + i] = row[l];
    }
}

// warp per list: allowed (filter bit set) vectors of the list
__global__ void k_list_allowed(IvfView v, const uint64_t* __restrict__ filter, uint32_t* __restrict__ cnt) {
    const int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (l >= v.nlist) return;
    const size_t b0 = static_cast<size_t>(v.sb_off[l]) * kSuperBlock;
    const uint32_t n = v.list_size[l];
    uint32_t c = 0;
    for (uint32_t j = lane; j < n; j += 32) {
        const uint32_t slot = v.ids[b0 + j];
        c += (filter[slot >> 6] >> (slot & 63)) & 1ull;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[l] = c;
}

// thread per query: the probe count
__global__ void k_probe_count(const uint32_t* __restrict__ ranked, const uint32_t* __restrict__ cnt, int nq, int nlist,
                              int min_probes, int wanted, int* __restrict__ out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const uint32_t* r = ranked + static_cast<size_t>(q) * nlist;
    long long seen = 0;
    int p = 0;
    for (; p < nlist; ++p) {
        if (p >= min_probes && seen >= wanted) break;
        seen += cnt[r[p]];
    }
    out[q] = p;
}

__global__ void k_take_columns(const uint32_t* __restrict__ list_in, const float* __restrict__ score_in, int nq,
                               int nlist, int P, uint32_t* __restrict__ list_out, float* __restrict__ score_out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(nq) * P) return;
    const size_t q = t / P, c = t % P;
    list_out[t] = list_in[q * nlist + c];
    score_out[t] = score_in[q * nlist + c];
}

int filtered_probes(const IvfView& v, const IvfSearchArgs& s, DevBuf<uint32_t>& probe, DevBuf<float>& pdist,
                    DevBuf<int>& nprobe_q, cudaStream_t st) {
    const int nq = s.nq, nlist = v.nlist;
    const int npow = next_pow2(nlist);
    const size_t smem = static_cast<size_t>(npow) * 8;
    require(smem <= 200 * 1024, "filtered queries on the GPU path need nlist <= 16384 (every list is ranked in "
                                "shared memory)", kUnsupported);
    DevBuf<float> scores(static_cast<size_t>(nq) * nlist, st);
    pair_scores(s.q, nq, v.centroids, nlist, v.dim, v.ip_metric, scores.get(), nlist, st);
    DevBuf<uint32_t> ranked(static_cast<size_t>(nq) * nlist, st);
    DevBuf<float> rscore(static_cast<size_t>(nq) * nlist, st);
    if (smem > 48 * 1024)
        QG_CUDA(cudaFuncSetAttribute(k_rank_lists, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    {
        KernelTimer kt("rank_lists", st);
        k_rank_lists<<<nq, 256, smem, st>>>(scores.get(), nlist, npow, ranked.get(), rscore.get());
        QG_LAUNCH_CHECK();
    }
    scores.release();
    DevBuf<uint32_t> cnt(nlist, st);
    k_list_allowed<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nlist) * 32, 256)), 256, 0, st>>>(v, s.filter,
                                                                                                    cnt.get());
    QG_LAUNCH_CHECK();
    nprobe_q.alloc(nq, st);
    k_probe_count<<<static_cast<unsigned>(ceil_div(nq, 128)), 128, 0, st>>>(ranked.get(), cnt.get(), nq, nlist,
                                                                            s.min_probes, s.wanted, nprobe_q.get());
    QG_LAUNCH_CHECK();
    std::vector<int> h(nq);
    QG_CUDA(cudaMemcpyAsync(h.data(), nprobe_q.get(), nq * sizeof(int), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    const int P = std::max(1, *std::max_element(h.begin(), h.end()));
    probe.alloc(static_cast<size_t>(nq) * P, st);
    pdist.alloc(static_cast<size_t>(nq) * P, st);
    k_take_columns<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * P, 256)), 256, 0, st>>>(
        ranked.get(), rscore.get(), nq, nlist, P, probe.get(), pdist.get());
    QG_LAUNCH_CHECK();
    return P;
}

} // namespace qg
