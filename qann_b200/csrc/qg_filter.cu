// Filtered IVF probing (reference src/ivf_index.cpp:501-521, with coarse_all
// :358-376): a query with an allowed-set filter ranks every list by its exact
// coarse score, probes at least max(nprobe, min_probes) lists, and keeps going,
// nearest first, until it has seen `wanted` allowed vectors. The reference
// stops on its TopK's size, which before the first trim (at 2k pushes) counts
// exactly the allowed vectors scanned; so the probe count of each query is the
// first p >= min_probes whose lists hold >= wanted allowed vectors. Each query
// may carry its own filter (a mixed batch of served requests); the walk reads
// only the ids of the lists the query goes on to scan.
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

// warp per query: its probe count. A query with a filter walks its lists
// nearest first, counting each list's allowed vectors, and stops at the first
// p >= min_probes with >= wanted seen (the reference stops on its TopK's size,
// which before the first trim counts exactly the allowed vectors scanned). A
// query without one probes its own nprobe.
__global__ void k_probe_walk(IvfView v, const uint32_t* __restrict__ ranked, int nq, const uint64_t* filter,
                             const uint64_t* const* filters, int min_probes, int wanted, const int* __restrict__ min_q,
                             const int* __restrict__ wanted_q, int nprobe, const int* __restrict__ nprobe_q,
                             int* __restrict__ out) {
    const int q = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int nlist = v.nlist;
    const uint64_t* f = filters ? filters[q] : filter;
    if (!f) {
        if (lane == 0) out[q] = min(nprobe_q ? nprobe_q[q] : nprobe, nlist);
        return;
    }
    const int mp = min_q ? min_q[q] : min_probes;
    const long long want = wanted_q ? wanted_q[q] : wanted;
    const uint32_t* r = ranked + static_cast<size_t>(q) * nlist;
    long long seen = 0;
    int p = 0;
    for (; p < nlist; ++p) {
        if (p >= mp && seen >= want) break;
        const uint32_t l = r[p];
        const size_t b0 = static_cast<size_t>(v.sb_off[l]) * kSuperBlock;
        const uint32_t n = v.list_size[l];
        uint32_t c = 0;
        for (uint32_t j = lane; j < n; j += 32) {
            const uint32_t slot = v.ids[b0 + j];
            if (slot != 0xFFFFFFFFu) c += (f[slot >> 6] >> (slot & 63)) & 1ull;
        }
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        seen += c;
    }
    if (lane == 0) out[q] = p;
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
        allow_large_smem<k_rank_lists>();
    {
        KernelTimer kt("rank_lists", st);
        k_rank_lists<<<nq, 256, smem, st>>>(scores.get(), nlist, npow, ranked.get(), rscore.get());
        QG_LAUNCH_CHECK();
    }
    scores.release();
    nprobe_q.alloc(nq, st);
    k_probe_walk<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * 32, 256)), 256, 0, st>>>(
        v, ranked.get(), nq, s.filter, s.pq.filter, s.min_probes, s.wanted, s.pq.min_probes, s.pq.wanted, s.nprobe,
        s.pq.nprobe, nprobe_q.get());
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
