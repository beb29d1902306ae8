// Filtered IVF probing (reference src/ivf_index.cpp:501-521, with coarse_all
// :358-376): a query with an allowed-set filter ranks every list by its exact
// coarse score, probes at least max(nprobe, min_probes) lists, and keeps going,
// nearest first, until it has seen `wanted` allowed vectors. The reference
// stops on its TopK's size, which before the first trim (at 2k pushes) counts
// exactly the allowed vectors scanned; so the probe count of each query is the
// first p >= min_probes whose lists hold >= wanted allowed vectors. Each query
// may carry its own filter (a mixed batch of served requests); the walk reads
// only the ids of the lists the query goes on to scan: the min_probes nearest
// ones in parallel, then one list at a time while fewer than `wanted` are seen.
#include "qg_device.cuh"
#include "qg_search.h"

#include <algorithm>
#include <atomic>
#include <vector>

namespace qg {

namespace {
std::atomic<int64_t> g_ranked_batches{0}, g_deep_walks{0};
void count_deep_walks(int64_t n) { g_deep_walks += n; }
}

void filtered_rank_counts(int64_t* batches, int64_t* deep) {
    *batches = g_ranked_batches.load();
    *deep = g_deep_walks.load();
}

// one block per query: every list sorted by (score, list) (float order, -0 == +0);
// 1024 threads, as the sort's stages are barrier-bound and the keys (up to
// 128 KB) hold the SM to one block anyway
__global__ void __launch_bounds__(1024) k_rank_lists(const float* __restrict__ scores, int nlist, int npow,
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

// Allowed vectors in the min_probes nearest lists of each filtered query, in
// parallel: kWalkBlocks blocks per query, a warp per list at a time, the id
// and bitmap loads of 4 strides of the list in flight together; the blocks'
// counts meet by atomics in seen[q] (zero at launch).
constexpr int kWalkBlocks = 16;
__global__ void __launch_bounds__(256) k_allowed_first(IvfView v, const uint32_t* __restrict__ ranked, int R, int nq,
                                                       const uint64_t* filter, const uint64_t* const* filters,
                                                       int min_probes, const int* __restrict__ min_q,
                                                       unsigned long long* __restrict__ seen) {
    const int q = blockIdx.x / kWalkBlocks, part = blockIdx.x % kWalkBlocks;
    const uint64_t* f = filters ? filters[q] : filter;
    if (q >= nq || !f) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int mp = min(min_q ? min_q[q] : min_probes, R);
    const uint32_t* r = ranked + static_cast<size_t>(q) * R;
    uint32_t c = 0;
    for (int i = part * nw + warp; i < mp; i += kWalkBlocks * nw) {
        const uint32_t l = r[i];
        const size_t b0 = static_cast<size_t>(v.sb_off[l]) * kSuperBlock;
        const uint32_t n = v.list_size[l];
        for (uint32_t j0 = 0; j0 < n; j0 += 128) {
            uint32_t slot[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t j = j0 + 32 * u + lane;
                slot[u] = j < n ? v.ids[b0 + j] : 0xFFFFFFFFu;
            }
            uint64_t w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) w[u] = slot[u] != 0xFFFFFFFFu ? f[slot[u] >> 6] : 0ull;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (slot[u] != 0xFFFFFFFFu) c += static_cast<uint32_t>((w[u] >> (slot[u] & 63)) & 1ull);
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0 && c) atomicAdd(seen + q, static_cast<unsigned long long>(c));
}

// warp per query: its probe count. A query with a filter walks its lists
// nearest first, counting each list's allowed vectors, and stops at the first
// p >= min_probes with >= wanted seen (the reference stops on its TopK's size,
// which before the first trim counts exactly the allowed vectors scanned). The
// min_probes nearest lists are counted in parallel beforehand (seen0), so the
// walk starts there and usually stops at once. A query without a filter
// probes its own nprobe. Only the R nearest lists are ranked: a walk that
// would go past them gives -1, and the caller ranks every list.
__global__ void k_probe_walk(IvfView v, const uint32_t* __restrict__ ranked, int R, int nq, const uint64_t* filter,
                             const uint64_t* const* filters, int min_probes, int wanted, const int* __restrict__ min_q,
                             const int* __restrict__ wanted_q, int nprobe, const int* __restrict__ nprobe_q,
                             const unsigned long long* __restrict__ seen0, int* __restrict__ out) {
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
    const uint32_t* r = ranked + static_cast<size_t>(q) * R;
    long long seen = static_cast<long long>(seen0[q]);
    int p = min(mp, R);   // lists [0, p) are counted in seen
    if (p < mp) {         // (the caller ranks at least min_probes lists; kept for safety)
        if (lane == 0) out[q] = -1;
        return;
    }
    for (; p < R; ++p) {
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
    const bool stopped = p < R || seen >= want || R == nlist;   // (p >= mp here)
    if (lane == 0) out[q] = stopped ? p : -1;
}

// With only the R nearest lists ranked (R well under nlist), every one of them
// is counted at once: a warp per list, its allowed vectors in cnt[q * R + i].
__global__ void __launch_bounds__(256) k_allowed_each(IvfView v, const uint32_t* __restrict__ ranked, int R, int nq,
                                                      const uint64_t* filter, const uint64_t* const* filters,
                                                      uint32_t* __restrict__ cnt) {
    const int q = blockIdx.x;
    const uint64_t* f = filters ? filters[q] : filter;
    if (q >= nq || !f) return;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= R) return;
    const uint32_t l = ranked[static_cast<size_t>(q) * R + i];
    const size_t b0 = static_cast<size_t>(v.sb_off[l]) * kSuperBlock;
    const uint32_t n = v.list_size[l];
    uint32_t c = 0;
    for (uint32_t j0 = 0; j0 < n; j0 += 128) {
        uint32_t slot[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t j = j0 + 32 * u + lane;
            slot[u] = j < n ? v.ids[b0 + j] : 0xFFFFFFFFu;
        }
        uint64_t w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) w[u] = slot[u] != 0xFFFFFFFFu ? f[slot[u] >> 6] : 0ull;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (slot[u] != 0xFFFFFFFFu) c += static_cast<uint32_t>((w[u] >> (slot[u] & 63)) & 1ull);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[static_cast<size_t>(q) * R + i] = c;
}

// warp per query, over the per-list counts of k_allowed_each: the first
// p >= min_probes whose lists [0, p) hold >= wanted allowed vectors (the
// stopping rule of k_probe_walk), found 32 lists at a time by a prefix sum;
// -1 when the R ranked lists are not enough. Unfiltered queries: their nprobe.
__global__ void k_probe_count(int nlist, int R, int nq, const uint64_t* filter, const uint64_t* const* filters,
                              int min_probes, int wanted, const int* __restrict__ min_q,
                              const int* __restrict__ wanted_q, int nprobe, const int* __restrict__ nprobe_q,
                              const uint32_t* __restrict__ cnt, int* __restrict__ out) {
    const int q = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    const uint64_t* f = filters ? filters[q] : filter;
    if (!f) {
        if (lane == 0) out[q] = min(nprobe_q ? nprobe_q[q] : nprobe, nlist);
        return;
    }
    const int mp = min_q ? min_q[q] : min_probes;
    const long long want = wanted_q ? wanted_q[q] : wanted;
    const uint32_t* c = cnt + static_cast<size_t>(q) * R;
    long long before = 0;   // allowed vectors in the lists ahead of this round
    int found = -1;
    for (int base = 0; base < R && found < 0; base += 32) {
        const int i = base + lane;
        long long incl = i < R ? c[i] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int p = i + 1;   // lists [0, p) hold before + incl
        const bool ok = i < R && p >= mp && before + incl >= want;
        const unsigned hit = __ballot_sync(0xffffffffu, ok);
        if (hit) found = base + __ffs(hit);
        before += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) out[q] = found;
}

__global__ void k_take_columns(const uint32_t* __restrict__ list_in, const float* __restrict__ score_in, int nq,
                               int R, int P, uint32_t* __restrict__ list_out, float* __restrict__ score_out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(nq) * P) return;
    const size_t q = t / P, c = t % P;
    list_out[t] = list_in[q * R + c];
    score_out[t] = score_in[q * R + c];
}

int filtered_probes(const IvfView& v, const IvfSearchArgs& s, DevBuf<uint32_t>& probe, DevBuf<float>& pdist,
                    DevBuf<int>& nprobe_q, cudaStream_t st) {
    const int nq = s.nq, nlist = v.nlist;
    const int npow = next_pow2(nlist);
    const size_t smem = static_cast<size_t>(npow) * 8;
    nprobe_q.alloc(nq, st);
    DevBuf<unsigned long long> seen(nq, st);
    std::vector<int> h(nq);
    DevBuf<uint32_t> ranked;
    DevBuf<float> rscore;
    // R nearest lists ranked per query (the coarse step's selection), and if a
    // walk goes past them, every list (exact scores and a full sort)
    int R = s.rank_depth > 0 && s.rank_depth < nlist ? std::max(s.rank_depth, s.nprobe) : nlist;
    g_ranked_batches += 1;
    for (;;) {
        if (R >= nlist) R = nlist;
        ranked.alloc(static_cast<size_t>(nq) * R, st);
        rscore.alloc(static_cast<size_t>(nq) * R, st);
        if (R < nlist) {
            nearest_lists(v, s, nq, R, ranked.get(), rscore.get(), st);
        } else {
            require(smem <= 200 * 1024, "filtered queries on the GPU path need nlist <= 16384 (every list is "
                                        "ranked in shared memory)", kUnsupported);
            DevBuf<float> scores(static_cast<size_t>(nq) * nlist, st);
            pair_scores(s.q, nq, v.centroids, nlist, v.dim, v.ip_metric, scores.get(), nlist, st);
            if (smem > 48 * 1024)
                allow_large_smem<k_rank_lists>();
            KernelTimer kt("rank_lists", st);
            k_rank_lists<<<nq, 1024, smem, st>>>(scores.get(), nlist, npow, ranked.get(), rscore.get());
            QG_LAUNCH_CHECK();
        }
        if (R < nlist) {
            // every ranked list counted at once, then a prefix sum per query
            DevBuf<uint32_t> cnt(static_cast<size_t>(nq) * R, st);
            KernelTimer kt("probe_walk", st);
            k_allowed_each<<<dim3(static_cast<unsigned>(nq), static_cast<unsigned>(ceil_div(R, 8))), 256, 0, st>>>(
                v, ranked.get(), R, nq, s.filter, s.pq.filter, cnt.get());
            QG_LAUNCH_CHECK();
            k_probe_count<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * 32, 256)), 256, 0, st>>>(
                nlist, R, nq, s.filter, s.pq.filter, s.min_probes, s.wanted, s.pq.min_probes, s.pq.wanted, s.nprobe,
                s.pq.nprobe, cnt.get(), nprobe_q.get());
            QG_LAUNCH_CHECK();
        } else {
            // every list ranked: the min_probes nearest counted at once, then the walk list by list
            QG_CUDA(cudaMemsetAsync(seen.get(), 0, nq * sizeof(unsigned long long), st));
            KernelTimer kt("probe_walk", st);
            k_allowed_first<<<static_cast<unsigned>(nq) * kWalkBlocks, 256, 0, st>>>(
                v, ranked.get(), R, nq, s.filter, s.pq.filter, s.min_probes, s.pq.min_probes, seen.get());
            QG_LAUNCH_CHECK();
            k_probe_walk<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * 32, 256)), 256, 0, st>>>(
                v, ranked.get(), R, nq, s.filter, s.pq.filter, s.min_probes, s.wanted, s.pq.min_probes, s.pq.wanted,
                s.nprobe, s.pq.nprobe, seen.get(), nprobe_q.get());
            QG_LAUNCH_CHECK();
        }
        QG_CUDA(cudaMemcpyAsync(h.data(), nprobe_q.get(), nq * sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        if (R == nlist || *std::min_element(h.begin(), h.end()) >= 0) break;
        R = nlist;   // some walk went past the ranked lists
        count_deep_walks(1);
    }
    const int P = std::max(1, *std::max_element(h.begin(), h.end()));
    probe.alloc(static_cast<size_t>(nq) * P, st);
    pdist.alloc(static_cast<size_t>(nq) * P, st);
    k_take_columns<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * P, 256)), 256, 0, st>>>(
        ranked.get(), rscore.get(), nq, R, P, probe.get(), pdist.get());
    QG_LAUNCH_CHECK();
    return P;
}

} // namespace qg
