// Device side of index training: grouping points by cluster in point order,
// cluster means, the state of mini-batch EMA k-means (e-means) between its
// steps, and the sample evaluation behind the cosine scoring decision. The
// drivers (qg_train_host.cpp) keep only the random draws on the host, so a
// training step is a chain of kernels on one stream with no host round trip.
//
// Every float operation that must match the reference's CPU build is written
// with an explicit round-to-nearest intrinsic (this library builds with
// -fmad=false), FMAs exactly where the reference's GCC build contracts.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_search.h"
#include "qg_train.h"

#include <cmath>

namespace qg {

// ---------------------------------------------------------------------------
// Grouping by label, stable. P problems of n labelled points each: `order`
// lists each problem's points cluster by cluster, in point order inside a
// cluster, and off[p][c] is where cluster c starts. The points are cut into
// chunks; one warp walks a chunk 32 points at a time and ranks equal labels
// among its lanes with __match_any_sync, so the order inside a chunk is kept,
// and chunks of a cluster are placed in chunk order by an exclusive prefix
// over the (problem, cluster, chunk) tallies.
// ---------------------------------------------------------------------------
namespace {

struct ChunkGrid {
    size_t chunk;   // points per chunk, a multiple of 32
    int nchunks;    // per problem
};

ChunkGrid chunk_grid(size_t n, int k, int P) {
    // keep the tally (P * k * nchunks words) near 8M entries at most
    const size_t cap = std::max<size_t>(1, (size_t{8} << 20) / (static_cast<size_t>(P) * k));
    const size_t nc = std::max<size_t>(1, std::min(cap, ceil_div(n, 32)));
    const size_t chunk = ceil_div(ceil_div(n, nc), 32) * 32;
    return {chunk, static_cast<int>(ceil_div(n, chunk))};
}

__global__ void k_group_tally(const uint32_t* __restrict__ labels, size_t n, int k, int P, size_t chunk, int nchunks,
                              uint32_t* __restrict__ tally) {
    const size_t w = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= static_cast<size_t>(P) * nchunks) return;
    const int p = static_cast<int>(w / nchunks), c = static_cast<int>(w % nchunks);
    const size_t i0 = static_cast<size_t>(c) * chunk, i1 = min(n, i0 + chunk);
    const uint32_t* lab = labels + static_cast<size_t>(p) * n;
    uint32_t* t = tally + static_cast<size_t>(p) * k * nchunks + c;
    for (size_t g = i0; g < i1; g += 32) {
        const size_t i = g + lane;
        const uint32_t l = i < i1 ? lab[i] : 0xFFFFFFFFu;
        const bool live = l < static_cast<uint32_t>(k);
        const unsigned act = __ballot_sync(0xffffffffu, live);
        if (live) {
            const unsigned peers = __match_any_sync(act, l);
            if (lane == __ffs(peers) - 1) t[static_cast<size_t>(l) * nchunks] += __popc(peers);
        }
        __syncwarp();
    }
}

// off[p][c] = first position of cluster c in problem p's part of `order`
__global__ void k_group_offsets(const uint32_t* __restrict__ start, size_t n, int k, int P, int nchunks,
                                uint32_t* __restrict__ off) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(P) * (k + 1)) return;
    const size_t p = t / (k + 1);
    const int c = static_cast<int>(t % (k + 1));
    off[t] = c == k ? static_cast<uint32_t>(n)
                    : static_cast<uint32_t>(start[(p * k + c) * nchunks] - p * n);
}

__global__ void k_group_place(const uint32_t* __restrict__ labels, size_t n, int k, int P, size_t chunk, int nchunks,
                              uint32_t* __restrict__ cursor, uint32_t* __restrict__ order) {
    const size_t w = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= static_cast<size_t>(P) * nchunks) return;
    const int p = static_cast<int>(w / nchunks), c = static_cast<int>(w % nchunks);
    const size_t i0 = static_cast<size_t>(c) * chunk, i1 = min(n, i0 + chunk);
    const uint32_t* lab = labels + static_cast<size_t>(p) * n;
    uint32_t* cur = cursor + static_cast<size_t>(p) * k * nchunks + c;
    const unsigned below = (1u << lane) - 1u;
    for (size_t g = i0; g < i1; g += 32) {
        const size_t i = g + lane;
        const uint32_t l = i < i1 ? lab[i] : 0xFFFFFFFFu;
        const bool live = l < static_cast<uint32_t>(k);
        const unsigned act = __ballot_sync(0xffffffffu, live);
        if (live) {
            const unsigned peers = __match_any_sync(act, l);
            const int first = __ffs(peers) - 1;
            uint32_t at = 0;
            if (lane == first) at = cur[static_cast<size_t>(l) * nchunks];
            at = __shfl_sync(peers, at, first);
            order[at + __popc(peers & below)] = static_cast<uint32_t>(i);
            if (lane == first) cur[static_cast<size_t>(l) * nchunks] = at + __popc(peers);
        }
        __syncwarp();
    }
}

// Exclusive prefix sums of uint32 in place: tiles of 4096 (4 per thread),
// tile totals scanned recursively, then added back.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan_tile(uint32_t* __restrict__ a, size_t n,
                                                             uint32_t* __restrict__ tile_sum) {
    __shared__ uint32_t warp_sum[kScanThreads / 32];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile + static_cast<size_t>(threadIdx.x) * kScanPer;
    uint32_t v[kScanPer], run = 0;
#pragma unroll
    for (int u = 0; u < kScanPer; ++u) {
        v[u] = base + u < n ? a[base + u] : 0u;
        run += v[u];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = run;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = warp_sum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;   // inclusive over warps
    }
    __syncthreads();
    uint32_t ex = inc - run + (warp > 0 ? warp_sum[warp - 1] : 0u);
#pragma unroll
    for (int u = 0; u < kScanPer; ++u) {
        if (base + u < n) a[base + u] = ex;
        ex += v[u];
    }
    if (threadIdx.x == kScanThreads - 1) tile_sum[blockIdx.x] = warp_sum[kScanThreads / 32 - 1];
}

__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* __restrict__ a, size_t n,
                                                            const uint32_t* __restrict__ tile_off) {
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
    const uint32_t add = tile_off[blockIdx.x];
    for (int u = threadIdx.x; u < kScanTile; u += kScanThreads)
        if (base + u < n) a[base + u] += add;
}

} // namespace

void exclusive_scan_u32(uint32_t* a, size_t n, cudaStream_t st) {
    if (n == 0) return;
    const size_t tiles = ceil_div(n, kScanTile);
    DevBuf<uint32_t> sums(tiles, st);
    k_scan_tile<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(a, n, sums.get());
    QG_LAUNCH_CHECK();
    if (tiles > 1) {
        exclusive_scan_u32(sums.get(), tiles, st);
        k_scan_add<<<static_cast<unsigned>(tiles), kScanThreads, 0, st>>>(a, n, sums.get());
        QG_LAUNCH_CHECK();
    }
}

void group_by_label(const uint32_t* labels, size_t n, int k, int P, uint32_t* order, uint32_t* off, cudaStream_t st) {
    require(static_cast<double>(n) * P < 4294967295.0, "grouping supports fewer than 2^32 points");
    if (n == 0) {
        QG_CUDA(cudaMemsetAsync(off, 0, static_cast<size_t>(P) * (k + 1) * sizeof(uint32_t), st));
        return;
    }
    const ChunkGrid g = chunk_grid(n, k, P);
    const size_t cells = static_cast<size_t>(P) * k * g.nchunks;
    DevBuf<uint32_t> tally(cells, st);
    QG_CUDA(cudaMemsetAsync(tally.get(), 0, cells * sizeof(uint32_t), st));
    const size_t warps = static_cast<size_t>(P) * g.nchunks;
    const unsigned blocks = static_cast<unsigned>(ceil_div(warps * 32, 256));
    k_group_tally<<<blocks, 256, 0, st>>>(labels, n, k, P, g.chunk, g.nchunks, tally.get());
    QG_LAUNCH_CHECK();
    exclusive_scan_u32(tally.get(), cells, st);
    k_group_offsets<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(P) * (k + 1), 256)), 256, 0, st>>>(
        tally.get(), n, k, P, g.nchunks, off);
    QG_LAUNCH_CHECK();
    k_group_place<<<blocks, 256, 0, st>>>(labels, n, k, P, g.chunk, g.nchunks, tally.get(), order);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Means of the member sums (float division by the count), made unit length
// for spherical k-means: the squared norm summed in double in dimension
// order, scale = float(1 / sqrt(sq)). An empty cluster's row is zero and
// raises *empty. Thread per (problem, cluster).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void unit_scale_row(float* row, int d, bool zero_when_empty) {
    double sq = 0.0;
    for (int l = 0; l < d; ++l) {
        const double v = static_cast<double>(row[l]);
        sq = __fma_rn(v, v, sq);   // the product is exact in double: fused or not, one rounding
    }
    if (sq > 0.0) {
        const float scale = __double2float_rn(__ddiv_rn(1.0, __dsqrt_rn(sq)));
        for (int l = 0; l < d; ++l) row[l] = __fmul_rn(row[l], scale);
    } else if (zero_when_empty) {
        for (int l = 0; l < d; ++l) row[l] = __fmul_rn(row[l], 0.0f);
    }
}

__global__ void k_cluster_means(const float* __restrict__ sums, const uint32_t* __restrict__ off, int k, int d, int P,
                                bool spherical, const float* __restrict__ fallback, float* __restrict__ out,
                                int* __restrict__ empty) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(P) * k) return;
    const size_t p = t / k;
    const int c = static_cast<int>(t % k);
    const uint32_t* o = off + p * (k + 1);
    const uint32_t cnt = o[c + 1] - o[c];
    float* row = out + t * d;
    const float* s = sums + t * d;
    if (cnt == 0) {
        for (int l = 0; l < d; ++l) row[l] = fallback ? fallback[t * d + l] : 0.0f;
        if (empty) atomicOr(empty, 1);
        return;
    }
    const float fc = __uint2float_rn(cnt);
    for (int l = 0; l < d; ++l) row[l] = __fdiv_rn(s[l], fc);
    if (spherical) unit_scale_row(row, d, false);
}

void cluster_means(const float* sums, const uint32_t* off, int k, int d, int P, bool spherical, const float* fallback,
                   float* out, int* empty, cudaStream_t st) {
    const size_t n = static_cast<size_t>(P) * k;
    if (n == 0) return;
    k_cluster_means<<<static_cast<unsigned>(ceil_div(n, 128)), 128, 0, st>>>(sums, off, k, d, P, spherical, fallback,
                                                                            out, empty);
    QG_LAUNCH_CHECK();
}

// rows made unit length in place or into dst (zero rows become zero)
__global__ void k_unit_rows(const float* __restrict__ src, size_t k, int d, float* __restrict__ dst) {
    const size_t j = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= k) return;
    float* row = dst + j * d;
    if (row != src + j * d)
        for (int l = 0; l < d; ++l) row[l] = src[j * d + l];
    unit_scale_row(row, d, true);
}

void unit_rows_dev(const float* src, size_t k, int d, float* dst, cudaStream_t st) {
    if (k == 0) return;
    k_unit_rows<<<static_cast<unsigned>(ceil_div(k, 128)), 128, 0, st>>>(src, k, d, dst);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// e-means state on the device: centroid positions, masses, and the closing
// pass's sums and counts. One step moves every cluster that received points
// toward the batch mean of its points with weight alpha * n_j / (mass_j +
// alpha * n_j), after all masses decayed by (1 - alpha).
// ---------------------------------------------------------------------------
__global__ void k_mass_decay(float* __restrict__ mass, int k, double keep) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < k) mass[j] = __double2float_rn(__dmul_rn(static_cast<double>(mass[j]), keep));
}

// warp per cluster
__global__ void k_ema_move(float* __restrict__ pos, float* __restrict__ mass, const float* __restrict__ sums,
                           const uint32_t* __restrict__ off, int k, int d, float alpha, bool replace) {
    const int j = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= k) return;
    const uint32_t cnt = off[j + 1] - off[j];
    if (cnt == 0) return;
    const float nj = __uint2float_rn(cnt);
    // the reference's build rounds alpha * n_j once and uses it for both the
    // new mass (a plain add, not fused) and the weight
    const float an = __fmul_rn(alpha, nj);
    const float grown = __fadd_rn(an, replace ? 0.0f : mass[j]);
    const float w = __fdiv_rn(an, grown);
    float* c = pos + static_cast<size_t>(j) * d;
    const float* s = sums + static_cast<size_t>(j) * d;
    for (int l = lane; l < d; l += 32) {
        const float mean = __fdiv_rn(s[l], nj);
        c[l] = w == 1.0f ? mean : __fmaf_rn(w, __fsub_rn(mean, c[l]), c[l]);
    }
    if (lane == 0) mass[j] = grown;
}

__global__ void k_pass_accumulate(float* __restrict__ close_sum, uint32_t* __restrict__ close_cnt,
                                  const float* __restrict__ sums, const uint32_t* __restrict__ off, int k, int d) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(k) * d) return;
    close_sum[t] = __fadd_rn(close_sum[t], sums[t]);
    if (t % d == 0) {
        const size_t j = t / d;
        close_cnt[j] += off[j + 1] - off[j];
    }
}

// Revival: cluster `to` takes a copy of donor `from` nudged by +-1e-4 per
// dimension (the donor moves the other way), and the two halve the donor's
// mass. The pairs are disjoint, so they run in parallel; warp per pair.
__global__ void k_split_into(float* __restrict__ pos, float* __restrict__ mass, const uint32_t* __restrict__ pairs,
                             int npairs, int d) {
    const int t = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= npairs) return;
    const uint32_t from = pairs[2 * t], to = pairs[2 * t + 1];
    float* a = pos + static_cast<size_t>(from) * d;
    float* c = pos + static_cast<size_t>(to) * d;
    bool same = true;
    for (int l = lane; l < d; l += 32) {
        const float nudge = (l & 1) == 0 ? 1e-4f : -1e-4f;
        const float v = a[l];
        const float va = __fmul_rn(v, __fsub_rn(1.0f, nudge));
        const float vc = __fmul_rn(v, __fadd_rn(1.0f, nudge));
        a[l] = va;
        c[l] = vc;
        same = same && va == vc;
    }
    same = __all_sync(0xffffffffu, same);
    if (lane == 0) {
        if (same) c[0] = nextafterf(c[0], INFINITY);
        const float half = __fdiv_rn(mass[from], 2.0f);
        mass[from] = half;
        mass[to] = half;
    }
}

// closing: clusters with points in the last pass move to their mean
__global__ void k_pass_close(float* __restrict__ pos, const float* __restrict__ close_sum,
                             const uint32_t* __restrict__ close_cnt, int k, int d) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(k) * d) return;
    const uint32_t cnt = close_cnt[t / d];
    if (cnt > 0) pos[t] = __fdiv_rn(close_sum[t], __uint2float_rn(cnt));
}

__global__ void k_fill_f32(float* __restrict__ a, size_t n, float v) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n) a[t] = v;
}

void EMeansState::init(int k_, int d_, cudaStream_t st) {
    k = k_;
    d = d_;
    const size_t kd = static_cast<size_t>(k) * d;
    pos.alloc(kd, st);
    mass.alloc(k, st);
    close_sum.alloc(kd, st);
    close_cnt.alloc(k, st);
    k_fill_f32<<<static_cast<unsigned>(ceil_div(k, 256)), 256, 0, st>>>(mass.get(), k, 1.0f / 65536.0f);
    QG_LAUNCH_CHECK();
    QG_CUDA(cudaMemsetAsync(close_sum.get(), 0, kd * sizeof(float), st));
    QG_CUDA(cudaMemsetAsync(close_cnt.get(), 0, k * sizeof(uint32_t), st));
}

void EMeansState::step(const float* sums, const uint32_t* off, double alpha, bool accumulate, cudaStream_t st) {
    const size_t kd = static_cast<size_t>(k) * d;
    if (accumulate) {
        k_pass_accumulate<<<static_cast<unsigned>(ceil_div(kd, 256)), 256, 0, st>>>(close_sum.get(), close_cnt.get(),
                                                                                     sums, off, k, d);
        QG_LAUNCH_CHECK();
    }
    const bool replace = alpha == 1.0;
    if (!replace) {
        k_mass_decay<<<static_cast<unsigned>(ceil_div(k, 256)), 256, 0, st>>>(mass.get(), k, 1.0 - alpha);
        QG_LAUNCH_CHECK();
    }
    k_ema_move<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(k) * 32, 256)), 256, 0, st>>>(
        pos.get(), mass.get(), sums, off, k, d, static_cast<float>(alpha), replace);
    QG_LAUNCH_CHECK();
}

void EMeansState::split(const std::vector<uint32_t>& pairs, cudaStream_t st) {
    const int np = static_cast<int>(pairs.size() / 2);
    if (np == 0) return;
    DevBuf<uint32_t> dp(pairs.size(), st);
    QG_CUDA(cudaMemcpyAsync(dp.get(), pairs.data(), pairs.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    // (a copy from pageable memory has left the host buffer when it returns)
    k_split_into<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(np) * 32, 256)), 256, 0, st>>>(
        pos.get(), mass.get(), dp.get(), np, d);
    QG_LAUNCH_CHECK();
}

void EMeansState::close(cudaStream_t st) {
    const size_t kd = static_cast<size_t>(k) * d;
    k_pass_close<<<static_cast<unsigned>(ceil_div(kd, 256)), 256, 0, st>>>(pos.get(), close_sum.get(),
                                                                          close_cnt.get(), k, d);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// The cosine PQ scoring decision (reference src/ivf_index.cpp:808-902): on a
// sample of the training rows, do inner-product tables or each list's own L2
// tables rank the true neighbours higher? Rows [0, nd) are scored and rows
// [n - nq, n) query them. A query probes its nearest lists by -q.c (ties by
// list) until they hold at least `want` sample rows; each sample row there
// gets three scores: exact -q.x, the inner-product LUT estimate (plus the
// list's 2 - 2 q.c) and the list's L2 LUT estimate. A query's hits are how
// many of its 10 best exact rows are among the 20 best of each estimate,
// all orders by (score, row) with -0 == +0.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ uint64_t score_key(float s, uint32_t i) {
    return (static_cast<uint64_t>(float_key_eq0(s)) << 32) | i;
}

// block per query: the cutoff key T of its probe prefix. Among lists with
// sample rows, keyed by (-q.c, list), T is the key at which the running count
// of sample rows first reaches `want` (all of them when the sample is
// smaller). A weighted radix select, 8 bits at a time from the top.
__global__ void __launch_bounds__(256) k_probe_cutoff(const float* __restrict__ scores, int nlist,
                                                      const uint32_t* __restrict__ off, uint32_t want,
                                                      uint64_t* __restrict__ cutoff) {
    __shared__ uint32_t hist[256];
    __shared__ uint64_t s_prefix, s_mask;
    __shared__ uint32_t s_need;
    __shared__ int s_all;
    const float* row = scores + static_cast<size_t>(blockIdx.x) * nlist;
    if (threadIdx.x == 0) {
        s_prefix = 0;
        s_mask = 0;
        s_need = want;
        s_all = 0;
    }
    for (int shift = 56; shift >= 0; shift -= 8) {
        hist[threadIdx.x] = 0;
        __syncthreads();
        const uint64_t prefix = s_prefix, mask = s_mask;
        for (int l = threadIdx.x; l < nlist; l += blockDim.x) {
            const uint32_t c = off[l + 1] - off[l];
            if (c == 0) continue;
            const uint64_t key = score_key(row[l], static_cast<uint32_t>(l));
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], c);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            int b = 0;
            for (; b < 256; ++b) {
                if (run + hist[b] >= s_need) break;
                run += hist[b];
            }
            if (b == 256) {
                s_all = 1;   // fewer sample rows than wanted: every list with rows
            } else {
                s_need -= run;
                s_prefix |= static_cast<uint64_t>(b) << shift;
                s_mask |= uint64_t{255} << shift;
            }
        }
        __syncthreads();
        if (s_all) break;
    }
    if (threadIdx.x == 0) cutoff[blockIdx.x] = s_all ? ~0ull : s_prefix;
}

constexpr int kPickWarps = 8;

struct PickShared {
    int dim, m, m_pad, sd;
};

// block per query (8 warps): the inner-product LUT of the query, then each
// warp takes probed lists, rounds the list's L2 table of q - center and
// scores the list's sample rows into the query's candidate arrays.
__global__ void __launch_bounds__(32 * kPickWarps) k_pick_score(
    const float* __restrict__ x, size_t n, int dim, int nq, const float* __restrict__ centers,
    const float* __restrict__ yt, int m, int sd, const uint8_t* __restrict__ codes, const float* __restrict__ scores,
    int nlist, const uint32_t* __restrict__ off, const uint32_t* __restrict__ members,
    const uint64_t* __restrict__ cutoff, size_t cap, uint64_t* __restrict__ k_exact, uint64_t* __restrict__ k_ip,
    uint64_t* __restrict__ k_l2, uint32_t* __restrict__ count) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int m_pad = (m + 3) & ~3;
    const int qi = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint4* lut_ip = reinterpret_cast<uint4*>(sm);
    uint4* lut_w = lut_ip + m_pad * (1 + warp);
    float* qv = reinterpret_cast<float*>(lut_ip + m_pad * (1 + kPickWarps));
    float* resid = qv + dim * (1 + warp);
    float* rmin = qv + dim * (1 + kPickWarps) + m * warp;
    __shared__ float s_ip_scale, s_ip_offset;
    const float* q = x + (n - nq + qi) * static_cast<size_t>(dim);
    for (int t = threadIdx.x; t < dim; t += blockDim.x) qv[t] = q[t];
    __syncthreads();
    if (warp == 0) {
        float sc, of;
        warp_quantize_lut(
            [&](int r, float* v) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = inner_term(qv, yt, r, sd, 16, j);
            },
            m, m_pad, rmin, lut_ip, sc, of);
        if (lane == 0) {
            s_ip_scale = sc;
            s_ip_offset = of;
        }
    }
    __syncthreads();
    const float ip_scale = s_ip_scale, ip_offset = s_ip_offset;
    const uint64_t cut = cutoff[qi];
    const float* srow = scores + static_cast<size_t>(qi) * nlist;
    const uint8_t* lip8 = reinterpret_cast<const uint8_t*>(lut_ip);
    const uint8_t* lw8 = reinterpret_cast<const uint8_t*>(lut_w);
    uint64_t* ke = k_exact + static_cast<size_t>(qi) * cap;
    uint64_t* kp = k_ip + static_cast<size_t>(qi) * cap;
    uint64_t* kl = k_l2 + static_cast<size_t>(qi) * cap;
    for (int l = warp; l < nlist; l += kPickWarps) {
        const uint32_t b0 = off[l], b1 = off[l + 1];
        if (b0 == b1 || score_key(srow[l], static_cast<uint32_t>(l)) > cut) continue;
        const float* c = centers + static_cast<size_t>(l) * dim;
        for (int t = lane; t < dim; t += 32) resid[t] = __fsub_rn(qv[t], c[t]);
        float qc = 0.0f;
        if (lane == 0) qc = exact_avx2<false>(qv, c, dim);
        const float base = __fmaf_rn(-2.0f, __shfl_sync(0xffffffffu, qc, 0), 2.0f);
        __syncwarp();
        float l2_scale, l2_offset;
        warp_quantize_lut(
            [&](int r, float* v) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = adc_term(resid, yt, r, sd, 16, j);
            },
            m, m_pad, rmin, lut_w, l2_scale, l2_offset);
        for (uint32_t e = b0 + lane; e < b1; e += 32) {
            const uint32_t i = members[e];
            const uint8_t* code = codes + static_cast<size_t>(i) * m;
            uint32_t a = 0, b = 0;
            for (int s = 0; s < m; ++s) {
                a += lip8[s * 16 + code[s]];
                b += lw8[s * 16 + code[s]];
            }
            const float s_ip = __fadd_rn(__fdiv_rn(__uint2float_rn(a), ip_scale), ip_offset);
            const float s_l2 = __fadd_rn(__fdiv_rn(__uint2float_rn(b), l2_scale), l2_offset);
            const float exact = -exact_avx2<false>(qv, x + static_cast<size_t>(i) * dim, dim);
            const uint32_t at = atomicAdd(count + qi, 1u);
            if (at < cap) {
                ke[at] = score_key(exact, i);
                kp[at] = score_key(__fadd_rn(base, s_ip), i);
                kl[at] = score_key(s_l2, i);
            }
        }
        __syncwarp();
    }
}

// block per query: the t smallest keys, ascending, by repeated block minima
// above the previous one (keys are distinct: the row is part of the key)
__device__ int block_smallest(const uint64_t* keys, uint32_t n, int t, uint32_t* out_rows, uint64_t* red) {
    uint64_t last = 0;
    bool first = true;
    int got = 0;
    for (; got < t; ++got) {
        uint64_t best = ~0ull;
        for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
            const uint64_t v = keys[e];
            if ((first || v > last) && v < best) best = v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t y = __shfl_xor_sync(0xffffffffu, best, o);
            best = y < best ? y : best;
        }
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t b = ~0ull;
            for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) b = red[w] < b ? red[w] : b;
            red[32] = b;
        }
        __syncthreads();
        best = red[32];
        __syncthreads();
        if (best == ~0ull) break;
        out_rows[got] = static_cast<uint32_t>(best);
        last = best;
        first = false;
    }
    return got;
}

__global__ void __launch_bounds__(256) k_pick_hits(const uint64_t* __restrict__ k_exact, const uint64_t* __restrict__ k_ip,
                                                   const uint64_t* __restrict__ k_l2, const uint32_t* __restrict__ count,
                                                   size_t cap, unsigned long long* __restrict__ hits) {
    __shared__ uint64_t red[33];
    __shared__ uint32_t top[10], best_ip[20], best_l2[20];
    const int qi = blockIdx.x;
    const uint32_t n = min(count[qi], static_cast<uint32_t>(cap));
    const size_t o = static_cast<size_t>(qi) * cap;
    const int nt = block_smallest(k_exact + o, n, 10, top, red);
    const int ni = block_smallest(k_ip + o, n, 20, best_ip, red);
    const int nl = block_smallest(k_l2 + o, n, 20, best_l2, red);
    if (threadIdx.x == 0) {
        unsigned long long hi = 0, hl = 0;
        for (int t = 0; t < nt; ++t) {
            for (int j = 0; j < ni; ++j) hi += best_ip[j] == top[t];
            for (int j = 0; j < nl; ++j) hl += best_l2[j] == top[t];
        }
        atomicAdd(hits, hi);
        atomicAdd(hits + 1, hl);
    }
}

} // namespace

bool cosine_ip_wins(const float* x, size_t n, int dim, const uint32_t* assign, const float* centroids,
                    const float* centers, int nlist, const float* yt, int m, int sd, cudaStream_t st) {
    constexpr size_t kSampleQueries = 200, kScoredRows = 20000;
    constexpr uint32_t kProbeRows = 2000;
    if (n < kSampleQueries + kProbeRows) return true;   // too small a sample to tell: keep inner product
    const size_t nq = kSampleQueries, nd = std::min(kScoredRows, n - nq);
    // codes of the scored rows, and the scored rows grouped by list in row order
    DevBuf<uint8_t> codes(nd * m, st);
    encode16(x, nd, dim, centers, assign, yt, m, sd, codes.get(), st);
    DevBuf<uint32_t> members(nd, st), off(static_cast<size_t>(nlist) + 1, st);
    group_by_label(assign, nd, nlist, 1, members.get(), off.get(), st);
    // -q.c of every sample query and list, in the reference's AVX2 order
    DevBuf<float> scores(nq * nlist, st);
    pair_scores(x + (n - nq) * dim, static_cast<int>(nq), centroids, nlist, dim, true, scores.get(), nlist, st);
    DevBuf<uint64_t> cut(nq, st);
    k_probe_cutoff<<<static_cast<unsigned>(nq), 256, 0, st>>>(scores.get(), nlist, off.get(), kProbeRows, cut.get());
    QG_LAUNCH_CHECK();
    // candidates are distinct scored rows: at most nd per query
    const size_t cap = nd;
    DevBuf<uint64_t> ke(nq * cap, st), kp(nq * cap, st), kl(nq * cap, st);
    DevBuf<uint32_t> count(nq, st);
    DevBuf<unsigned long long> hits(2, st);
    QG_CUDA(cudaMemsetAsync(count.get(), 0, nq * sizeof(uint32_t), st));
    QG_CUDA(cudaMemsetAsync(hits.get(), 0, 2 * sizeof(unsigned long long), st));
    const int m_pad = (m + 3) & ~3;
    const size_t smem = static_cast<size_t>(m_pad) * 16 * (1 + kPickWarps) +
                        sizeof(float) * (static_cast<size_t>(dim) * (1 + kPickWarps) + static_cast<size_t>(m) * kPickWarps);
    require(smem <= 200 * 1024, "the cosine scoring decision supports dim and m up to about 4096", kUnsupported);
    if (smem > 48 * 1024) allow_large_smem<k_pick_score>();
    k_pick_score<<<static_cast<unsigned>(nq), 32 * kPickWarps, smem, st>>>(
        x, n, dim, static_cast<int>(nq), centers, yt, m, sd, codes.get(), scores.get(), nlist, off.get(),
        members.get(), cut.get(), cap, ke.get(), kp.get(), kl.get(), count.get());
    QG_LAUNCH_CHECK();
    k_pick_hits<<<static_cast<unsigned>(nq), 256, 0, st>>>(ke.get(), kp.get(), kl.get(), count.get(), cap, hits.get());
    QG_LAUNCH_CHECK();
    unsigned long long h[2] = {0, 0};
    QG_CUDA(cudaMemcpyAsync(h, hits.get(), sizeof(h), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    return h[0] >= h[1];   // L2 tables only when they rank strictly better
}

} // namespace qg
