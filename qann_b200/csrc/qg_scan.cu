// The code scan with fused top-k' selection (reference src/ivf_index.cpp:421-641,
// src/topk.hpp), and the orchestration of one IVF fast-scan search.
//
// A block takes one query and a chunk of its probes. The chunk's lists are cut
// into work items of at most 8 superblocks (64 vectors each), in probe order.
// Warps run independently: a warp takes the next 4 items, builds their uint8
// LUTs with its 32 lanes (mode L2: B + C + A rounded, as build_quantize_lut;
// mode L2-ADC: the residual's ADC table rounded; modes IP / cosine-IP use the
// query's one LUT and skip this), and its 4 octets (8 lanes each) scan one
// item each with register-resident 4-bit lookups.
//
// Selection keeps the k' smallest candidates by key64 = key(dist) << 32 |
// push index, the push index being the vector's position in the query's
// sequence of probed lists: exactly the set the reference's TopK keeps
// (distance first, first pushed among ties). Each warp buffers the candidates
// that beat the block's threshold; when its buffer fills it keeps its own k'
// best and lowers the block threshold to its k'-th key (an upper bound of the
// block's k'-th, so the pruning is exact). Deleted (or filtered-out) vectors
// are skipped before they can enter, as the reference's push() does. The
// integer pre-test `sum <= S*` is exact: S* is the largest sum whose distance
// is <= the threshold distance (sum_limit). At the end the warps' lists are
// merged and the k' survivors' slots are looked up from their push index.
#include "qg_device.cuh"
#include "qg_search.h"

#include <algorithm>

namespace qg {

namespace {
constexpr int kItemSb = 8;       // superblocks per work item
constexpr int kMaxChunk = 256;   // probes per block at most
constexpr int kItemsPerWarp = 4;
}

// The 16 entries of LUT rows rounded and packed: round-half-even of
// (t - min) * scale, as nearbyint / cvtps do, through the 1.5 * 2^23 addend
// (every value here lies in [0, 64), where float spacing at that magnitude is 1).
__device__ __forceinline__ uint4 round_row(const float* v, float mn, float scale) {
    uint32_t b[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        b[j] = __float_as_uint(__fadd_rn(__fmul_rn(__fsub_rn(v[j], mn), scale), 12582912.0f));
    return make_uint4(prmt(prmt(b[0], b[1], 0x0040), prmt(b[2], b[3], 0x0040), 0x5410),
                      prmt(prmt(b[4], b[5], 0x0040), prmt(b[6], b[7], 0x0040), 0x5410),
                      prmt(prmt(b[8], b[9], 0x0040), prmt(b[10], b[11], 0x0040), 0x5410),
                      prmt(prmt(b[12], b[13], 0x0040), prmt(b[14], b[15], 0x0040), 0x5410));
}

// LUT of one list by one warp (rows cached in registers for m <= 64; larger
// m recomputes rows in the second pass). Same arithmetic as quantize_lut.
template <class RowFn>
__device__ __forceinline__ void warp_lut3(RowFn row, int m, int m_pad, float* row_min, uint4* lut_out, float& scale_out,
                                          float& offset_out) {
    const int lane = threadIdx.x & 31;
    float v0[16], v1[16];
    float widest = 0.0f;
    auto ranges = [&](int r, float* v) {
        float lo = v[0], hi = v[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            lo = fminf(lo, v[j]);
            hi = fmaxf(hi, v[j]);
        }
        row_min[r] = lo;
        const float w = __fsub_rn(hi, lo);
        widest = widest < w ? w : widest;
    };
    if (m <= 64) {
        if (lane < m) {
            row(lane, v0);
            ranges(lane, v0);
        }
        if (lane + 32 < m) {
            row(lane + 32, v1);
            ranges(lane + 32, v1);
        }
    } else {
        for (int r = lane; r < m; r += 32) {
            row(r, v0);
            ranges(r, v0);
        }
    }
    widest = warp_max(widest);
    __syncwarp();
    float part = 0.0f;
    if (lane < 4)
        for (int r = lane; r < m; r += 4) part = __fadd_rn(part, row_min[r]);
    const float p0 = __shfl_sync(0xffffffffu, part, 0), p1 = __shfl_sync(0xffffffffu, part, 1);
    const float p2 = __shfl_sync(0xffffffffu, part, 2), p3 = __shfl_sync(0xffffffffu, part, 3);
    const float offset = __fadd_rn(__fadd_rn(p0, p1), __fadd_rn(p2, p3));
    const float scale = widest > 0.0f ? __fdiv_rn(static_cast<float>(kLutMax), widest) : 1.0f;
    if (m <= 64) {
        if (lane < m) lut_out[lane] = round_row(v0, row_min[lane], scale);
        if (lane + 32 < m) lut_out[lane + 32] = round_row(v1, row_min[lane + 32], scale);
    } else {
        for (int r = lane; r < m; r += 32) {
            row(r, v0);
            lut_out[r] = round_row(v0, row_min[r], scale);
        }
    }
    for (int r = m + lane; r < m_pad; r += 32) lut_out[r] = make_uint4(0, 0, 0, 0);
    scale_out = scale;
    offset_out = offset;
    __syncwarp();
}

__device__ __forceinline__ int upper_index(const uint32_t* pre, int n, uint32_t x) {
    // the largest i in [0, n) with pre[i] <= x (pre nondecreasing, pre[0] <= x)
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Keys only, one warp, n a power of two.
__device__ __forceinline__ void warp_sort_keys(uint64_t* key, int n) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncwarp();
            for (int t = lane; t < (n >> 1); t += 32) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t k0 = key[lo], k1 = key[hi];
                if (up ? (k1 < k0) : (k0 < k1)) {
                    key[lo] = k1;
                    key[hi] = k0;
                }
            }
        }
    }
    __syncwarp();
}

struct ScanLayout {
    int wcap;    // per-warp candidate buffer (keys)
    int nw;      // warps per block
    size_t bytes;
};

__host__ __device__ inline ScanLayout scan_layout(int kp, int m_pad, int qtab_len, int pch, bool shared_lut, int nw) {
    ScanLayout L;
    L.nw = nw;
    int w = 1;
    while (w < kp + kItemsPerWarp * kSuperBlock) w <<= 1;
    L.wcap = w;
    size_t b = static_cast<size_t>(nw) * w * 8;                                          // candidate buffers
    b += shared_lut ? static_cast<size_t>(m_pad) * 16
                    : static_cast<size_t>(nw) * kItemsPerWarp * m_pad * 16;              // LUTs
    b += shared_lut ? 0 : static_cast<size_t>(nw) * m_pad * 4;                           // row minimums
    b += static_cast<size_t>(nw) * kItemsPerWarp * 8;                                    // per-warp scale / offset
    b += static_cast<size_t>(qtab_len) * 4;
    b += static_cast<size_t>(pch) * 4 * 6 + 4 * 2;                                       // per-probe arrays
    L.bytes = b;
    return L;
}

template <int NW>
__global__ void __launch_bounds__(NW * 32, 2) k_scan(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    constexpr int NT = NW * 32;
    const IvfView& v = a.v;
    const int qi = blockIdx.x / a.nchunks;
    const int chunk = blockIdx.x - qi * a.nchunks;
    const int p0 = chunk * a.pch;
    const int np = min(a.nprobe_q ? a.nprobe_q[qi] : a.P, p0 + a.pch) - p0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t* qfilter = a.filters ? a.filters[qi] : a.filter;
    if (np <= 0) {   // a query whose probes end before this chunk
        for (int i = tid; i < a.kp; i += NT) {
            a.out_key[static_cast<size_t>(blockIdx.x) * a.kp + i] = ~0ull;
            a.out_slot[static_cast<size_t>(blockIdx.x) * a.kp + i] = 0xFFFFFFFFu;
        }
        return;
    }
    const int oct = lane >> 3, r = lane & 7;
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int qtab_len = v.mode == kModeL2 ? v.m * 16 : (v.mode == kModeL2Adc ? v.dim : 0);
    const ScanLayout lay = scan_layout(a.kp, v.m_pad, qtab_len, a.pch, shared_lut, NW);
    const int wcap = lay.wcap;

    uint64_t* wbuf_all = reinterpret_cast<uint64_t*>(sm);
    uint4* lut_all = reinterpret_cast<uint4*>(wbuf_all + static_cast<size_t>(NW) * wcap);
    float* rmin_all = reinterpret_cast<float*>(
        lut_all + (shared_lut ? static_cast<size_t>(v.m_pad) : static_cast<size_t>(NW) * kItemsPerWarp * v.m_pad));
    float* wscale_all = rmin_all + (shared_lut ? 0 : NW * v.m_pad);
    float* woffset_all = wscale_all + NW * kItemsPerWarp;
    float* qtab = woffset_all + NW * kItemsPerWarp;
    float* p_scale = qtab + qtab_len;
    float* p_offset = p_scale + a.pch;
    uint32_t* p_list = reinterpret_cast<uint32_t*>(p_offset + a.pch);
    uint32_t* p_size = p_list + a.pch;
    uint32_t* p_push = p_size + a.pch;
    uint32_t* p_itpre = p_push + a.pch;   // np + 1 item prefix (pch + 2 slots)
    __shared__ int s_next, s_overflow;
    __shared__ int s_wcount[NW];
    __shared__ unsigned long long s_thr;
    __shared__ uint32_t red[NW];

    const size_t qp = static_cast<size_t>(qi) * a.P;
    if (tid == 0) {
        s_next = 0;
        s_overflow = 0;
        s_thr = ~0ull;
    }
    if (tid < NW) s_wcount[tid] = 0;
    uint32_t before = 0;
    for (int p = tid; p < p0; p += NT) before += v.list_size[a.probe[qp + p]];
    for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
    if (lane == 0) red[warp] = before;
    for (int p = tid; p < np; p += NT) {
        const uint32_t l = a.probe[qp + p0 + p];
        p_list[p] = l;
        p_size[p] = v.list_size[l];
    }
    if (v.mode == kModeL2)
        for (int t = tid; t < v.m * 16; t += NT) qtab[t] = a.qC[static_cast<size_t>(qi) * v.m * 16 + t];
    if (v.mode == kModeL2Adc)
        for (int t = tid; t < v.dim; t += NT) qtab[t] = a.q[static_cast<size_t>(qi) * v.dim + t];
    if (shared_lut) {
        for (int rr = tid; rr < v.m_pad; rr += NT) lut_all[rr] = a.qlut[static_cast<size_t>(qi) * v.m_pad + rr];
        for (int p = tid; p < np; p += NT) {
            p_scale[p] = a.qscale[qi];
            p_offset[p] = __fadd_rn(a.qoffset[qi], a.pterm[qp + p0 + p]);
        }
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t b = 0, it = 0;
        for (int w = 0; w < NW; ++w) b += red[w];
        for (int p = 0; p < np; ++p) {
            p_push[p] = b;
            b += p_size[p];
            p_itpre[p] = it;
            it += (((p_size[p] + kSuperBlock - 1) / kSuperBlock) + kItemSb - 1) / kItemSb;
        }
        p_itpre[np] = it;
    }
    __syncthreads();
    const uint32_t total_items = p_itpre[np];

    uint64_t* wbuf = wbuf_all + static_cast<size_t>(warp) * wcap;
    uint4* wlut = lut_all + (shared_lut ? 0 : static_cast<size_t>(warp) * kItemsPerWarp * v.m_pad);
    float* wrmin = rmin_all + warp * v.m_pad;
    float* wscale = wscale_all + warp * kItemsPerWarp;
    float* woffset = woffset_all + warp * kItemsPerWarp;
    const unsigned octmask = 0xFFu << (oct * 8);

    // candidate buffer of this warp: trims keep the warp's k' best and lower the block threshold
    auto warp_trim = [&]() {
        __syncwarp();
        const int n = min(s_wcount[warp], wcap);
        int npow = 2;
        while (npow < n) npow <<= 1;
        for (int i = n + lane; i < npow; i += 32) wbuf[i] = ~0ull;
        warp_sort_keys(wbuf, npow);
        if (lane == 0) {
            if (n >= a.kp) atomicMin(&s_thr, static_cast<unsigned long long>(wbuf[a.kp - 1]));
            s_wcount[warp] = min(n, a.kp);
        }
        __syncwarp();
    };

    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = static_cast<uint32_t>(atomicAdd(&s_next, kItemsPerWarp));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total_items) break;
        const int nit = static_cast<int>(min(static_cast<uint32_t>(kItemsPerWarp), total_items - base));
        // this octet's item: probe, superblock range
        const bool has = oct < nit;
        const uint32_t item = base + min(oct, nit - 1);
        const int p = upper_index(p_itpre, np, item);
        const uint32_t l = p_list[p];
        const uint32_t nsb_list = (p_size[p] + kSuperBlock - 1) / kSuperBlock;
        const uint32_t sb0 = (item - p_itpre[p]) * kItemSb;
        const int cnt = has ? static_cast<int>(min(static_cast<uint32_t>(kItemSb), nsb_list - sb0)) : 0;
        float scale, offset;
        const uint4* L;
        if (shared_lut) {
            scale = p_scale[p];
            offset = p_offset[p];
            L = wlut;
        } else {
            // LUTs of the (up to 4) items, built by the whole warp one after another
            for (int j = 0; j < nit; ++j) {
                const uint32_t it_j = base + j;
                const int pj = upper_index(p_itpre, np, it_j);
                const uint32_t lj = p_list[pj];
                float s, o;
                if (v.mode == kModeL2) {
                    const float A = a.pterm[qp + p0 + pj];
                    const float* B = v.B + static_cast<size_t>(lj) * v.m * 16;
                    warp_lut3(
                        [&](int rr, float* out) {
                            const float4* b4 = reinterpret_cast<const float4*>(B + rr * 16);
                            const float4* c4 = reinterpret_cast<const float4*>(qtab + rr * 16);
#pragma unroll
                            for (int u = 0; u < 4; ++u) {
                                const float4 bb = __ldg(b4 + u), cc = c4[u];
                                out[4 * u + 0] = __fadd_rn(bb.x, cc.x);
                                out[4 * u + 1] = __fadd_rn(bb.y, cc.y);
                                out[4 * u + 2] = __fadd_rn(bb.z, cc.z);
                                out[4 * u + 3] = __fadd_rn(bb.w, cc.w);
                            }
                            if (rr == 0) {
#pragma unroll
                                for (int jj = 0; jj < 16; ++jj) out[jj] = __fadd_rn(out[jj], A);
                            }
                        },
                        v.m, v.m_pad, wrmin, wlut + static_cast<size_t>(j) * v.m_pad, s, o);
                } else {
                    // the residual (q - center) is formed per element inside the table
                    // loop, as compute_adc_table reads it (reference src/ivf_index.cpp:594-610)
                    const float* ctr = v.resid + static_cast<size_t>(lj) * v.dim;
                    warp_lut3(
                        [&](int rr, float* out) {
#pragma unroll
                            for (int jj = 0; jj < 16; ++jj) {
                                float acc = 0.0f;
                                for (int u = 0; u < v.sd; ++u) {
                                    const int e = rr * v.sd + u;
                                    const float diff = __fsub_rn(__fsub_rn(qtab[e], ctr[e]), v.pq_t[e * 16 + jj]);
                                    acc = __fmaf_rn(diff, diff, acc);
                                }
                                out[jj] = acc;
                            }
                        },
                        v.m, v.m_pad, wrmin, wlut + static_cast<size_t>(j) * v.m_pad, s, o);
                }
                if (lane == 0) {
                    wscale[j] = s;
                    woffset[j] = o;
                }
            }
            __syncwarp();
            scale = wscale[min(oct, nit - 1)];
            offset = woffset[min(oct, nit - 1)];
            L = wlut + static_cast<size_t>(min(oct, nit - 1)) * v.m_pad;
        }
        // the integer limit of this item's list for the current threshold
        unsigned long long thr_seen = s_thr;
        int smax = sum_limit_fast(static_cast<uint32_t>(thr_seen >> 32), scale, offset);
        int maxcnt = cnt;
        for (int o = 8; o < 32; o <<= 1) maxcnt = max(maxcnt, __shfl_xor_sync(0xffffffffu, maxcnt, o));
        const uint32_t size = p_size[p], push0 = p_push[p];
        for (int j = 0; j < maxcnt; ++j) {
            if (j < cnt) {
                const unsigned long long thr = s_thr;
                if (thr != thr_seen) {
                    thr_seen = thr;
                    smax = sum_limit_fast(static_cast<uint32_t>(thr >> 32), scale, offset);
                }
                const uint32_t sbl = sb0 + j;
                const size_t sbg = static_cast<size_t>(v.sb_off[l]) + sbl;
                uint32_t sums[8];
                octet_sums(v.codes + sbg * static_cast<size_t>(2 * v.m_pad), L, v.m_pad, r, sums);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const uint32_t pos = sbl * kSuperBlock + 8 * r + i;
                    if (pos < size && static_cast<int>(sums[i]) <= smax) {
                        const float dist = fs_dist(sums[i], scale, offset);
                        const uint64_t key = (static_cast<uint64_t>(float_key(dist)) << 32) | (push0 + pos);
                        if (key < thr) {
                            const uint32_t slot = v.ids[sbg * kSuperBlock + 8 * r + i];
                            const bool ok = qfilter ? ((qfilter[slot >> 6] >> (slot & 63)) & 1ull)
                                                    : !(v.deleted && ((v.deleted[slot >> 6] >> (slot & 63)) & 1ull));
                            if (ok) {
                                const int idx = atomicAdd(&s_wcount[warp], 1);
                                if (idx < wcap) wbuf[idx] = key;
                                else s_overflow = 1;
                            }
                        }
                    }
                }
            }
            __syncwarp();
            if (s_wcount[warp] > wcap - kItemsPerWarp * kSuperBlock) warp_trim();
        }
        (void)octmask;
    }
    // ---- merge the warps' lists: each keeps its k' best, then the block sorts them all ----
    warp_trim();
    __syncthreads();
    const int region = NW * wcap;
    for (int i = tid; i < region; i += NT) {
        const int w = i / wcap, e = i - w * wcap;
        if (e >= s_wcount[w]) wbuf_all[i] = ~0ull;
    }
    bitonic_sort_keys(wbuf_all, region);
    int kept = 0;
    for (int w = 0; w < NW; ++w) kept += s_wcount[w];
    kept = min(kept, a.kp);
    const size_t ob = static_cast<size_t>(blockIdx.x) * a.kp;
    for (int i = tid; i < a.kp; i += NT) {
        if (i < kept) {
            const uint64_t key = wbuf_all[i];
            const uint32_t push = static_cast<uint32_t>(key);
            const int pp = upper_index(p_push, np, push);
            const uint32_t pos = push - p_push[pp];
            const size_t sbg = static_cast<size_t>(v.sb_off[p_list[pp]]) + pos / kSuperBlock;
            a.out_key[ob + i] = key;
            a.out_slot[ob + i] = v.ids[sbg * kSuperBlock + pos % kSuperBlock];
        } else {
            a.out_key[ob + i] = ~0ull;
            a.out_slot[ob + i] = 0xFFFFFFFFu;
        }
    }
    if (tid == 0 && s_overflow) atomicExch(a.err, 1);
}

int scan_cap(int kp) { return scan_layout(kp, 4, 0, 1, true, 1).wcap; }

template <int NW>
static void launch_scan(const ScanArgs& a, size_t smem, unsigned blocks, cudaStream_t st) {
    allow_large_smem<k_scan<NW>>();
    KernelTimer kt("scan", st);
    k_scan<NW><<<blocks, NW * 32, smem, st>>>(a);
    QG_LAUNCH_CHECK();
}

void ivf_candidates(const IvfView& v, const IvfSearchArgs& s, uint64_t* out_key, uint32_t* out_slot, cudaStream_t st) {
    const int nq = s.nq, kp = s.kp;
    if (nq == 0) return;
    int P = s.nprobe;
    DevBuf<uint32_t> probe;
    DevBuf<float> pdist;
    DevBuf<int> nprobe_q;
    const int* probes_of = s.pq.nprobe;   // unfiltered mixed batch: each query's own nprobe (<= P)
    if (s.filter || s.any_filter) {
        // every list ranked, then each query's own probe count (reference src/ivf_index.cpp:501-521)
        P = filtered_probes(v, s, probe, pdist, nprobe_q, st);
        probes_of = nprobe_q.get();
    } else {
        // coarse: all pair scores, then the P nearest lists per query
        DevBuf<float> scores(static_cast<size_t>(nq) * v.nlist, st);
        pair_scores(s.q, nq, v.centroids, v.nlist, v.dim, v.ip_metric, scores.get(), v.nlist, st);
        probe.alloc(static_cast<size_t>(nq) * P, st);
        pdist.alloc(static_cast<size_t>(nq) * P, st);
        // (score, list) compared as the reference's heap of (float, uint16_t) pairs does: -0 == +0
        select_rows(scores.get(), v.nlist, nq, v.nlist, P, probe.get(), pdist.get(), st, nullptr, nullptr, 0, true);
    }

    DevBuf<float> pterm(static_cast<size_t>(nq) * P, st);
    probe_terms(v, s.q, nq, P, probe.get(), pdist.get(), pterm.get(), st);
    DevBuf<float> qC, qscale, qoffset;
    DevBuf<uint4> qlut;
    if (v.mode == kModeL2) qC.alloc(static_cast<size_t>(nq) * v.m * 16, st);
    if (v.mode == kModeIP || v.mode == kModeCosIP) {
        qlut.alloc(static_cast<size_t>(nq) * v.m_pad, st);
        qscale.alloc(nq, st);
        qoffset.alloc(nq, st);
    }
    if (v.mode != kModeL2Adc) query_tables(v, s.q, nq, qC.get(), qlut.get(), qscale.get(), qoffset.get(), st);

    // chunks: enough blocks to fill the GPU several times over, at most kMaxChunk probes each
    const int sms = s.sm_count > 0 ? s.sm_count : 148;
    int nchunks = std::clamp(static_cast<int>(ceil_div(static_cast<size_t>(4 * sms), nq)), 1, P);
    nchunks = std::max(nchunks, static_cast<int>(ceil_div(P, kMaxChunk)));
    const int pch = static_cast<int>(ceil_div(P, nchunks));
    nchunks = static_cast<int>(ceil_div(P, pch));
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int qtab_len = v.mode == kModeL2 ? v.m * 16 : (v.mode == kModeL2Adc ? v.dim : 0);
    // warps per block: 8 when the candidate buffers and LUTs fit in ~100 KB, fewer otherwise
    int nw = 8;
    while (nw > 1 && scan_layout(kp, v.m_pad, qtab_len, pch, shared_lut, nw).bytes > 100 * 1024) nw >>= 1;
    const ScanLayout lay = scan_layout(kp, v.m_pad, qtab_len, pch, shared_lut, nw);
    require(lay.bytes <= 227 * 1024, "fast-scan shared memory exceeds the B200 limit for this m / k * k_factor",
            kUnsupported);

    const bool direct = nchunks == 1;
    const size_t nout = static_cast<size_t>(nq) * nchunks * kp;
    DevBuf<uint64_t> ckey;
    DevBuf<uint32_t> cslot;
    if (!direct) {
        ckey.alloc(nout, st);
        cslot.alloc(nout, st);
    }
    ScanArgs a{};
    a.v = v;
    a.q = s.q;
    a.probe = probe.get();
    a.pterm = pterm.get();
    a.qC = qC.get();
    a.qlut = qlut.get();
    a.qscale = qscale.get();
    a.qoffset = qoffset.get();
    a.filter = s.filter;
    a.filters = s.pq.filter;
    a.nprobe_q = probes_of;
    a.P = P;
    a.pch = pch;
    a.nchunks = nchunks;
    a.kp = kp;
    a.cap = lay.wcap;
    a.out_key = direct ? out_key : ckey.get();
    a.out_slot = direct ? out_slot : cslot.get();
    a.err = s.d_err;
    const unsigned blocks = static_cast<unsigned>(nq * nchunks);
    switch (nw) {
        case 8: launch_scan<8>(a, lay.bytes, blocks, st); break;
        case 4: launch_scan<4>(a, lay.bytes, blocks, st); break;
        case 2: launch_scan<2>(a, lay.bytes, blocks, st); break;
        default: launch_scan<1>(a, lay.bytes, blocks, st); break;
    }
    if (!direct) merge_candidates(ckey.get(), cslot.get(), nq, nchunks, kp, out_key, out_slot, st);
}

} // namespace qg
