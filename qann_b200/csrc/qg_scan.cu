// The code scan with fused top-k' selection (reference src/ivf_index.cpp:421-641,
// src/topk.hpp), and the orchestration of one IVF fast-scan search.
//
// A block of 256 threads takes one query and a chunk of its probes, in probe
// order, in groups of 16 probes. For each group the 8 warps build the lists'
// uint8 LUTs in shared memory (mode L2: B + C + A rounded, as
// build_quantize_lut; mode L2-ADC: the ADC table of the residual rounded;
// modes IP / cosine-IP share the query's one LUT and skip this), then the 32
// octets (8 threads each) take the group's superblocks (64 vectors) in turn.
//
// Selection keeps the k' smallest candidates by key64 = key(dist) << 32 |
// push index, the push index being the vector's position in the query's
// sequence of probed lists: exactly the set the reference's TopK keeps
// (distance first, first pushed among ties). Candidates enter a shared buffer
// when key64 beats the current k'-th key; the buffer is sorted and cut back
// to k' when it fills, which lowers the threshold. Deleted (or filtered-out)
// vectors are skipped before they can enter, as the reference's push() does.
// The integer pre-test `sum <= S*` is exact: S* is the largest sum whose
// distance is <= the threshold distance (sum_limit). Only keys are buffered;
// the slots of the k' survivors are looked up from their push index at the end.
#include "qg_device.cuh"
#include "qg_search.h"

#include <algorithm>

namespace qg {

namespace {
constexpr int kGroup = 16;      // probes per LUT group (L2 modes)
constexpr int kMaxChunk = 256;  // probes per block at most
constexpr int kScanThreads = 256;
}

// LUT of one list by one warp; rows cached in registers when m <= 64 so the
// table is produced once (the reference fuses the sum into rounding the same
// way; the arithmetic per entry is unchanged).
template <class RowFn>
__device__ __forceinline__ void warp_lut(RowFn row, int m, int m_pad, float* row_min, uint4* lut_out, float& scale_out,
                                         float& offset_out) {
    const int lane = threadIdx.x & 31;
    if (m > 64) {
        warp_quantize_lut(row, m, m_pad, row_min, lut_out, scale_out, offset_out);
        return;
    }
    float v0[16], v1[16];
    const int r0 = lane, r1 = lane + 32;
    float widest = 0.0f;
    if (r0 < m) {
        row(r0, v0);
        float lo = v0[0], hi = v0[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            lo = fminf(lo, v0[j]);
            hi = fmaxf(hi, v0[j]);
        }
        row_min[r0] = lo;
        const float w = __fsub_rn(hi, lo);
        widest = widest < w ? w : widest;
    }
    if (r1 < m) {
        row(r1, v1);
        float lo = v1[0], hi = v1[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            lo = fminf(lo, v1[j]);
            hi = fmaxf(hi, v1[j]);
        }
        row_min[r1] = lo;
        const float w = __fsub_rn(hi, lo);
        widest = widest < w ? w : widest;
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
    auto emit = [&](int r, const float* v) {
        if (r >= m_pad) return;
        if (r >= m) {
            lut_out[r] = make_uint4(0, 0, 0, 0);
            return;
        }
        const float mn = row_min[r];
        int q[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) q[j] = __float2int_rn(__fmul_rn(__fsub_rn(v[j], mn), scale));
        lut_out[r] = make_uint4(pack4(q[0], q[1], q[2], q[3]), pack4(q[4], q[5], q[6], q[7]),
                                pack4(q[8], q[9], q[10], q[11]), pack4(q[12], q[13], q[14], q[15]));
    };
    emit(r0, v0);
    emit(r1, v1);
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

template <int NT>
__global__ void __launch_bounds__(NT, 3) k_scan(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    constexpr int NW = NT / 32, NOCT = NT / 8;
    const IvfView& v = a.v;
    const int qi = blockIdx.x / a.nchunks;
    const int chunk = blockIdx.x - qi * a.nchunks;
    const int p0 = chunk * a.pch;
    const int np = min(a.P, p0 + a.pch) - p0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int G = shared_lut ? a.pch : kGroup;
    const int nlut = shared_lut ? 1 : kGroup;
    const int qtab_len = v.mode == kModeL2 ? v.m * 16 : (v.mode == kModeL2Adc ? v.dim : 0);

    uint64_t* ckey = reinterpret_cast<uint64_t*>(sm);
    uint4* lut = reinterpret_cast<uint4*>(ckey + a.cap);
    float* rmin_all = reinterpret_cast<float*>(lut + static_cast<size_t>(nlut) * v.m_pad);
    float* qtab = rmin_all + (shared_lut ? 0 : NW * v.m_pad);
    float* p_scale = qtab + qtab_len;
    float* p_offset = p_scale + a.pch;
    int* p_smax = reinterpret_cast<int*>(p_offset + a.pch);
    uint32_t* p_list = reinterpret_cast<uint32_t*>(p_smax + a.pch);
    uint32_t* p_size = p_list + a.pch;
    uint32_t* p_push = p_size + a.pch;
    uint32_t* g_sbpre = p_push + a.pch;   // G + 1
    __shared__ int s_count, s_overflow;
    __shared__ uint64_t s_thr;
    __shared__ uint32_t red[NW];

    const size_t qp = static_cast<size_t>(qi) * a.P;
    if (tid == 0) {
        s_count = 0;
        s_overflow = 0;
        s_thr = ~0ull;
    }
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
        for (int r = tid; r < v.m_pad; r += NT) lut[r] = a.qlut[static_cast<size_t>(qi) * v.m_pad + r];
        for (int p = tid; p < np; p += NT) {
            p_scale[p] = a.qscale[qi];
            p_offset[p] = __fadd_rn(a.qoffset[qi], a.pterm[qp + p0 + p]);
        }
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t b = 0;
        for (int w = 0; w < NW; ++w) b += red[w];
        for (int p = 0; p < np; ++p) {
            p_push[p] = b;
            b += p_size[p];
        }
    }

    const int oct = tid >> 3, r = tid & 7;
    for (int g0 = 0; g0 < np; g0 += G) {
        const int gn = min(G, np - g0);
        if (!shared_lut) {
            float* rmin = rmin_all + warp * v.m_pad;
            for (int p = warp; p < gn; p += NW) {
                const uint32_t l = p_list[g0 + p];
                float s, o;
                if (v.mode == kModeL2) {
                    const float A = a.pterm[qp + p0 + g0 + p];
                    const float* B = v.B + static_cast<size_t>(l) * v.m * 16;
                    warp_lut(
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
                                for (int j = 0; j < 16; ++j) out[j] = __fadd_rn(out[j], A);
                            }
                        },
                        v.m, v.m_pad, rmin, lut + static_cast<size_t>(p) * v.m_pad, s, o);
                } else {
                    // the residual (q - center) is formed per element inside the table
                    // loop, as compute_adc_table reads it (reference src/ivf_index.cpp:594-610)
                    const float* ctr = v.resid + static_cast<size_t>(l) * v.dim;
                    warp_lut(
                        [&](int rr, float* out) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                float acc = 0.0f;
                                for (int u = 0; u < v.sd; ++u) {
                                    const int e = rr * v.sd + u;
                                    const float diff = __fsub_rn(__fsub_rn(qtab[e], ctr[e]), v.pq_t[e * 16 + j]);
                                    acc = __fmaf_rn(diff, diff, acc);
                                }
                                out[j] = acc;
                            }
                        },
                        v.m, v.m_pad, rmin, lut + static_cast<size_t>(p) * v.m_pad, s, o);
                }
                if (lane == 0) {
                    p_scale[g0 + p] = s;
                    p_offset[g0 + p] = o;
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t sb = 0;
            for (int p = 0; p < gn; ++p) {
                g_sbpre[p] = sb;
                sb += (p_size[g0 + p] + kSuperBlock - 1) / kSuperBlock;
            }
            g_sbpre[gn] = sb;
        }
        {
            const uint32_t tk = static_cast<uint32_t>(s_thr >> 32);
            for (int p = tid; p < gn; p += NT) p_smax[g0 + p] = sum_limit(tk, p_scale[g0 + p], p_offset[g0 + p]);
        }
        __syncthreads();
        const int total = static_cast<int>(g_sbpre[gn]);
        for (int base = 0; base < total; base += NOCT) {
            const int item = base + oct;
            if (item < total) {
                const int pl = upper_index(g_sbpre, gn, static_cast<uint32_t>(item));
                const int p = g0 + pl;
                const int sbl = item - static_cast<int>(g_sbpre[pl]);
                const uint32_t l = p_list[p];
                const size_t sbg = static_cast<size_t>(v.sb_off[l]) + sbl;
                const uint4* L = lut + static_cast<size_t>(shared_lut ? 0 : pl) * v.m_pad;
                uint32_t sums[8];
                octet_sums(v.codes + sbg * static_cast<size_t>(2 * v.m_pad), L, v.m_pad, r, sums);
                const int smax = p_smax[p];
                const uint32_t size = p_size[p];
                const float scale = p_scale[p], offset = p_offset[p];
                const uint64_t thr = s_thr;
                const uint32_t push0 = p_push[p];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const uint32_t pos = static_cast<uint32_t>(sbl) * kSuperBlock + 8 * r + i;
                    if (pos < size && static_cast<int>(sums[i]) <= smax) {
                        const float dist = fs_dist(sums[i], scale, offset);
                        const uint64_t key = (static_cast<uint64_t>(float_key(dist)) << 32) | (push0 + pos);
                        if (key < thr) {
                            const uint32_t slot = v.ids[sbg * kSuperBlock + 8 * r + i];
                            const bool ok = a.filter ? ((a.filter[slot >> 6] >> (slot & 63)) & 1ull)
                                                     : !(v.deleted && ((v.deleted[slot >> 6] >> (slot & 63)) & 1ull));
                            if (ok) {
                                const int idx = atomicAdd(&s_count, 1);
                                if (idx < a.cap) ckey[idx] = key;
                                else s_overflow = 1;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            if (s_count > a.cap - NOCT * kSuperBlock) {
                const int n = min(s_count, a.cap);
                const int npow = max(2, next_pow2(n));
                for (int i = n + tid; i < npow; i += NT) ckey[i] = ~0ull;
                bitonic_sort_keys(ckey, npow);
                if (tid == 0) {
                    if (n >= a.kp) s_thr = ckey[a.kp - 1];
                    s_count = min(n, a.kp);
                }
                __syncthreads();
                const uint32_t tk = static_cast<uint32_t>(s_thr >> 32);
                for (int p = tid; p < gn; p += NT) p_smax[g0 + p] = sum_limit(tk, p_scale[g0 + p], p_offset[g0 + p]);
                __syncthreads();
            }
        }
    }
    // ---- output: this chunk's k' best, sorted by key64, with their slots ---------
    const int n = min(s_count, a.cap);
    if (n > 0) {
        const int npow = max(2, next_pow2(n));
        for (int i = n + tid; i < npow; i += NT) ckey[i] = ~0ull;
        bitonic_sort_keys(ckey, npow);
    }
    const int kept = min(n, a.kp);
    const size_t ob = static_cast<size_t>(blockIdx.x) * a.kp;
    for (int i = tid; i < a.kp; i += NT) {
        if (i < kept) {
            const uint64_t key = ckey[i];
            const uint32_t push = static_cast<uint32_t>(key);
            const int p = upper_index(p_push, np, push);
            const uint32_t pos = push - p_push[p];
            const size_t sbg = static_cast<size_t>(v.sb_off[p_list[p]]) + pos / kSuperBlock;
            a.out_key[ob + i] = key;
            a.out_slot[ob + i] = v.ids[sbg * kSuperBlock + pos % kSuperBlock];
        } else {
            a.out_key[ob + i] = ~0ull;
            a.out_slot[ob + i] = 0xFFFFFFFFu;
        }
    }
    if (tid == 0 && s_overflow) atomicExch(a.err, 1);
}

static size_t scan_smem_bytes(const IvfView& v, int pch, int cap) {
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int nlut = shared_lut ? 1 : kGroup;
    const int nw = kScanThreads / 32;
    const int qtab = v.mode == kModeL2 ? v.m * 16 : (v.mode == kModeL2Adc ? v.dim : 0);
    const int G = shared_lut ? pch : kGroup;
    size_t b = static_cast<size_t>(cap) * 8;
    b += static_cast<size_t>(nlut) * v.m_pad * 16;
    b += shared_lut ? 0 : static_cast<size_t>(nw) * v.m_pad * 4;
    b += static_cast<size_t>(qtab) * 4;
    b += static_cast<size_t>(pch) * 4 * 6 + static_cast<size_t>(G + 1) * 4;
    return b;
}

int scan_cap(int kp) {
    // room for k' kept entries plus one full round of candidates (32 octets of
    // a 256-thread block, 64 vectors each)
    return next_pow2(kp + (kScanThreads / 8) * kSuperBlock);
}

void ivf_candidates(const IvfView& v, const IvfSearchArgs& s, uint64_t* out_key, uint32_t* out_slot, cudaStream_t st) {
    const int nq = s.nq, P = s.nprobe, kp = s.kp;
    if (nq == 0) return;
    // coarse: all pair scores, then the P nearest lists per query
    DevBuf<float> scores(static_cast<size_t>(nq) * v.nlist, st);
    pair_scores(s.q, nq, v.centroids, v.nlist, v.dim, v.ip_metric, scores.get(), v.nlist, st);
    DevBuf<uint32_t> probe(static_cast<size_t>(nq) * P, st);
    DevBuf<float> pdist(static_cast<size_t>(nq) * P, st);
    // (score, list) compared as the reference's heap of (float, uint16_t) pairs does: -0 == +0
    select_rows(scores.get(), v.nlist, nq, v.nlist, P, probe.get(), pdist.get(), st, nullptr, nullptr, 0, true);
    scores.release();

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
    const int cap = scan_cap(kp);
    const size_t smem = scan_smem_bytes(v, pch, cap);
    require(smem <= 227 * 1024, "fast-scan shared memory exceeds the B200 limit for this m / k * k_factor",
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
    a.P = P;
    a.pch = pch;
    a.nchunks = nchunks;
    a.kp = kp;
    a.cap = cap;
    a.out_key = direct ? out_key : ckey.get();
    a.out_slot = direct ? out_slot : cslot.get();
    a.err = s.d_err;
    QG_CUDA(cudaFuncSetAttribute(k_scan<kScanThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    {
        KernelTimer kt("scan", st);
        k_scan<kScanThreads><<<static_cast<unsigned>(nq * nchunks), kScanThreads, smem, st>>>(a);
        QG_LAUNCH_CHECK();
    }
    if (!direct) merge_candidates(ckey.get(), cslot.get(), nq, nchunks, kp, out_key, out_slot, st);
}

} // namespace qg
