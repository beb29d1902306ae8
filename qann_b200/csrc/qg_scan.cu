// The code scan with fused top-k' selection (reference src/ivf_index.cpp:421-641,
// src/topk.hpp), and the orchestration of one IVF fast-scan search.
//
// Work units are (query, chunk of at most 256 of its probes). The kernel is
// persistent: a block takes the next unit from a global counter until none
// is left. Inside a unit the block walks the probes in groups of `lc` lists.
// For each group the warps first build the lists' uint8 LUTs into one half
// of a double-buffered LUT ring (mode L2: B + C + A rounded as
// build_quantize_lut; mode L2-ADC: the residual's ADC table rounded; modes IP
// and cosine-IP share the query's one LUT and only set each list's
// scale / offset). Then every octet (8 lanes) of every warp takes superblocks
// (64 vectors) of the group from a shared counter, so uneven lists spread
// over all octets. A warp that finds no superblock left goes on to build the
// next group's LUTs in the other half: one block barrier per group.
//
// Selection keeps the k' smallest candidates by key64 = key(dist) << 32 |
// push index, the push index being the vector's position in the query's
// sequence of probed lists: exactly the set the reference's TopK keeps
// (distance first, first pushed among ties). Each warp appends the candidates
// that beat the block's threshold to its own buffer; when the buffer is
// nearly full it keeps its k' best (radix select) and lowers the block
// threshold to its k'-th key (an upper bound of the block's k'-th, so the
// pruning is exact). Deleted (or filtered-out) vectors are skipped before
// they can enter, as the reference's push() does. The integer pre-test
// `sum <= S*` is exact: S* is the largest sum whose distance is <= the
// threshold distance (sum_limit). At the end of a unit the warps' survivors
// are gathered, cut to k', sorted, and their slots looked up from the push
// index.
#include "qg_device.cuh"
#include "qg_search.h"
#include "qg_sm100.cuh"
#include "qg_train.h"

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

namespace qg {

namespace {
constexpr int kMaxChunk = 256;   // probes per work unit at most
constexpr int kMinChunk = 8;     // probes per work unit at least, when the query has that many
constexpr int kSbPerWarp = 4;    // superblocks a warp takes at a time, one per octet
// Row stride (floats) of the query's table C in shared memory: 80 bytes puts
// the 16-byte reads of 8 lanes (one row each) on distinct banks.
constexpr int kQtabStride = 20;
constexpr int kFirstGroup = 2;   // lists in the first LUT group (at most LC)
}

// LUT of one list by one warp. Same arithmetic as quantize_lut. Lane l forms
// rows l and l + 32 (of each round of 64 rows) together in straight-line code,
// so that their table loads are in flight at once, and keeps the last round's
// two rows in registers for the rounding pass; with m > 64 the earlier rounds'
// rows are formed again there. The row minima meet in shared memory, where
// four lanes sum them in the reference's order (each lane's rows r = lane
// mod 4 in order, then (p0 + p1) + (p2 + p3)), eight loads ahead.
// thr_hi: the block's current threshold key (0xFFFFFFFF: none yet). When even
// a zero sum's distance is above it, no vector of the list can become a
// candidate (distances grow with the sum and the threshold only falls), so
// the LUT entries are left unwritten: the scan never reads them, because its
// sum limit for such a list is -1.
template <class RowFn>
__device__ __forceinline__ bool warp_lut3(RowFn row, int m, int m_pad, float* row_min, uint4* lut_out, float& scale_out,
                                          float& offset_out, uint32_t thr_hi) {
    const int lane = threadIdx.x & 31;
    float widest = 0.0f;
    float va[16], vb[16];   // rows base + lane and base + 32 + lane of the last round
    float mina = 0.0f, minb = 0.0f;
    auto range = [&](const float* v, float& lo_out) {
        float lo = v[0], hi = v[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            lo = fminf(lo, v[j]);
            hi = fmaxf(hi, v[j]);
        }
        lo_out = lo;
        return __fsub_rn(hi, lo);
    };
    auto low = [&](const float* v) {
        float lo = v[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) lo = fminf(lo, v[j]);
        return lo;
    };
    // one round (m <= 64): the rows stay in registers, and their maxima are
    // formed only once the list is known not to be hopeless
    const bool one_round = m <= 64;
    int base = 0;
    for (;; base += 64) {
        const int ra = base + lane, rb = ra + 32;
        row(min(ra, m - 1), va);   // (lanes past the last row form row m - 1 again, unused)
        row(min(rb, m - 1), vb);
        if (one_round) {
            mina = low(va);
            minb = low(vb);
        } else {
            const float wa = range(va, mina), wb = range(vb, minb);
            if (ra < m) widest = widest < wa ? wa : widest;
            if (rb < m) widest = widest < wb ? wb : widest;
        }
        if (ra < m) row_min[ra] = mina;
        if (rb < m) row_min[rb] = minb;
        if (base + 64 >= m) break;
    }
    __syncwarp();
    float part = 0.0f;
    if (lane < 4)
        for (int r0 = lane; r0 < m; r0 += 32) {
            float t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t[u] = r0 + 4 * u < m ? row_min[r0 + 4 * u] : 0.0f;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (r0 + 4 * u < m) part = __fadd_rn(part, t[u]);
        }
    const float p0 = __shfl_sync(0xffffffffu, part, 0), p1 = __shfl_sync(0xffffffffu, part, 1);
    const float p2 = __shfl_sync(0xffffffffu, part, 2), p3 = __shfl_sync(0xffffffffu, part, 3);
    const float offset = __fadd_rn(__fadd_rn(p0, p1), __fadd_rn(p2, p3));
    if (one_round) {
        // a zero sum's distance is 0 + offset for any scale > 0 and NaN (key
        // 0xFFFFFFFF, above every threshold but the open one) for scale 0, so a
        // list whose 0 + offset is above the threshold is hopeless at any scale
        if (thr_hi != 0xFFFFFFFFu && float_key(__fadd_rn(0.0f, offset)) > thr_hi) {
            scale_out = 1.0f;
            offset_out = offset;
            __syncwarp();
            return false;
        }
        float hia = va[0], hib = vb[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            hia = fmaxf(hia, va[j]);
            hib = fmaxf(hib, vb[j]);
        }
        const float wa = __fsub_rn(hia, mina), wb = __fsub_rn(hib, minb);
        if (lane < m) widest = widest < wa ? wa : widest;
        if (lane + 32 < m) widest = widest < wb ? wb : widest;
    }
    widest = warp_max(widest);
    const float scale = widest > 0.0f ? __fdiv_rn(static_cast<float>(kLutMax), widest) : 1.0f;
    const bool live = thr_hi == 0xFFFFFFFFu || float_key(fs_dist0(scale, offset)) <= thr_hi;   // (warp-uniform)
    if (live) {
        float v0[16];
        for (int r = lane; r < base; r += 32) {   // rounds before the last one
            row(r, v0);
            lut_out[r] = round_row(v0, row_min[r], scale);
        }
        if (base + lane < m) lut_out[base + lane] = round_row(va, mina, scale);
        if (base + 32 + lane < m) lut_out[base + 32 + lane] = round_row(vb, minb, scale);
        for (int r = m + lane; r < m_pad; r += 32) lut_out[r] = make_uint4(0, 0, 0, 0);
    }
    scale_out = scale;
    offset_out = offset;
    __syncwarp();
    return live;
}

// Mode L2: the LUT of B[list] + C[query] (+ A on row 0), as build_quantize_lut
// sums them (reference src/fast_scan.cpp:243-254).
__device__ __forceinline__ bool warp_lut_l2(const float* __restrict__ B, const float* qtab, float A, int m, int m_pad,
                                         float* row_min, uint4* lut_out, float* scale_out, float* offset_out,
                                         uint32_t thr_hi) {
    float sc, of;
    const bool live = warp_lut3(
        [&](int rr, float* o) {
            const float4* b4 = reinterpret_cast<const float4*>(B + rr * 16);
            const float4* c4 = reinterpret_cast<const float4*>(qtab + rr * kQtabStride);
#pragma unroll
            for (int u = 0; u < 4; ++u) {   // packed FP32 adds, rounding per component as __fadd_rn
                const float4 bb = __ldg(b4 + u), cc = c4[u];
                const float2 lo = __fadd2_rn(make_float2(bb.x, bb.y), make_float2(cc.x, cc.y));
                const float2 hi = __fadd2_rn(make_float2(bb.z, bb.w), make_float2(cc.z, cc.w));
                o[4 * u + 0] = lo.x;
                o[4 * u + 1] = lo.y;
                o[4 * u + 2] = hi.x;
                o[4 * u + 3] = hi.y;
            }
            if (rr == 0) {
                const float2 a2 = make_float2(A, A);
#pragma unroll
                for (int jj = 0; jj < 16; jj += 2) {
                    const float2 t = __fadd2_rn(make_float2(o[jj], o[jj + 1]), a2);
                    o[jj] = t.x;
                    o[jj + 1] = t.y;
                }
            }
        },
        m, m_pad, row_min, lut_out, sc, of, thr_hi);
    *scale_out = sc;
    *offset_out = of;
    return live;
}

// Mode L2-ADC: the LUT of the residual's ADC table; the residual (q - center)
// is formed per element inside the table loop, as compute_adc_table reads it
// (reference src/ivf_index.cpp:594-610).
__device__ __forceinline__ bool warp_lut_adc(const float* __restrict__ ctr, const float* q, const float* __restrict__ pq_t,
                                          int sd, int m, int m_pad, float* row_min, uint4* lut_out, float* scale_out,
                                          float* offset_out, uint32_t thr_hi) {
    float sc, of;
    const bool live = warp_lut3(
        [&](int rr, float* o) {
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
                float acc = 0.0f;
                for (int u = 0; u < sd; ++u) {
                    const int e = rr * sd + u;
                    const float diff = __fsub_rn(__fsub_rn(q[e], ctr[e]), pq_t[e * 16 + jj]);
                    acc = __fmaf_rn(diff, diff, acc);
                }
                o[jj] = acc;
            }
        },
        m, m_pad, row_min, lut_out, sc, of, thr_hi);
    *scale_out = sc;
    *offset_out = of;
    return live;
}

// octet_sums over a superblock staged in shared memory.
__device__ __forceinline__ void octet_sums_shared(const uint4* sb, const uint4* __restrict__ lut, int m_pad, int r,
                                                  uint32_t sums[8]) {
    uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    const int nq = m_pad >> 2;
    int q = 0;
    for (; q + 2 <= nq; q += 2) {
        const uint4 w0 = sb[q * 8 + r], w1 = sb[(q + 1) * 8 + r];
        octet_step(w0, lut + 4 * q, a0, b0, a1, b1);
        octet_step(w1, lut + 4 * (q + 1), a0, b0, a1, b1);
    }
    if (q < nq) octet_step(sb[q * 8 + r], lut + 4 * q, a0, b0, a1, b1);
    sums[0] = a0 & 0xFFFFu;
    sums[1] = b0 & 0xFFFFu;
    sums[2] = a0 >> 16;
    sums[3] = b0 >> 16;
    sums[4] = a1 & 0xFFFFu;
    sums[5] = b1 & 0xFFFFu;
    sums[6] = a1 >> 16;
    sums[7] = b1 >> 16;
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

// Shared memory of one block. The LUT ring shares its space with the
// end-of-unit gather of candidates and their final sort.
struct ScanLayout {
    int nw, lc, wcap, lut_stride;   // lut_stride: uint4s per LUT (m_pad + 2: 32 bytes keep
                                    // consecutive LUTs of a warp's octets on distinct banks)
    size_t off_wbuf, off_hist, off_rmin, off_group, off_probe, off_qtab, off_stage, off_cbar, bytes;
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~static_cast<size_t>(15); }

__host__ __device__ inline ScanLayout scan_layout(int kp, int m_pad, int qtab_len, int pch, bool shared_lut, int nw,
                                                  int lc, bool staged) {
    ScanLayout L;
    L.nw = nw;
    L.lc = lc;
    L.wcap = (kp + kSbPerWarp * kSuperBlock + 31) & ~31;
    L.lut_stride = m_pad + 2;
    const size_t lut = shared_lut ? static_cast<size_t>(m_pad) * 16 : static_cast<size_t>(2) * lc * L.lut_stride * 16;
    const size_t gather = static_cast<size_t>(nw) * kp * 8;
    const size_t sortb = static_cast<size_t>(next_pow2(kp < 2 ? 2 : kp)) * 8;
    size_t b = align16(lut > gather ? (lut > sortb ? lut : sortb) : (gather > sortb ? gather : sortb));
    L.off_wbuf = b;
    b += static_cast<size_t>(nw) * L.wcap * 8;
    L.off_hist = b;
    b += static_cast<size_t>(nw) * 256 * 4;
    L.off_rmin = b;
    b += shared_lut ? 0 : static_cast<size_t>(nw) * m_pad * 4;
    L.off_group = b;
    b += static_cast<size_t>(2) * lc * 8;                         // scale, offset of both halves
    L.off_probe = b;
    b += static_cast<size_t>(pch) * 16 + static_cast<size_t>(pch + 1) * 4;   // list, size, push, first superblock, prefix
    b = align16(b);
    L.off_qtab = b;
    b += static_cast<size_t>(qtab_len) * 4;
    b = (b + 127) & ~static_cast<size_t>(127);
    L.off_stage = b;   // staged: per warp, two stages of kSbPerWarp superblocks
    b += staged ? static_cast<size_t>(nw) * 2 * kSbPerWarp * m_pad * 32 : 0;
    L.off_cbar = b;    // staged: per warp, one mbarrier per stage
    b += staged ? static_cast<size_t>(nw) * 2 * 8 : 0;
    L.bytes = align16(b);
    return L;
}

// kMinB: blocks per SM the register budget is sized for (the dense shapes
// trade registers for more resident warps, which hide the scan's latencies).
template <int NW, bool kStaged, int kMinB = (kStaged ? 1 : 2)>
__global__ void __launch_bounds__(NW * 32, kMinB) k_scan(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    constexpr int NT = NW * 32;
    constexpr unsigned kFull = 0xffffffffu;
    const IvfView& v = a.v;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int oct = lane >> 3, r = lane & 7;
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int qtab_len = v.mode == kModeL2 ? v.m * kQtabStride : (v.mode == kModeL2Adc ? v.dim : 0);
    const ScanLayout lay = scan_layout(a.kp, v.m_pad, qtab_len, a.pch, shared_lut, NW, a.lc, kStaged);
    const int wcap = lay.wcap, LC = lay.lc, LS = lay.lut_stride, kp = a.kp;
    const uint32_t sb_bytes = static_cast<uint32_t>(v.m_pad) * 32;   // one superblock of codes
    uint8_t* cstage = sm + lay.off_stage + static_cast<size_t>(warp) * 2 * kSbPerWarp * sb_bytes;
    uint64_t* cbar = reinterpret_cast<uint64_t*>(sm + lay.off_cbar) + 2 * warp;
    int cst = 0;         // stage the next take fills
    uint32_t cpar = 0;   // bit s: parity of stage s's next completion

    uint4* lut_ring = reinterpret_cast<uint4*>(sm);
    uint64_t* gath = reinterpret_cast<uint64_t*>(sm);
    uint64_t* wbuf = reinterpret_cast<uint64_t*>(sm + lay.off_wbuf) + static_cast<size_t>(warp) * wcap;
    int* hist = reinterpret_cast<int*>(sm + lay.off_hist) + warp * 256;
    float* wrmin = reinterpret_cast<float*>(sm + lay.off_rmin) + warp * v.m_pad;
    float* g_scale = reinterpret_cast<float*>(sm + lay.off_group);   // [2][LC]
    float* g_offset = g_scale + 2 * LC;
    uint32_t* p_list = reinterpret_cast<uint32_t*>(sm + lay.off_probe);
    uint32_t* p_size = p_list + a.pch;
    uint32_t* p_push = p_size + a.pch;
    uint32_t* p_sboff = p_push + a.pch;   // each probe's first superblock in the code array
    uint32_t* p_sbpre = p_sboff + a.pch;  // pch + 1
    float* qtab = reinterpret_cast<float*>(sm + lay.off_qtab);
    __shared__ int s_unit, s_overflow, s_abort;
    __shared__ int s_next[2], s_build[2];
    __shared__ unsigned long long s_thr;
    __shared__ int s_wcount[NW];
    __shared__ uint32_t s_red[NW], s_red2[NW];

    if (tid == 0) s_abort = 0;
    if (kStaged && lane == 0) {
        sm100::mbar_init(&cbar[0], 1);
        sm100::mbar_init(&cbar[1], 1);
        sm100::fence_barrier_init();
    }
    for (;;) {
        __syncthreads();   // the previous unit is done with every shared array
        if (tid == 0) s_unit = atomicAdd(a.work, 1);
        __syncthreads();
        const int unit = s_unit;
        if (unit >= a.nunits) break;
        const int qi = unit / a.nchunks;
        const int chunk = unit - qi * a.nchunks;
        const int p0 = chunk * a.pch;
        const int np = min(a.nprobe_q ? a.nprobe_q[qi] : a.P, p0 + a.pch) - p0;
        const size_t ob = static_cast<size_t>(unit) * kp;
        if (np <= 0) {   // a query whose probes end before this chunk
            for (int i = tid; i < kp; i += NT) {
                a.out_key[ob + i] = ~0ull;
                a.out_slot[ob + i] = 0xFFFFFFFFu;
            }
            continue;
        }
        const uint64_t* qfilter = a.filters ? a.filters[qi] : a.filter;
        const size_t qp = static_cast<size_t>(qi) * a.P;

        // ---- the unit's probes, tables and counters ----
        uint32_t before = 0;   // vectors pushed by the query's earlier chunks
        for (int p = tid; p < p0; p += NT) before += v.list_size[a.probe[qp + p]];
        for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(kFull, before, o);
        if (lane == 0) s_red[warp] = before;
        for (int p = tid; p < np; p += NT) {
            const uint32_t l = a.probe[qp + p0 + p];
            p_list[p] = l;
            p_size[p] = v.list_size[l];
            p_sboff[p] = v.sb_off[l];
        }
        if (v.mode == kModeL2)
            for (int t = tid; t < v.m * 16; t += NT)
                qtab[(t >> 4) * kQtabStride + (t & 15)] = a.qC[static_cast<size_t>(qi) * v.m * 16 + t];
        if (v.mode == kModeL2Adc)
            for (int t = tid; t < v.dim; t += NT) qtab[t] = a.q[static_cast<size_t>(qi) * v.dim + t];
        if (shared_lut)
            for (int rr = tid; rr < v.m_pad; rr += NT) lut_ring[rr] = a.qlut[static_cast<size_t>(qi) * v.m_pad + rr];
        if (tid == 0) {
            s_overflow = 0;
            s_thr = a.qthr ? *reinterpret_cast<volatile unsigned long long*>(a.qthr + qi) : ~0ull;
            s_next[0] = 0;
            s_next[1] = 0;
            s_build[0] = 0;
        }
        __syncthreads();
        if (warp == 0) {
            // push offsets and superblock prefix of the unit's probes
            uint32_t run_push = 0, run_sb = 0;
            for (int w = 0; w < NW; ++w) run_push += s_red[w];
            for (int base = 0; base < np; base += 32) {
                const int p = base + lane;
                const uint32_t sz = p < np ? p_size[p] : 0;
                // superblocks held on this device (none for another shard's list)
                const uint32_t nsb = p < np ? v.sb_off[p_list[p] + 1] - p_sboff[p] : 0;
                uint32_t ip = sz, is = nsb;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t1 = __shfl_up_sync(kFull, ip, o), t2 = __shfl_up_sync(kFull, is, o);
                    if (lane >= o) {
                        ip += t1;
                        is += t2;
                    }
                }
                if (p < np) {
                    p_push[p] = run_push + ip - sz;
                    p_sbpre[p] = run_sb + is - nsb;
                }
                run_push += __shfl_sync(kFull, ip, 31);
                run_sb += __shfl_sync(kFull, is, 31);
            }
            if (lane == 0) p_sbpre[np] = run_sb;
        }

        // LUTs (or scale / offset) of group g into half g & 1. Warps take the
        // lists from a counter, so warps that finish scanning group g - 1 early
        // build more of them. A list none of whose vectors can beat the block
        // threshold (even a zero sum's distance is above it) gets scale -1 (real
        // scales are >= 0) and no LUT; the group's scan skips its superblocks.
        // Groups of LC lists, the first one of 2 only: its keys meet no threshold
        // yet, so the block's bound on the k'-th key after it (below) comes
        // sooner. (2 to 4 lists measured best for 8 x 32, 8 x 16 and 4 x 8 shapes
        // alike, 2 by a little.)
        const int first = min(LC, kFirstGroup);
        auto group_start = [&](int g) { return g == 0 ? 0 : min(np, first + (g - 1) * LC); };
        auto build_group = [&](int g) {
            const int h = g & 1, gp0 = group_start(g), nc = group_start(g + 1) - gp0;
            if (tid == 0) {
                s_next[h] = 0;        // its last user, group g - 2, is done
                s_build[h ^ 1] = 0;   // group g + 1's; its last user, group g - 1, is done
            }
            for (;;) {
                int j = 0;
                if (lane == 0) j = atomicAdd(&s_build[h], 1);
                j = __shfl_sync(kFull, j, 0);
                if (j >= nc) break;
                const int p = gp0 + j;
                uint32_t thr_now = 0;   // the same in every lane
                if (lane == 0) thr_now = static_cast<uint32_t>(*reinterpret_cast<volatile unsigned long long*>(&s_thr) >> 32);
                thr_now = __shfl_sync(kFull, thr_now, 0);
                if (shared_lut) {
                    if (lane == 0) {
                        const float sc = a.qscale[qi], of = __fadd_rn(a.qoffset[qi], a.pterm[qp + p0 + p]);
                        const bool live = thr_now == 0xFFFFFFFFu || float_key(fs_dist0(sc, of)) <= thr_now;
                        g_scale[h * LC + j] = live ? sc : -1.0f;
                        g_offset[h * LC + j] = of;
                    }
                    continue;
                }
                const uint32_t lj = p_list[p];
                uint4* out = lut_ring + static_cast<size_t>(h * LC + j) * LS;
                float sc, of;
                bool live;
                if (v.mode == kModeL2)
                    live = warp_lut_l2(v.B + static_cast<size_t>(lj) * v.m * 16, qtab, a.pterm[qp + p0 + p], v.m,
                                       v.m_pad, wrmin, out, &sc, &of, thr_now);
                else
                    live = warp_lut_adc(v.resid + static_cast<size_t>(lj) * v.dim, qtab, v.pq_t, v.sd, v.m, v.m_pad,
                                        wrmin, out, &sc, &of, thr_now);
                if (lane == 0) {
                    g_scale[h * LC + j] = live ? sc : -1.0f;
                    g_offset[h * LC + j] = of;
                }
            }
        };

        // (all threads, after a block barrier; the per-warp histograms serve as one)
        auto seed_threshold = [&]() {
            int total = 0;
            for (int w = 0; w < NW; ++w) total += s_wcount[w];
            if (total <= kp) return;   // (block-uniform)
            constexpr int kBins = NW * 256 < 1024 ? NW * 256 : 1024;
            int* bh = reinterpret_cast<int*>(sm + lay.off_hist);
            const uint64_t* wb0 = reinterpret_cast<const uint64_t*>(sm + lay.off_wbuf);
            uint32_t lo = ~0u, hi = 0;
            for (int w = 0; w < NW; ++w)
                for (int i = tid; i < s_wcount[w]; i += NT) {
                    const uint32_t k = static_cast<uint32_t>(wb0[static_cast<size_t>(w) * wcap + i] >> 32);
                    lo = min(lo, k);
                    hi = max(hi, k);
                }
            for (int t = tid; t < kBins; t += NT) bh[t] = 0;
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(kFull, lo, o));
                hi = max(hi, __shfl_xor_sync(kFull, hi, o));
            }
            if (lane == 0) {
                s_red[warp] = lo;
                s_red2[warp] = hi;
            }
            __syncthreads();
            for (int w = 0; w < NW; ++w) {
                lo = min(lo, s_red[w]);
                hi = max(hi, s_red2[w]);
            }
            if (lo == hi) {   // (block-uniform)
                if (tid == 0) {
                    atomicMin(&s_thr, (static_cast<unsigned long long>(lo) << 32) | 0xFFFFFFFFull);
                    if (a.qthr) atomicMin(a.qthr + qi, (static_cast<unsigned long long>(lo) << 32) | 0xFFFFFFFFull);
                }
                return;
            }
            const KeyBins kb(lo, static_cast<uint64_t>(hi - lo) + 1, kBins);
            for (int w = 0; w < NW; ++w)
                for (int i = tid; i < s_wcount[w]; i += NT) {
                    const uint32_t k = static_cast<uint32_t>(wb0[static_cast<size_t>(w) * wcap + i] >> 32);
                    atomicAdd(&bh[kb.bin(k)], 1);
                }
            __syncthreads();
            if (warp == 0) {   // lane l owns bins kPer l .. kPer l + kPer - 1
                constexpr int kPer = kBins / 32;
                int own = 0;
                for (int b = 0; b < kPer; ++b) own += bh[kPer * lane + b];
                int incl = own;
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl += t;
                }
                const int excl = incl - own;
                if (excl < kp && kp <= incl) {
                    int acc = excl, bin = kPer * lane + kPer - 1;
                    for (int b = 0; b < kPer; ++b) {
                        acc += bh[kPer * lane + b];
                        if (acc >= kp) {
                            bin = kPer * lane + b;
                            break;
                        }
                    }
                    // every key counted in bins <= bin is <= kb.last(bin)
                    const uint32_t T = static_cast<uint32_t>(min(kb.last(bin), static_cast<uint64_t>(hi)));
                    atomicMin(&s_thr, (static_cast<unsigned long long>(T) << 32) | 0xFFFFFFFFull);
                    if (a.qthr) atomicMin(a.qthr + qi, (static_cast<unsigned long long>(T) << 32) | 0xFFFFFFFFull);
                }
            }
            __syncthreads();   // warp 0 is done with the histograms before any trim reuses them
        };

        const int ngroups = np <= first ? 1 : 1 + (np - first + LC - 1) / LC;
        build_group(0);
        int wcount = 0;   // entries in this warp's buffer (the same in every lane)
        for (int g = 0; g < ngroups; ++g) {
            if (a.qthr && tid == 0)   // the bound the query's other chunks reached meanwhile
                atomicMin(&s_thr, *reinterpret_cast<volatile unsigned long long*>(a.qthr + qi));
            __syncthreads();   // group g's LUTs and the unit's prefix arrays are complete
            // After the first two groups: the warps' buffers together hold the
            // block's k' best keys so far, so the k'-th smallest of their union
            // bounds the unit's final k'-th key. Its high half, rounded up to the
            // end of a histogram interval, lowers the threshold: much tighter than
            // any single warp's k'-th, so about half as many later takes reach
            // the candidate path. (At later groups it cost more barriers than it
            // saved.)
            if (NW >= 4 && (g == 1 || g == 2)) seed_threshold();
            const int h = g & 1, gp0 = group_start(g), nc = group_start(g + 1) - gp0;
            // The group's superblocks without those of skipped lists, numbered
            // 0..total-1 list after list: list lane (and lane + 32 when LC = 64)
            // starts at st0 (st1); empty and skipped lists hold ~0u, which no
            // index reaches. Every warp forms these in its own registers.
            uint32_t st0 = 0, st1 = 0, total = 0;
            {
                uint32_t n0 = 0, n1 = 0;
                if (lane < nc && !(g_scale[h * LC + lane] < 0.0f))
                    n0 = p_sbpre[gp0 + lane + 1] - p_sbpre[gp0 + lane];
                if (lane + 32 < nc && !(g_scale[h * LC + lane + 32] < 0.0f))
                    n1 = p_sbpre[gp0 + lane + 33] - p_sbpre[gp0 + lane + 32];
                uint32_t i0 = n0, i1 = n1;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t0 = __shfl_up_sync(kFull, i0, o), t1 = __shfl_up_sync(kFull, i1, o);
                    if (lane >= o) {
                        i0 += t0;
                        i1 += t1;
                    }
                }
                const uint32_t tot0 = __shfl_sync(kFull, i0, 31);
                total = tot0 + __shfl_sync(kFull, i1, 31);
                st0 = n0 ? i0 - n0 : ~0u;
                st1 = n1 ? tot0 + i1 - n1 : ~0u;
            }
            int cur = -1;   // this octet's current list (index into the unit's probes)
            uint32_t list_sb = 0, size = 0, push0 = 0, thr_hi = 0;
            float scale = 1.0f, offset = 0.0f;
            int smax = 0;
            const uint4* L = lut_ring;
            // A take: the warp's next kSbPerWarp superblocks of the group, one per
            // octet: ti (valid while < total), its probe tp and the index tf of
            // that list's first superblock. Staged, the octets' leaders start
            // bulk copies of the taken superblocks into stage `cst`.
            auto take = [&](uint32_t& ti, int& tp, uint32_t& tf) -> bool {
                int base = 0;
                if (lane == 0) base = atomicAdd(&s_next[h], kSbPerWarp);
                base = __shfl_sync(kFull, base, 0);
                if (static_cast<uint32_t>(base) >= total) return false;
                ti = base + oct;
                // the list of each octet's superblock: the last list starting at or before it
                int jl = 0;
#pragma unroll
                for (int o = 0; o < kSbPerWarp; ++o) {
                    const uint32_t t = base + o;
                    const unsigned b1 = LC > 32 ? __ballot_sync(kFull, st1 <= t) : 0u;
                    const unsigned b0 = __ballot_sync(kFull, st0 <= t);
                    const int j = b1 ? 63 - __clz(b1) : 31 - __clz(b0);
                    if (o == oct) jl = j;
                }
                const uint32_t f0 = __shfl_sync(kFull, st0, jl & 31), f1 = __shfl_sync(kFull, st1, jl & 31);
                tf = jl < 32 ? f0 : f1;
                tp = ti < total ? gp0 + jl : -1;
                if constexpr (kStaged) {
                    const uint32_t nvalid = min(static_cast<uint32_t>(kSbPerWarp), total - base);
                    if (lane == 0) sm100::mbar_expect_tx(&cbar[cst], nvalid * sb_bytes);
                    __syncwarp();
                    if (r == 0 && tp >= 0) {
                        const size_t sbg = static_cast<size_t>(p_sboff[tp]) + (ti - tf);
                        sm100::bulk_load(cstage + static_cast<size_t>(cst * kSbPerWarp + oct) * sb_bytes,
                                         v.codes + sbg * static_cast<size_t>(2 * v.m_pad), sb_bytes, &cbar[cst]);
                    }
                    cst ^= 1;
                }
                return true;
            };
            // The sums of take (i, p) and its candidates; codes from `src` (the
            // stage in shared memory, or global memory).
            auto process = [&](uint32_t i, int p, uint32_t first, int stage) {
                const uint64_t thr = *reinterpret_cast<volatile unsigned long long*>(&s_thr);
                uint32_t sums[8];
                uint32_t cmask = 0, sbl = 0;
                size_t sbg = 0;
                if (p >= 0) {
                    if (p != cur) {
                        cur = p;
                        list_sb = p_sboff[p];
                        size = p_size[p];
                        push0 = p_push[p];
                        scale = g_scale[h * LC + p - gp0];
                        offset = g_offset[h * LC + p - gp0];
                        L = shared_lut ? lut_ring : lut_ring + static_cast<size_t>(h * LC + p - gp0) * LS;
                        thr_hi = static_cast<uint32_t>(thr >> 32);
                        smax = sum_limit_fast(thr_hi, scale, offset);
                    } else if (static_cast<uint32_t>(thr >> 32) != thr_hi) {
                        thr_hi = static_cast<uint32_t>(thr >> 32);
                        smax = sum_limit_fast(thr_hi, scale, offset);
                    }
                    sbl = i - first;
                    sbg = static_cast<size_t>(list_sb) + sbl;
                    if (smax < 0) {   // no vector of the list can pass (its LUT may be unbuilt)
#pragma unroll
                        for (int e = 0; e < 8; ++e) sums[e] = 0;
                    } else if constexpr (kStaged) {
                        octet_sums_shared(reinterpret_cast<const uint4*>(
                                              cstage + static_cast<size_t>(stage * kSbPerWarp + oct) * sb_bytes),
                                          L, v.m_pad, r, sums);
                    } else {
                        octet_sums_padded(v.codes + sbg * static_cast<size_t>(2 * v.m_pad), L, v.m_pad, r, sums);
                    }
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const uint32_t pos = sbl * kSuperBlock + 8 * r + e;
                        if (pos < size && static_cast<int>(sums[e]) <= smax) cmask |= 1u << e;
                    }
                }
                if (__any_sync(kFull, cmask != 0)) {
                    // keys of this lane's passing vectors; slots (and their filter
                    // or deletion bits) are read only when a filter or deletions
                    // exist, all loads of the lane in flight together
                    uint64_t keys[8];
                    uint32_t kmask = 0;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        keys[e] = ~0ull;
                        if ((cmask >> e) & 1u) {
                            const uint32_t pos = sbl * kSuperBlock + 8 * r + e;
                            const float dist = fs_dist(sums[e], scale, offset);
                            keys[e] = (static_cast<uint64_t>(float_key(dist)) << 32) | (push0 + pos);
                            if (keys[e] < thr) kmask |= 1u << e;
                        }
                    }
                    const uint64_t* bits = qfilter ? qfilter : v.deleted;
                    if (bits && kmask) {
                        uint32_t slot[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e)
                            slot[e] = (kmask >> e) & 1u ? v.ids[sbg * kSuperBlock + 8 * r + e] : 0u;
                        uint64_t word[8];
#pragma unroll
                        for (int e = 0; e < 8; ++e) word[e] = (kmask >> e) & 1u ? bits[slot[e] >> 6] : 0ull;
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const bool set = (word[e] >> (slot[e] & 63)) & 1ull;
                            // a filter lists the allowed slots; the deletion bitmap the removed ones
                            if (set != (qfilter != nullptr)) kmask &= ~(1u << e);
                        }
                    }
                    // append: this lane's keys after those of the lanes below it
                    const int mine = __popc(kmask);
                    int incl = mine;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(kFull, incl, o);
                        if (lane >= o) incl += t;
                    }
                    int idx = wcount + incl - mine;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        if ((kmask >> e) & 1u) {
                            if (idx < wcap) wbuf[idx] = keys[e];
                            else s_overflow = 1;
                            ++idx;
                        }
                    }
                    wcount += __shfl_sync(kFull, incl, 31);
                    if (wcount > wcap - kSbPerWarp * kSuperBlock && wcount > kp) {
                        __syncwarp();
                        // keys above the block threshold cannot be among the unit's
                        // k' best (the block holds k' keys at or below it, the one it
                        // equals included): drop them first, and select only if more
                        // than k' remain
                        const uint64_t lim = *reinterpret_cast<volatile unsigned long long*>(&s_thr);
                        wcount = warp_keep_upto(wbuf, min(wcount, wcap), lim);
                        if (wcount > kp) {
                            const uint64_t kth = warp_select_keep(wbuf, wcount, kp, hist);
                            if (lane == 0) {
                                atomicMin(&s_thr, static_cast<unsigned long long>(kth));
                                if (a.qthr) atomicMin(a.qthr + qi, static_cast<unsigned long long>(kth));
                            }
                            wcount = kp;
                        }
                    }
                }
            };
            uint32_t i0 = 0, i1 = 0, f0 = 0, f1 = 0;
            int q0 = -1, q1 = -1;
            int s0 = cst;
            bool v0 = take(i0, q0, f0);
            while (v0) {
                if constexpr (kStaged) {
                    const bool v1 = take(i1, q1, f1);   // the next take's copies overlap this one's sums
                    if (!sm100::mbar_wait(&cbar[s0], (cpar >> s0) & 1u, &s_abort)) {
                        s_abort = 1;
                        atomicExch(a.err, 2);
                    }
                    cpar ^= 1u << s0;
                    process(i0, q0, f0, s0);
                    __syncwarp();   // stage s0 is free again
                    s0 ^= 1;
                    i0 = i1;
                    q0 = q1;
                    f0 = f1;
                    v0 = v1;
                } else {
                    process(i0, q0, f0, 0);
                    v0 = take(i0, q0, f0);
                }
            }
            if (lane == 0) s_wcount[warp] = min(wcount, wcap);   // for the next group's threshold bound
            // out of superblocks of group g: build group g + 1 in the other half
            if (g + 1 < ngroups) build_group(g + 1);
        }

        // ---- the unit's k' best: each warp's own, gathered, cut to k', sorted ----
        __syncwarp();
        // keys above the block threshold first (as at a trim), so that fewer
        // reach warp 0's cut below
        wcount = warp_keep_upto(wbuf, min(wcount, wcap), *reinterpret_cast<volatile unsigned long long*>(&s_thr));
        if (wcount > kp) {
            warp_select_keep(wbuf, min(wcount, wcap), kp, hist);
            wcount = kp;
        }
        if (lane == 0) s_wcount[warp] = min(wcount, wcap);
        __syncthreads();   // every warp is done with the LUT ring: gather over it
        int off = 0, total = 0;
        for (int w = 0; w < NW; ++w) {
            if (w < warp) off += s_wcount[w];
            total += s_wcount[w];
        }
        for (int i = lane; i < s_wcount[warp]; i += 32) gath[off + i] = wbuf[i];
        __syncthreads();
        const int kept = min(total, kp);
        if (kept <= 256) {   // warp 0 alone cuts to k' and sorts in registers; one barrier
            if (warp == 0) {
                if (total > kp) warp_select_keep(gath, total, kp, hist);
                warp_sort_keys(gath, kept);
            }
            __syncthreads();
        } else {
            if (total > kp) {
                if (warp == 0) warp_select_keep(gath, total, kp, hist);
                __syncthreads();
            }
            const int ns = next_pow2(kept);
            for (int i = kept + tid; i < ns; i += NT) gath[i] = ~0ull;
            bitonic_sort_keys(gath, ns);
        }
        for (int i = tid; i < kp; i += NT) {
            if (i < kept) {
                const uint64_t key = gath[i];
                const uint32_t push = static_cast<uint32_t>(key);
                const int pp = upper_index(p_push, np, push);
                const uint32_t pos = push - p_push[pp];
                const size_t sbg = static_cast<size_t>(p_sboff[pp]) + pos / kSuperBlock;
                a.out_key[ob + i] = key;
                a.out_slot[ob + i] = v.ids[sbg * kSuperBlock + pos % kSuperBlock];
            } else {
                a.out_key[ob + i] = ~0ull;
                a.out_slot[ob + i] = 0xFFFFFFFFu;
            }
        }
        if (tid == 0 && s_overflow) atomicExch(a.err, 1);
    }
}

template <int NW, bool kStaged, int kMinB = (kStaged ? 1 : 2)>
static void launch_scan(const ScanArgs& a, size_t smem, cudaStream_t st) {
    allow_large_smem<k_scan<NW, kStaged, kMinB>>();
    int per_sm = 0;
    QG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan<NW, kStaged, kMinB>, NW * 32, smem));
    require(per_sm > 0, "fast-scan launch configuration does not fit on the device", kUnsupported);
    const unsigned blocks = static_cast<unsigned>(std::min<long long>(a.nunits, static_cast<long long>(per_sm) * sm_count()));
    KernelTimer kt("scan", st);
    k_scan<NW, kStaged, kMinB><<<blocks, NW * 32, smem, st>>>(a);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Scan shapes and their autotuner. A shape is (warps per block, lists per LUT
// group, codes read from global memory or staged through shared memory by
// bulk copies). Every shape gives the same results; the autotuner times the
// candidates on the first large search of each problem key and keeps the
// fastest for the rest of the process.
// ---------------------------------------------------------------------------
namespace {
struct ScanShape {
    int nw = 0, lc = 0;
    bool staged = false;
    bool dense = false;   // unstaged, registers sized for 3 (8 warps) or 5 (4 warps) blocks per SM
};

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int>, ScanShape> g_tuned;   // (mode, m_pad, kp, log2 P, log2 nq, variant) -> shape
std::atomic<int> g_autotune{1};    // 0: the first fitting unstaged shape, 1: tune
std::atomic<int> g_force{-1};      // -1: any; 0: unstaged (two-block) only; 1: staged only; 2: dense only
std::atomic<int> g_last_shape{0};  // the last scan's shape: warps * 1000 + lists per group * 10 + staged
}

void set_scan_autotune(int on) { g_autotune.store(on); }
int scan_autotune() { return g_autotune.load(); }
void set_scan_variant(int v) { g_force.store(v); }
int scan_variant() { return g_force.load(); }
int scan_last_shape() { return g_last_shape.load(); }
int scan_tuned_shapes() {
    std::lock_guard<std::mutex> g(g_tune_mu);
    return static_cast<int>(g_tuned.size());
}

// Candidate shapes whose shared memory fits: up to three unstaged ones for two
// blocks per SM (or one, when none fits that), the dense unstaged ones whose
// shared memory allows their block count, and a staged one.
static std::vector<ScanShape> scan_shapes(int kp, int m_pad, int qtab_len, int pch, bool shared_lut) {
    static constexpr int kUnstaged[][2] = {{8, 32}, {8, 16}, {4, 32}, {4, 16}, {8, 8}, {4, 8}, {2, 8}, {2, 4}, {1, 4}, {1, 1}};
    static constexpr int kStagedShapes[][2] = {{8, 16}, {8, 8}, {4, 32}, {4, 16}, {4, 8}};
    std::vector<ScanShape> out;
    const int force = g_force.load();
    auto fits = [&](const auto& table, bool staged, size_t limit, size_t most) {
        size_t added = 0;
        for (const auto& sh : table) {
            if (added == most) break;
            const int lc = shared_lut ? 64 : sh[1];
            const bool dup = std::any_of(out.begin(), out.end(), [&](const ScanShape& o) {
                return o.nw == sh[0] && o.lc == lc && o.staged == staged && !o.dense;
            });
            if (!dup && scan_layout(kp, m_pad, qtab_len, pch, shared_lut, sh[0], lc, staged).bytes <= limit) {
                out.push_back({sh[0], lc, staged, false});
                ++added;
            }
        }
        return added > 0;
    };
    if ((force == -1 || force == 0) && !fits(kUnstaged, false, 110 * 1024, 3)) fits(kUnstaged, false, 226 * 1024, 1);
    if (force == -1 || force == 2) {
        // dense: 8 warps x 3 blocks or 4 warps x 5 blocks per SM, the widest
        // LUT group whose shared memory allows that many blocks
        static constexpr int kDense[][3] = {{8, 3, 32}, {8, 3, 16}, {8, 3, 8}, {4, 5, 16}, {4, 5, 8}};
        int added8 = 0, added4 = 0;
        for (const auto& d : kDense) {
            int& added = d[0] == 8 ? added8 : added4;
            const int lc = shared_lut ? 64 : d[2];
            const size_t limit = (227 * 1024) / d[1] - 1024;
            if (added == 0 && scan_layout(kp, m_pad, qtab_len, pch, shared_lut, d[0], lc, false).bytes <= limit) {
                out.push_back({d[0], lc, false, true});
                added = 1;
            }
        }
    }
    if (force == -1 || force == 1) fits(kStagedShapes, true, 226 * 1024, 1);
    if (out.empty()) fits(kUnstaged, false, 226 * 1024, 1);   // (a forced kind that fits nowhere)
    return out;
}

static void run_scan(const ScanShape& sh, ScanArgs a, const IvfView& v, int qtab_len, cudaStream_t st) {
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    a.lc = sh.lc;
    const size_t smem = scan_layout(a.kp, v.m_pad, qtab_len, a.pch, shared_lut, sh.nw, sh.lc, sh.staged).bytes;
    QG_CUDA(cudaMemsetAsync(a.work, 0, sizeof(int), st));
    if (a.qthr)   // (every timed run of the autotuner starts from no bound too)
        QG_CUDA(cudaMemsetAsync(a.qthr, 0xFF, static_cast<size_t>(a.nunits / a.nchunks) * sizeof(unsigned long long), st));
    if (sh.staged) {
        switch (sh.nw) {
            case 8: launch_scan<8, true>(a, smem, st); break;
            default: launch_scan<4, true>(a, smem, st); break;
        }
    } else if (sh.dense) {
        if (sh.nw == 8) launch_scan<8, false, 3>(a, smem, st);
        else launch_scan<4, false, 5>(a, smem, st);
    } else {
        switch (sh.nw) {
            case 8: launch_scan<8, false>(a, smem, st); break;
            case 4: launch_scan<4, false>(a, smem, st); break;
            case 2: launch_scan<2, false>(a, smem, st); break;
            default: launch_scan<1, false>(a, smem, st); break;
        }
    }
}

// Times each candidate once on this search's own inputs (its outputs are
// the same every time) and returns the fastest.
static ScanShape tune_scan(const std::vector<ScanShape>& cands, const ScanArgs& a, const IvfView& v, int qtab_len,
                           cudaStream_t st) {
    cudaEvent_t e0, e1;
    QG_CUDA(cudaEventCreate(&e0));
    QG_CUDA(cudaEventCreate(&e1));
    ScanShape best = cands.front();
    float best_ms = 0.0f;
    // every candidate timed twice, in two rounds, its faster run kept: the
    // first launches of a search meet cold caches and one-time setup
    std::vector<float> fastest(cands.size(), 0.0f);
    for (int round = 0; round < 2; ++round)
        for (size_t c = 0; c < cands.size(); ++c) {
            QG_CUDA(cudaEventRecord(e0, st));
            run_scan(cands[c], a, v, qtab_len, st);
            QG_CUDA(cudaEventRecord(e1, st));
            QG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (round == 0 || ms < fastest[c]) fastest[c] = ms;
        }
    for (size_t c = 0; c < cands.size(); ++c)
        if (c == 0 || fastest[c] < best_ms) {
            best_ms = fastest[c];
            best = cands[c];
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// The query-major scan (k_scan) of nq queries: probe / pterm rows of
// `stride` entries, each query scanning its first probes_of[q] (or Pn) of
// them, at most Pn; tables qC (mode L2) or qlut / qscale / qoffset (IP
// modes), raw queries q (mode L2-ADC). Outputs each query's k' best keys and
// slots, sorted.
static void scan_query_major(const IvfView& v, const IvfSearchArgs& s, int nq, int stride, int Pn,
                             const uint32_t* probe, const float* pterm, const float* qC, const uint4* qlut,
                             const float* qscale, const float* qoffset, const float* q, const int* probes_of,
                             uint64_t* out_key, uint32_t* out_slot, cudaStream_t st) {
    const int kp = s.kp;
    if (nq == 0) return;
    // chunks: enough blocks to fill the GPU several times over, at most kMaxChunk probes each
    const int sms = s.sm_count > 0 ? s.sm_count : 148;
    const int P = Pn;
    // (and at least kMinChunk probes a chunk, so the merge stays small for small batches)
    int nchunks = std::clamp(static_cast<int>(ceil_div(static_cast<size_t>(4 * sms), nq)), 1,
                             std::max(1, P / kMinChunk));
    nchunks = std::max(nchunks, static_cast<int>(ceil_div(P, kMaxChunk)));
    const int pch = static_cast<int>(ceil_div(P, nchunks));
    nchunks = static_cast<int>(ceil_div(P, pch));
    const bool shared_lut = v.mode == kModeIP || v.mode == kModeCosIP;
    const int qtab_len = v.mode == kModeL2 ? v.m * kQtabStride : (v.mode == kModeL2Adc ? v.dim : 0);
    const std::vector<ScanShape> cands = scan_shapes(kp, v.m_pad, qtab_len, pch, shared_lut);
    require(!cands.empty(), "fast-scan shared memory exceeds the B200 limit for this m / k * k_factor", kUnsupported);

    const bool direct = nchunks == 1;
    const size_t nout = static_cast<size_t>(nq) * nchunks * kp;
    DevBuf<uint64_t> ckey;
    DevBuf<uint32_t> cslot;
    DevBuf<unsigned long long> qthr;
    if (!direct) {
        ckey.alloc(nout, st);
        cslot.alloc(nout, st);
        qthr.alloc(nq, st);
    }
    DevBuf<int> work(1, st);
    QG_CUDA(cudaMemsetAsync(work.get(), 0, sizeof(int), st));
    ScanArgs a{};
    a.v = v;
    a.q = q;
    a.probe = probe;
    a.pterm = pterm;
    a.qC = qC;
    a.qlut = qlut;
    a.qscale = qscale;
    a.qoffset = qoffset;
    a.filter = s.filter;
    a.filters = s.pq.filter;
    a.nprobe_q = probes_of;
    a.P = stride;
    a.pch = pch;
    a.nchunks = nchunks;
    a.kp = kp;
    a.nunits = nq * nchunks;
    a.work = work.get();
    a.qthr = direct ? nullptr : qthr.get();
    a.out_key = direct ? out_key : ckey.get();
    a.out_slot = direct ? out_slot : cslot.get();
    a.err = s.d_err;
    // the shape: tuned once per problem key on a search large enough to fill
    // the GPU several times over, else the first candidate. Batch size and
    // probe count enter the key by their power of two (served batches, whose
    // largest nprobe or filtered probe count changes from batch to batch,
    // would otherwise tune nearly every batch); a shape tuned for another
    // member of the bucket is kept when it is among this search's candidates.
    const int nq_bucket = 31 - __builtin_clz(static_cast<unsigned>(std::max(1, nq)));
    const int p_bucket = 31 - __builtin_clz(static_cast<unsigned>(std::max(1, P)));
    const auto key = std::make_tuple(v.mode, v.m_pad, kp, p_bucket, nq_bucket, g_force.load());
    ScanShape shape = cands.front();
    bool tuned = !g_autotune.load();
    if (!tuned) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        const auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            const ScanShape t = it->second;
            if (std::any_of(cands.begin(), cands.end(), [&](const ScanShape& c) {
                    return c.nw == t.nw && c.lc == t.lc && c.staged == t.staged && c.dense == t.dense;
                }))
                shape = t;
            tuned = true;
        }
    }
    const bool big = static_cast<long long>(nq) * P >= 4 * 148 * 256;
    if (!tuned && cands.size() > 1 && big && !s.capture) {
        shape = tune_scan(cands, a, v, qtab_len, st);
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tuned[key] = shape;
    }
    g_last_shape.store(shape.nw * 1000 + shape.lc * 10 + (shape.staged ? 1 : shape.dense ? 2 : 0));
    run_scan(shape, a, v, qtab_len, st);
    if (!direct) merge_candidates(ckey.get(), cslot.get(), nq, nchunks, kp, out_key, out_slot, st);
}

void nearest_lists(const IvfView& v, const IvfSearchArgs& s, int nq, int P, uint32_t* probe, float* pdist,
                   cudaStream_t st) {
    if (nq == 0) return;
    // exact pair scores, then the P nearest lists per query by (score, list),
    // compared as the reference's heap of (float, uint16_t) pairs does: -0 == +0
    auto exact_coarse = [&](const float* qs, int n, uint32_t* pr, float* pd) {
        DevBuf<float> scores(static_cast<size_t>(n) * v.nlist, st);
        pair_scores(qs, n, v.centroids, v.nlist, v.dim, v.ip_metric, scores.get(), v.nlist, st);
        select_rows(scores.get(), v.nlist, n, v.nlist, P, pr, pd, st, nullptr, nullptr, 0, true);
    };
    // batches of at most one query per SM (and captured ones) read nothing
    // back mid-search: their recheck holds every list, so none is redone
    const bool no_readback = s.d_err && (s.capture || nq <= s.sm_count);
    if (!use_tensor_coarse(nq, v.nlist, v.dim) ||
        !coarse_mm_supported(v.nlist, v.dim, P, v.cent_f16 != nullptr, no_readback)) {
        exact_coarse(s.q, nq, probe, pdist);
        return;
    }
    std::vector<int> redo;
    coarse_probes_mm(v, s.q, nq, P, probe, pdist, redo, st, no_readback ? s.d_err + 2 : nullptr);
    if (!s.capture) count_tensor_coarse(nq, static_cast<int64_t>(redo.size()));
    if (redo.empty()) return;
    // queries with too many near-ties: the exact path, results copied into place
    const size_t m = redo.size();
    std::vector<uint32_t> hidx(redo.begin(), redo.end());
    DevBuf<uint32_t> idx(m, st);
    QG_CUDA(cudaMemcpyAsync(idx.get(), hidx.data(), m * 4, cudaMemcpyHostToDevice, st));
    DevBuf<float> qs(m * v.dim, st);
    gather_rows(s.q, idx.get(), m, v.dim, qs.get(), st);
    DevBuf<uint32_t> pr(m * P, st);
    DevBuf<float> pd(m * P, st);
    exact_coarse(qs.get(), static_cast<int>(m), pr.get(), pd.get());
    for (size_t j = 0; j < m; ++j) {
        QG_CUDA(cudaMemcpyAsync(probe + static_cast<size_t>(redo[j]) * P, pr.get() + j * P, P * 4,
                                cudaMemcpyDeviceToDevice, st));
        QG_CUDA(cudaMemcpyAsync(pdist + static_cast<size_t>(redo[j]) * P, pd.get() + j * P, P * 4,
                                cudaMemcpyDeviceToDevice, st));
    }
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
        // the nearest lists ranked, then each query's own probe count (reference src/ivf_index.cpp:501-521)
        P = filtered_probes(v, s, probe, pdist, nprobe_q, st);
        probes_of = nprobe_q.get();
    } else {
        probe.alloc(static_cast<size_t>(nq) * P, st);
        pdist.alloc(static_cast<size_t>(nq) * P, st);
        nearest_lists(v, s, nq, P, probe.get(), pdist.get(), st);
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

    const bool per_query = s.pq.k || s.pq.kp || s.pq.nprobe;
    if (tensor_scan_applies(v, s, P, per_query)) {
        // wave 0: the first F probes of every query, query-major; wave 1 on the tensor cores
        const int F = tensor_scan_first(P);
        DevBuf<int> first(nq, st);
        fill_i32(first.get(), nq, F, st);
        DevBuf<uint64_t> key0(static_cast<size_t>(nq) * kp, st);
        DevBuf<uint32_t> slot0(static_cast<size_t>(nq) * kp, st);
        scan_query_major(v, s, nq, P, F, probe.get(), pterm.get(), qC.get(), qlut.get(), qscale.get(), qoffset.get(),
                         s.q, first.get(), key0.get(), slot0.get(), st);
        std::vector<int> redo;
        tensor_scan_candidates(v, nq, P, kp, probe.get(), pterm.get(), qC.get(), key0.get(), out_key, out_slot, redo,
                               s.d_err, st);
        if (!redo.empty()) {
            // queries whose candidates overflowed: the query-major scan over all their probes
            const size_t r = redo.size();
            std::vector<uint32_t> hidx(redo.begin(), redo.end());
            DevBuf<uint32_t> idx(r, st);
            QG_CUDA(cudaMemcpyAsync(idx.get(), hidx.data(), r * 4, cudaMemcpyHostToDevice, st));
            DevBuf<uint32_t> pr(r * P, st);
            DevBuf<float> pt(r * P, st), qc(r * v.m * 16, st);
            gather_rows(reinterpret_cast<const float*>(probe.get()), idx.get(), r, P, reinterpret_cast<float*>(pr.get()),
                        st);
            gather_rows(pterm.get(), idx.get(), r, P, pt.get(), st);
            gather_rows(qC.get(), idx.get(), r, v.m * 16, qc.get(), st);
            DevBuf<uint64_t> rk(r * kp, st);
            DevBuf<uint32_t> rs(r * kp, st);
            IvfSearchArgs sr = s;   // (an unfiltered batch of uniform settings, re-indexed)
            sr.pq = PerQuery{};
            sr.nq = static_cast<int>(r);
            scan_query_major(v, sr, static_cast<int>(r), P, P, pr.get(), pt.get(), qc.get(), nullptr, nullptr, nullptr,
                             nullptr, nullptr, rk.get(), rs.get(), st);
            for (size_t j = 0; j < r; ++j) {
                QG_CUDA(cudaMemcpyAsync(out_key + static_cast<size_t>(redo[j]) * kp, rk.get() + j * kp, kp * 8,
                                        cudaMemcpyDeviceToDevice, st));
                QG_CUDA(cudaMemcpyAsync(out_slot + static_cast<size_t>(redo[j]) * kp, rs.get() + j * kp, kp * 4,
                                        cudaMemcpyDeviceToDevice, st));
            }
            QG_CUDA(cudaStreamSynchronize(st));   // the index buffers above outlive their copies
        }
        return;
    }
    scan_query_major(v, s, nq, P, P, probe.get(), pterm.get(), qC.get(), qlut.get(), qscale.get(), qoffset.get(), s.q,
                     probes_of, out_key, out_slot, st);
}

} // namespace qg
