// The fast-scan on the tensor cores, list-major (reference src/ivf_index.cpp:421-641
// and src/fast_scan.cpp:256-338 compute the same sums one query at a time).
//
// A fast-scan sum is a lookup: sum(v, q) = sum_s LUT_q[s][code(v, s)]. Written
// as a product it is one-hot(v) . LUT_q over K = 16 m bytes, where one-hot(v)
// has a 1 at byte 16 s + code(v, s). So the sums of a list's vectors against
// every query that probes the list are one integer GEMM:
//
//     D[vector, query] = OneHot[vector, K] x LUT[query, K]^T      (u8 x u8 -> s32)
//
// exact in 32-bit integers (entries <= 63, so sums <= 63 m), the same
// numbers the lookups give. A large batch probes each list from hundreds of
// queries, which fills the GEMM's N dimension.
//
// The search runs in two waves. Wave 0 scans each query's first F probes with
// the query-major kernel (qg_scan.cu) and yields its k' best keys there; the
// k'-th of them bounds the query's final k'-th key from above. Wave 1 covers
// the remaining probes list by list:
//
//   1. pairs (query, probe) whose list cannot hold a key under the bound are
//      dropped by a lower bound on the LUT's zero-sum distance (row minima of
//      B and C, the same summation order as the LUT's offset, so the bound
//      never exceeds it);
//   2. the other pairs are grouped by list (stable), and cut into units of up
//      to kTsQ queries of one list;
//   3. k_tscan, persistent, takes units: its 16 warps round the unit's LUTs
//      (B[list] + C[query] + A on row 0, as build_quantize_lut does) straight
//      into the MMA's B operand, then for each 128-vector tile of the list
//      expand the 4-bit codes into the one-hot A operand, one thread issues
//      tcgen05.mma kind::i8 into TMEM, and the warps read the sums back with
//      tcgen05.ld and append every key under its query's bound;
//   4. per query, wave 0's k' keys and wave 1's candidates are cut to the k'
//      smallest and sorted.
//
// Keys are those of the query-major kernel, key(dist) << 32 | push index, the
// push index being the vector's position in the query's probe sequence, so
// the k' kept are exactly those the reference's TopK keeps. Queries whose
// candidates outgrow their buffer are redone by the query-major kernel.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_search.h"
#include "qg_sm100.cuh"
#include "qg_train.h"

#include <algorithm>
#include <atomic>

namespace qg {

namespace {

constexpr int kTsQ = 64;          // queries per unit: the MMA's N
constexpr int kTsV = 128;         // vectors per tile: the MMA's M (TMEM lanes)
constexpr int kTsWarps = 16;
constexpr int kTsThreads = kTsWarps * 32;
constexpr int kTsMaxM = 64;       // subspaces supported (K = 16 * 64 bytes at most)
constexpr uint32_t kTmemCols = 64;
constexpr int kTsFirst = 16;      // probes per query in wave 0

std::atomic<int> g_tensor_scan{1};   // 0 never, 1 when it pays, 2 whenever supported
std::atomic<long long> g_tscan_calls{0}, g_tscan_redone{0};

struct TScanArgs {
    IvfView v;
    int P, F, m8;              // probes per query, the first F scanned by wave 0, m rounded up to 8
    const uint32_t* probe;     // nq * P
    const float* pterm;        // nq * P: A terms
    const uint32_t* push;      // nq * P: vectors of the query's probes before this one
    const float* qC;           // nq * m * 16
    const uint64_t* bound;     // nq: upper bound on the query's k'-th key (~0: none)
    const uint32_t* members;   // wave-1 pairs grouped by list
    const uint32_t* units;     // per unit: list, first member, count
    const uint32_t* nunits;    // (device) number of units
    int* work;                 // next unit (zero at launch)
    uint64_t* cand;            // nq * cap candidate keys
    uint32_t* ccount;          // nq
    uint32_t cap;
    int* err;                  // [2]: a tensor-core wait ran out
    unsigned long long* stats; // kTsStats counters of this search
};

// Work counters of the tensor-core scan (summed over searches, for tuning):
// units, (unit, vector tile) steps, LUTs rounded, LUTs skipped as hopeless,
// candidate keys appended, wave-1 pairs, pairs left after the prefilter.
enum { kStUnits, kStTiles, kStLutLive, kStLutDead, kStCand, kStPairs, kStPairsKept, kTsStats };
std::atomic<long long> g_tscan_stat[kTsStats];

// Candidate keys a query may collect in wave 1 before it is redone by the
// query-major kernel.
uint32_t tscan_cap(int kp) { return static_cast<uint32_t>(std::min(16384, std::max(2048, 32 * kp))); }

size_t tscan_smem(int m, int m8) {
    const size_t K = static_cast<size_t>(16) * m8;
    size_t b = 1024;                                  // alignment slack for the operand tiles
    b += kTsV * K + kTsQ * K;                         // one-hot tile, LUT tile
    b += static_cast<size_t>(m) * 16 * 4;             // the list's B rows
    b += static_cast<size_t>(kTsWarps) * m * 4;       // per-warp row minima
    b += kTsQ * (4 * 6 + 8);                          // per-query slots
    b += 64;                                          // mbarrier, TMEM address
    return b;
}

// A one-hot 16-byte chunk: byte `code` set to 1.
__device__ __forceinline__ uint4 one_hot(uint32_t code) {
    const uint32_t val = 1u << ((code & 3u) * 8);
    const uint32_t w = code >> 2;
    return make_uint4(w == 0 ? val : 0u, w == 1 ? val : 0u, w == 2 ? val : 0u, w == 3 ? val : 0u);
}

// Byte offset of 16-byte chunk `s` of row `r` in a K-major tile of `rows`
// rows, 128-byte swizzle (the layout TMA's SWIZZLE_128B writes): K atoms of
// 128 bytes are rows * 128 bytes apart; within an atom chunk c of row r sits
// at c ^ (r % 8).
__device__ __forceinline__ uint32_t sw_chunk(int rows, int r, int s) {
    return static_cast<uint32_t>((s >> 3) * rows * 128 + r * 128 + (((s & 7) ^ (r & 7)) << 4));
}

__global__ void __launch_bounds__(kTsThreads, 1) k_tscan(TScanArgs a) {
    using namespace sm100;
    extern __shared__ uint8_t smraw[];
    const IvfView& v = a.v;
    const int m = v.m, m8 = a.m8, K = 16 * m8;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t* tiles = smraw + ((1024 - (smem_u32(smraw) & 1023)) & 1023);
    uint8_t* sA = tiles;                          // kTsV x K one-hot
    uint8_t* sB = sA + static_cast<size_t>(kTsV) * K;   // kTsQ x K LUTs
    float* blist = reinterpret_cast<float*>(sB + static_cast<size_t>(kTsQ) * K);
    float* rmin = blist + m * 16 + warp * m;
    uint32_t* s_q = reinterpret_cast<uint32_t*>(blist + m * 16 + kTsWarps * m);
    uint32_t* s_push = s_q + kTsQ;
    int* s_smax = reinterpret_cast<int*>(s_push + kTsQ);
    float* s_scale = reinterpret_cast<float*>(s_smax + kTsQ);
    float* s_offset = s_scale + kTsQ;
    float* s_aterm = s_offset + kTsQ;
    uint64_t* s_bound = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(s_aterm + kTsQ) + 7) & ~static_cast<uintptr_t>(7));
    uint64_t* mbar = s_bound + kTsQ;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    __shared__ int s_unit;
    __shared__ int s_abort;

    if (tid == 0) {
        mbar_init(mbar, 1);
        s_abort = 0;
        fence_barrier_init();
    }
    if (warp == 0) tmem_alloc(tslot, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = idesc_u8_s32(kTsV, kTsQ);
    const int span = a.P - a.F;
    uint32_t phase = 0;
    bool failed = false;   // a tensor-core wait ran out (the same in every thread)
    const uint32_t tot_units = *a.nunits;

    for (;;) {
        __syncthreads();   // the previous unit is done with every shared array
        if (tid == 0) {
            const int u = atomicAdd(a.work, 1);
            s_unit = static_cast<uint32_t>(u) < tot_units ? u : -1;
        }
        __syncthreads();
        const int unit = s_unit;
        if (unit < 0) break;
        const uint32_t l = a.units[3 * unit], first = a.units[3 * unit + 1], cnt = a.units[3 * unit + 2];
        if (tid == 0) atomicAdd(a.stats + kStUnits, 1ull);
        for (int j = tid; j < kTsQ; j += kTsThreads) {
            if (j < static_cast<int>(cnt)) {
                const uint32_t pair = a.members[first + j];
                const uint32_t q = pair / span, p = a.F + pair % span;
                s_q[j] = q;
                s_push[j] = a.push[static_cast<size_t>(q) * a.P + p];
                s_aterm[j] = a.pterm[static_cast<size_t>(q) * a.P + p];
                s_bound[j] = a.bound[q];
            } else {
                s_q[j] = 0xFFFFFFFFu;
            }
            s_smax[j] = -1;
        }
        for (int t = tid; t < m * 16; t += kTsThreads) blist[t] = v.B[static_cast<size_t>(l) * m * 16 + t];
        __syncthreads();

        // ---- LUTs of the unit's queries, rounded into the B operand ----
        for (int j = warp; j < static_cast<int>(cnt); j += kTsWarps) {
            const uint32_t q = s_q[j];
            const float A = s_aterm[j];
            const uint32_t thr_hi = static_cast<uint32_t>(s_bound[j] >> 32);
            const float* C = a.qC + static_cast<size_t>(q) * m * 16;
            auto row = [&](int r, float* o) {
                const float4* b4 = reinterpret_cast<const float4*>(blist + r * 16);
                const float4* c4 = reinterpret_cast<const float4*>(C + r * 16);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 bb = b4[u], cc = __ldg(c4 + u);
                    const float2 lo = __fadd2_rn(make_float2(bb.x, bb.y), make_float2(cc.x, cc.y));
                    const float2 hi = __fadd2_rn(make_float2(bb.z, bb.w), make_float2(cc.z, cc.w));
                    o[4 * u + 0] = lo.x;
                    o[4 * u + 1] = lo.y;
                    o[4 * u + 2] = hi.x;
                    o[4 * u + 3] = hi.y;
                }
                if (r == 0) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) o[e] = __fadd_rn(o[e], A);
                }
            };
            // each lane holds its rows (lane, lane + 32; m <= 64) between the range
            // pass and the rounding pass
            float ta[16], tb[16];
            const int ra = lane, rb = lane + 32;
            float widest = 0.0f;
            auto ranges = [&](int r, const float* t) {
                float lo = t[0], hi = t[0];
#pragma unroll
                for (int e = 1; e < 16; ++e) {
                    lo = fminf(lo, t[e]);
                    hi = fmaxf(hi, t[e]);
                }
                rmin[r] = lo;
                const float w = __fsub_rn(hi, lo);
                widest = widest < w ? w : widest;
            };
            if (ra < m) {
                row(ra, ta);
                ranges(ra, ta);
            }
            if (rb < m) {
                row(rb, tb);
                ranges(rb, tb);
            }
            widest = warp_max(widest);
            __syncwarp();
            float part = 0.0f;
            if (lane < 4)
                for (int r = lane; r < m; r += 4) part = __fadd_rn(part, rmin[r]);
            const float p0 = __shfl_sync(0xffffffffu, part, 0), p1 = __shfl_sync(0xffffffffu, part, 1);
            const float p2 = __shfl_sync(0xffffffffu, part, 2), p3 = __shfl_sync(0xffffffffu, part, 3);
            const float offset = __fadd_rn(__fadd_rn(p0, p1), __fadd_rn(p2, p3));
            const float scale = widest > 0.0f ? __fdiv_rn(static_cast<float>(kLutMax), widest) : 1.0f;
            // a list none of whose sums can reach under the bound: no LUT, no candidates
            const bool live = thr_hi == 0xFFFFFFFFu || float_key(fs_dist0(scale, offset)) <= thr_hi;
            if (live) {
                const uint4 z = make_uint4(0, 0, 0, 0);
                if (ra < m8) *reinterpret_cast<uint4*>(sB + sw_chunk(kTsQ, j, ra)) = ra < m ? round_row(ta, rmin[ra], scale) : z;
                if (rb < m8) *reinterpret_cast<uint4*>(sB + sw_chunk(kTsQ, j, rb)) = rb < m ? round_row(tb, rmin[rb], scale) : z;
            }
            if (lane == 0) {
                s_scale[j] = scale;
                s_offset[j] = offset;
                s_smax[j] = live ? sum_limit_fast(thr_hi, scale, offset) : -1;
                atomicAdd(a.stats + (live ? kStLutLive : kStLutDead), 1ull);
            }
            __syncwarp();
        }

        // ---- the list's vectors, 128 at a time ----
        const uint32_t sb0 = v.sb_off[l], nsb = v.sb_off[l + 1] - sb0, size = v.list_size[l];
        const int ntiles = static_cast<int>((nsb + 1) / 2);
        const int m_pad = v.m_pad, ngroups = m8 / 4;
        for (int t = 0; t < ntiles; ++t) {
            // one-hot rows: item (superblock half h, octet row r, subspace group g, component c)
            const int items = 2 * 8 * ngroups * 4;
            for (int it = tid; it < items; it += kTsThreads) {
                const int c = it & 3, g = (it >> 2) % ngroups, hr = (it >> 2) / ngroups;
                const int h = hr >> 3, r = hr & 7;
                const uint32_t sbi = 2u * t + h;
                const int s = 4 * g + c;
                uint32_t word = 0;
                const bool present = sbi < nsb && s < m;
                if (present) {
                    const uint4 w4 = __ldg(v.codes + (static_cast<size_t>(sb0) + sbi) * (2 * m_pad) + g * 8 + r);
                    word = c == 0 ? w4.x : c == 1 ? w4.y : c == 2 ? w4.z : w4.w;
                }
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int row_v = h * 64 + 8 * r + i;
                    const uint4 chunk = present ? one_hot((word >> (4 * i)) & 15u) : make_uint4(0, 0, 0, 0);
                    *reinterpret_cast<uint4*>(sA + sw_chunk(kTsV, row_v, s)) = chunk;
                }
            }
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                atomicAdd(a.stats + kStTiles, 1ull);
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
                const int ksteps = K / 32;
                for (int ks = 0; ks < ksteps; ++ks) {
                    const int kb = ks >> 2, kin = ks & 3;
                    mma_u8(tmem, sw128_desc(a0 + kb * kTsV * 128 + kin * 32), sw128_desc(b0 + kb * kTsQ * 128 + kin * 32),
                           idesc, ks > 0);
                }
                mma_commit(mbar);
            }
            const bool ok = mbar_wait(mbar, phase, &s_abort);
            phase ^= 1u;
            if (!__syncthreads_and(ok)) {   // (block-uniform)
                failed = true;
                if (tid == 0) atomicExch(a.err, 2);
                break;
            }
            tc_fence_after();
            // ---- sums back from TMEM: warp w reads lanes 32 (w % 4) .., columns 16 (w / 4) .. ----
            const int quad = warp & 3, cb = warp >> 2;
            uint32_t sums[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(quad * 32) << 16) + static_cast<uint32_t>(cb * 16), sums);
            const uint32_t pos = static_cast<uint32_t>(t) * kTsV + quad * 32 + lane;
            const bool valid = pos < size;
            const unsigned below = (1u << lane) - 1u;
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int col = cb * 16 + e;
                const int smax = s_smax[col];
                bool pass = valid && smax >= 0 && static_cast<int>(sums[e]) <= smax;
                uint64_t key = 0;
                if (pass) {
                    const float dist = fs_dist(sums[e], s_scale[col], s_offset[col]);
                    key = (static_cast<uint64_t>(float_key(dist)) << 32) | (s_push[col] + pos);
                    pass = key < s_bound[col];
                    if (pass && v.deleted) {
                        const uint32_t slot = v.ids[(static_cast<size_t>(sb0) + pos / kSuperBlock) * kSuperBlock +
                                                    pos % kSuperBlock];
                        pass = !((v.deleted[slot >> 6] >> (slot & 63)) & 1ull);
                    }
                }
                const unsigned mask = __ballot_sync(0xffffffffu, pass);
                if (mask) {
                    const uint32_t q = s_q[col];
                    const int lead = __ffs(mask) - 1;
                    uint32_t at = 0;
                    if (lane == lead) {
                        at = atomicAdd(a.ccount + q, static_cast<uint32_t>(__popc(mask)));
                        atomicAdd(a.stats + kStCand, static_cast<unsigned long long>(__popc(mask)));
                    }
                    at = __shfl_sync(0xffffffffu, at, lead) + __popc(mask & below);
                    if (pass && at < a.cap) a.cand[static_cast<size_t>(q) * a.cap + at] = key;
                }
            }
            tc_fence_before();
            __syncthreads();   // TMEM and the one-hot tile are free for the next tile
        }
        if (failed) break;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, kTmemCols);
    }
}

// Per query: the push offset of every probe (vectors of the probes before
// it, in probe order). Warp per query.
__global__ void k_push_offsets(const uint32_t* __restrict__ probe, const uint32_t* __restrict__ list_size, int nq,
                               int P, uint32_t* __restrict__ push) {
    const int q = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (q >= nq) return;
    uint32_t run = 0;
    for (int b = 0; b < P; b += 32) {
        const int p = b + lane;
        const uint32_t sz = p < P ? list_size[probe[static_cast<size_t>(q) * P + p]] : 0u;
        uint32_t inc = sz;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (p < P) push[static_cast<size_t>(q) * P + p] = run + inc - sz;
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
}

// Row minima: out[i * m + s] = min over the 16 entries of row s of table i.
__global__ void k_row_minima(const float* __restrict__ t, size_t n, int m, float* __restrict__ out) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n * m) return;
    const float4* r = reinterpret_cast<const float4*>(t + i * 16);
    float lo = r[0].x;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const float4 x = r[u];
        lo = fminf(lo, fminf(fminf(x.x, x.y), fminf(x.z, x.w)));
    }
    out[i] = lo;
}

// Wave-1 pairs: label = the probe's list, or nlist (left out) when the
// list holds no superblocks here or cannot hold a key under the query's
// bound. The test: each LUT row's minimum is at least fl(minB + minC)
// (+ A on row 0: fl(fl(B + C) + A) is monotone in B + C), and the offset sums
// the row minima in the same order with monotone float adds, so the bound
// below never exceeds the LUT's zero-sum distance.
__global__ void k_pair_labels(IvfView v, int nq, int P, int F, const uint32_t* __restrict__ probe,
                              const float* __restrict__ pterm, const float* __restrict__ minB,
                              const float* __restrict__ minC, const uint64_t* __restrict__ bound,
                              uint32_t* __restrict__ label) {
    const int span = P - F;
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(nq) * span) return;
    const size_t q = t / span;
    const int p = F + static_cast<int>(t % span);
    const uint32_t l = probe[q * P + p];
    uint32_t out = l;
    if (v.sb_off[l + 1] == v.sb_off[l]) {
        out = static_cast<uint32_t>(v.nlist);
    } else {
        const uint32_t thr_hi = static_cast<uint32_t>(bound[q] >> 32);
        if (thr_hi != 0xFFFFFFFFu) {
            const float* mb = minB + static_cast<size_t>(l) * v.m;
            const float* mc = minC + q * v.m;
            float part[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (int r = 0; r < v.m; ++r) {
                float lo = __fadd_rn(mb[r], mc[r]);
                if (r == 0) lo = __fadd_rn(lo, pterm[q * P + p]);
                part[r & 3] = __fadd_rn(part[r & 3], lo);
            }
            const float off = __fadd_rn(__fadd_rn(part[0], part[1]), __fadd_rn(part[2], part[3]));
            if (float_key(__fadd_rn(0.0f, off)) > thr_hi) out = static_cast<uint32_t>(v.nlist);
        }
    }
    label[t] = out;
}

// Units: per list, ceil(members / kTsQ) of them.
__global__ void k_unit_counts(const uint32_t* __restrict__ off, int nlist, uint32_t* __restrict__ ucount) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < nlist) ucount[l] = (off[l + 1] - off[l] + kTsQ - 1) / kTsQ;
}

__global__ void k_unit_table(const uint32_t* __restrict__ off, const uint32_t* __restrict__ ubase, int nlist,
                             uint32_t* __restrict__ units, uint32_t* __restrict__ nunits) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlist) return;
    const uint32_t c = off[l + 1] - off[l], nu = (c + kTsQ - 1) / kTsQ, b = ubase[l];
    for (uint32_t u = 0; u < nu; ++u) {
        units[3 * (b + u) + 0] = static_cast<uint32_t>(l);
        units[3 * (b + u) + 1] = off[l] + u * kTsQ;
        units[3 * (b + u) + 2] = min(static_cast<uint32_t>(kTsQ), c - u * kTsQ);
    }
    if (l == nlist - 1) *nunits = b + nu;
}

__global__ void k_wave0_bounds(const uint64_t* __restrict__ key0, int nq, int kp, uint64_t* __restrict__ bound) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nq) bound[q] = key0[static_cast<size_t>(q) * kp + kp - 1];
}

// Per query: wave 0's k' keys and wave 1's candidates cut to the k'
// smallest, sorted, with their slots (the push index located among the
// query's probes). Queries whose candidates overflowed are listed in redo.
__global__ void __launch_bounds__(256) k_tscan_final(IvfView v, int P, const uint32_t* __restrict__ probe,
                                                     const uint32_t* __restrict__ push, const uint64_t* __restrict__ key0,
                                                     const uint64_t* __restrict__ cand,
                                                     const uint32_t* __restrict__ ccount, uint32_t cap, int kp,
                                                     uint64_t* __restrict__ out_key, uint32_t* __restrict__ out_slot,
                                                     uint32_t* __restrict__ redo, uint32_t* __restrict__ nredo) {
    extern __shared__ __align__(16) uint8_t sm[];
    __shared__ int hist[256];
    const int q = blockIdx.x;
    uint64_t* buf = reinterpret_cast<uint64_t*>(sm);
    const uint32_t c = ccount[q];
    uint64_t* ok = out_key + static_cast<size_t>(q) * kp;
    uint32_t* os = out_slot + static_cast<size_t>(q) * kp;
    if (c > cap) {
        if (threadIdx.x == 0) redo[atomicAdd(nredo, 1u)] = static_cast<uint32_t>(q);
        return;
    }
    const int n = kp + static_cast<int>(c);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        buf[i] = i < kp ? key0[static_cast<size_t>(q) * kp + i] : cand[static_cast<size_t>(q) * cap + (i - kp)];
    __syncthreads();
    if (n > kp) {
        if (threadIdx.x < 32) warp_select_keep(buf, n, kp, hist);
        __syncthreads();
    }
    const int ns = next_pow2(kp < 2 ? 2 : kp);
    for (int i = kp + threadIdx.x; i < ns; i += blockDim.x) buf[i] = ~0ull;
    __syncthreads();
    bitonic_sort_keys(buf, ns);
    const uint32_t* pq = push + static_cast<size_t>(q) * P;
    for (int i = threadIdx.x; i < kp; i += blockDim.x) {
        const uint64_t key = buf[i];
        ok[i] = key;
        if (key == ~0ull) {
            os[i] = 0xFFFFFFFFu;
            continue;
        }
        const uint32_t ps = static_cast<uint32_t>(key);
        int lo = 0, hi = P - 1;   // the last probe whose push offset is <= ps
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pq[mid] <= ps) lo = mid;
            else hi = mid - 1;
        }
        // (empty lists share their offset with the next probe: the last such probe holds ps)
        const uint32_t l = probe[static_cast<size_t>(q) * P + lo], pos = ps - pq[lo];
        os[i] = v.ids[(static_cast<size_t>(v.sb_off[l]) + pos / kSuperBlock) * kSuperBlock + pos % kSuperBlock];
    }
}

__global__ void k_fill_i32(int* a, int n, int v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

} // namespace

void fill_i32(int* a, int n, int value, cudaStream_t st) {
    if (n <= 0) return;
    k_fill_i32<<<static_cast<unsigned>(ceil_div(n, 256)), 256, 0, st>>>(a, n, value);
    QG_LAUNCH_CHECK();
}

void set_tensor_scan(int mode) { g_tensor_scan.store(mode); }
int tensor_scan() { return g_tensor_scan.load(); }
void tensor_scan_counts(int64_t* calls, int64_t* redone) {
    if (calls) *calls = g_tscan_calls.load();
    if (redone) *redone = g_tscan_redone.load();
}

bool tensor_scan_stat(const std::string& name, int64_t* value) {
    static const char* names[kTsStats] = {"units", "tiles", "luts_live", "luts_hopeless", "candidates", "pairs",
                                          "pairs_kept"};
    for (int i = 0; i < kTsStats; ++i)
        if (name == names[i]) {
            *value = g_tscan_stat[i].load();
            return true;
        }
    return false;
}

int tensor_scan_first(int P) { return std::min(P, kTsFirst); }

static int kp_of(const IvfSearchArgs& s) { return s.kp; }

bool tensor_scan_applies(const IvfView& v, const IvfSearchArgs& s, int P, bool per_query) {
    const int mode = g_tensor_scan.load();
    if (mode == 0 || s.capture || per_query || s.filter || s.any_filter) return false;
    if (v.mode != kModeL2 || v.m > kTsMaxM || v.m < 1) return false;
    if (tscan_smem(v.m, (v.m + 7) & ~7) > 227 * 1024) return false;
    const int F = std::min(P, kTsFirst);
    if (P - F < 1) return false;
    if (static_cast<size_t>(kp_of(s) + tscan_cap(kp_of(s))) * 8 > 200 * 1024) return false;   // the final cut's keys
    // Mode 1 ("when it pays") does not pick it: measured on the 1.2M x 100
    // angular batch (10,000 queries, nprobe 256, k' 200) the two waves took
    // 9.8 ms against 6.9 ms for the query-major kernel alone. Per (unit, tile)
    // step the one-hot expansion, the barriers around the MMA and the L2
    // latency of the LUT inputs keep 16 warps at 28 % issue, and 56 % of the
    // LUTs turn out hopeless only after their range pass.
    return mode == 2;
}

// Wave 0 by `scan0` (the query-major kernel on each query's first F probes,
// results sorted into key0 / slot0 per query), then wave 1 here. The outputs
// are the k' best keys and slots of each query, sorted; queries whose
// candidates overflow are listed for the caller to redo.
void tensor_scan_candidates(const IvfView& v, int nq, int P, int kp, const uint32_t* probe, const float* pterm,
                            const float* qC, const uint64_t* key0, uint64_t* out_key, uint32_t* out_slot,
                            std::vector<int>& redo_q, int* d_err, cudaStream_t st) {
    redo_q.clear();
    g_tscan_calls.fetch_add(1);
    const int F = std::min(P, kTsFirst), span = P - F, m = v.m, m8 = (m + 7) & ~7;
    const size_t npairs = static_cast<size_t>(nq) * span;
    require(npairs < (size_t{1} << 31), "too many (query, list) pairs for the tensor-core scan", kUnsupported);
    DevBuf<uint32_t> push(static_cast<size_t>(nq) * P, st);
    KernelTimer prep_timer("tscan_prep", st);   // push offsets .. unit table
    k_push_offsets<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * 32, 256)), 256, 0, st>>>(
        probe, v.list_size, nq, P, push.get());
    QG_LAUNCH_CHECK();
    DevBuf<uint64_t> bound(nq, st);
    k_wave0_bounds<<<static_cast<unsigned>(ceil_div(nq, 256)), 256, 0, st>>>(key0, nq, kp, bound.get());
    QG_LAUNCH_CHECK();
    DevBuf<float> minB(static_cast<size_t>(v.nlist) * m, st), minC(static_cast<size_t>(nq) * m, st);
    k_row_minima<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(v.nlist) * m, 256)), 256, 0, st>>>(
        v.B, v.nlist, m, minB.get());
    QG_LAUNCH_CHECK();
    k_row_minima<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nq) * m, 256)), 256, 0, st>>>(qC, nq, m,
                                                                                                    minC.get());
    QG_LAUNCH_CHECK();
    DevBuf<uint32_t> label(npairs, st), members(npairs, st), off(static_cast<size_t>(v.nlist) + 2, st);
    k_pair_labels<<<static_cast<unsigned>(ceil_div(npairs, 256)), 256, 0, st>>>(
        v, nq, P, F, probe, pterm, minB.get(), minC.get(), bound.get(), label.get());
    QG_LAUNCH_CHECK();
    minB.release();
    minC.release();
    group_by_label(label.get(), npairs, v.nlist + 1, 1, members.get(), off.get(), st);
    label.release();
    DevBuf<uint32_t> ubase(v.nlist, st), nunits(1, st);
    k_unit_counts<<<static_cast<unsigned>(ceil_div(v.nlist, 256)), 256, 0, st>>>(off.get(), v.nlist, ubase.get());
    QG_LAUNCH_CHECK();
    exclusive_scan_u32(ubase.get(), v.nlist, st);
    // at most ceil(pairs / kTsQ) + nlist units
    const size_t max_units = npairs / kTsQ + v.nlist + 1;
    DevBuf<uint32_t> units(3 * max_units, st);
    k_unit_table<<<static_cast<unsigned>(ceil_div(v.nlist, 256)), 256, 0, st>>>(off.get(), ubase.get(), v.nlist,
                                                                                units.get(), nunits.get());
    QG_LAUNCH_CHECK();
    prep_timer.stop();

    const uint32_t cap = tscan_cap(kp);
    DevBuf<uint64_t> cand(static_cast<size_t>(nq) * cap, st);
    DevBuf<uint32_t> ccount(nq, st);
    QG_CUDA(cudaMemsetAsync(ccount.get(), 0, nq * sizeof(uint32_t), st));
    DevBuf<int> work(1, st);
    QG_CUDA(cudaMemsetAsync(work.get(), 0, sizeof(int), st));
    DevBuf<unsigned long long> stats(kTsStats, st);
    QG_CUDA(cudaMemsetAsync(stats.get(), 0, kTsStats * sizeof(unsigned long long), st));
    TScanArgs a{};
    a.v = v;
    a.P = P;
    a.F = F;
    a.m8 = m8;
    a.probe = probe;
    a.pterm = pterm;
    a.push = push.get();
    a.qC = qC;
    a.bound = bound.get();
    a.members = members.get();
    a.units = units.get();
    a.nunits = nunits.get();
    a.work = work.get();
    a.cand = cand.get();
    a.ccount = ccount.get();
    a.cap = cap;
    a.err = d_err;
    a.stats = stats.get();
    const size_t smem = tscan_smem(m, m8);
    allow_large_smem<k_tscan>();
    {
        KernelTimer kt("tscan", st);
        k_tscan<<<static_cast<unsigned>(sm_count()), kTsThreads, smem, st>>>(a);
        QG_LAUNCH_CHECK();
    }
    DevBuf<uint32_t> redo(nq, st), nredo(1, st);
    QG_CUDA(cudaMemsetAsync(nredo.get(), 0, sizeof(uint32_t), st));
    const size_t fsmem = static_cast<size_t>(kp + cap) * 8;
    if (fsmem > 48 * 1024) allow_large_smem<k_tscan_final>();
    {
        KernelTimer kt("tscan_final", st);
        k_tscan_final<<<static_cast<unsigned>(nq), 256, fsmem, st>>>(v, P, probe, push.get(), key0, cand.get(),
                                                                     ccount.get(), cap, kp, out_key, out_slot,
                                                                     redo.get(), nredo.get());
        QG_LAUNCH_CHECK();
    }
    uint32_t nr = 0, kept = 0;
    unsigned long long hs[kTsStats] = {};
    QG_CUDA(cudaMemcpyAsync(&nr, nredo.get(), sizeof(nr), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaMemcpyAsync(&kept, off.get() + v.nlist, sizeof(kept), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaMemcpyAsync(hs, stats.get(), sizeof(hs), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    hs[kStPairs] = npairs;
    hs[kStPairsKept] = kept;
    for (int i = 0; i < kTsStats; ++i) g_tscan_stat[i].fetch_add(static_cast<long long>(hs[i]));
    if (nr) {
        std::vector<uint32_t> h(nr);
        QG_CUDA(cudaMemcpyAsync(h.data(), redo.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        redo_q.assign(h.begin(), h.end());
        std::sort(redo_q.begin(), redo_q.end());
        g_tscan_redone.fetch_add(nr);
    }
}

} // namespace qg
