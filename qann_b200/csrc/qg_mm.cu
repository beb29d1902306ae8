// Exact top-k by a BF16 tensor-core filter and an FP32 recheck: flat search
// (reference src/flat_index.cpp:33-64), nearest-centroid assignment
// (reference src/kmeans.cpp:34-115) and any other "k smallest exact scores of
// each query over a set of rows", with results identical to the exact path.
//
// Why it is exact. Let s be a pair's exact score as the reference computes it
// (squared L2 or -dot in float, AVX2 order) and ŝ its tensor-core estimate
// from bf16-rounded inputs accumulated in FP32. Input rounding contributes at
// most (2u + u^2) sum|q_i x_i| (u = 2^-8), accumulation and the reference's
// own float rounding at most d 2^-19 of the same scale, and sum|q_i x_i| <=
// |q||x| <= (|q|^2 + |x|^2) / 2. So |ŝ - s| <= e = C (|q|^2 + |x|^2) for L2
// and C/2 (|q|^2 + |x|^2) for inner product, C = 2^-7 + 2^-14 + d 2^-19 (the
// 2^-14 absorbs the float rounding of the bound arithmetic itself). Each query
// keeps a running exact top-k; T, its k-th exact score, bounds the final
// k-th score from above. A row whose lower bound ŝ - e exceeds T cannot enter
// the top-k; every other row is rescored exactly and merged. The rows are
// taken in chunks of growing size so that T tightens between them.
//
// The filter kernel (k_mm_filter) is persistent and warp-specialised: warp 0
// loads 128-row query tiles and 256-row base tiles with TMA (128-byte swizzle,
// K-major bf16), warp 1 issues tcgen05.mma into one of two TMEM accumulators
// (128 lanes x 256 columns each), and 8 or 16 epilogue warps (the schedule
// autotuner's pick) read the accumulator with tcgen05.ld, form the lower
// bound with one FMA and append the rows that pass to the query's candidate
// list.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_sm100.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace qg {

namespace {

constexpr int BM = 128;         // queries per tile (TMEM lanes)
constexpr int BN = 256;         // base rows per tile (accumulator columns)
constexpr int KA = 64;          // bf16 elements per 128-byte swizzle row
constexpr int kStages = 2;      // base tile buffers
// epilogue warps: EPI / 4 per TMEM lane quadrant, each on BN / (EPI / 4) columns of a tile
// (8 or 16, picked per problem by the filter's autotuner)
template <int EPI>
constexpr int filter_threads() { return (2 + EPI) * 32; }
constexpr uint32_t kTmemCols = 2 * BN;
constexpr int kMaxKBlocks = 2;  // d <= 128

struct MmArgs {
    int nq;
    int n0, n1;          // base rows [n0, n1) of this launch
    int kblocks;         // 64-element K blocks of the padded rows
    int ksteps;          // 16-element MMA steps covering d
    int mtiles, ntiles;
    const float* xterm;  // per base row: its part of the lower bound
    const float* thr;    // per query: a row passes when fma(-mult, acc, xterm) <= thr
    float mult;
    const uint64_t* allow;   // base rows that may be returned, or null
    const uint64_t* deny;    // base rows that may not, or null
    uint32_t* cand_count;    // per query
    uint32_t* cand_row;      // per query, cap entries
    int cap;
    int* err;
    float* store;            // store mode: the raw products acc(q, row) at store[q * ld + row - n0], no filtering
    size_t ld;
    int f16;                 // operands are F16 (else BF16)
};

size_t filter_smem_bytes(int kblocks) {
    return 1024 + static_cast<size_t>(kblocks) * BM * 128 + static_cast<size_t>(kStages) * kblocks * BN * 128 + 256;
}

} // namespace

// Tile schedule: each CTA takes a contiguous range of tile indices, walked in
// groups of kGroupN base tiles; within a group the query tile changes every
// kGroupN tiles. A base tile thus comes from HBM once and from L2 for every
// later query tile, and the single-buffered query tile reloads only once
// per group.
constexpr int kGroupN = 8;
__device__ __forceinline__ void tile_coords(int t, int mtiles, int ntiles, int& mt, int& nt) {
    const int group = t / (mtiles * kGroupN);
    const int rem = t - group * mtiles * kGroupN;
    const int gsize = min(kGroupN, ntiles - group * kGroupN);
    mt = rem / gsize;
    nt = group * kGroupN + (rem - mt * gsize);
}

template <int EPI>
__global__ void __launch_bounds__(filter_threads<EPI>(), 1)
    k_mm_filter(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, MmArgs a) {
    static_assert(EPI == 8 || EPI == 16, "8 or 16 epilogue warps");
    using namespace sm100;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(16) float s_xt[EPI][32];   // epilogue: each warp's current run of row terms
    uint8_t* base = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const uint32_t a_bytes = static_cast<uint32_t>(a.kblocks) * BM * 128;
    const uint32_t b_bytes = static_cast<uint32_t>(a.kblocks) * BN * 128;
    uint8_t* sA = base;
    uint8_t* sB = base + a_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kStages * b_bytes);
    uint64_t* full_b = bars;        // [kStages] TMA -> MMA
    uint64_t* empty_b = bars + 2;   // [kStages] MMA -> TMA
    uint64_t* full_a = bars + 4;    // TMA -> MMA
    uint64_t* empty_a = bars + 5;   // MMA -> TMA
    uint64_t* tfull = bars + 6;     // [2] MMA -> epilogue
    uint64_t* tempty = bars + 8;    // [2] epilogue -> MMA
    uint64_t* mma_done = bars + 10; // teardown
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 11);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_b[s], 1);
            mbar_init(&empty_b[s], 1);
        }
        mbar_init(full_a, 1);
        mbar_init(empty_a, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI);
        }
        mbar_init(mma_done, 1);
        *abort = 0;
        fence_barrier_init();
    }
    if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int total = a.mtiles * a.ntiles;
    const int per = (total + gridDim.x - 1) / gridDim.x;   // this CTA's tiles: [t_begin, t_end)
    const int t_begin = min(total, blockIdx.x * per), t_end = min(total, t_begin + per);
    auto fail = [&] {
        *abort = 1;
        atomicExch(a.err, 2);
    };

    if (warp == 0) {
        if (lane == 0) {
            int it = 0, aloads = 0, cur_m = -1;
            for (int t = t_begin; t < t_end && !*abort; ++t) {
                int mt, nt;
                tile_coords(t, a.mtiles, a.ntiles, mt, nt);
                if (mt != cur_m) {
                    if (aloads > 0 && !mbar_wait(empty_a, (aloads - 1) & 1, abort)) {
                        fail();
                        break;
                    }
                    mbar_expect_tx(full_a, a_bytes);
                    for (int kb = 0; kb < a.kblocks; ++kb)
                        tma_load_2d(&tmA, sA + kb * BM * 128, full_a, kb * KA, mt * BM);
                    ++aloads;
                    cur_m = mt;
                }
                const int s = it % kStages;
                if (it >= kStages && !mbar_wait(&empty_b[s], ((it / kStages) - 1) & 1, abort)) {
                    fail();
                    break;
                }
                mbar_expect_tx(&full_b[s], b_bytes);
                for (int kb = 0; kb < a.kblocks; ++kb)
                    tma_load_2d(&tmB, sB + s * b_bytes + kb * BN * 128, &full_b[s], kb * KA, a.n0 + nt * BN);
                ++it;
            }
            // no copy may land after the CTA is gone: wait for the last load of each buffer
            volatile int never = 0;
            for (int s = 0; s < kStages && s < it; ++s) {
                const int last = it - 1 - ((it - 1 - s) % kStages);   // last use of stage s
                mbar_wait(&full_b[s], (last / kStages) & 1, &never);
            }
            if (aloads > 0) mbar_wait(full_a, (aloads - 1) & 1, &never);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = a.f16 ? idesc_f16_f32(BM, BN) : idesc_bf16_f32(BM, BN);
            int it = 0, aloads = 0, cur_m = -1, ti = 0;
            for (int t = t_begin; t < t_end && !*abort; ++t) {
                int mt, nt;
                tile_coords(t, a.mtiles, a.ntiles, mt, nt);
                (void)nt;
                if (mt != cur_m) {
                    if (cur_m >= 0) mma_commit(empty_a);   // the old query tile is free once its MMAs finish
                    if (!mbar_wait(full_a, aloads & 1, abort)) {
                        fail();
                        break;
                    }
                    ++aloads;
                    cur_m = mt;
                }
                const int acc = ti & 1;
                if (ti >= 2 && !mbar_wait(&tempty[acc], ((ti >> 1) - 1) & 1, abort)) {
                    fail();
                    break;
                }
                const int s = it % kStages;
                if (!mbar_wait(&full_b[s], (it / kStages) & 1, abort)) {
                    fail();
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB + s * b_bytes);
                for (int ks = 0; ks < a.ksteps; ++ks) {
                    const int kb = ks >> 2, kin = ks & 3;
                    mma_bf16(tmem + acc * BN, sw128_desc(a0 + kb * BM * 128 + kin * 32),
                             sw128_desc(b0 + kb * BN * 128 + kin * 32), idesc, ks > 0);
                }
                mma_commit(&empty_b[s]);
                mma_commit(&tfull[acc]);
                ++it;
                ++ti;
            }
            // every MMA done before TMEM is freed
            volatile int never = 0;
            mma_commit(mma_done);
            mbar_wait(mma_done, 0, &never);
        }
    } else {
        const int ew = warp - 2;      // 0..EPI-1
        const int quad = warp & 3;    // this warp's TMEM lanes: 32 * quad ..
        constexpr int kCols = BN / (EPI / 4);   // this warp's columns of a tile
        const int col0 = (ew >> 2) * kCols;
        const int row_in_tile = quad * 32 + lane;
        int ti = 0;
        for (int t = t_begin; t < t_end; ++t) {
            int mt, nt;
            tile_coords(t, a.mtiles, a.ntiles, mt, nt);
            const int acc = ti & 1;
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&tfull[acc], (ti >> 1) & 1, abort));
            if (!ok) {
                if (lane == 0) fail();
                break;
            }
            tc_fence_after();
            const int qi = mt * BM + row_in_tile;
            const bool live = qi < a.nq;
            const float thr = live && !a.store ? a.thr[qi] : 0.0f;
            for (int c = 0; c < kCols; c += 32) {
                uint32_t v[32];
                tmem_ld32(tmem + (static_cast<uint32_t>(quad * 32) << 16) + static_cast<uint32_t>(acc * BN + col0 + c),
                          v);
                const int r0 = a.n0 + nt * BN + col0 + c;   // base row of v[0]
                if (a.store) {
                    if (live) {
                        float* dst = a.store + static_cast<size_t>(qi) * a.ld + (r0 - a.n0);
                        if (r0 + 32 <= a.n1 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                            // a whole 32-column run: 16-byte stores, a quarter of the store instructions
#pragma unroll
                            for (int j = 0; j < 32; j += 4)
                                *reinterpret_cast<float4*>(dst + j) =
                                    make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (r0 + j < a.n1) dst[j] = __uint_as_float(v[j]);
                        }
                    }
                    continue;
                }
                // the run's row terms, staged for broadcast reads
                float* sx = s_xt[ew];
                __syncwarp();   // the previous run's reads are done
                sx[lane] = r0 + lane < a.n1 ? a.xterm[r0 + lane] : 0.0f;
                __syncwarp();
                // the smallest lb of this lane's run: when it is above thr, no
                // row of the run passes, and the element loop runs only when
                // some lane's run may hold one
                float lbmin = __int_as_float(0x7f800000);
#pragma unroll
                for (int j = 0; j < 32; j += 4) {
                    const float4 x4 = *reinterpret_cast<const float4*>(sx + j);
                    const float l0 = __fmaf_rn(-a.mult, __uint_as_float(v[j]), x4.x);
                    const float l1 = __fmaf_rn(-a.mult, __uint_as_float(v[j + 1]), x4.y);
                    const float l2 = __fmaf_rn(-a.mult, __uint_as_float(v[j + 2]), x4.z);
                    const float l3 = __fmaf_rn(-a.mult, __uint_as_float(v[j + 3]), x4.w);
                    lbmin = fminf(lbmin, fminf(fminf(l0, l1), fminf(l2, l3)));
                }
                const bool maybe = live && lbmin <= thr;
                if (!__any_sync(0xffffffffu, maybe)) continue;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float xj = sx[j];
                    const int row = r0 + j;
                    const float lb = __fmaf_rn(-a.mult, __uint_as_float(v[j]), xj);
                    if (maybe && row < a.n1 && lb <= thr) {
                        const bool allowed = (!a.allow || ((a.allow[row >> 6] >> (row & 63)) & 1ull)) &&
                                             (!a.deny || !((a.deny[row >> 6] >> (row & 63)) & 1ull));
                        if (allowed) {
                            const uint32_t pos = atomicAdd(&a.cand_count[qi], 1u);
                            if (pos < static_cast<uint32_t>(a.cap))
                                a.cand_row[static_cast<size_t>(qi) * a.cap + pos] = static_cast<uint32_t>(row);
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[acc]);
            ++ti;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_free(tmem, kTmemCols);
    }
}

// Rows to bf16 (round to nearest even), zero-padded to dpad, and each row's
// float sum of squares. One warp per row.
__global__ void k_mm_prep(const float* __restrict__ x, size_t n, int d, int dpad, __nv_bfloat16* __restrict__ xb,
                          float* __restrict__ x2) {
    const size_t r = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float s = 0.0f;
    for (int j = lane; j < dpad; j += 32) {
        const float v = j < d ? x[r * d + j] : 0.0f;
        s = __fmaf_rn(v, v, s);
        xb[r * dpad + j] = __float2bfloat16_rn(v);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x2[r] = s;
}

// Rows to f16 after scaling each by a power of two, 2^e with e = 14 -
// exponent(max |x_i|), so the largest element lands in [2^13, 2^14) (exact
// scaling, round to nearest even), zero-padded to dpad; each row's float sum
// of squares (unscaled) and e. One warp per row.
__global__ void k_mm_prep16(const float* __restrict__ x, size_t n, int d, int dpad, __half* __restrict__ xh,
                            float* __restrict__ x2, int* __restrict__ xe) {
    const size_t r = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    float s = 0.0f, mx = 0.0f;
    for (int j = lane; j < d; j += 32) {
        const float v = x[r * d + j];
        s = __fmaf_rn(v, v, s);
        mx = fmaxf(mx, fabsf(v));
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    int ex = 0;
    if (mx > 0.0f) frexpf(mx, &ex);
    const int e = mx > 0.0f ? 14 - ex : 0;
    for (int j = lane; j < dpad; j += 32) {
        const float v = j < d ? ldexpf(x[r * d + j], e) : 0.0f;
        xh[r * dpad + j] = __float2half_rn(v);
    }
    if (lane == 0) {
        x2[r] = s;
        xe[r] = e;
    }
}

__global__ void k_mm_terms(const float* __restrict__ sq, size_t n, float coef, float* __restrict__ out) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) out[i] = coef * sq[i];
}

// Each query's pass threshold from its running list: T - rowterm rounded up
// (T = the k-th exact score, +inf while fewer than k rows are known).
__global__ void k_mm_thresholds(const uint64_t* __restrict__ run_key, int nq, int k, const float* __restrict__ q2,
                                float qcoef, float* __restrict__ thr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const uint64_t key = run_key[static_cast<size_t>(i) * k + k - 1];
    if (key == ~0ull) {
        thr[i] = __int_as_float(0x7f800000);
        return;
    }
    const double T = static_cast<double>(key_float(static_cast<uint32_t>(key >> 32)));
    thr[i] = __double2float_ru(T - static_cast<double>(qcoef) * static_cast<double>(q2[i]));
}

// Exact scores of a query's new candidates merged into its running top-k
// (by (score, row), -0 == +0). One block per query.
__global__ void __launch_bounds__(256) k_mm_merge(const float* __restrict__ q, int d, const float* __restrict__ rows,
                                                  bool ip, int k, int cap, const uint32_t* __restrict__ cand_count,
                                                  const uint32_t* __restrict__ cand_row, uint64_t* __restrict__ run_key,
                                                  uint32_t* __restrict__ run_slot, int* __restrict__ overflow) {
    extern __shared__ uint8_t sm_raw[];
    const int qi = blockIdx.x;
    uint32_t cnt = cand_count[qi];
    if (cnt == 0) return;
    if (cnt > static_cast<uint32_t>(cap)) {
        if (threadIdx.x == 0) overflow[qi] = 1;
        cnt = cap;
    }
    float* qv = reinterpret_cast<float*>(sm_raw);
    uint64_t* keys = reinterpret_cast<uint64_t*>(sm_raw + ((static_cast<size_t>(d) * 4 + 15) & ~size_t{15}));
    const int n = k + static_cast<int>(cnt);
    const int npow = next_pow2(n);
    for (int t = threadIdx.x; t < d; t += blockDim.x) qv[t] = q[static_cast<size_t>(qi) * d + t];
    __syncthreads();
    for (int i = threadIdx.x; i < npow; i += blockDim.x) {
        uint64_t key = ~0ull;
        if (i < k) {
            key = run_key[static_cast<size_t>(qi) * k + i];
        } else if (i < n) {
            const uint32_t row = cand_row[static_cast<size_t>(qi) * cap + (i - k)];
            const float s = exact_score(qv, rows + static_cast<size_t>(row) * d, d, ip);
            key = (static_cast<uint64_t>(float_key_eq0(s)) << 32) | row;
        }
        keys[i] = key;
    }
    if (n <= 512 && blockDim.x == 256) {
        // (block-uniform) the k smallest without a sort network: each of the
        // 8 warps sorts a run of up to 64 keys in registers, a key's rank is
        // the number of keys below it in every run (binary searches), and a
        // key of rank below k goes to its place. Keys are unique but for the
        // all-ones key of empty running places, which takes no place.
        __syncthreads();
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int n_w = max(0, min(64, n - 64 * warp));
        if (n_w > 0) warp_sort_keys_reg<2>(keys + 64 * warp, n_w);
        __syncthreads();
        auto below = [&](uint64_t key) {
            int rank = 0;
            for (int w = 0; w < 8; ++w) {
                const int len = max(0, min(64, n - 64 * w));
                const uint64_t* rw = keys + 64 * w;
                int pos = 0;
#pragma unroll
                for (int step = 64; step > 0; step >>= 1)
                    if (pos + step <= len && rw[pos + step - 1] < key) pos += step;
                rank += pos;
            }
            return rank;
        };
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int e = 32 * i + lane;
            if (e >= n_w) continue;
            const uint64_t key = keys[64 * warp + e];
            if (key == ~0ull) continue;
            const int rank = below(key);
            if (rank < k) {
                run_key[static_cast<size_t>(qi) * k + rank] = key;
                run_slot[static_cast<size_t>(qi) * k + rank] = static_cast<uint32_t>(key);
            }
        }
        if (static_cast<int>(threadIdx.x) < k) {
            const int valid = below(~0ull);
            for (int i = threadIdx.x; i < k; i += blockDim.x)
                if (i >= valid) {
                    run_key[static_cast<size_t>(qi) * k + i] = ~0ull;
                    run_slot[static_cast<size_t>(qi) * k + i] = 0xFFFFFFFFu;
                }
        }
        return;
    }
    bitonic_sort_keys(keys, npow);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        run_key[static_cast<size_t>(qi) * k + i] = keys[i];
        run_slot[static_cast<size_t>(qi) * k + i] = keys[i] == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(keys[i]);
    }
}

// k_mm_merge for k <= 24 and rows with an even dim at 8-byte alignment: one
// warp per query (8 per block). Candidates go in rounds of 8, scored exactly
// by 4-lane groups (exact_avx2_group4, the same bits as exact_score); lanes
// 0..k-1 hold the running top-k keys, lanes k..k+7 the round's, and one
// register sort of the 32 keys keeps the k smallest in lanes 0..k-1.
__global__ void __launch_bounds__(256) k_mm_merge_warp(const float* __restrict__ q, int d, const float* __restrict__ rows,
                                                       bool ip, int k, int nq, int cap,
                                                       const uint32_t* __restrict__ cand_count,
                                                       const uint32_t* __restrict__ cand_row,
                                                       uint64_t* __restrict__ run_key, uint32_t* __restrict__ run_slot,
                                                       int* __restrict__ overflow) {
    extern __shared__ __align__(16) uint8_t sm_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qi = blockIdx.x * 8 + warp;
    if (qi >= nq) return;
    uint32_t cnt = cand_count[qi];
    if (cnt == 0) return;
    if (cnt > static_cast<uint32_t>(cap)) {
        if (lane == 0) overflow[qi] = 1;
        cnt = cap;
    }
    const int dp = (d + 3) & ~3;
    float* qv = reinterpret_cast<float*>(sm_raw) + warp * dp;
    uint64_t* keys = reinterpret_cast<uint64_t*>(reinterpret_cast<float*>(sm_raw) + 8 * dp) + warp * 32;
    for (int t = lane; t < d; t += 32) qv[t] = q[static_cast<size_t>(qi) * d + t];
    uint64_t mine = lane < k ? run_key[static_cast<size_t>(qi) * k + lane] : ~0ull;
    __syncwarp();
    const uint32_t* cq = cand_row + static_cast<size_t>(qi) * cap;
    const int grp = lane >> 2;
    for (uint32_t c0 = 0; c0 < cnt; c0 += 8) {
        const uint32_t i = c0 + grp;
        const bool act = i < cnt;
        const uint32_t row = act ? cq[i] : 0u;   // idle groups score row 0 unused
        const float* rp = rows + static_cast<size_t>(row) * d;
        const float s = ip ? -exact_avx2_group4<false>(qv, rp, d) : exact_avx2_group4<true>(qv, rp, d);
        const uint64_t key = act ? (static_cast<uint64_t>(float_key_eq0(s)) << 32) | row : ~0ull;
        // group g's key to lane k + g
        const uint64_t got = __shfl_sync(0xffffffffu, key, 4 * ((lane - k) & 7));
        keys[lane] = lane < k ? mine : (lane < k + 8 ? got : ~0ull);
        __syncwarp();
        warp_sort_keys_reg<1>(keys, 32);
        __syncwarp();
        mine = lane < k ? keys[lane] : ~0ull;
    }
    if (lane < k) {
        run_key[static_cast<size_t>(qi) * k + lane] = mine;
        run_slot[static_cast<size_t>(qi) * k + lane] = mine == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(mine);
    }
}

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    require(fn != nullptr, "cuTensorMapEncodeTiled is not available", kCudaError);
    return fn;
}

// bf16 or f16 rows (dpad elements, row stride dpad * 2 bytes) read as boxes of 64 x box_rows, 128-byte swizzle.
CUtensorMap make_map(const void* ptr, size_t rows, int dpad, int box_rows, bool f16 = false) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(dpad), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(dpad) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(KA), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(&m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                   const_cast<void*>(ptr), dims,
                                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    require(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed", kCudaError);
    return m;
}

} // namespace

bool mm_supported(int dim) { return dim >= 1 && dim <= kMaxKBlocks * KA; }

void mm_prepare(const float* rows, size_t n, int dim, MmRows& out, cudaStream_t st) {
    require(mm_supported(dim), "the tensor-core filter supports dim <= 128", kUnsupported);
    out.n = n;
    out.dim = dim;
    out.dpad = (dim + 7) & ~7;
    out.bf16.alloc(std::max<size_t>(1, n * out.dpad), st);
    out.sq.alloc(std::max<size_t>(1, n), st);
    if (n) {
        k_mm_prep<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, st>>>(
            rows, n, dim, out.dpad, reinterpret_cast<__nv_bfloat16*>(out.bf16.get()), out.sq.get());
        QG_LAUNCH_CHECK();
    }
}

// ---------------------------------------------------------------------------
// The filter's schedule and its autotuner. The epilogue limits the filter, so
// its warp count is the schedule choice: 8 epilogue warps (two per TMEM lane
// quadrant, 128 columns of a tile each) or 16 (four per quadrant, 64 columns
// each). On the first launch of a problem (store or filter mode, K blocks,
// query tiles and base tiles by their power of two) with at least 8 tiles per
// SM, both are timed twice on the launch's own inputs and the faster kept for
// the rest of the process; a filter run appends candidates, so their counts are
// cleared before each timed run, and the last timed run's candidates are the
// launch's result. Both give the same candidate sets. Launches that must not
// wait on the host (the coarse step without read-back, graph capture) use the
// problem's pick if there is one, else 8.
// ---------------------------------------------------------------------------
namespace {
std::mutex g_ftune_mu;
std::map<uint64_t, int> g_ftune;   // problem key -> epilogue warps
std::atomic<int> g_ftune_on{1}, g_ftune_last{8}, g_ftune_force{0};   // force: 0, or 8 / 16 epilogue warps

template <int EPI>
void launch_filter_epi(const CUtensorMap& tmA, const CUtensorMap& tmB, const MmArgs& a, size_t smem, cudaStream_t st) {
    allow_large_smem<k_mm_filter<EPI>>();
    const int tiles = a.mtiles * a.ntiles;
    k_mm_filter<EPI><<<static_cast<unsigned>(std::min(tiles, sm_count())), filter_threads<EPI>(), smem, st>>>(tmA, tmB,
                                                                                                            a);
    QG_LAUNCH_CHECK();
}

void launch_filter_as(int epi, const CUtensorMap& tmA, const CUtensorMap& tmB, const MmArgs& a, size_t smem,
                      cudaStream_t st) {
    if (epi == 16) launch_filter_epi<16>(tmA, tmB, a, smem, st);
    else launch_filter_epi<8>(tmA, tmB, a, smem, st);
    g_ftune_last.store(epi);
}

void launch_filter(const CUtensorMap& tmA, const CUtensorMap& tmB, const MmArgs& a, size_t smem, cudaStream_t st,
                   bool may_tune) {
    if (const int f = g_ftune_force.load()) {
        launch_filter_as(f, tmA, tmB, a, smem, st);
        return;
    }
    const uint64_t key = (static_cast<uint64_t>(a.store != nullptr) << 48) | (static_cast<uint64_t>(a.kblocks) << 40) |
                         (static_cast<uint64_t>(next_pow2(a.mtiles)) << 20) | static_cast<uint64_t>(next_pow2(a.ntiles));
    {
        std::lock_guard<std::mutex> g(g_ftune_mu);
        const auto it = g_ftune.find(key);
        if (it != g_ftune.end()) {
            launch_filter_as(it->second, tmA, tmB, a, smem, st);
            return;
        }
    }
    if (!may_tune || !g_ftune_on.load() || a.mtiles * a.ntiles < 8 * sm_count()) {
        launch_filter_as(8, tmA, tmB, a, smem, st);
        return;
    }
    cudaEvent_t e0, e1;
    QG_CUDA(cudaEventCreate(&e0));
    QG_CUDA(cudaEventCreate(&e1));
    constexpr int kCand[2] = {8, 16};
    float fastest[2] = {0.0f, 0.0f};
    for (int round = 0; round < 2; ++round)
        for (int c = 0; c < 2; ++c) {
            if (!a.store) QG_CUDA(cudaMemsetAsync(a.cand_count, 0, static_cast<size_t>(a.nq) * sizeof(uint32_t), st));
            QG_CUDA(cudaEventRecord(e0, st));
            launch_filter_as(kCand[c], tmA, tmB, a, smem, st);
            QG_CUDA(cudaEventRecord(e1, st));
            QG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            QG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (round == 0 || ms < fastest[c]) fastest[c] = ms;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(g_ftune_mu);
    g_ftune[key] = fastest[1] < fastest[0] ? 16 : 8;
}
} // namespace

void set_filter_autotune(int on) { g_ftune_on.store(on); }
int filter_autotune() { return g_ftune_on.load(); }
int64_t filter_tuned_problems() {
    std::lock_guard<std::mutex> g(g_ftune_mu);
    return static_cast<int64_t>(g_ftune.size());
}
int filter_last_epilogue_warps() { return g_ftune_last.load(); }
void set_filter_epilogue_warps(int warps) { g_ftune_force.store(warps); }
int filter_epilogue_warps() { return g_ftune_force.load(); }

static void mm_topk_block(const float* q, size_t nq, const float* rows, const MmRows& base, bool ip, size_t k,
                          const uint64_t* allow, const uint64_t* deny, uint64_t* out_key, uint32_t* out_slot,
                          std::vector<int>& overflow_q, size_t q_first, cudaStream_t st);

void mm_topk(const float* q, size_t nq, const float* rows, const MmRows& base, bool ip, size_t k, const uint64_t* allow,
             const uint64_t* deny, uint64_t* out_key, uint32_t* out_slot, std::vector<int>& overflow_q, cudaStream_t st) {
    overflow_q.clear();
    // query blocks bound the candidate lists (block x cap rows) and the bf16 query copies
    const size_t QB = 65536;
    for (size_t q0 = 0; q0 < nq; q0 += QB) {
        const size_t nb = std::min(QB, nq - q0);
        mm_topk_block(q + q0 * base.dim, nb, rows, base, ip, k, allow, deny, out_key + q0 * k, out_slot + q0 * k,
                      overflow_q, q0, st);
    }
}

static void mm_topk_block(const float* q, size_t nq, const float* rows, const MmRows& base, bool ip, size_t k,
                          const uint64_t* allow, const uint64_t* deny, uint64_t* out_key, uint32_t* out_slot,
                          std::vector<int>& overflow_q, size_t q_first, cudaStream_t st) {
    const size_t n = base.n;
    const int d = base.dim;
    if (nq == 0 || k == 0) return;
    require(n < (size_t{1} << 31), "the tensor-core filter supports fewer than 2^31 rows", kUnsupported);
    MmRows qb;
    mm_prepare(q, nq, d, qb, st);
    const double C = std::ldexp(1.0, -7) + std::ldexp(1.0, -14) + d * std::ldexp(1.0, -19);
    const float coef = static_cast<float>(ip ? -0.5 * C : 1.0 - C);   // of |x|^2 and of |q|^2
    DevBuf<float> xterm(std::max<size_t>(1, n), st), thr(nq, st);
    k_mm_terms<<<static_cast<unsigned>(ceil_div(std::max<size_t>(1, n), 256)), 256, 0, st>>>(base.sq.get(), n, coef,
                                                                                            xterm.get());
    QG_LAUNCH_CHECK();

    // seed: the exact top-k of the first rows, which gives the first filter
    // chunk its threshold. The exact tiles run far below the tensor cores, so
    // the seed is a small share of the rows: 1/256 of them, at least 64 (and
    // 4k) and at most 4,096 (and 4k). Nearest-centroid assignment against
    // 4,096 to 16,384 centroids otherwise spends most of its time here.
    const size_t seed_lo = std::max<size_t>(64, 4 * k), seed_hi = std::max<size_t>(4096, 4 * k);
    const size_t seed = std::min(n, std::clamp<size_t>(n / 256, seed_lo, seed_hi));
    flat_candidates(q, nq, rows, seed, d, ip, k, allow, deny, out_key, out_slot, st, /*allow_mm=*/false);
    if (seed == n) return;

    const int cap = static_cast<int>(std::clamp<size_t>(4 * k, 1024, 4096));
    // chunks grow 4x while about 3k new rows pass per chunk stay well under the cap, else 2x
    const size_t growth = 12 * k <= static_cast<size_t>(cap) ? 4 : 2;
    DevBuf<uint32_t> cnt(nq, st), crow(nq * static_cast<size_t>(cap), st);
    DevBuf<int> ovf(nq, st), err(1, st);
    QG_CUDA(cudaMemsetAsync(ovf.get(), 0, nq * sizeof(int), st));
    QG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    const int kblocks = (base.dpad + KA - 1) / KA;
    const CUtensorMap tmA = make_map(reinterpret_cast<const __nv_bfloat16*>(qb.bf16.get()), nq, qb.dpad, BM);
    const CUtensorMap tmB = make_map(reinterpret_cast<const __nv_bfloat16*>(base.bf16.get()), n, base.dpad, BN);
    // more than half an SM's shared memory: one CTA per SM, so no two CTAs wait on each other's TMEM
    const size_t smem = std::max<size_t>(filter_smem_bytes(kblocks), 116 * 1024);
    const size_t merge_smem = ((static_cast<size_t>(d) * 4 + 15) & ~size_t{15}) + static_cast<size_t>(next_pow2(static_cast<int>(k) + cap)) * 8;
    require(merge_smem <= 200 * 1024, "k too large for the tensor-core filter", kUnsupported);
    allow_large_smem<k_mm_merge>();
    // small k: a warp per query merges the candidates (8 queries per block)
    const bool warp_merge = k <= 24 && (d & 1) == 0 && (reinterpret_cast<uintptr_t>(rows) & 7) == 0;
    MmArgs a{};
    a.nq = static_cast<int>(nq);
    a.kblocks = kblocks;
    a.ksteps = (d + 15) / 16;
    a.mtiles = static_cast<int>(ceil_div(nq, BM));
    a.xterm = xterm.get();
    a.thr = thr.get();
    a.mult = ip ? 1.0f : 2.0f;
    a.allow = allow;
    a.deny = deny;
    a.cand_count = cnt.get();
    a.cand_row = crow.get();
    a.cap = cap;
    a.err = err.get();
    size_t n0 = seed, chunk = (growth - 1) * seed;
    while (n0 < n) {
        const size_t n1 = std::min(n, n0 + chunk);
        k_mm_thresholds<<<static_cast<unsigned>(ceil_div(nq, 256)), 256, 0, st>>>(out_key, static_cast<int>(nq),
                                                                                  static_cast<int>(k), qb.sq.get(),
                                                                                  coef, thr.get());
        QG_LAUNCH_CHECK();
        QG_CUDA(cudaMemsetAsync(cnt.get(), 0, nq * sizeof(uint32_t), st));
        a.n0 = static_cast<int>(n0);
        a.n1 = static_cast<int>(n1);
        a.ntiles = static_cast<int>(ceil_div(n1 - n0, BN));
        {
            KernelTimer kt("mm_filter", st);
            launch_filter(tmA, tmB, a, smem, st, /*may_tune=*/true);
        }
        if (warp_merge) {
            const size_t wsm = 8 * static_cast<size_t>((d + 3) & ~3) * 4 + 8 * 32 * 8;
            k_mm_merge_warp<<<static_cast<unsigned>(ceil_div(nq, 8)), 256, wsm, st>>>(
                q, d, rows, ip, static_cast<int>(k), static_cast<int>(nq), cap, cnt.get(), crow.get(), out_key,
                out_slot, ovf.get());
        } else {
            k_mm_merge<<<static_cast<unsigned>(nq), 256, merge_smem, st>>>(q, d, rows, ip, static_cast<int>(k), cap,
                                                                          cnt.get(), crow.get(), out_key, out_slot,
                                                                          ovf.get());
        }
        QG_LAUNCH_CHECK();
        n0 = n1;
        chunk = std::min<size_t>(n0 * (growth - 1), size_t{1} << 21);
    }
    int herr = 0;
    std::vector<int> hovf(nq);
    QG_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaMemcpyAsync(hovf.data(), ovf.get(), nq * sizeof(int), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    require(herr == 0, "tensor-core filter: a pipeline wait timed out", kRuntimeError);
    for (size_t i = 0; i < nq; ++i)
        if (hovf[i]) overflow_q.push_back(static_cast<int>(q_first + i));
}


// ---------------------------------------------------------------------------
// Coarse assignment through the tensor cores (reference src/ivf_index.cpp:
// 305-419, which ranks lists by the exact distance, ties by list). The store
// mode of k_mm_filter gives acc(q, c), the F16 dot product of a query and a
// centroid (each row scaled by a power of two first, undone exactly after)
// accumulated in FP32. With e = C (|q|^2 + |c|^2) as in mm_topk (C from
// f16's unit roundoff 2^-11), each exact score lies in [lb, ub] = [s^ - e,
// s^ + e] (s^ = |q|^2 + |c|^2 - 2 acc for L2, -acc for inner product, e
// halved). T, the P-th smallest ub,
// bounds the P-th exact score from above, so only centroids with lb <= T can
// be among the P nearest: k_coarse_recheck scores those exactly, in the
// reference's order, and keeps the P smallest by (score, list), -0 == +0.
// ---------------------------------------------------------------------------
namespace {

// A threshold T at or above the k-th smallest (1-based) of the n uint32 keys
// in shared memory, by one block. 0xFFFFFFFF marks an unbounded key, above
// every other. [kmin, kmax] is the range of the nfin bounded keys; they are
// counted into kCoarseBins nearly equal key intervals (KeyBins), and T is the last key of the
// first interval whose running count reaches k, so at least k keys are <= T
// and T lies within one interval of the k-th smallest. (A T above the k-th
// smallest only admits more candidates to the exact step.) hist: kCoarseBins
// ints of shared scratch, zero on entry; two barriers.
constexpr int kCoarseBins = 1024;
__device__ uint32_t block_threshold_u32(const uint32_t* keys, int n, int k, uint32_t kmin, uint32_t kmax, int nfin,
                                        int* hist, uint32_t* s_t) {
    if (nfin < k) return 0xFFFFFFFFu;   // (block-uniform) the k-th smallest is unbounded
    if (kmax == kmin) return kmin;
    const KeyBins kb(kmin, static_cast<uint64_t>(kmax - kmin) + 1, kCoarseBins);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t key = keys[i];
        if (key != 0xFFFFFFFFu) atomicAdd(&hist[kb.bin(key)], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {   // warp 0: lane l owns bins 32 l .. 32 l + 31
        const int lane = threadIdx.x;
        constexpr int kPer = kCoarseBins / 32;
        int own = 0;
#pragma unroll 8
        for (int b = 0; b < kPer; ++b) own += hist[kPer * lane + b];
        int incl = own;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - own;
        if (excl < k && k <= incl) {
            int acc = excl, bin = kPer * lane + kPer - 1;
            for (int b = 0; b < kPer; ++b) {
                acc += hist[kPer * lane + b];
                if (acc >= k) {
                    bin = kPer * lane + b;
                    break;
                }
            }
            // every key counted in bins <= bin is <= kb.last(bin)
            *s_t = static_cast<uint32_t>(min(kb.last(bin), static_cast<uint64_t>(kmax)));
        }
    }
    __syncthreads();
    return *s_t;
}

} // namespace

// x * 2^e rounded to nearest, which is what ldexpf returns: one multiply by
// 2^e when that is a normal float (the product is then the correctly rounded
// x * 2^e), ldexpf itself otherwise.
__device__ __forceinline__ float scale_pow2(float x, int e) {
    return (e >= -126 && e <= 127) ? __fmul_rn(x, __int_as_float((e + 127) << 23)) : ldexpf(x, e);
}

// The P smallest of the cnt distinct keys key[0, cnt) written in order, key by
// key, for P <= cnt <= 32 K x warps: each warp sorts a run of up to 32 K keys
// in registers; a key's rank is then the number of keys below it in each run
// (binary searches over the sorted runs; its own run counts its place in it),
// and a key of rank < P goes to place rank. One block barrier.
template <int K>
__device__ void ranked_out(uint64_t* key, int cnt, int P, const float* score_of, uint32_t* probe_q, float* pdist_q) {
    constexpr int R = 32 * K;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int n_w = max(0, min(R, cnt - R * warp));
    if (n_w > 0) warp_sort_keys_reg<K>(key + R * warp, n_w);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int e = R * warp + i * 32 + lane;
        if (e >= cnt) continue;
        const uint64_t k = key[e];
        int rank = 0;
        for (int w = 0; w < nw; ++w) {
            const int len = max(0, min(R, cnt - R * w));
            const uint64_t* run = key + R * w;
            int pos = 0;   // keys of the run below k
#pragma unroll
            for (int step = R; step > 0; step >>= 1)
                if (pos + step <= len && run[pos + step - 1] < k) pos += step;
            rank += pos;
        }
        if (rank < P) {
            const uint32_t j = static_cast<uint32_t>(k);
            probe_q[rank] = j;
            pdist_q[rank] = score_of[j];
        }
    }
}

__global__ void __launch_bounds__(256, 6) k_coarse_recheck(const float* __restrict__ q, const float* __restrict__ q2,
                                                        const int* __restrict__ qexp, const float* __restrict__ cent,
                                                        const float* __restrict__ c2, const int* __restrict__ cexp,
                                                        int nlist, int d, bool ip, float c_up, float c_lo,
                                                        const float* __restrict__ accm, size_t ld, int P, int cap,
                                                        uint32_t* __restrict__ probe, float* __restrict__ pdist,
                                                        int* __restrict__ redo,
                                                        unsigned long long* __restrict__ ncand) {
    extern __shared__ __align__(16) uint8_t sm_raw[];
    const int qi = blockIdx.x;
    uint64_t* ckey = reinterpret_cast<uint64_t*>(sm_raw);             // cap
    float* qv = reinterpret_cast<float*>(ckey + cap);                   // d, 16-byte aligned
    uint32_t* ub = reinterpret_cast<uint32_t*>(qv + ((d + 3) & ~3));    // nlist
    __shared__ int hist[kCoarseBins], s_count, s_wfin[8];
    __shared__ uint32_t s_wmin[8], s_wmax[8], s_t;
    const float* arow = accm + static_cast<size_t>(qi) * ld;
    const float qq = q2[qi];
    const int qe = qexp[qi];
    // norms where float squares lose relative accuracy (underflow or near
    // overflow): the relative bound does not hold, so such a query takes the
    // exact path and such a list is always rescored
    auto extreme = [](float x2) { return (x2 > 0.0f && x2 < 0x1p-60f) || !(x2 < 0x1p60f); };
    const bool all = extreme(qq);   // rescored in full here when there is no exact path to send it to
    if (all && redo) {
        if (threadIdx.x == 0) redo[qi] = 1;
        return;
    }
    for (int t = threadIdx.x; t < d; t += blockDim.x) qv[t] = q[static_cast<size_t>(qi) * d + t];
    for (int t = threadIdx.x; t < kCoarseBins; t += blockDim.x) hist[t] = 0;
    // upper bounds, rounded up at every step (c_up >= 1 + C for L2, >= C / 2
    // for inner product; the f16 row scaling is undone exactly by scale_pow2).
    // Four lists per thread and step, read as 16-byte vectors.
    auto upper = [&](float acc_j, float c2j, int cej) -> uint32_t {
        const float s = __fadd_ru(qq, c2j);
        const float a = scale_pow2(acc_j, -(qe + cej));
        const float hi = ip ? __fmaf_ru(c_up, s, -a) : __fmaf_ru(-2.0f, a, __fmul_ru(c_up, s));
        return extreme(c2j) ? 0xFFFFFFFFu : float_key(hi);
    };
    // (and the range and count of the bounded ones, for the threshold)
    uint32_t kmin = 0xFFFFFFFFu, kmax = 0;
    int nfin = 0;
    auto keep = [&](int j, uint32_t u) {
        ub[j] = u;
        if (u != 0xFFFFFFFFu) {
            kmin = min(kmin, u);
            kmax = max(kmax, u);
            ++nfin;
        }
    };
    const int n4 = nlist & ~3;
    for (int j = 4 * threadIdx.x; j < n4; j += 4 * blockDim.x) {
        const float4 av = *reinterpret_cast<const float4*>(arow + j);
        const float4 cv = *reinterpret_cast<const float4*>(c2 + j);
        const int4 ev = *reinterpret_cast<const int4*>(cexp + j);
        keep(j, upper(av.x, cv.x, ev.x));
        keep(j + 1, upper(av.y, cv.y, ev.y));
        keep(j + 2, upper(av.z, cv.z, ev.z));
        keep(j + 3, upper(av.w, cv.w, ev.w));
    }
    for (int j = n4 + threadIdx.x; j < nlist; j += blockDim.x) keep(j, upper(arow[j], c2[j], cexp[j]));
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        nfin += __shfl_xor_sync(0xffffffffu, nfin, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_wmin[threadIdx.x >> 5] = kmin;
        s_wmax[threadIdx.x >> 5] = kmax;
        s_wfin[threadIdx.x >> 5] = nfin;
    }
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (int w = 0; w < 8; ++w) {
        kmin = min(kmin, s_wmin[w]);
        kmax = max(kmax, s_wmax[w]);
    }
    nfin = 0;
    for (int w = 0; w < 8; ++w) nfin += s_wfin[w];
    const uint32_t T = block_threshold_u32(ub, nlist, P, kmin, kmax, nfin, hist, &s_t);
    // candidates: lower bound, rounded down (c_lo <= 1 - C for L2; for inner
    // product the margin c_up is subtracted from a sum rounded up), <= T
    auto lower_in = [&](float acc_j, float c2j, int cej) -> bool {
        const float a = scale_pow2(acc_j, -(qe + cej));
        const float lo = ip ? __fmaf_rd(-c_up, __fadd_ru(qq, c2j), -a)
                            : __fmaf_rd(-2.0f, a, __fmul_rd(c_lo, __fadd_rd(qq, c2j)));
        return all || float_key(lo) <= T || extreme(c2j);
    };
    auto push = [&](int j) {
        const int pos = atomicAdd(&s_count, 1);
        if (pos < cap) ckey[pos] = static_cast<uint64_t>(j);
    };
    for (int j = 4 * threadIdx.x; j < n4; j += 4 * blockDim.x) {
        const float4 av = *reinterpret_cast<const float4*>(arow + j);
        const float4 cv = *reinterpret_cast<const float4*>(c2 + j);
        const int4 ev = *reinterpret_cast<const int4*>(cexp + j);
        if (lower_in(av.x, cv.x, ev.x)) push(j);
        if (lower_in(av.y, cv.y, ev.y)) push(j + 1);
        if (lower_in(av.z, cv.z, ev.z)) push(j + 2);
        if (lower_in(av.w, cv.w, ev.w)) push(j + 3);
    }
    for (int j = n4 + threadIdx.x; j < nlist; j += blockDim.x)
        if (lower_in(arow[j], c2[j], cexp[j])) push(j);
    __syncthreads();
    const int cnt = s_count;
    if (threadIdx.x == 0 && ncand) atomicAdd(ncand, static_cast<unsigned long long>(cnt));
    if (cnt > cap) {   // too many near-ties: this query takes the exact path (cap >= nlist when redo is null)
        if (threadIdx.x == 0 && redo) redo[qi] = 1;
        return;
    }
    // exact scores, one candidate per 8-lane group; each list's score is kept
    // by list (over its upper bound, no longer needed) for the output
    float* score_of = reinterpret_cast<float*>(ub);
    if ((d & 1) == 0 && (reinterpret_cast<uintptr_t>(cent) & 7) == 0) {
        // rows 8-byte aligned: one candidate per 4-lane group, one 32-byte
        // sector of its row per step
        const int ngrp = blockDim.x >> 2, grp = threadIdx.x >> 2;
        const int rounds = (cnt + ngrp - 1) / ngrp;   // (block-uniform)
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = rd * ngrp + grp;
            const bool act = i < cnt;
            const int j = act ? static_cast<int>(ckey[i]) : 0;   // idle groups score row 0 unused
            const float* row = cent + static_cast<size_t>(j) * d;
            const float sc = ip ? -exact_avx2_group4<false>(qv, row, d) : exact_avx2_group4<true>(qv, row, d);
            if (act && (threadIdx.x & 3) == 0) {
                ckey[i] = (static_cast<uint64_t>(float_key_eq0(sc)) << 32) | static_cast<uint32_t>(j);
                score_of[j] = sc;
            }
        }
    } else {
        const int ngrp = blockDim.x >> 3, grp = threadIdx.x >> 3;
        const int rounds = (cnt + ngrp - 1) / ngrp;   // (block-uniform)
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = rd * ngrp + grp;
            const bool act = i < cnt;
            const int j = act ? static_cast<int>(ckey[i]) : 0;   // idle groups score row 0 unused
            const float* row = cent + static_cast<size_t>(j) * d;
            const float sc = ip ? -exact_avx2_group8<false, true>(qv, row, d) : exact_avx2_group8<true, true>(qv, row, d);
            if (act && (threadIdx.x & 7) == 0) {
                ckey[i] = (static_cast<uint64_t>(float_key_eq0(sc)) << 32) | static_cast<uint32_t>(j);
                score_of[j] = sc;
            }
        }
    }
    __syncthreads();
    // the P smallest by (score, list), in order
    if (cnt <= 32 * (static_cast<int>(blockDim.x) >> 5)) {
        ranked_out<1>(ckey, cnt, P, score_of, probe + static_cast<size_t>(qi) * P, pdist + static_cast<size_t>(qi) * P);
        return;
    }
    if (cnt <= 64 * (static_cast<int>(blockDim.x) >> 5)) {
        ranked_out<2>(ckey, cnt, P, score_of, probe + static_cast<size_t>(qi) * P, pdist + static_cast<size_t>(qi) * P);
        return;
    }
    if (cnt > P) {
        if (threadIdx.x < 32) warp_select_keep(ckey, cnt, P, hist);
        __syncthreads();
    }
    const int ns = next_pow2(P < 2 ? 2 : P);
    for (int i = P + threadIdx.x; i < ns; i += blockDim.x) ckey[i] = ~0ull;
    bitonic_sort_keys(ckey, ns);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const uint32_t j = static_cast<uint32_t>(ckey[i]);
        probe[static_cast<size_t>(qi) * P + i] = j;
        pdist[static_cast<size_t>(qi) * P + i] = score_of[j];
    }
}

static size_t coarse_recheck_smem(int nlist, int d, int cap) {
    return static_cast<size_t>(cap) * 8 + static_cast<size_t>((d + 3) & ~3) * 4 + static_cast<size_t>(nlist) * 4;
}

static int coarse_cap(int nlist, int P) {
    return std::min(next_pow2(nlist), std::max(1024, next_pow2(4 * P)));
}

bool coarse_mm_supported(int nlist, int dim, int P, bool cent_prepared, bool no_readback) {
    const int cap = no_readback ? next_pow2(nlist) : coarse_cap(nlist, P);
    return cent_prepared && mm_supported(dim) && P >= 1 && P <= nlist && nlist <= 16384 &&
           coarse_recheck_smem(nlist, dim, cap) <= 200 * 1024;
}

void coarse_probes_mm(const IvfView& v, const float* q, int nq, int P, uint32_t* probe, float* pdist,
                      std::vector<int>& redo_q, cudaStream_t st, int* err_dev) {
    const bool no_readback = err_dev != nullptr;
    redo_q.clear();
    if (nq == 0) return;
    const int d = v.dim, nlist = v.nlist;
    const size_t QB = 65536;   // query blocks bound the score matrix
    for (size_t q0 = 0; q0 < static_cast<size_t>(nq); q0 += QB) {
        const int nb = static_cast<int>(std::min(QB, static_cast<size_t>(nq) - q0));
        DevBuf<uint16_t> qh;
        DevBuf<float> qsq;
        DevBuf<int> qexp;
        int qdpad = 0;
        prepare_f16_rows(q + q0 * d, nb, d, qh, qsq, qexp, qdpad, st);
        const size_t ld = (static_cast<size_t>(nlist) + 3) & ~size_t{3};
        DevBuf<float> accm(static_cast<size_t>(nb) * ld, st);
        DevBuf<int> redo, err;
        DevBuf<unsigned long long> ncand;
        if (!no_readback) {
            redo.alloc(nb, st);
            err.alloc(1, st);
            ncand.alloc(1, st);
            QG_CUDA(cudaMemsetAsync(ncand.get(), 0, sizeof(unsigned long long), st));
            QG_CUDA(cudaMemsetAsync(redo.get(), 0, nb * sizeof(int), st));
            QG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
        }
        const int kblocks = (qdpad + KA - 1) / KA;
        const CUtensorMap tmA = make_map(qh.get(), nb, qdpad, BM, true);
        const CUtensorMap tmB = make_map(v.cent_f16, nlist, v.cent_dpad, BN, true);
        const size_t smem = std::max<size_t>(filter_smem_bytes(kblocks), 116 * 1024);
        MmArgs a{};
        a.nq = nb;
        a.n0 = 0;
        a.n1 = nlist;
        a.kblocks = kblocks;
        a.ksteps = (d + 15) / 16;
        a.mtiles = static_cast<int>(ceil_div(static_cast<size_t>(nb), BM));
        a.ntiles = static_cast<int>(ceil_div(static_cast<size_t>(nlist), BN));
        a.err = no_readback ? err_dev : err.get();
        a.store = accm.get();
        a.ld = ld;
        a.f16 = 1;
        {
            KernelTimer kt("coarse_mm", st);
            launch_filter(tmA, tmB, a, smem, st, /*may_tune=*/!no_readback);
        }
        const int cap = no_readback ? next_pow2(nlist) : coarse_cap(nlist, P);   // no read-back: every list fits
        const size_t rsm = coarse_recheck_smem(nlist, d, cap);
        allow_large_smem<k_coarse_recheck>();
        // f16 inputs: unit roundoff 2^-11 in place of bf16's 2^-8 (subnormal
        // rounding of the scaled rows is far below the 2^-14 term)
        const double C = std::ldexp(1.0, -10) + std::ldexp(1.0, -14) + d * std::ldexp(1.0, -19);
        // the bound's factors as floats rounded outwards
        const float c_up = v.ip_metric ? std::nextafter(static_cast<float>(0.5 * C), 1.0f)
                                       : std::nextafter(static_cast<float>(1.0 + C), 2.0f);
        const float c_lo = std::nextafter(static_cast<float>(1.0 - C), 0.0f);
        {
            KernelTimer kt("coarse_recheck", st);
            k_coarse_recheck<<<static_cast<unsigned>(nb), 256, rsm, st>>>(
                q + q0 * d, qsq.get(), qexp.get(), v.centroids, v.cent_sq, v.cent_exp, nlist, d, v.ip_metric, c_up,
                c_lo, accm.get(), ld, P, cap, probe + q0 * P, pdist + q0 * P, redo.get(), ncand.get());
            QG_LAUNCH_CHECK();
        }
        if (no_readback) continue;   // the caller reads the flag with the results
        int herr = 0;
        unsigned long long hcand = 0;
        std::vector<int> hredo(nb);
        QG_CUDA(cudaMemcpyAsync(&hcand, ncand.get(), sizeof(hcand), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaMemcpyAsync(hredo.data(), redo.get(), nb * sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        require(herr == 0, "tensor-core coarse step: a pipeline wait timed out", kRuntimeError);
        count_tensor_coarse_candidates(static_cast<int64_t>(hcand));
        for (int i = 0; i < nb; ++i)
            if (hredo[i]) redo_q.push_back(static_cast<int>(q0) + i);
    }
}

void prepare_f16_rows(const float* rows, size_t n, int dim, DevBuf<uint16_t>& f16, DevBuf<float>& sq,
                      DevBuf<int>& exps, int& dpad, cudaStream_t st) {
    require(mm_supported(dim), "the tensor-core path supports dim <= 128", kUnsupported);
    dpad = (dim + 7) & ~7;
    f16.alloc(std::max<size_t>(1, n * dpad), st);
    sq.alloc(std::max<size_t>(1, n), st);
    exps.alloc(std::max<size_t>(1, n), st);
    if (n) {
        k_mm_prep16<<<static_cast<unsigned>(ceil_div(n * 32, 256)), 256, 0, st>>>(
            rows, n, dim, dpad, reinterpret_cast<__half*>(f16.get()), sq.get(), exps.get());
        QG_LAUNCH_CHECK();
    }
}

} // namespace qg
