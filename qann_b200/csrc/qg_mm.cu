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
// (128 lanes x 256 columns each), and 8 epilogue warps read the accumulator
// with tcgen05.ld, form the lower bound with one FMA and append the rows that
// pass to the query's candidate list.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_sm100.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace qg {

namespace {

constexpr int BM = 128;         // queries per tile (TMEM lanes)
constexpr int BN = 256;         // base rows per tile (accumulator columns)
constexpr int KA = 64;          // bf16 elements per 128-byte swizzle row
constexpr int kStages = 2;      // base tile buffers
constexpr int kEpiWarps = 8;    // two per TMEM lane quadrant, each on half the columns
constexpr int kThreads = (2 + kEpiWarps) * 32;
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
};

size_t filter_smem_bytes(int kblocks) {
    return 1024 + static_cast<size_t>(kblocks) * BM * 128 + static_cast<size_t>(kStages) * kblocks * BN * 128 + 256;
}

} // namespace

__global__ void __launch_bounds__(kThreads, 1)
    k_mm_filter(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, MmArgs a) {
    using namespace sm100;
    extern __shared__ uint8_t smem_raw[];
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
            mbar_init(&tempty[b], kEpiWarps);
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
    auto fail = [&] {
        *abort = 1;
        atomicExch(a.err, 2);
    };

    if (warp == 0) {
        if (lane == 0) {
            int it = 0, aloads = 0, cur_m = -1;
            for (int t = blockIdx.x; t < total && !*abort; t += gridDim.x) {
                const int mt = t / a.ntiles, nt = t - mt * a.ntiles;
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
            const uint32_t idesc = idesc_bf16_f32(BM, BN);
            int it = 0, aloads = 0, cur_m = -1, ti = 0;
            for (int t = blockIdx.x; t < total && !*abort; t += gridDim.x) {
                const int mt = t / a.ntiles;
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
        const int ew = warp - 2;      // 0..7
        const int quad = warp & 3;    // this warp's TMEM lanes: 32 * quad ..
        const int col0 = (ew >> 2) * (BN / 2);
        const int row_in_tile = quad * 32 + lane;
        int ti = 0;
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            const int mt = t / a.ntiles, nt = t - mt * a.ntiles;
            const int acc = ti & 1;
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&tfull[acc], (ti >> 1) & 1, abort));
            if (!ok) {
                if (lane == 0) fail();
                break;
            }
            tc_fence_after();
            const int qi = mt * BM + row_in_tile;
            const bool live = qi < a.nq;
            const float thr = live ? a.thr[qi] : 0.0f;
            for (int c = 0; c < BN / 2; c += 32) {
                uint32_t v[32];
                tmem_ld32(tmem + (static_cast<uint32_t>(quad * 32) << 16) + static_cast<uint32_t>(acc * BN + col0 + c),
                          v);
                const int r0 = a.n0 + nt * BN + col0 + c;   // base row of v[0]
                const float xt = r0 + lane < a.n1 ? a.xterm[r0 + lane] : 0.0f;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const float xj = __shfl_sync(0xffffffffu, xt, j);
                    const int row = r0 + j;
                    const float lb = __fmaf_rn(-a.mult, __uint_as_float(v[j]), xj);
                    if (live && row < a.n1 && lb <= thr) {
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
    bitonic_sort_keys(keys, npow);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        run_key[static_cast<size_t>(qi) * k + i] = keys[i];
        run_slot[static_cast<size_t>(qi) * k + i] = keys[i] == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(keys[i]);
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

// bf16 rows (dpad elements, row stride dpad * 2 bytes) read as boxes of 64 x box_rows, 128-byte swizzle.
CUtensorMap make_map(const __nv_bfloat16* ptr, size_t rows, int dpad, int box_rows) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(dpad), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(dpad) * 2};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(KA), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims,
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

    // seed: the exact top-k of the first rows
    const size_t seed = std::min(n, std::max<size_t>(4096, 4 * k));
    flat_candidates(q, nq, rows, seed, d, ip, k, allow, deny, out_key, out_slot, st, /*allow_mm=*/false);
    if (seed == n) return;

    const int cap = static_cast<int>(std::clamp<size_t>(4 * k, 1024, 4096));
    DevBuf<uint32_t> cnt(nq, st), crow(nq * static_cast<size_t>(cap), st);
    DevBuf<int> ovf(nq, st), err(1, st);
    QG_CUDA(cudaMemsetAsync(ovf.get(), 0, nq * sizeof(int), st));
    QG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    const int kblocks = (base.dpad + KA - 1) / KA;
    const CUtensorMap tmA = make_map(reinterpret_cast<const __nv_bfloat16*>(qb.bf16.get()), nq, qb.dpad, BM);
    const CUtensorMap tmB = make_map(reinterpret_cast<const __nv_bfloat16*>(base.bf16.get()), n, base.dpad, BN);
    // more than half an SM's shared memory: one CTA per SM, so no two CTAs wait on each other's TMEM
    const size_t smem = std::max<size_t>(filter_smem_bytes(kblocks), 116 * 1024);
    allow_large_smem<k_mm_filter>();
    const size_t merge_smem = ((static_cast<size_t>(d) * 4 + 15) & ~size_t{15}) + static_cast<size_t>(next_pow2(static_cast<int>(k) + cap)) * 8;
    require(merge_smem <= 200 * 1024, "k too large for the tensor-core filter", kUnsupported);
    allow_large_smem<k_mm_merge>();
    const int sms = sm_count();
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
    size_t n0 = seed, chunk = seed;
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
        const int tiles = a.mtiles * a.ntiles;
        {
            KernelTimer kt("mm_filter", st);
            k_mm_filter<<<static_cast<unsigned>(std::min(tiles, sms)), kThreads, smem, st>>>(tmA, tmB, a);
            QG_LAUNCH_CHECK();
        }
        k_mm_merge<<<static_cast<unsigned>(nq), 256, merge_smem, st>>>(q, d, rows, ip, static_cast<int>(k), cap,
                                                                      cnt.get(), crow.get(), out_key, out_slot,
                                                                      ovf.get());
        QG_LAUNCH_CHECK();
        n0 = n1;
        chunk = std::min<size_t>(chunk * 2, size_t{1} << 21);
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

} // namespace qg
