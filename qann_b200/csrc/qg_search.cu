// The IVF fast-scan + refine query path on the GPU.
//
// One search call runs, on one stream:
//   k_normalize       cosine queries to unit length (reference src/index.cpp:193-218)
//   coarse            every (query, centroid) exact score in the reference's
//                     AVX2 order, then the nprobe smallest by (score, list)
//                     (reference src/ivf_index.cpp:305-356)
//   k_probe_terms     per-probe distance terms A / base (reference :526-529, :577-579)
//   k_query_tables    per-query C table, or the per-query uint8 LUT for inner
//                     product scoring (reference :436-456)
//   k_scan            per (query, probe chunk): LUT build in shared memory,
//                     4-bit lookups from registers, fused top-k' selection
//                     (reference :421-641 and src/topk.hpp)
//   k_merge           per query: the k' best of its chunks
//   k_finalize_ivf /  the k results, sorted by (distance, id) (reference
//   k_refine_scores + src/topk.hpp:53-77), or re-ranked with exact distances
//   k_refine_select   from the raw rows (reference src/refine_index.cpp:112-140)
#include "qg_device.cuh"
#include "qg_search.h"

#include <algorithm>
#include <vector>

namespace qg {

// ---------------------------------------------------------------------------
// Cosine normalisation: one thread per row, the row's sum of squares in
// double in index order (each `sum += x * x` one double FMA, as the
// reference's GCC build contracts it), scale = float(1 / sqrt(sum)), x * scale.
// ---------------------------------------------------------------------------
__global__ void k_normalize(const float* __restrict__ x, float* __restrict__ y, int n, int d, int* zero_row) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = x + static_cast<size_t>(i) * d;
    double s = 0.0;
    for (int j = 0; j < d; ++j) {
        const double v = static_cast<double>(r[j]);
        s = __fma_rn(v, v, s);
    }
    const double len = __dsqrt_rn(s);
    float* o = y + static_cast<size_t>(i) * d;
    if (len == 0.0) {
        atomicExch(zero_row, 1);
        for (int j = 0; j < d; ++j) o[j] = 0.0f;
        return;
    }
    const float scale = __double2float_rn(__ddiv_rn(1.0, len));
    for (int j = 0; j < d; ++j) o[j] = __fmul_rn(r[j], scale);
}

// ---------------------------------------------------------------------------
// All-pairs exact scores, out[i * nb + j] = score(a_i, b_j), in the AVX2
// chain order of exact_avx2 (qg_common.cuh). Tiles of 16 rows of a x 32 rows
// of b; each thread keeps the 32 chain accumulators of two pairs while the
// 32-float chunks of the rows stream through shared memory.
// ---------------------------------------------------------------------------
namespace {
constexpr int kTA = 16, kTB = 32;
}

template <bool kIP>
__global__ void __launch_bounds__(256) k_pair_scores(const float* __restrict__ A, int na, const float* __restrict__ Bm,
                                                     int nb, int d, float* __restrict__ out, size_t ld_out) {
    // rows padded to 34 floats: 8-byte loads stay aligned, and the 16 B rows a
    // half-warp reads fall on distinct bank pairs
    __shared__ __align__(8) float sa[kTA][34];
    __shared__ __align__(8) float sb[kTB][34];
    const int ta = threadIdx.x >> 4;          // 0..15: row of a
    const int tb = threadIdx.x & 15;          // pairs (tb) and (tb + 16) of b
    const int a0 = blockIdx.y * kTA, b0 = blockIdx.x * kTB;
    // acc[p][j][h]: accumulator j of AVX2 lanes 2h and 2h + 1, advanced as one
    // packed pair (each component rounds as the scalar FMA does)
    float2 acc[2][4][4];
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 4; ++h) acc[p][j][h] = make_float2(0.0f, 0.0f);
    auto step = [&](float2& c, const float* qa, const float* qb, int e) {
        const float2 x = *reinterpret_cast<const float2*>(qa + e), y = *reinterpret_cast<const float2*>(qb + e);
        if (kIP) {
            c = __ffma2_rn(x, y, c);
        } else {
            const float2 df = sub2(x, y);
            c = __ffma2_rn(df, df, c);
        }
    };

    const int n32 = d & ~31;
    auto stage = [&](int base, int len) {
        for (int e = threadIdx.x; e < kTA * 32; e += 256) {
            const int r = e >> 5, c = e & 31;
            const int gi = a0 + r;
            sa[r][c] = (gi < na && c < len) ? A[static_cast<size_t>(gi) * d + base + c] : 0.0f;
        }
        for (int e = threadIdx.x; e < kTB * 32; e += 256) {
            const int r = e >> 5, c = e & 31;
            const int gj = b0 + r;
            sb[r][c] = (gj < nb && c < len) ? Bm[static_cast<size_t>(gj) * d + base + c] : 0.0f;
        }
    };
    for (int base = 0; base < n32; base += 32) {
        stage(base, 32);
        __syncthreads();
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const float* qa = sa[ta];
            const float* qb = sb[tb + 16 * p];
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int h = 0; h < 4; ++h) step(acc[p][j][h], qa, qb, 8 * j + 2 * h);
        }
        __syncthreads();
    }
    const int rem = d - n32;
    if (rem > 0) {
        stage(n32, rem);
        __syncthreads();
    }
    const int rem8 = rem & ~7;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const float* qa = sa[ta];
        const float* qb = sb[tb + 16 * p];
        for (int u = 0; u < rem8; u += 8)   // 8-float steps into accumulator 0
#pragma unroll
            for (int h = 0; h < 4; ++h) step(acc[p][0][h], qa, qb, u + 2 * h);
        float s[8];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            s[2 * h] = __fadd_rn(__fadd_rn(acc[p][0][h].x, acc[p][1][h].x), __fadd_rn(acc[p][2][h].x, acc[p][3][h].x));
            s[2 * h + 1] =
                __fadd_rn(__fadd_rn(acc[p][0][h].y, acc[p][1][h].y), __fadd_rn(acc[p][2][h].y, acc[p][3][h].y));
        }
        float r = __fadd_rn(__fadd_rn(__fadd_rn(s[0], s[4]), __fadd_rn(s[1], s[5])),
                            __fadd_rn(__fadd_rn(s[2], s[6]), __fadd_rn(s[3], s[7])));
        r = exact_tail<!kIP>(qa, qb, rem8, rem, r);   // the n % 8 tail as the reference build computes it
        const int gi = a0 + ta, gj = b0 + tb + 16 * p;
        if (gi < na && gj < nb) out[static_cast<size_t>(gi) * ld_out + gj] = kIP ? -r : r;
    }
}

void pair_scores(const float* A, int na, const float* B, int nb, int d, bool ip, float* out, size_t ld_out,
                 cudaStream_t st) {
    if (na == 0 || nb == 0) return;
    dim3 grid(static_cast<unsigned>(ceil_div(nb, kTB)), static_cast<unsigned>(ceil_div(na, kTA)));
    KernelTimer kt("pair_scores", st);
    if (ip) k_pair_scores<true><<<grid, 256, 0, st>>>(A, na, B, nb, d, out, ld_out);
    else k_pair_scores<false><<<grid, 256, 0, st>>>(A, na, B, nb, d, out, ld_out);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// The P smallest of each row by (key(score), column), sorted. One block per
// row: a 4-pass radix select finds the P-th key T, an ordered compaction takes
// every key < T and the first ties at T in column order, then a bitonic sort.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool col_allowed(const uint64_t* allow, const uint64_t* deny, size_t c) {
    return (!allow || ((allow[c >> 6] >> (c & 63)) & 1ull)) && (!deny || !((deny[c >> 6] >> (c & 63)) & 1ull));
}

// Columns refused by allow / deny (bitmaps over col_base + column, either may
// be null) rank last and come out as column 0xFFFFFFFF with score +inf.
// With `staged`, the row's keys are formed once into shared memory (ncols
// words after the P slots) and every pass reads them there: for the small
// batches of serving, whose few blocks would otherwise wait on L2 once per pass.
__global__ void __launch_bounds__(1024) k_select_rows(const float* __restrict__ scores, size_t ld, int ncols, int P,
                                                      const uint64_t* __restrict__ allow, const uint64_t* __restrict__ deny,
                                                      size_t col_base, bool eq0, bool staged, uint32_t* __restrict__ out_col,
                                                      float* __restrict__ out_score) {
    extern __shared__ uint8_t sm_raw[];
    const int Pp = next_pow2(P);
    uint64_t* skey = reinterpret_cast<uint64_t*>(sm_raw);
    int64_t* sval = reinterpret_cast<int64_t*>(skey + Pp);
    uint32_t* rkey = reinterpret_cast<uint32_t*>(sval + Pp);   // staged: the row's keys
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_mask, s_remaining;
    __shared__ uint32_t warp_cnt[2][32];
    const float* row = scores + static_cast<size_t>(blockIdx.x) * ld;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_prefix = 0;
        s_mask = 0;
        s_remaining = static_cast<uint32_t>(P);
    }
    auto key_of = [&](int c) -> uint32_t {
        return col_allowed(allow, deny, col_base + c) ? (eq0 ? float_key_eq0(row[c]) : float_key(row[c])) : 0xFFFFFFFFu;
    };
    if (staged)
        for (int c = tid; c < ncols; c += blockDim.x) rkey[c] = key_of(c);   // (the first pass's barrier orders these)
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = tid; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        const uint32_t prefix = s_prefix, mask = s_mask;
        for (int c0 = 0; c0 < ncols; c0 += blockDim.x) {   // (trip count block-uniform)
            const int c = c0 + tid;
            const uint32_t k = c < ncols ? (staged ? rkey[c] : key_of(c)) : 0xFFFFFFFFu;
            const int bin = c < ncols && (k & mask) == prefix ? static_cast<int>((k >> shift) & 255u) : -1;
            // lanes of a warp that share a bin add once (early passes put most keys in a few bins)
            const unsigned same = __match_any_sync(0xffffffffu, bin);
            if (bin >= 0 && (tid & 31) == __ffs(same) - 1) atomicAdd(&hist[bin], static_cast<uint32_t>(__popc(same)));
        }
        __syncthreads();
        if (tid < 32) {   // warp 0: the bin holding the remaining-th key, lane l owning bins 8 l .. 8 l + 7
            const uint32_t rem = s_remaining;
            uint32_t cb[8], own = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                cb[j] = hist[8 * tid + j];
                own += cb[j];
            }
            uint32_t incl = own;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= o) incl += t;
            }
            const uint32_t excl = incl - own;
            if (excl < rem && rem <= incl) {
                uint32_t left = rem - excl, b = 8 * tid + 7;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (cb[j] >= left) {
                        b = 8 * tid + j;
                        break;
                    }
                    left -= cb[j];
                }
                s_remaining = left;
                s_prefix = prefix | (b << shift);
                s_mask = mask | (255u << shift);
            }
        }
        __syncthreads();
    }
    const uint32_t T = s_prefix;
    const uint32_t need_eq = s_remaining;   // ties at T to take, in column order
    // the P columns: keys below T, then the first need_eq ties at T in column
    // order. Each warp owns a contiguous run of columns: it counts its own,
    // the warps' counts give each one its offsets, and it writes in order.
    const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    const int span = ((ncols + nwarps - 1) / nwarps + 31) & ~31;
    const int c_begin = min(ncols, warp * span), c_end = min(ncols, c_begin + span);
    auto key_at = [&](int c) -> uint32_t { return staged ? rkey[c] : key_of(c); };
    uint32_t n_lt = 0, n_eq = 0;
    for (int c0 = c_begin; c0 < c_end; c0 += 32) {
        const int c = c0 + lane;
        const uint32_t k = c < c_end ? key_at(c) : 0xFFFFFFFFu;
        n_lt += __popc(__ballot_sync(0xffffffffu, c < c_end && k < T));
        n_eq += __popc(__ballot_sync(0xffffffffu, c < c_end && k == T));
    }
    if (lane == 0) {
        warp_cnt[0][warp] = n_lt;
        warp_cnt[1][warp] = n_eq;
    }
    __syncthreads();
    uint32_t off_lt = 0, off_eq = 0;
    for (int w = 0; w < warp; ++w) {
        off_lt += warp_cnt[0][w];
        off_eq += warp_cnt[1][w];
    }
    const uint32_t below = (1u << lane) - 1u;
    for (int c0 = c_begin; c0 < c_end; c0 += 32) {
        const int c = c0 + lane;
        const uint32_t k = c < c_end ? key_at(c) : 0xFFFFFFFFu;
        const bool lt = c < c_end && k < T;
        const bool eq = c < c_end && k == T;
        const uint32_t blt = __ballot_sync(0xffffffffu, lt), beq = __ballot_sync(0xffffffffu, eq);
        if (lt) {
            const uint32_t pos = off_lt + __popc(blt & below);
            skey[pos] = static_cast<uint64_t>(k);
            sval[pos] = c;
        }
        if (eq) {
            const uint32_t r = off_eq + __popc(beq & below);
            if (r < need_eq) {
                const uint32_t pos = (static_cast<uint32_t>(P) - need_eq) + r;
                skey[pos] = static_cast<uint64_t>(k);
                sval[pos] = c;
            }
        }
        off_lt += __popc(blt);
        off_eq += __popc(beq);
    }
    // in (key, column) order: up to 1,024 of them, each one's rank is the count
    // of smaller pairs (all distinct) and it goes straight to its place, with
    // no sorting stages; beyond that a bitonic sort
    if (P <= 1024) {   // (block-uniform)
        __syncthreads();
        for (int i = tid; i < P; i += blockDim.x) {
            const uint64_t ki = skey[i];
            const int64_t vi = sval[i];
            int rank = 0;
            for (int j = 0; j < P; ++j) rank += pair_less(skey[j], sval[j], ki, vi);
            const uint32_t col = static_cast<uint32_t>(vi);
            const bool ok = col_allowed(allow, deny, col_base + col);
            out_col[static_cast<size_t>(blockIdx.x) * P + rank] = ok ? col : 0xFFFFFFFFu;
            out_score[static_cast<size_t>(blockIdx.x) * P + rank] = ok ? row[col] : __int_as_float(0x7f800000);
        }
        return;
    }
    for (int i = P + tid; i < Pp; i += blockDim.x) {
        skey[i] = ~0ull;
        sval[i] = INT64_MAX;
    }
    bitonic_sort(skey, sval, Pp);
    for (int i = tid; i < P; i += blockDim.x) {
        const uint32_t col = static_cast<uint32_t>(sval[i]);
        const bool ok = col_allowed(allow, deny, col_base + col);
        out_col[static_cast<size_t>(blockIdx.x) * P + i] = ok ? col : 0xFFFFFFFFu;
        out_score[static_cast<size_t>(blockIdx.x) * P + i] =
            ok ? row[col] : __int_as_float(0x7f800000);
    }
}

// select_rows for P = 1: a warp per row keeps the smallest (key, column)
// pair of its row (a column that is not allowed has the all-ones key, as in
// k_select_rows) and writes its column and score, or -1 and +inf when the
// pick is not allowed.
__global__ void __launch_bounds__(256) k_select_min_rows(const float* __restrict__ scores, size_t ld, int nrows,
                                                         int ncols, const uint64_t* __restrict__ allow,
                                                         const uint64_t* __restrict__ deny, size_t col_base, bool eq0,
                                                         uint32_t* __restrict__ out_col, float* __restrict__ out_score) {
    const int r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= nrows) return;
    const float* row = scores + static_cast<size_t>(r) * ld;
    uint64_t best = ~0ull;
    for (int c = lane; c < ncols; c += 32) {
        const uint32_t k = col_allowed(allow, deny, col_base + c) ? (eq0 ? float_key_eq0(row[c]) : float_key(row[c]))
                                                                  : 0xFFFFFFFFu;
        const uint64_t kc = (static_cast<uint64_t>(k) << 32) | static_cast<uint32_t>(c);
        best = kc < best ? kc : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint32_t lo = __shfl_xor_sync(0xffffffffu, static_cast<uint32_t>(best), o);
        const uint32_t hi = __shfl_xor_sync(0xffffffffu, static_cast<uint32_t>(best >> 32), o);
        const uint64_t other = (static_cast<uint64_t>(hi) << 32) | lo;
        best = other < best ? other : best;
    }
    if (lane == 0) {
        const uint32_t col = static_cast<uint32_t>(best);
        const bool ok = ncols > 0 && col_allowed(allow, deny, col_base + col);
        out_col[r] = ok ? col : 0xFFFFFFFFu;
        out_score[r] = ok ? row[col] : __int_as_float(0x7f800000);
    }
}

void select_rows(const float* scores, size_t ld, int nrows, int ncols, int P, uint32_t* out_col, float* out_score,
                 cudaStream_t st, const uint64_t* allow, const uint64_t* deny, size_t col_base, bool eq0) {
    if (nrows > 0 && P == 1) {
        KernelTimer kt("select_rows", st);
        k_select_min_rows<<<static_cast<unsigned>(ceil_div(static_cast<size_t>(nrows), 8)), 256, 0, st>>>(
            scores, ld, nrows, ncols, allow, deny, col_base, eq0, out_col, out_score);
        QG_LAUNCH_CHECK();
        return;
    }
    if (nrows == 0) return;
    // few rows (serving's small batches): 1,024 threads a row and the row's
    // keys staged in shared memory; many rows: 256 threads, keys from L2
    const bool few = nrows < 2 * sm_count();
    const size_t base = static_cast<size_t>(next_pow2(P)) * 16;
    const bool staged = few && base + static_cast<size_t>(ncols) * 4 <= 160 * 1024;
    const size_t smem = base + (staged ? static_cast<size_t>(ncols) * 4 : 0);
    if (smem > 48 * 1024)
        allow_large_smem<k_select_rows>();
    KernelTimer kt("select_rows", st);
    k_select_rows<<<nrows, few ? 1024 : 256, smem, st>>>(scores, ld, ncols, P, allow, deny, col_base, eq0, staged,
                                                          out_col, out_score);
    QG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Per-probe distance terms.
//   mode L2 / L2-ADC : A (the probe's exact coarse distance, or the exact
//                      distance to the list's residual center when the index has them)
//   mode IP          : offset term = A = -(q . c)
//   mode cosine-IP   : base = (A + 1) - |e|^2 (reference src/ivf_index.cpp:577-579)
// ---------------------------------------------------------------------------
// One (query, probe) pair per lane group of G: the exact distance to the
// list's residual center in exact_avx2's order, by 8 lanes (each reads its
// row as 32-byte segments, so the rows cross L2 once) or, for rows of an even
// dim at 8-byte alignment, by 4 (each lane two AVX2 lanes, one 32-byte sector
// of the row per group step; half the lane instructions).
template <int G>
__global__ void k_probe_terms(IvfView v, const float* __restrict__ q, int nq, int P, const uint32_t* __restrict__ probe,
                              const float* __restrict__ pdist, float* __restrict__ term) {
    static_assert(G == 4 || G == 8, "lane groups of 4 or 8");
    const size_t n = static_cast<size_t>(nq) * P;
    const size_t i0 = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
    const bool in = i0 < n;   // (whole warps call the group scorer together)
    const size_t i = in ? i0 : 0;
    const int qi = static_cast<int>(i / P);
    const uint32_t list = probe[i];
    float A = pdist[i];
    if (v.has_resid) {
        const float* qa = q + static_cast<size_t>(qi) * v.dim;
        const float* rc = v.resid + static_cast<size_t>(list) * v.dim;
        A = G == 4 ? exact_avx2_group4<true>(qa, rc, v.dim) : exact_avx2_group8<true, true>(qa, rc, v.dim);
    }
    if (v.mode == kModeCosIP) A = __fsub_rn(__fadd_rn(A, 1.0f), v.sqnorm[list]);
    if (in && (threadIdx.x & (G - 1)) == 0) term[i] = A;
}

// ---------------------------------------------------------------------------
// Per-query tables: C (mode L2, reference src/pq.cpp:186-204), or the inner
// table rounded to the query's uint8 LUT (modes IP / cosine-IP; IP halves the
// table first, reference src/ivf_index.cpp:448-456). One block per query.
// ---------------------------------------------------------------------------
__global__ void k_query_tables(IvfView v, const float* __restrict__ q, float* __restrict__ qC, uint4* __restrict__ qlut,
                               float* __restrict__ qscale, float* __restrict__ qoffset) {
    extern __shared__ float tab[];   // m * 16 floats, then m floats of row minimums
    const int qi = blockIdx.x;
    const float* qv = q + static_cast<size_t>(qi) * v.dim;
    const int T = v.m * 16;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        float c = inner_term(qv, v.pq_t, t >> 4, v.sd, 16, t & 15);
        if (v.mode == kModeIP) c = __fmul_rn(c, 0.5f);
        tab[t] = c;
        if (v.mode == kModeL2) qC[static_cast<size_t>(qi) * T + t] = c;
    }
    if (v.mode == kModeL2 || v.mode == kModeL2Adc) return;
    __syncthreads();
    if (threadIdx.x < 32) {
        float s, o;
        warp_quantize_lut(
            [&](int r, float* out) {
#pragma unroll
                for (int j = 0; j < 16; ++j) out[j] = tab[r * 16 + j];
            },
            v.m, v.m_pad, tab + T, qlut + static_cast<size_t>(qi) * v.m_pad, s, o);
        if (threadIdx.x == 0) {
            qscale[qi] = s;
            qoffset[qi] = o;
        }
    }
}

// ---------------------------------------------------------------------------
// Merge: the k' smallest key64 of a query's chunk outputs, sorted. The buffer
// holds the current best k' and the next batch of entries.
// ---------------------------------------------------------------------------
// The k' best of a query's chunk lists (each sorted, ~0 for empty entries):
// a block-wide radix select of the k'-th smallest valid key, 8 bits a pass
// from the top and stopping once every key of the chosen bin is kept, then
// the survivors compacted and sorted. One block per query.
// ---------------------------------------------------------------------------
// Every pass reads 4 keys a thread before it bins them, so that the loads of
// a pass (from L2) overlap instead of each waiting for the last.
__global__ void __launch_bounds__(1024) k_merge(const uint64_t* __restrict__ in_key, const uint32_t* __restrict__ in_slot,
                                                int nchunks, int kp, int npow, uint64_t* __restrict__ out_key,
                                                uint32_t* __restrict__ out_slot) {
    extern __shared__ uint8_t sm_raw[];
    uint64_t* key = reinterpret_cast<uint64_t*>(sm_raw);   // npow
    int64_t* val = reinterpret_cast<int64_t*>(key + npow);
    __shared__ int hist[256], s_pick[3], s_valid, s_count;
    const int qi = blockIdx.x;
    const int total = nchunks * kp;
    const uint64_t* ik = in_key + static_cast<size_t>(qi) * total;
    const uint32_t* is = in_slot + static_cast<size_t>(qi) * total;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_valid = 0;
        s_count = 0;
    }
    __syncthreads();
    constexpr int U = 4;   // keys in flight per thread
    const int step = U * blockDim.x;
    int mine = 0;
    for (int b0 = 0; b0 < total; b0 += step) {
        uint64_t kk[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = b0 + u * blockDim.x + threadIdx.x;
            kk[u] = e < total ? ik[e] : ~0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) mine += kk[u] != ~0ull;
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if (lane == 0) atomicAdd(&s_valid, mine);
    __syncthreads();
    uint64_t lim = ~0ull - 1;   // every valid key
    if (s_valid > kp) {
        uint64_t prefix = 0, mask = 0;
        int need = kp, shift = 56;
        for (;; shift -= 8) {
            for (int j = threadIdx.x; j < 256; j += blockDim.x) hist[j] = 0;
            __syncthreads();
            for (int b0 = 0; b0 < total; b0 += step) {   // (trip count is block-uniform)
                uint64_t kk[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = b0 + u * blockDim.x + threadIdx.x;
                    kk[u] = e < total ? ik[e] : ~0ull;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint64_t k = kk[u];
                    const bool in = k != ~0ull && (k & mask) == prefix;
                    const int bin = in ? static_cast<int>((k >> shift) & 255) : -1;
                    const unsigned same = __match_any_sync(0xffffffffu, bin);
                    if (in && lane == __ffs(same) - 1) atomicAdd(&hist[bin], __popc(same));
                }
            }
            __syncthreads();
            if (threadIdx.x < 32) {
                int c[8], own = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    c[j] = hist[8 * lane + j];
                    own += c[j];
                }
                int incl = own;
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const int excl = incl - own;
                if (excl < need && need <= incl) {
                    int acc = excl;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        if (acc + c[j] >= need) {
                            s_pick[0] = 8 * lane + j;
                            s_pick[1] = acc;
                            s_pick[2] = c[j];
                            break;
                        }
                        acc += c[j];
                    }
                }
            }
            __syncthreads();
            need -= s_pick[1];
            prefix |= static_cast<uint64_t>(s_pick[0]) << shift;
            mask |= 0xFFull << shift;
            const bool done = s_pick[2] == need || shift == 0;
            __syncthreads();
            if (done) break;
        }
        lim = prefix | ((1ull << shift) - 1);
    }
    // the survivors (at most kp), then sorted
    for (int b0 = 0; b0 < total; b0 += step) {
        uint64_t kk[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = b0 + u * blockDim.x + threadIdx.x;
            kk[u] = e < total ? ik[e] : ~0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = b0 + u * blockDim.x + threadIdx.x;
            if (kk[u] != ~0ull && kk[u] <= lim) {
                const int pos = atomicAdd(&s_count, 1);
                if (pos < npow) {
                    key[pos] = kk[u];
                    val[pos] = static_cast<int64_t>(is[e]);
                }
            }
        }
    }
    __syncthreads();
    for (int i = min(s_count, npow) + threadIdx.x; i < npow; i += blockDim.x) {
        key[i] = ~0ull;
        val[i] = INT64_MAX;
    }
    bitonic_sort(key, val, npow);
    for (int i = threadIdx.x; i < kp; i += blockDim.x) {
        out_key[static_cast<size_t>(qi) * kp + i] = key[i];
        out_slot[static_cast<size_t>(qi) * kp + i] = key[i] == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(val[i]);
    }
}

// ---------------------------------------------------------------------------
// IVF results: the first k of the k' list, sorted by (distance key, id) as
// take_sorted does (reference src/topk.hpp:53-77), ids mapped through labels.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_finalize_ivf(const uint64_t* __restrict__ key_in, const uint32_t* __restrict__ slot_in,
                                                      int kp, int k, const int64_t* __restrict__ labels, bool cosine,
                                                      int64_t* __restrict__ out_ids, float* __restrict__ out_d,
                                                      const int* __restrict__ k_q) {
    extern __shared__ uint8_t sm_raw[];
    const int kpow = max(2, next_pow2(k));
    uint64_t* key = reinterpret_cast<uint64_t*>(sm_raw);
    int64_t* val = reinterpret_cast<int64_t*>(key + kpow);
    const int qi = blockIdx.x;
    const int kq = k_q ? min(k_q[qi], k) : k;   // the query's first kq candidates by key64
    for (int i = threadIdx.x; i < kpow; i += blockDim.x) {
        const uint64_t k64 = i < kq && i < kp ? key_in[static_cast<size_t>(qi) * kp + i] : ~0ull;
        if (k64 == ~0ull) {
            key[i] = ~0ull;
            val[i] = INT64_MAX;
        } else {
            const uint32_t slot = slot_in[static_cast<size_t>(qi) * kp + i];
            key[i] = k64 >> 32;
            val[i] = labels ? labels[slot] : static_cast<int64_t>(slot);
        }
    }
    bitonic_sort(key, val, kpow);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const size_t o = static_cast<size_t>(qi) * k + i;
        if (key[i] == ~0ull) {
            out_ids[o] = -1;
            out_d[o] = __int_as_float(0x7f800000);
        } else {
            const float d = key_float(static_cast<uint32_t>(key[i]));
            out_ids[o] = val[i];
            out_d[o] = cosine ? __fmul_rn(d, 0.5f) : d;
        }
    }
}

// ---------------------------------------------------------------------------
// Re-rank (reference src/refine_index.cpp:112-140): the exact score of every
// candidate from the raw rows, then the k smallest by (score, slot), compared
// as floats (so -0 == +0), ids mapped through the refine index's labels.
// Two kernels: every candidate of the batch scored at once, an 8-lane group
// per candidate reading its row with 128-byte loads (so a batch of one query
// spreads its gathers over the whole GPU as a large batch does), each score
// kept as key(score) << 32 | slot; then per query those keys sorted.
// ---------------------------------------------------------------------------
template <bool kIP, int G>
__global__ void __launch_bounds__(256) k_refine_scores(const float* __restrict__ q, int dim,
                                                       const float* __restrict__ rows,
                                                       const uint64_t* __restrict__ key_in,
                                                       const uint32_t* __restrict__ slot_in, int nq, int kp,
                                                       const int* __restrict__ kp_q, uint64_t* __restrict__ scored) {
    static_assert(G == 4 || G == 8, "lane groups of 4 or 8");
    const size_t g = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;   // candidate, query-major
    const size_t total = static_cast<size_t>(nq) * kp;
    // whole G-lane groups take part in the shuffles; groups past the end, and
    // empty candidates, score the query against itself unused
    const bool in = g < total;
    const size_t gi = in ? g : 0;
    const int qi = static_cast<int>(gi / kp), c = static_cast<int>(gi % kp);
    const int kpq = kp_q ? min(kp_q[qi], kp) : kp;   // the query's first kpq candidates by key64
    const bool ok = in && c < kpq && key_in[gi] != ~0ull;
    const uint32_t sl = ok ? slot_in[gi] : 0u;
    const float* qv = q + static_cast<size_t>(qi) * dim;
    const float* row = ok ? rows + static_cast<size_t>(sl) * dim : qv;
    float d;
    if constexpr (G == 4) d = kIP ? -exact_avx2_group4<false>(qv, row, dim) : exact_avx2_group4<true>(qv, row, dim);
    else d = kIP ? -exact_avx2_group8<false, true>(qv, row, dim) : exact_avx2_group8<true, true>(qv, row, dim);
    if (in && (threadIdx.x & (G - 1)) == 0)
        scored[gi] = ok ? (static_cast<uint64_t>(float_key_eq0(d)) << 32) | sl : ~0ull;
}

__global__ void __launch_bounds__(1024) k_refine_select(const float* __restrict__ q, int dim,
                                                        const float* __restrict__ rows,
                                                        const uint64_t* __restrict__ scored, int kp, int k, bool ip,
                                                        const int64_t* __restrict__ labels, bool cosine,
                                                        int64_t* __restrict__ out_ids, float* __restrict__ out_d,
                                                        const int* __restrict__ k_q) {
    extern __shared__ uint64_t rkey[];
    const int kpow = max(2, next_pow2(kp));
    const int qi = blockIdx.x;
    const int kq = k_q ? min(k_q[qi], k) : k;
    for (int i = threadIdx.x; i < kpow; i += blockDim.x)
        rkey[i] = i < kp ? scored[static_cast<size_t>(qi) * kp + i] : ~0ull;
    bitonic_sort_keys(rkey, kpow);
    const float* qv = q + static_cast<size_t>(qi) * dim;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const size_t o = static_cast<size_t>(qi) * k + i;
        if (i >= kq || rkey[i] == ~0ull) {
            out_ids[o] = -1;
            out_d[o] = __int_as_float(0x7f800000);
        } else {
            const uint32_t slot = static_cast<uint32_t>(rkey[i]);
            // recompute: float_key_eq0 folded -0 into +0, and the reference returns the value itself
            const float d = exact_score(qv, rows + static_cast<size_t>(slot) * dim, dim, ip);
            out_ids[o] = labels ? labels[slot] : static_cast<int64_t>(slot);
            out_d[o] = cosine ? __fmul_rn(d, 0.5f) : d;
        }
    }
}

// k_refine_select for kp <= 256 K with 8 warps: each warp sorts a run of up
// to 32 K candidate keys in registers; a key's rank is then the number of
// keys below it in each run (binary searches over the sorted runs; its own run
// counts its place in it), and the keys of rank below k are written at their
// rank. The keys are unique but for the all-ones key of empty candidates,
// which takes no place. One block barrier, where the bitonic sort takes one per
// stage.
template <int K>
__global__ void __launch_bounds__(256) k_refine_select_ranked(const float* __restrict__ q, int dim,
                                                              const float* __restrict__ rows,
                                                              const uint64_t* __restrict__ scored, int kp, int k,
                                                              bool ip, const int64_t* __restrict__ labels, bool cosine,
                                                              int64_t* __restrict__ out_ids, float* __restrict__ out_d,
                                                              const int* __restrict__ k_q) {
    constexpr int R = 32 * K, NW = 8;
    __shared__ uint64_t rkey[NW * R];
    const int qi = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kq = k_q ? min(k_q[qi], k) : k;
    const uint64_t* src = scored + static_cast<size_t>(qi) * kp;
    uint64_t* run = rkey + R * warp;
    const int n_w = max(0, min(R, kp - R * warp));
    for (int i = lane; i < n_w; i += 32) run[i] = src[R * warp + i];
    __syncwarp();
    if (n_w > 0) warp_sort_keys_reg<K>(run, n_w);
    __syncthreads();
    auto below = [&](uint64_t key) {   // keys < key over all runs
        int rank = 0;
        for (int w = 0; w < NW; ++w) {
            const int len = max(0, min(R, kp - R * w));
            const uint64_t* rw = rkey + R * w;
            int pos = 0;
#pragma unroll
            for (int step = R; step > 0; step >>= 1)
                if (pos + step <= len && rw[pos + step - 1] < key) pos += step;
            rank += pos;
        }
        return rank;
    };
    const float* qv = q + static_cast<size_t>(qi) * dim;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int e = i * 32 + lane;
        if (e >= n_w) continue;
        const uint64_t key = run[e];
        if (key == ~0ull) continue;
        const int rank = below(key);
        if (rank >= kq) continue;
        const size_t o = static_cast<size_t>(qi) * k + rank;
        const uint32_t slot = static_cast<uint32_t>(key);
        // recompute: float_key_eq0 folded -0 into +0, and the reference returns the value itself
        const float d = exact_score(qv, rows + static_cast<size_t>(slot) * dim, dim, ip);
        out_ids[o] = labels ? labels[slot] : static_cast<int64_t>(slot);
        out_d[o] = cosine ? __fmul_rn(d, 0.5f) : d;
    }
    if (static_cast<int>(threadIdx.x) < k) {
        const int filled = min(kq, below(~0ull));   // places taken by real candidates
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            if (i >= filled) {
                out_ids[static_cast<size_t>(qi) * k + i] = -1;
                out_d[static_cast<size_t>(qi) * k + i] = __int_as_float(0x7f800000);
            }
    }
}

// ---------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------
void normalize_rows(const float* x, float* y, int n, int d, int* d_zero, cudaStream_t st) {
    if (n == 0) return;
    k_normalize<<<static_cast<unsigned>(ceil_div(n, 128)), 128, 0, st>>>(x, y, n, d, d_zero);
    QG_LAUNCH_CHECK();
}

// Rows times an orthonormal rotation (reference src/rotation.cpp:165-187):
// out[i][j] accumulates fma(x[i][k], R[k][j], acc) for k = 0..d-1 in order,
// from +0. A block computes 32 rows x 32 columns, staging 32-deep slices of
// the rows and of R in shared memory; each thread owns 4 rows of one column.
__global__ void __launch_bounds__(256) k_rotate(const float* __restrict__ x, size_t n, int d,
                                                const float* __restrict__ R, float* __restrict__ out) {
    __shared__ float xs[32][33];
    __shared__ float rs[32][32];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const size_t r0 = static_cast<size_t>(blockIdx.x) * 32;
    const int c0 = blockIdx.y * 32;
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int k0 = 0; k0 < d; k0 += 32) {
        for (int t = threadIdx.x; t < 32 * 32; t += 256) {
            const int a = t >> 5, b = t & 31;
            const size_t row = r0 + a;
            xs[a][b] = row < n && k0 + b < d ? x[row * d + k0 + b] : 0.0f;
            rs[a][b] = k0 + a < d && c0 + b < d ? R[static_cast<size_t>(k0 + a) * d + c0 + b] : 0.0f;
        }
        __syncthreads();
        const int kn = min(32, d - k0);   // no padded terms: fma(0, r, -0) would turn -0 into +0
        for (int kk = 0; kk < kn; ++kk) {
            const float rv = rs[kk][tx];
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = __fmaf_rn(xs[ty * 4 + i][kk], rv, acc[i]);
        }
        __syncthreads();
    }
    const int c = c0 + tx;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const size_t row = r0 + ty * 4 + i;
        if (row < n && c < d) out[row * d + c] = acc[i];
    }
}

void rotate_rows(const float* R, const float* x, size_t n, int d, float* out, cudaStream_t st) {
    if (n == 0) return;
    const dim3 grid(static_cast<unsigned>(ceil_div(n, 32)), static_cast<unsigned>(ceil_div(d, 32)));
    k_rotate<<<grid, 256, 0, st>>>(x, n, d, R, out);
    QG_LAUNCH_CHECK();
}


void probe_terms(const IvfView& v, const float* q, int nq, int P, const uint32_t* probe, const float* pdist, float* term,
                 cudaStream_t st) {
    const size_t n = static_cast<size_t>(nq) * P;
    if (n == 0) return;
    KernelTimer kt("probe_terms", st);
    const bool g4 = v.has_resid && (v.dim & 1) == 0 && (reinterpret_cast<uintptr_t>(q) & 7) == 0 &&
                    (reinterpret_cast<uintptr_t>(v.resid) & 7) == 0;
    if (g4) k_probe_terms<4><<<static_cast<unsigned>(ceil_div(n * 4, 256)), 256, 0, st>>>(v, q, nq, P, probe, pdist, term);
    else k_probe_terms<8><<<static_cast<unsigned>(ceil_div(n * 8, 256)), 256, 0, st>>>(v, q, nq, P, probe, pdist, term);
    QG_LAUNCH_CHECK();
}

void query_tables(const IvfView& v, const float* q, int nq, float* qC, uint4* qlut, float* qscale, float* qoffset,
                  cudaStream_t st) {
    if (nq == 0) return;
    const size_t smem = static_cast<size_t>(v.m) * 17 * 4;
    if (smem > 48 * 1024)
        allow_large_smem<k_query_tables>();
    KernelTimer kt("query_tables", st);
    k_query_tables<<<nq, 128, smem, st>>>(v, q, qC, qlut, qscale, qoffset);
    QG_LAUNCH_CHECK();
}

void merge_candidates(const uint64_t* in_key, const uint32_t* in_slot, int nq, int nchunks, int kp, uint64_t* out_key,
                      uint32_t* out_slot, cudaStream_t st) {
    if (nq == 0) return;
    const int npow = next_pow2(std::max(2, kp));
    const size_t msm = static_cast<size_t>(npow) * 16;
    if (msm > 48 * 1024)
        allow_large_smem<k_merge>();
    KernelTimer kt("merge", st);
    // few queries (serving's small batches): 1,024 threads a query
    k_merge<<<nq, nq < 2 * sm_count() ? 1024 : 256, msm, st>>>(in_key, in_slot, nchunks, kp, npow, out_key, out_slot);
    QG_LAUNCH_CHECK();
}

void finalize_ivf(const uint64_t* key, const uint32_t* slot, int nq, int kp, int k, const int64_t* labels, bool cosine,
                  int64_t* out_ids, float* out_d, cudaStream_t st, const int* k_q) {
    if (nq == 0 || k == 0) return;
    const int kpow = std::max(2, next_pow2(k));
    k_finalize_ivf<<<nq, 128, static_cast<size_t>(kpow) * 16, st>>>(key, slot, kp, k, labels, cosine, out_ids, out_d,
                                                                      k_q);
    QG_LAUNCH_CHECK();
}

void refine_candidates(const float* q, int nq, int dim, const float* rows, const uint64_t* key, const uint32_t* slot,
                       int kp, int k, bool ip, const int64_t* labels, bool cosine, int64_t* out_ids, float* out_d,
                       cudaStream_t st, const int* kp_q, const int* k_q) {
    if (nq == 0 || k == 0) return;
    const int kpow = std::max(2, next_pow2(kp));
    const size_t ssm = static_cast<size_t>(kpow) * 8;
    require(ssm <= 200 * 1024, "re-rank shared memory exceeds the B200 limit for this k * k_factor", kUnsupported);
    const size_t total = static_cast<size_t>(nq) * kp;
    DevBuf<uint64_t> scored(total, st);
    KernelTimer kt("refine", st);
    // rows of an even dim at 8-byte alignment: one candidate per 4-lane group
    const bool g4 = (dim & 1) == 0 && (reinterpret_cast<uintptr_t>(q) & 7) == 0 &&
                    (reinterpret_cast<uintptr_t>(rows) & 7) == 0;
    const unsigned blocks = static_cast<unsigned>(ceil_div(total * (g4 ? 4 : 8), size_t{256}));
    if (g4 && ip)
        k_refine_scores<true, 4><<<blocks, 256, 0, st>>>(q, dim, rows, key, slot, nq, kp, kp_q, scored.get());
    else if (g4)
        k_refine_scores<false, 4><<<blocks, 256, 0, st>>>(q, dim, rows, key, slot, nq, kp, kp_q, scored.get());
    else if (ip)
        k_refine_scores<true, 8><<<blocks, 256, 0, st>>>(q, dim, rows, key, slot, nq, kp, kp_q, scored.get());
    else
        k_refine_scores<false, 8><<<blocks, 256, 0, st>>>(q, dim, rows, key, slot, nq, kp, kp_q, scored.get());
    QG_LAUNCH_CHECK();
    if (ssm > 48 * 1024)
        allow_large_smem<k_refine_select>();
    if (kp <= 256) {
        k_refine_select_ranked<1><<<nq, 256, 0, st>>>(q, dim, rows, scored.get(), kp, k, ip, labels, cosine, out_ids,
                                                       out_d, k_q);
    } else if (kp <= 512) {
        k_refine_select_ranked<2><<<nq, 256, 0, st>>>(q, dim, rows, scored.get(), kp, k, ip, labels, cosine, out_ids,
                                                       out_d, k_q);
    } else {
        // few queries (serving's small batches): 1,024 threads a query for the sort
        const int threads = nq < 2 * sm_count() ? 1024 : 256;
        k_refine_select<<<nq, threads, ssm, st>>>(q, dim, rows, scored.get(), kp, k, ip, labels, cosine, out_ids,
                                                  out_d, k_q);
    }
    QG_LAUNCH_CHECK();
}

} // namespace qg
