// Device building blocks of the search path: block-wide bitonic sort, the
// bit-exact uint8 LUT quantisation, the reference's PQ table terms, and the
// register-resident 4-bit lookup of the code scan.
#pragma once

#include "qg_common.cuh"

namespace qg {

inline constexpr int kLutMax = 63;   // reference src/fast_scan.hpp:36-39

// ---------------------------------------------------------------------------
// Block-wide bitonic sort of n (a power of two) (key, val) pairs in shared
// memory, ascending by (key, val). Every thread of the block must call it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool pair_less(uint64_t ka, int64_t va, uint64_t kb, int64_t vb) {
    return ka < kb || (ka == kb && va < vb);
}

__device__ __noinline__ static void bitonic_sort(uint64_t* key, int64_t* val, int n) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int t = threadIdx.x; t < (n >> 1); t += blockDim.x) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t k0 = key[lo], k1 = key[hi];
                const int64_t v0 = val[lo], v1 = val[hi];
                const bool swap = up ? pair_less(k1, v1, k0, v0) : pair_less(k0, v0, k1, v1);
                if (swap) {
                    key[lo] = k1; key[hi] = k0;
                    val[lo] = v1; val[hi] = v0;
                }
            }
        }
    }
    __syncthreads();
}

// Keys only (unique keys need no tie-break).
__device__ __noinline__ static void bitonic_sort_keys(uint64_t* key, int n) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int t = threadIdx.x; t < (n >> 1); t += blockDim.x) {
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
    __syncthreads();
}

// One warp sorts n <= 32 * K keys in registers (a network of 32 * K, the
// places past n holding all-ones keys that sort last): element
// e = i * 32 + lane sits in register i of lane `lane`. Partners within a
// lane's registers compare in place, partners across lanes through two 32-bit
// shuffles; no block barrier. Keys in shared memory, read and written by the
// calling warp only (the caller orders them with the other warps).
template <int K>
__device__ __forceinline__ void warp_sort_keys_reg(uint64_t* key, int n) {
    const int lane = threadIdx.x & 31;
    uint64_t r[K];
#pragma unroll
    for (int i = 0; i < K; ++i) r[i] = i * 32 + lane < n ? key[i * 32 + lane] : ~0ull;
    constexpr int N = 32 * K;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {   // partners in this lane's registers
                const int rs = stride >> 5;
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    if (i & rs) continue;
                    const int e = i * 32 + lane;
                    const bool up = (e & size) == 0;
                    const uint64_t a = r[i], b = r[i | rs];
                    const bool sw = up ? (b < a) : (a < b);
                    r[i] = sw ? b : a;
                    r[i | rs] = sw ? a : b;
                }
            } else {              // partners in lane ^ stride
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    const int e = i * 32 + lane;
                    const bool up = (e & size) == 0;
                    const uint32_t lo = __shfl_xor_sync(0xffffffffu, static_cast<uint32_t>(r[i]), stride);
                    const uint32_t hi = __shfl_xor_sync(0xffffffffu, static_cast<uint32_t>(r[i] >> 32), stride);
                    const uint64_t o = (static_cast<uint64_t>(hi) << 32) | lo;
                    const bool lower = (lane & stride) == 0;
                    const bool take_min = lower == up;
                    r[i] = take_min ? (o < r[i] ? o : r[i]) : (o > r[i] ? o : r[i]);
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < K; ++i)
        if (i * 32 + lane < n) key[i * 32 + lane] = r[i];
}

// warp_sort_keys_reg for n <= 256 keys; false (nothing done) when n is larger.
__device__ __forceinline__ bool warp_sort_keys(uint64_t* key, int n) {
    if (n <= 32) warp_sort_keys_reg<1>(key, n);
    else if (n <= 64) warp_sort_keys_reg<2>(key, n);
    else if (n <= 128) warp_sort_keys_reg<4>(key, n);
    else if (n <= 256) warp_sort_keys_reg<8>(key, n);
    else return false;
    __syncwarp();
    return true;
}

__host__ __device__ __forceinline__ int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// One warp keeps the `keep` smallest of the n distinct keys buf[0, n) in
// buf[0, keep) (in no particular order) and returns the largest kept key.
// Radix select, 8 bits at a time from the top: each pass counts the keys
// that share the prefix chosen so far by their next digit, and takes the
// digit whose bin holds the keep-th key; it stops once every key of that
// bin is kept. hist: 256 ints of warp-private shared scratch. n > keep >= 1.
__device__ __noinline__ static uint64_t warp_select_keep(uint64_t* buf, int n, int keep, int* hist) {
    const int lane = threadIdx.x & 31;
    constexpr unsigned kFull = 0xffffffffu;
    uint64_t prefix = 0, mask = 0;
    int need = keep;   // keys still to take among those that match the prefix
    int shift = 56;
    for (;; shift -= 8) {
#pragma unroll
        for (int j = 0; j < 8; ++j) hist[8 * lane + j] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const uint64_t k = buf[i];
            if ((k & mask) == prefix) atomicAdd(&hist[static_cast<int>(k >> shift) & 255], 1);
        }
        __syncwarp();
        int c[8], own = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            c[j] = hist[8 * lane + j];
            own += c[j];
        }
        int incl = own;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const int excl = incl - own;
        const unsigned owner = __ballot_sync(kFull, excl < need && need <= incl);
        const int ol = __ffs(owner) - 1;
        int digit = 0, below = 0, cnt = 0;
        if (lane == ol) {
            int acc = excl;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (cnt == 0 && acc + c[j] >= need) {
                    digit = 8 * lane + j;
                    below = acc;
                    cnt = c[j];
                }
                acc += c[j];
            }
        }
        digit = __shfl_sync(kFull, digit, ol);
        below = __shfl_sync(kFull, below, ol);
        cnt = __shfl_sync(kFull, cnt, ol);
        need -= below;
        prefix |= static_cast<uint64_t>(digit) << shift;
        mask |= 0xFFull << shift;
        __syncwarp();
        if (cnt == need || shift == 0) break;   // (at shift 0 the bin is one key)
    }
    // kept: every key whose bits above `shift` do not exceed the prefix
    const uint64_t lim = prefix | ((1ull << shift) - 1);
    int out = 0;
    uint64_t kmax = 0;
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        uint64_t k = 0;
        bool in = false;
        if (i < n) {
            k = buf[i];
            in = k <= lim;
        }
        const unsigned bal = __ballot_sync(kFull, in);
        __syncwarp();
        if (in) {
            buf[out + __popc(bal & ((1u << lane) - 1))] = k;
            kmax = k > kmax ? k : kmax;
        }
        out += __popc(bal);
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t t = __shfl_xor_sync(kFull, kmax, o);
        kmax = t > kmax ? t : kmax;
    }
    __syncwarp();
    return kmax;
}


// Keeps, in order, the keys of buf[0, n) at or below lim (by one warp, in
// place) and returns how many there are.
__device__ __noinline__ static int warp_keep_upto(uint64_t* buf, int n, uint64_t lim) {
    const int lane = threadIdx.x & 31;
    constexpr unsigned kFull = 0xffffffffu;
    int out = 0;
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        const uint64_t k = i < n ? buf[i] : ~0ull;
        const bool in = i < n && k <= lim;
        const unsigned bal = __ballot_sync(kFull, in);
        __syncwarp();
        if (in) buf[out + __popc(bal & ((1u << lane) - 1))] = k;
        out += __popc(bal);
    }
    __syncwarp();
    return out;
}

// ---------------------------------------------------------------------------
// Block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Rounding an m x 16 float table to uint8 entries, bit-exact with the
// reference's quantize_lut (reference src/fast_scan.cpp:18-46 scalar,
// :164-192 AVX2; both give the same bytes):
//   row minimum / maximum over its 16 entries (exact in any order),
//   widest = max over rows of (max - min),
//   scale  = 63 / widest (IEEE division), or 1 when every row is constant,
//   offset = (p0 + p1) + (p2 + p3), p[i % 4] summing the row minimums in row order,
//   lut    = round-half-even((x - min) * scale), subtract and multiply rounded apart.
// Implemented for one warp working on a table in shared memory; the LUT rows
// are written as four 32-bit words (entries 0-3, 4-7, 8-11, 12-15).
// row_min: m floats of warp-private shared scratch.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
    return static_cast<uint32_t>(a) | (static_cast<uint32_t>(b) << 8) | (static_cast<uint32_t>(c) << 16) |
           (static_cast<uint32_t>(d) << 24);
}

// The table row r is produced on demand by row(r, v) (16 floats), which lets
// callers fuse the table sum (B + C + A) into the rounding as the reference's
// build_quantize_lut does. Returns scale / offset to every lane.
template <class RowFn>
__device__ void warp_quantize_lut(RowFn row, int m, int m_pad, float* row_min, uint4* lut_out, float& scale_out,
                                  float& offset_out) {
    const int lane = threadIdx.x & 31;
    float widest = 0.0f;
    for (int r = lane; r < m; r += 32) {
        float v[16];
        row(r, v);
        float lo = v[0], hi = v[0];
#pragma unroll
        for (int j = 1; j < 16; ++j) {
            lo = fminf(lo, v[j]);
            hi = fmaxf(hi, v[j]);
        }
        row_min[r] = lo;
        const float w = __fsub_rn(hi, lo);
        widest = widest < w ? w : widest;   // std::max(widest, w)
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
    for (int r = lane; r < m_pad; r += 32) {
        if (r >= m) {
            lut_out[r] = make_uint4(0, 0, 0, 0);
            continue;
        }
        float v[16];
        row(r, v);
        const float mn = row_min[r];
        int q[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) q[j] = __float2int_rn(__fmul_rn(__fsub_rn(v[j], mn), scale));
        lut_out[r] = make_uint4(pack4(q[0], q[1], q[2], q[3]), pack4(q[4], q[5], q[6], q[7]),
                                pack4(q[8], q[9], q[10], q[11]), pack4(q[12], q[13], q[14], q[15]));
    }
    scale_out = scale;
    offset_out = offset;
    __syncwarp();
}

// ---------------------------------------------------------------------------
// PQ table terms, bit-exact with the reference (reference src/pq.cpp):
//   inner (C): out[s][k] = sum_j ((-2 * q[s*sd+j]) * y[s][j][k])   (:186-204)
//   list  (B): out[s][k] = sum_j y * (y + 2 * c[s*sd+j])            (:206-223)
//   adc      : out[s][k] = sum_j (q - y)^2                          (:165-184)
// y is the transposed codebook, m * sd * K floats. The reference's release
// build (GCC, C++, -mfma; CMakeLists.txt:63-68) fuses each `out += a * b`
// into one FMA (GCC's default -ffp-contract=fast in C++ modes), so these do too.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float inner_term(const float* q, const float* yt, int s, int sd, int K, int k) {
    float out = 0.0f;
    for (int j = 0; j < sd; ++j) {
        out = __fmaf_rn(__fmul_rn(-2.0f, q[s * sd + j]), yt[(s * sd + j) * K + k], out);
    }
    return out;
}

__device__ __forceinline__ float list_term(const float* c, const float* yt, int s, int sd, int K, int k) {
    float out = 0.0f;
    for (int j = 0; j < sd; ++j) {
        const float y = yt[(s * sd + j) * K + k];
        out = __fmaf_rn(y, __fadd_rn(y, __fmul_rn(2.0f, c[s * sd + j])), out);
    }
    return out;
}

__device__ __forceinline__ float adc_term(const float* r, const float* yt, int s, int sd, int K, int k) {
    float out = 0.0f;
    for (int j = 0; j < sd; ++j) {
        const float diff = __fsub_rn(r[s * sd + j], yt[(s * sd + j) * K + k]);
        out = __fmaf_rn(diff, diff, out);
    }
    return out;
}

// ---------------------------------------------------------------------------
// 4-bit lookups from registers. prmt.b32 picks four bytes out of eight by
// four 4-bit selectors; a selector with its top bit set yields the sign of the
// picked byte (0x00 for LUT entries, which are <= 63). So with the 16-entry
// row as words L0..L3:
//   prmt(L0, L1, codes)          = entry c for codes c < 8, 0 otherwise
//   prmt(L2, L3, codes ^ 0x8888) = entry c for codes c >= 8, 0 otherwise
// and their sum is the lookup of four codes at once, one byte each.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

// The 16 entries of LUT rows rounded and packed: round-half-even of
// (t - min) * scale, as nearbyint / cvtps do, through the 1.5 * 2^23 addend
// (every value here lies in [0, 64), where float spacing at that magnitude is 1).
// Two entries per packed FP32 instruction: each component rounds as the scalar
// __fadd_rn / __fmul_rn does, and t - min is t + (-min) exactly.
__device__ __forceinline__ uint4 round_row(const float* v, float mn, float scale) {
    const float2 neg = make_float2(-mn, -mn), sc = make_float2(scale, scale);
    const float2 magic = make_float2(12582912.0f, 12582912.0f);
    uint32_t b[16];
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
        const float2 t = __fadd2_rn(__fmul2_rn(__fadd2_rn(make_float2(v[j], v[j + 1]), neg), sc), magic);
        b[j] = __float_as_uint(t.x);
        b[j + 1] = __float_as_uint(t.y);
    }
    return make_uint4(prmt(prmt(b[0], b[1], 0x0040), prmt(b[2], b[3], 0x0040), 0x5410),
                      prmt(prmt(b[4], b[5], 0x0040), prmt(b[6], b[7], 0x0040), 0x5410),
                      prmt(prmt(b[8], b[9], 0x0040), prmt(b[10], b[11], 0x0040), 0x5410),
                      prmt(prmt(b[12], b[13], 0x0040), prmt(b[14], b[15], 0x0040), 0x5410));
}

// Device code layout (built from the file format's blocks by pack_superblocks, qg_index.cu):
// a list is stored in superblocks of 64 vectors. Octet lane r (0..7) owns
// vectors 8r..8r+7; its word for subspace s holds their codes, vector 8r+i
// in nibble i. Words are interleaved so each 16-byte load of the 8 lanes is
// one 128-byte line: uint4 index (s/4)*8 + r holds subspaces s..s+3.
inline constexpr int kSuperBlock = 64;

// Sums of the 8 vectors of one octet lane over m_pad subspaces (m_pad % 4 == 0).
// lut: m_pad rows as uint4 (shared memory). Sums are exact uint16 values
// (m_pad * 63 <= 64512).
__device__ __forceinline__ void octet_step(const uint4& w, const uint4* __restrict__ lut, uint32_t& a0, uint32_t& b0,
                                           uint32_t& a1, uint32_t& b1) {
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
    uint32_t g0 = 0, g1 = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const uint4 L = lut[t];
        const uint32_t c = ws[t];
        const uint32_t cx = c ^ 0x88888888u;
        g0 += prmt(L.x, L.y, c) + prmt(L.z, L.w, cx);
        g1 += prmt(L.x, L.y, c >> 16) + prmt(L.z, L.w, cx >> 16);
    }
    // bytes 0, 2 and 1, 3 of the byte sums widened into 16-bit fields by one
    // byte permute each (selector nibble 4 picks a zero byte of the second operand)
    a0 += prmt(g0, 0u, 0x4240u);
    b0 += prmt(g0, 0u, 0x4341u);
    a1 += prmt(g1, 0u, 0x4240u);
    b1 += prmt(g1, 0u, 0x4341u);
}

__device__ __forceinline__ void octet_sums(const uint4* __restrict__ sb, const uint4* __restrict__ lut, int m_pad,
                                           int r, uint32_t sums[8]) {
    uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    const int nq = m_pad >> 2;
    // two 16-byte code words in use and the next two in flight
    const uint4 zero = make_uint4(0, 0, 0, 0);
    uint4 c0 = nq > 0 ? __ldg(sb + r) : zero;
    uint4 c1 = nq > 1 ? __ldg(sb + 8 + r) : zero;
    int q = 0;
    for (; q + 2 <= nq; q += 2) {
        const uint4 n0 = q + 2 < nq ? __ldg(sb + (q + 2) * 8 + r) : zero;
        const uint4 n1 = q + 3 < nq ? __ldg(sb + (q + 3) * 8 + r) : zero;
        octet_step(c0, lut + 4 * q, a0, b0, a1, b1);
        octet_step(c1, lut + 4 * (q + 1), a0, b0, a1, b1);
        c0 = n0;
        c1 = n1;
    }
    if (q < nq) octet_step(c0, lut + 4 * q, a0, b0, a1, b1);
    sums[0] = a0 & 0xFFFFu;
    sums[1] = b0 & 0xFFFFu;
    sums[2] = a0 >> 16;
    sums[3] = b0 >> 16;
    sums[4] = a1 & 0xFFFFu;
    sums[5] = b1 & 0xFFFFu;
    sums[6] = a1 >> 16;
    sums[7] = b1 >> 16;
}

// octet_sums for code arrays padded by kCodePad uint4 past their last
// superblock: the loads two words ahead need no bounds tests (those past the
// superblock read the next one or the padding, and are never used).
inline constexpr int kCodePad = 16;
__device__ __forceinline__ void octet_sums_padded(const uint4* __restrict__ sb, const uint4* __restrict__ lut,
                                                  int m_pad, int r, uint32_t sums[8]) {
    uint32_t a0 = 0, b0 = 0, a1 = 0, b1 = 0;
    const int nq = m_pad >> 2;
    const uint4* p = sb + r;
    uint4 c0 = __ldg(p), c1 = __ldg(p + 8);
    int q = 0;
    for (; q + 2 <= nq; q += 2) {
        const uint4 n0 = __ldg(p + (q + 2) * 8), n1 = __ldg(p + (q + 3) * 8);
        octet_step(c0, lut + 4 * q, a0, b0, a1, b1);
        octet_step(c1, lut + 4 * (q + 1), a0, b0, a1, b1);
        c0 = n0;
        c1 = n1;
    }
    if (q < nq) octet_step(c0, lut + 4 * q, a0, b0, a1, b1);
    sums[0] = a0 & 0xFFFFu;
    sums[1] = b0 & 0xFFFFu;
    sums[2] = a0 >> 16;
    sums[3] = b0 >> 16;
    sums[4] = a1 & 0xFFFFu;
    sums[5] = b1 & 0xFFFFu;
    sums[6] = a1 >> 16;
    sums[7] = b1 >> 16;
}

// Fast-scan distance of an integer sum: sums / scale + offset, an IEEE
// division then an add (reference src/ivf_index.cpp:496).
__device__ __forceinline__ float fs_dist(uint32_t sum, float scale, float offset) {
    return __fadd_rn(__fdiv_rn(static_cast<float>(sum), scale), offset);
}

// fs_dist(0, scale, offset) without the division: 0 / scale is +0 for any
// scale > 0 (+inf included), and the LUT scales are >= 0 (0 / 0 gives the
// canonical NaN, as here).
__device__ __forceinline__ float fs_dist0(float scale, float offset) {
    return scale > 0.0f ? __fadd_rn(0.0f, offset) : __int_as_float(0x7fffffff);
}

// Largest integer sum whose distance has key <= thr_key, or -1 when none;
// 65535 when every sum passes. Distances grow monotonically with the sum, so
// the exact float test `key(dist(S)) <= thr_key` becomes `S <= result`.
__device__ __forceinline__ int sum_limit(uint32_t thr_key, float scale, float offset) {
    if (thr_key == 0xFFFFFFFFu) return 65535;
    // binary search of the monotone predicate over [-1, 65535]: 17 steps
    int lo = -1, hi = 65535;   // invariant: pred(lo) true (or lo == -1), pred(hi + 1) false
    if (float_key(fs_dist(65535u, scale, offset)) <= thr_key) return 65535;
    while (lo < hi - 1) {
        const int mid = (lo + hi) >> 1;
        if (float_key(fs_dist(static_cast<uint32_t>(mid), scale, offset)) <= thr_key) lo = mid;
        else hi = mid;
    }
    return lo;
}

// sum_limit from an estimate: floor((thr - offset) * scale) is within a unit
// or two of the answer unless the subtraction cancels badly; a short exact
// walk settles it, with the binary search as the fallback.
__device__ __forceinline__ int sum_limit_fast(uint32_t thr_key, float scale, float offset) {
    if (thr_key == 0xFFFFFFFFu) return 65535;
    const float x = __fmul_rn(__fsub_rn(key_float(thr_key), offset), scale);
    auto pass = [&](int t) { return float_key(fs_dist(static_cast<uint32_t>(t), scale, offset)) <= thr_key; };
    // far outside the sum range: distances are monotone in the sum, so one
    // end decides it (a list whose smallest distance is above the threshold
    // is the common case once the threshold has tightened)
    if (!(x > -4.0f)) return float_key(fs_dist0(scale, offset)) <= thr_key ? sum_limit(thr_key, scale, offset) : -1;
    if (!(x < 65540.0f)) return pass(65535) ? 65535 : sum_limit(thr_key, scale, offset);
    int s = max(-1, min(65535, __float2int_rd(x)));
    for (int it = 0; it < 4; ++it) {
        if (s >= 0 && !pass(s)) {
            --s;
        } else if (s < 65535 && pass(s + 1)) {
            ++s;
        } else {
            return s;   // pass(s) (or s == -1) and !pass(s + 1) (or s == 65535)
        }
    }
    return sum_limit(thr_key, scale, offset);
}

// nbins nearly equal intervals over the keys lo .. lo + span - 1, found by a
// multiply-high instead of a 64-bit division per key. With span > nbins,
// mul = floor(2^32 nbins / span) < 2^32 and bin(x) = floor((x - lo) mul / 2^32)
// <= floor(nbins (span - 1) / span) < nbins; otherwise every key has its own
// interval (mul = 0). last(b), the largest key whose interval is <= b, is
// lo + ceil((b + 1) 2^32 / mul) - 1 (x mul < (b + 1) 2^32), so a threshold
// taken there is at or above every key counted in intervals 0 .. b.
struct KeyBins {
    uint32_t lo, mul;
    __device__ __forceinline__ KeyBins(uint32_t lo_, uint64_t span, int nbins)
        : lo(lo_),
          mul(span > static_cast<uint64_t>(nbins)
                  ? static_cast<uint32_t>((static_cast<uint64_t>(nbins) << 32) / span)
                  : 0u) {}
    __device__ __forceinline__ int bin(uint32_t key) const {
        const uint32_t x = key - lo;
        return static_cast<int>(mul ? __umulhi(x, mul) : x);
    }
    __device__ __forceinline__ uint64_t last(int b) const {
        return static_cast<uint64_t>(lo) +
               (mul ? ((static_cast<uint64_t>(b + 1) << 32) + mul - 1) / mul - 1 : static_cast<uint64_t>(b));
    }
};

} // namespace qg
