// Shared device/host helpers for the qann B200 search path.
//
// Numerics contract: every float operation whose result must match the
// reference CPU build bit for bit is written with explicit round-to-nearest
// intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, __fmaf_rn) and the library is
// compiled with -fmad=false, so a multiply and an add are fused exactly where
// the reference's release build (GCC, C++, -mavx2 -mfma, whose default
// -ffp-contract=fast fuses `x += a * b`) fuses them, and nowhere else.
#pragma once

#include "qg_cuda.h"

#include <cstddef>
#include <cstdint>
#include <cstring>

namespace qg {

// ---------------------------------------------------------------------------
// Ordered float keys (reference src/topk.hpp:82-91): a float maps to a uint32
// that sorts the same way (negative floats flipped, positives with the sign
// bit set). -0.0f sorts just below +0.0f, as in the reference's TopK.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t float_key(float f) {
#ifdef __CUDA_ARCH__
    const uint32_t b = __float_as_uint(f);
#else
    uint32_t b;
    std::memcpy(&b, &f, 4);
#endif
    return b ^ (static_cast<uint32_t>(static_cast<int32_t>(b) >> 31) | 0x80000000u);
}

__host__ __device__ __forceinline__ float key_float(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k ^ 0x80000000u) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    std::memcpy(&f, &b, 4);
    return f;
#endif
}

// Key for comparisons the reference does on float values with operator<
// (std::sort / nth_element over (float, slot) pairs, e.g. RefineIndex::rerank):
// there -0.0f == +0.0f, so both map to +0's key.
__host__ __device__ __forceinline__ uint32_t float_key_eq0(float f) {
    return float_key(f == 0.0f ? 0.0f : f);
}

// ---------------------------------------------------------------------------
// Exact distances in the reference's AVX2+FMA accumulation order
// (reference src/distance.cpp:66-96 l2_distance_avx2, :138-151
// inner_product_avx2). Four 8-lane accumulators over 32-float steps, an
// 8-float step into accumulator 0, the lane sum
// ((a0+a1)+(a2+a3)) per lane, then the hsum256 tree
// ((l0+l4)+(l1+l5)) + ((l2+l6)+(l3+l7)), then the n % 8 tail as the
// reference's release build (GCC -O3 -mavx2 -mfma) computes `result += d * d`:
// with 4 or more elements left, four products rounded and added in order
// (its vectorised epilogue), then one FMA per remaining element.
//
// chain(j, L): the FMA chain of accumulator j, lane L.
// ---------------------------------------------------------------------------
// Packed FP32 (sm_100): each component of __fadd2_rn / __ffma2_rn rounds as
// the scalar __fadd_rn / __fmaf_rn does, and x - y is x + (-y) exactly, so
// pairs of independent chains advance two per instruction with the same bits.
__device__ __forceinline__ float2 sub2(float2 x, float2 y) { return __fadd2_rn(x, make_float2(-y.x, -y.y)); }

template <bool kL2>
__device__ __forceinline__ float exact_tail(const float* __restrict__ a, const float* __restrict__ b, int i, int n,
                                            float r) {
    if (n - i >= 4) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float p;
            if (kL2) {
                const float d = __fsub_rn(a[i + e], b[i + e]);
                p = __fmul_rn(d, d);
            } else {
                p = __fmul_rn(a[i + e], b[i + e]);
            }
            r = __fadd_rn(r, p);
        }
        i += 4;
    }
    for (; i < n; ++i) {
        if (kL2) {
            const float d = __fsub_rn(a[i], b[i]);
            r = __fmaf_rn(d, d, r);
        } else {
            r = __fmaf_rn(a[i], b[i], r);
        }
    }
    return r;
}

template <bool kL2>
__device__ __forceinline__ float exact_avx2(const float* __restrict__ a, const float* __restrict__ b, int n) {
    const int n32 = n & ~31;
    const int n8 = n & ~7;     // end of the 8-float steps
    float t[4];
#pragma unroll
    for (int L = 0; L < 4; ++L) {
        float s[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int lane = L + 4 * h;
            // accumulators 0/1 and 2/3 advance as packed pairs
            float2 acc01 = make_float2(0.f, 0.f), acc23 = make_float2(0.f, 0.f);
            int i = 0;
            for (; i < n32; i += 32) {
                const float2 x01 = make_float2(a[i + lane], a[i + 8 + lane]);
                const float2 x23 = make_float2(a[i + 16 + lane], a[i + 24 + lane]);
                const float2 y01 = make_float2(b[i + lane], b[i + 8 + lane]);
                const float2 y23 = make_float2(b[i + 16 + lane], b[i + 24 + lane]);
                if (kL2) {
                    const float2 d01 = sub2(x01, y01), d23 = sub2(x23, y23);
                    acc01 = __ffma2_rn(d01, d01, acc01);
                    acc23 = __ffma2_rn(d23, d23, acc23);
                } else {
                    acc01 = __ffma2_rn(x01, y01, acc01);
                    acc23 = __ffma2_rn(x23, y23, acc23);
                }
            }
            float acc0 = acc01.x;
            const float acc1 = acc01.y, acc2 = acc23.x, acc3 = acc23.y;
            for (; i < n8; i += 8) {
                if (kL2) {
                    const float d = __fsub_rn(a[i + lane], b[i + lane]);
                    acc0 = __fmaf_rn(d, d, acc0);
                } else {
                    acc0 = __fmaf_rn(a[i + lane], b[i + lane], acc0);
                }
            }
            s[h] = __fadd_rn(__fadd_rn(acc0, acc1), __fadd_rn(acc2, acc3));
        }
        t[L] = __fadd_rn(s[0], s[1]);
    }
    float r = __fadd_rn(__fadd_rn(t[0], t[1]), __fadd_rn(t[2], t[3]));
    return exact_tail<kL2>(a, b, n8, n, r);
}

// exact_avx2 with all 32 accumulators advanced together: each 32-float step
// of a and b is eight 16-byte loads (both 16-byte aligned, n % 4 == 0). Every
// accumulator's FMA chain runs in the same order as in exact_avx2, so the
// result is the same to the bit; the loads of a step are all in flight at once.
template <bool kL2>
__device__ __forceinline__ float exact_avx2_vec(const float* __restrict__ a, const float* __restrict__ b, int n) {
    const int n32 = n & ~31;
    const int n8 = n & ~7;
    float acc[32];   // acc[8 * j + L]: accumulator j, AVX2 lane L
#pragma unroll
    for (int e = 0; e < 32; ++e) acc[e] = 0.0f;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const float4* b4 = reinterpret_cast<const float4*>(b);
    auto step4 = [&](const float4& av, const float4& bv, int base) {   // two chains per packed instruction
        const float2 x01 = make_float2(av.x, av.y), x23 = make_float2(av.z, av.w);
        const float2 y01 = make_float2(bv.x, bv.y), y23 = make_float2(bv.z, bv.w);
        float2 c01 = make_float2(acc[base], acc[base + 1]), c23 = make_float2(acc[base + 2], acc[base + 3]);
        if (kL2) {
            const float2 d01 = sub2(x01, y01), d23 = sub2(x23, y23);
            c01 = __ffma2_rn(d01, d01, c01);
            c23 = __ffma2_rn(d23, d23, c23);
        } else {
            c01 = __ffma2_rn(x01, y01, c01);
            c23 = __ffma2_rn(x23, y23, c23);
        }
        acc[base] = c01.x;
        acc[base + 1] = c01.y;
        acc[base + 2] = c23.x;
        acc[base + 3] = c23.y;
    };
    for (int i = 0; i < n32; i += 32) {
        float4 av[8], bv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            av[k] = __ldg(a4 + (i >> 2) + k);
            bv[k] = __ldg(b4 + (i >> 2) + k);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) step4(av[k], bv[k], 4 * k);
    }
    for (int i = n32; i < n8; i += 8) {   // 8-float steps into accumulator 0
        const float4 a0 = __ldg(a4 + (i >> 2)), a1 = __ldg(a4 + (i >> 2) + 1);
        const float4 b0 = __ldg(b4 + (i >> 2)), b1 = __ldg(b4 + (i >> 2) + 1);
        step4(a0, b0, 0);
        step4(a1, b1, 4);
    }
    float s[8];
#pragma unroll
    for (int L = 0; L < 8; ++L) s[L] = __fadd_rn(__fadd_rn(acc[L], acc[8 + L]), __fadd_rn(acc[16 + L], acc[24 + L]));
    const float r = __fadd_rn(__fadd_rn(__fadd_rn(s[0], s[4]), __fadd_rn(s[1], s[5])),
                              __fadd_rn(__fadd_rn(s[2], s[6]), __fadd_rn(s[3], s[7])));
    return exact_tail<kL2>(a, b, n8, n, r);
}

// exact_avx2 of one row by the 4 lanes of an aligned lane group: lane h runs
// AVX2 lanes 2h and 2h + 1 (their four FMA chains, packed, over one 8-byte load
// of a and of b per step), so each step of the group reads one 32-byte sector
// of b. Lanes h and h ^ 2 add their lane sums pairwise and lanes h and h ^ 1
// add those, which is exact_avx2's tree ((s0 + s4) + (s1 + s5)) + ((s2 + s6) +
// (s3 + s7)) (float addition of two operands is commutative, so every lane
// ends with the same bits); every lane adds the tail. All 32 lanes of the warp
// call it together. a and b 8-byte aligned, n even; a in any address space, b
// global memory read through the read-only path.
template <bool kL2>
__device__ __forceinline__ float exact_avx2_group4(const float* a, const float* __restrict__ b, int n) {
    const int h = threadIdx.x & 3;
    const int n32 = n & ~31, n8 = n & ~7;
    float2 acc[4];   // accumulator j of AVX2 lanes 2h and 2h + 1
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = make_float2(0.f, 0.f);
    auto step = [&](int e, int j) {
        const float2 x = *reinterpret_cast<const float2*>(a + e);
        const float2 y = __ldg(reinterpret_cast<const float2*>(b + e));
        if (kL2) {
            const float2 dv = sub2(x, y);
            acc[j] = __ffma2_rn(dv, dv, acc[j]);
        } else {
            acc[j] = __ffma2_rn(x, y, acc[j]);
        }
    };
    int i = 0;
    for (; i < n32; i += 32) {
#pragma unroll
        for (int j = 0; j < 4; ++j) step(i + 8 * j + 2 * h, j);
    }
    for (; i < n8; i += 8) step(i + 2 * h, 0);   // 8-float steps into accumulator 0
    const float s0 = __fadd_rn(__fadd_rn(acc[0].x, acc[1].x), __fadd_rn(acc[2].x, acc[3].x));   // AVX2 lane 2h
    const float s1 = __fadd_rn(__fadd_rn(acc[0].y, acc[1].y), __fadd_rn(acc[2].y, acc[3].y));   // AVX2 lane 2h + 1
    const float o0 = __shfl_xor_sync(0xffffffffu, s0, 2, 4), o1 = __shfl_xor_sync(0xffffffffu, s1, 2, 4);
    const float u = __fadd_rn(__fadd_rn(s0, o0), __fadd_rn(s1, o1));
    const float r = __fadd_rn(u, __shfl_xor_sync(0xffffffffu, u, 1, 4));
    return exact_tail<kL2>(a, b, n8, n, r);
}

// exact_avx2 of one row by the 8 lanes of an aligned lane group: lane L of the
// group runs AVX2 lane L's four FMA chains (elements i + 8 j + L), the groups'
// lane sums meet in exact_avx2's tree order through shuffles, and every lane
// adds the tail. All 32 lanes of the warp call it together. Same bits as
// exact_avx2<kL2>(a, b, n). kLdg: b is global memory read through the
// read-only path (else any address space).
template <bool kL2, bool kLdg>
__device__ __forceinline__ float exact_avx2_group8(const float* a, const float* __restrict__ b, int n) {
    const int L = threadIdx.x & 7;
    const int n32 = n & ~31, n8 = n & ~7;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    int i = 0;
    auto term = [&](int e, float acc) {
        const float be = kLdg ? __ldg(b + e) : b[e];
        if (kL2) {
            const float d = __fsub_rn(a[e], be);
            return __fmaf_rn(d, d, acc);
        }
        return __fmaf_rn(a[e], be, acc);
    };
    for (; i < n32; i += 32) {
        acc0 = term(i + L, acc0);
        acc1 = term(i + 8 + L, acc1);
        acc2 = term(i + 16 + L, acc2);
        acc3 = term(i + 24 + L, acc3);
    }
    for (; i < n8; i += 8) acc0 = term(i + L, acc0);
    const float sl = __fadd_rn(__fadd_rn(acc0, acc1), __fadd_rn(acc2, acc3));
    const float t = __fadd_rn(sl, __shfl_down_sync(0xffffffffu, sl, 4, 8));   // lanes 0..3: s_L + s_{L+4}
    const float t0 = __shfl_sync(0xffffffffu, t, 0, 8), t1 = __shfl_sync(0xffffffffu, t, 1, 8);
    const float t2 = __shfl_sync(0xffffffffu, t, 2, 8), t3 = __shfl_sync(0xffffffffu, t, 3, 8);
    const float r = __fadd_rn(__fadd_rn(t0, t1), __fadd_rn(t2, t3));
    return exact_tail<kL2>(a, b, n8, n, r);
}

// The score the reference's DenseIndex ranks by (reference
// include/vecengine/index.hpp:269-271): squared L2, or -(a . b) for inner product.
__device__ __forceinline__ float exact_score(const float* a, const float* b, int n, bool ip) {
    return ip ? -exact_avx2<false>(a, b, n) : exact_avx2<true>(a, b, n);
}

} // namespace qg
