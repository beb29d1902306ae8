// Device steps of training: assignment for small codebooks, member sums in
// point order, distances to the own centroid, and row gathers. The host side
// (qg_train_host.cpp) replays the reference's random choices and bookkeeping
// around them.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_train.h"

namespace qg {

// thread per (problem, point): k exact distances, first index of the minimum
// (the reference's nearest_centroid keeps the first strictly smaller one;
// reference src/kmeans.cpp:102-115)
__global__ void k_assign_small(const float* __restrict__ x, size_t n, int d, const float* __restrict__ c, int k, int P,
                               uint32_t* __restrict__ assign) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * P) return;
    const size_t p = t / n;
    const float* pt = x + t * d;
    const float* cp = c + p * static_cast<size_t>(k) * d;
    float best = 3.402823466e+38f;   // FLT_MAX, the reference's starting value
    uint32_t bi = 0;
    for (int j = 0; j < k; ++j) {
        const float dist = exact_avx2<true>(pt, cp + static_cast<size_t>(j) * d, d);
        if (dist < best) {
            best = dist;
            bi = static_cast<uint32_t>(j);
        }
    }
    assign[t] = bi;
}

void assign_small(const float* x, size_t n, int d, const float* c, int k, int P, uint32_t* assign, cudaStream_t st) {
    if (n == 0) return;
    k_assign_small<<<static_cast<unsigned>(ceil_div(n * P, 128)), 128, 0, st>>>(x, n, d, c, k, P, assign);
    QG_LAUNCH_CHECK();
}

// thread per (problem, centroid, dim): a sequential float sum over the
// centroid's members in the order given
__global__ void k_member_sums(const float* __restrict__ x, size_t n, int d, const uint32_t* __restrict__ order,
                              const uint32_t* __restrict__ off, int k, int P, float* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t per = static_cast<size_t>(k) * d;
    if (t >= per * P) return;
    const size_t p = t / per;
    const int c = static_cast<int>((t % per) / d);
    const int l = static_cast<int>(t % d);
    const uint32_t* o = order + p * n;
    const uint32_t* f = off + p * (k + 1);
    const float* xp = x + p * n * d;
    float s = 0.0f;
    for (uint32_t i = f[c]; i < f[c + 1]; ++i) s = __fadd_rn(s, xp[static_cast<size_t>(o[i]) * d + l]);
    out[t] = s;
}

void member_sums(const float* x, size_t n, int d, const uint32_t* order, const uint32_t* off, int k, int P, float* out,
                 cudaStream_t st) {
    const size_t total = static_cast<size_t>(k) * d * P;
    if (total == 0) return;
    k_member_sums<<<static_cast<unsigned>(ceil_div(total, 128)), 128, 0, st>>>(x, n, d, order, off, k, P, out);
    QG_LAUNCH_CHECK();
}

__global__ void k_own_dist(const float* __restrict__ x, size_t n, int d, const float* __restrict__ c, int k,
                           const uint32_t* __restrict__ assign, int P, float* __restrict__ dist) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * P) return;
    const size_t p = t / n;
    dist[t] = exact_avx2<true>(x + t * d, c + (p * k + assign[t]) * static_cast<size_t>(d), d);
}

void own_dist(const float* x, size_t n, int d, const float* c, int k, const uint32_t* assign, int P, float* dist,
              cudaStream_t st) {
    if (n == 0) return;
    k_own_dist<<<static_cast<unsigned>(ceil_div(n * P, 128)), 128, 0, st>>>(x, n, d, c, k, assign, P, dist);
    QG_LAUNCH_CHECK();
}

__global__ void k_gather_rows(const float* __restrict__ src, const uint32_t* __restrict__ idx, size_t n, int d,
                              float* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * d) return;
    const size_t i = t / d;
    out[t] = src[static_cast<size_t>(idx[i]) * d + (t % d)];
}

void gather_rows(const float* src, const uint32_t* idx, size_t n, int d, float* out, cudaStream_t st) {
    if (n == 0) return;
    k_gather_rows<<<static_cast<unsigned>(ceil_div(n * d, 256)), 256, 0, st>>>(src, idx, n, d, out);
    QG_LAUNCH_CHECK();
}

__global__ void k_residuals(const float* __restrict__ x, size_t n, int d, const float* __restrict__ centers,
                            const uint32_t* __restrict__ assign, float* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * d) return;
    const size_t i = t / d;
    out[t] = __fsub_rn(x[t], centers[static_cast<size_t>(assign[i]) * d + (t % d)]);
}

void residuals(const float* x, size_t n, int d, const float* centers, const uint32_t* assign, float* out,
               cudaStream_t st) {
    if (n == 0) return;
    k_residuals<<<static_cast<unsigned>(ceil_div(n * d, 256)), 256, 0, st>>>(x, n, d, centers, assign, out);
    QG_LAUNCH_CHECK();
}

__global__ void k_split_columns(const float* __restrict__ x, size_t n, int dim, int d, int P, float* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * dim) return;
    const size_t i = t / dim;
    const int col = static_cast<int>(t % dim);
    const int p = col / d, l = col % d;
    out[(static_cast<size_t>(p) * n + i) * d + l] = x[t];
}

void split_columns(const float* x, size_t n, int dim, int d, int P, float* out, cudaStream_t st) {
    if (n == 0) return;
    (void)P;
    k_split_columns<<<static_cast<unsigned>(ceil_div(n * dim, 256)), 256, 0, st>>>(x, n, dim, d, P, out);
    QG_LAUNCH_CHECK();
}

} // namespace qg
