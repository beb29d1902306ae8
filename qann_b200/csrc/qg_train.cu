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

// mean[j] = (double(x[0][j]) + double(x[1][j]) + ...) / n, in row order. One
// thread per column; loads run 8 rows ahead of the dependent adds.
__global__ void k_col_means(const float* __restrict__ x, size_t n, int d, double* __restrict__ mean) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d) return;
    double s = 0.0;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = x[(i + u) * d + j];
#pragma unroll
        for (int u = 0; u < 8; ++u) s = __dadd_rn(s, static_cast<double>(v[u]));
    }
    for (; i < n; ++i) s = __dadd_rn(s, static_cast<double>(x[i * d + j]));
    mean[j] = __ddiv_rn(s, static_cast<double>(n));
}

// cov[t] = sum over rows in order of fma(xc[p], xc[q], cov), xc = double(x) -
// mean, for the pair t = (p, q) = (pairs[t] >> 16, pairs[t] & 0xFFFF). Rows
// are centred into shared memory `tile` rows at a time.
__global__ void __launch_bounds__(256) k_cov_upper(const float* __restrict__ x, size_t n, int d,
                                                   const double* __restrict__ mean, const uint32_t* __restrict__ pairs,
                                                   int npairs, int tile, double* __restrict__ cov) {
    extern __shared__ double xs[];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = t < npairs;
    const int p = live ? static_cast<int>(pairs[t] >> 16) : 0;
    const int q = live ? static_cast<int>(pairs[t] & 0xFFFFu) : 0;
    double acc = 0.0;
    for (size_t i0 = 0; i0 < n; i0 += tile) {
        const int rows = static_cast<int>(n - i0 < static_cast<size_t>(tile) ? n - i0 : tile);
        __syncthreads();
        for (int e = threadIdx.x; e < rows * d; e += blockDim.x) {
            const int j = e % d;
            xs[e] = __dsub_rn(static_cast<double>(x[i0 * d + e]), mean[j]);
        }
        __syncthreads();
        if (live)
            for (int r = 0; r < rows; ++r) acc = __fma_rn(xs[r * d + p], xs[r * d + q], acc);
    }
    if (live) cov[t] = acc;
}

std::vector<double> covariance(const float* x, size_t n, int d, cudaStream_t st) {
    require(n > 0, "training set must not be empty");
    require(d <= 6144, "the GPU rotation training supports dim <= 6144", kUnsupported);
    DevBuf<double> mean(d, st);
    k_col_means<<<static_cast<unsigned>(ceil_div(d, 32)), 32, 0, st>>>(x, n, d, mean.get());
    QG_LAUNCH_CHECK();
    std::vector<uint32_t> pairs;
    pairs.reserve(static_cast<size_t>(d) * (d + 1) / 2);
    for (int p = 0; p < d; ++p)
        for (int q = p; q < d; ++q) pairs.push_back(static_cast<uint32_t>(p) << 16 | static_cast<uint32_t>(q));
    const int np = static_cast<int>(pairs.size());
    DevBuf<uint32_t> dp(np, st);
    QG_CUDA(cudaMemcpyAsync(dp.get(), pairs.data(), np * 4, cudaMemcpyHostToDevice, st));
    DevBuf<double> dc(np, st);
    const int tile = std::max(1, std::min(64, 6144 / d));   // <= 48 KB of centred rows
    k_cov_upper<<<static_cast<unsigned>(ceil_div(np, 256)), 256, static_cast<size_t>(tile) * d * 8, st>>>(
        x, n, d, mean.get(), dp.get(), np, tile, dc.get());
    QG_LAUNCH_CHECK();
    std::vector<double> upper(np);
    QG_CUDA(cudaMemcpyAsync(upper.data(), dc.get(), np * 8, cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    const double scale = n > 1 ? 1.0 / static_cast<double>(n - 1) : 1.0;
    std::vector<double> cov(static_cast<size_t>(d) * d);
    for (int t = 0; t < np; ++t) {
        const size_t p = pairs[t] >> 16, q = pairs[t] & 0xFFFFu;
        cov[p * d + q] = upper[t] * scale;
        cov[q * d + p] = cov[p * d + q];
    }
    return cov;
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
