// GPU kernels of training (k-means / e-means / PQ codebooks) and the host
// entry points that drive them.
#pragma once

#include "qg_cuda.h"

#include <cstdint>
#include <optional>
#include <vector>

namespace qg {

// ---- device steps (qg_train.cu); P independent problems of n points x d dims
// and k centroids each, packed problem-major. -----------------------------------

// assign[p][i] = nearest centroid (squared L2 in the reference's AVX2 order,
// first index on ties), for small k (PQ codebooks).
void assign_small(const float* x, size_t n, int d, const float* c, int k, int P, uint32_t* assign, cudaStream_t st);

// out[p][c][l] = x[order[off[c]]][l] + x[order[off[c] + 1]][l] + ... summed in
// float from 0 in the order given (the reference adds members in point order).
// order / off are per problem: order P x n, off P x (k + 1).
void member_sums(const float* x, size_t n, int d, const uint32_t* order, const uint32_t* off, int k, int P, float* out,
                 cudaStream_t st);

// dist[p][i] = squared L2 (AVX2 order) of point i to centroid assign[p][i].
void own_dist(const float* x, size_t n, int d, const float* c, int k, const uint32_t* assign, int P, float* dist,
              cudaStream_t st);

// rows[i] = src[idx[i]] (n rows of d floats).
void gather_rows(const float* src, const uint32_t* idx, size_t n, int d, float* out, cudaStream_t st);
// out[i] = x[i] - centers[assign[i]]
void residuals(const float* x, size_t n, int d, const float* centers, const uint32_t* assign, float* out,
               cudaStream_t st);
// out[p][i][0..d) = x[i][p*d .. (p+1)*d): the subspace columns, problem-major
void split_columns(const float* x, size_t n, int dim, int d, int P, float* out, cudaStream_t st);

// The sample covariance of n rows (reference src/rotation.cpp:77-104): column
// means summed in double in row order, then cov[p][q] (p <= q) accumulated as
// fma(x[p] - mean[p], x[q] - mean[q], cov) over the rows in order, scaled by
// 1 / (n - 1) (1 for n = 1) and mirrored. Returned on the host, d x d.
std::vector<double> covariance(const float* x, size_t n, int d, cudaStream_t st);

// ---- clustering steps on the device (qg_cluster.cu) ------------------------------

// Exclusive prefix sums of n uint32 values in place (the total must fit in 32 bits).
void exclusive_scan_u32(uint32_t* a, size_t n, cudaStream_t st);

// Points grouped by label, stable: for each of P problems of n points,
// order[p * n + j] lists the problem's point indices cluster by cluster, in
// point order within a cluster; off[p * (k + 1) + c] is where cluster c
// starts (off[.. + k] = n). Labels of k or more are left out.
void group_by_label(const uint32_t* labels, size_t n, int k, int P, uint32_t* order, uint32_t* off, cudaStream_t st);

// out[p][c] = sums[p][c] / float(count) (counts from off), made unit length
// (norm in double) when spherical. A cluster without points gets the row of
// `fallback` (when given) or zeros, and sets *empty (when given).
void cluster_means(const float* sums, const uint32_t* off, int k, int d, int P, bool spherical, const float* fallback,
                   float* out, int* empty, cudaStream_t st);

// dst[j] = src[j] scaled to unit length (norm in double; zero rows stay
// zero); dst may be src.
void unit_rows_dev(const float* src, size_t k, int d, float* dst, cudaStream_t st);

// e-means state between steps (positions, masses, the closing pass's sums).
struct EMeansState {
    int k = 0, d = 0;
    DevBuf<float> pos, mass, close_sum;
    DevBuf<uint32_t> close_cnt;
    void init(int k, int d, cudaStream_t st);   // masses 2^-16, pass sums zero
    // one mini-batch: member sums and cluster offsets of the batch, the step's alpha
    void step(const float* sums, const uint32_t* off, double alpha, bool accumulate, cudaStream_t st);
    void split(const std::vector<uint32_t>& pairs, cudaStream_t st);   // (donor, starved) pairs
    void close(cudaStream_t st);   // clusters seen in the closing pass move to its means
};

// The cosine PQ scoring decision on the training sample (reference
// src/ivf_index.cpp:808-902): true when inner-product tables find at least as
// many of the sample queries' true neighbours as per-list L2 tables. x: the
// n training rows (normalised), assign: their lists, centroids: coarse
// centroids, centers: residual centers, yt: transposed codebook (m x sd x 16).
bool cosine_ip_wins(const float* x, size_t n, int dim, const uint32_t* assign, const float* centroids,
                    const float* centers, int nlist, const float* yt, int m, int sd, cudaStream_t st);

// ---- host algorithms (qg_train_host.cpp, qg_rotation.cpp) -----------------------

// Jacobi eigen-decomposition of a symmetric d x d matrix (eigenvectors as columns).
void symmetric_eigen(std::vector<double> a, size_t d, std::vector<double>& values, std::vector<double>& vectors);
// The PCA-balanced rotation (d x d, row-major) for m subspaces from a covariance.
std::vector<float> balanced_rotation(std::vector<double> cov, size_t d, size_t m);

struct KMeansOut {
    std::vector<float> centroids;     // P * k * d
    DevBuf<float> centroids_dev;      // the same, on the device
    DevBuf<uint32_t> assign;          // P * n, on the device
};

// Lloyd's k-means (reference src/kmeans.cpp:174-252) for P problems at once
// (x_dev: P x n x d); problem p starts from seeds[p], or a random seed.
KMeansOut kmeans_lloyd(const float* x_dev, size_t n, int d, int k, size_t iters,
                       const std::vector<std::optional<uint32_t>>& seeds, bool spherical, int P, cudaStream_t st);

// e-means (reference src/kmeans.cpp:280-414), one problem.
KMeansOut emeans(const float* x_dev, size_t n, int d, int k, size_t passes, std::optional<uint32_t> seed,
                 bool spherical, cudaStream_t st);

// PQ codes (K = 16) of x - centers[assign] (qg_build.cu).
void encode16(const float* x, size_t n, int dim, const float* centers, const uint32_t* assign, const float* yt, int m,
              int sd, uint8_t* codes, cudaStream_t st);

} // namespace qg
