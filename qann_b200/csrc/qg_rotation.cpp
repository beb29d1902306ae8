// PCA-balanced rotation for IVF-PQ, host side (reference src/rotation.cpp).
// The mean and the covariance of the training rows come from the GPU
// (qg_train.cu covariance()); this file diagonalises the covariance and
// deals the eigenvectors out to the PQ subspaces.
//
// The reference's optimised build forms fused multiply-adds from its
// expressions (GCC's default floating-point contraction with -mfma); they
// are written out here with std::fma, and this file is compiled without
// contraction, so the rotation comes out bit-identical.
#include "qg_train.h"
#include "qg_error.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace qg {

// Cyclic Jacobi eigen-decomposition of a symmetric d x d matrix (reference
// src/rotation.cpp:20-69; the method of Numerical Recipes 11.1): sweeps of
// plane rotations, each zeroing one off-diagonal entry, until the
// off-diagonal mass falls below 1e-24 of the total (at most 100 sweeps).
// vectors holds the eigenvectors as columns.
void symmetric_eigen(std::vector<double> a, size_t d, std::vector<double>& values, std::vector<double>& vectors) {
    vectors.assign(d * d, 0.0);
    for (size_t i = 0; i < d; ++i) vectors[i * d + i] = 1.0;
    double total = 0.0;
    for (double x : a) total = std::fma(x, x, total);

    auto rotate_pair = [](double& x, double& y, double c, double s) {
        const double xv = x, yv = y;
        x = std::fma(c, xv, -(s * yv));   // c x - s y
        y = std::fma(s, xv, c * yv);      // s x + c y
    };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (size_t p = 0; p < d; ++p)
            for (size_t q = p + 1; q < d; ++q) off = std::fma(a[p * d + q], a[p * d + q], off);
        if (off <= 1e-24 * total) break;
        for (size_t p = 0; p < d; ++p) {
            for (size_t q = p + 1; q < d; ++q) {
                const double apq = a[p * d + q];
                if (apq == 0.0) continue;
                // t = tan of the angle: the smaller root of t^2 + 2 theta t - 1 = 0
                const double theta = (a[q * d + q] - a[p * d + p]) / (2.0 * apq);
                const double t = std::abs(theta) > 1e150
                                     ? 1.0 / (2.0 * theta)
                                     : (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(std::fma(theta, theta, 1.0)));
                const double c = 1.0 / std::sqrt(std::fma(t, t, 1.0));
                const double s = t * c;
                for (size_t k = 0; k < d; ++k) rotate_pair(a[k * d + p], a[k * d + q], c, s);   // a J
                for (size_t k = 0; k < d; ++k) rotate_pair(a[p * d + k], a[q * d + k], c, s);   // J^T a
                for (size_t k = 0; k < d; ++k) rotate_pair(vectors[k * d + p], vectors[k * d + q], c, s);
            }
        }
    }
    values.resize(d);
    for (size_t i = 0; i < d; ++i) values[i] = a[i * d + i];
}

// The rotation from the (scaled, symmetric) covariance (reference
// src/rotation.cpp:71-130): eigenvalues largest first, each eigenvector into
// the subspace with room whose sum of log-eigenvalues is smallest so far, so
// that the subspaces carry balanced variance products. R is d x d row-major;
// column best * (d / m) + slot holds the eigenvector.
std::vector<float> balanced_rotation(std::vector<double> cov, size_t d, size_t m) {
    std::vector<double> values, vectors;
    symmetric_eigen(std::move(cov), d, values, vectors);
    std::vector<size_t> order(d);
    std::iota(order.begin(), order.end(), size_t{0});
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return values[x] > values[y]; });
    const size_t width = d / m;
    std::vector<size_t> filled(m, 0);
    std::vector<double> log_sum(m, 0.0);
    std::vector<float> r(d * d);
    for (size_t e : order) {
        size_t best = m;
        for (size_t b = 0; b < m; ++b)
            if (filled[b] < width && (best == m || log_sum[b] < log_sum[best])) best = b;
        log_sum[best] += std::log(std::max(values[e], 1e-12));
        const size_t col = best * width + filled[best]++;
        for (size_t row = 0; row < d; ++row) r[row * d + col] = static_cast<float>(vectors[row * d + e]);
    }
    return r;
}

} // namespace qg
