// Training on the GPU: the host side. It replays the reference's random
// choices (libstdc++ mt19937, uniform_int_distribution, shuffle,
// uniform_real_distribution, in the reference's call order) and its scalar
// bookkeeping (counts, divisions, e-means' mass and step schedule, reseeding),
// and sends the heavy steps — assignment, member sums, distances, encoding —
// to the GPU (qg_train.cu, qg_build.cu, qg_search.cu). The float arithmetic
// here is written out operation by operation (this file is built with
// -ffp-contract=off) with std::fma where the reference's release build
// (GCC, C++, -mfma) contracts a multiply into an add.
//
//   kmeans_lloyd           reference src/kmeans.cpp:174-252 (+ reseed :117-172)
//   emeans                 reference src/kmeans.cpp:254-414
//   PQ codebook training   reference src/pq.cpp:41-73
//   IVFIndex::train        reference src/ivf_index.cpp:725-806
//   pick_cosine_inner_product  reference src/ivf_index.cpp:808-902
#include "qg_ops.h"
#include "qg_search.h"
#include "qg_train.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <numbers>
#include <numeric>
#include <queue>
#include <random>

namespace qg {

namespace {

uint32_t seed_or_random(std::optional<uint32_t> s) { return s ? *s : std::random_device{}(); }

template <class T>
void h2d(T* dst, const T* src, size_t n, cudaStream_t st) {
    if (n) QG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

template <class T>
void d2h(T* dst, const T* src, size_t n, cudaStream_t st) {
    if (n) QG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
}

// unit-length copy of each row (reference src/kmeans.cpp:258-266); the double
// sum of squares is exact per product, so fused or not it is the same value
void unit_rows(const float* c, size_t k, size_t d, float* out) {
    for (size_t j = 0; j < k; ++j) {
        double sq = 0;
        for (size_t l = 0; l < d; ++l) sq += double(c[j * d + l]) * c[j * d + l];
        const float scale = sq > 0 ? static_cast<float>(1.0 / std::sqrt(sq)) : 0.0f;
        for (size_t l = 0; l < d; ++l) out[j * d + l] = c[j * d + l] * scale;
    }
}

size_t round_power_of_two(double v) {
    if (v <= 1) return 1;
    const size_t low = size_t{1} << static_cast<int>(std::floor(std::log2(v)));
    const size_t high = 2 * low;
    return v / double(low) < double(high) / v ? low : high;
}

// stable counting sort of labels: order (n) and offsets (k + 1)
void bucket(const uint32_t* labels, size_t n, int k, uint32_t* order, uint32_t* off, uint32_t* counts) {
    std::fill(counts, counts + k, 0u);
    for (size_t i = 0; i < n; ++i) ++counts[labels[i]];
    off[0] = 0;
    for (int c = 0; c < k; ++c) off[c + 1] = off[c] + counts[c];
    std::vector<uint32_t> cur(off, off + k);
    for (size_t i = 0; i < n; ++i) order[cur[labels[i]]++] = static_cast<uint32_t>(i);
}

// nearest centroid of each row on the GPU, results on the host
void assign_dev(const float* x_dev, size_t n, int d, const float* c_dev, int k, uint32_t* out_host, DevBuf<uint32_t>& tmp,
                cudaStream_t st) {
    tmp.alloc(std::max<size_t>(n, 1), st);
    assign_nearest(x_dev, n, c_dev, k, d, tmp.get(), st);
    d2h(out_host, tmp.get(), n, st);
}

} // namespace

// ---------------------------------------------------------------------------
// Lloyd
// ---------------------------------------------------------------------------
KMeansOut kmeans_lloyd(const float* x_dev, size_t n, int d, int k, size_t iters,
                       const std::vector<std::optional<uint32_t>>& seeds, bool spherical, int P, cudaStream_t st) {
    if (n < static_cast<size_t>(k)) throw Error(kInvalidArgument, "kmeans: need at least k points");
    const size_t kd = static_cast<size_t>(k) * d;
    // initial centroids: k distinct rows by a partial Fisher-Yates of mt19937(seed)
    std::vector<uint32_t> init(static_cast<size_t>(P) * k);
    for (int p = 0; p < P; ++p) {
        std::mt19937 rng(seed_or_random(seeds[p]));
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        for (int i = 0; i < k; ++i) {
            std::uniform_int_distribution<size_t> dist(i, n - 1);
            const size_t pick = dist(rng);
            std::swap(idx[i], idx[pick]);
            init[static_cast<size_t>(p) * k + i] = static_cast<uint32_t>(p * n + idx[i]);
        }
    }
    DevBuf<float> cent(P * kd, st);
    {
        DevBuf<uint32_t> di(init.size(), st);
        h2d(di.get(), init.data(), init.size(), st);
        gather_rows(x_dev, di.get(), init.size(), d, cent.get(), st);
    }
    KMeansOut out;
    out.centroids.resize(P * kd);
    out.assign.resize(static_cast<size_t>(P) * n);
    DevBuf<uint32_t> asg(static_cast<size_t>(P) * n, st), dorder(static_cast<size_t>(P) * n, st),
        doff(static_cast<size_t>(P) * (k + 1), st);
    DevBuf<float> sums(P * kd, st), dist;
    std::vector<uint32_t> order(static_cast<size_t>(P) * n), off(static_cast<size_t>(P) * (k + 1)), counts(k);
    std::vector<size_t> sizes(static_cast<size_t>(P) * k);
    std::vector<float> nc(P * kd);
    const bool small = k <= 64;
    auto assign_all = [&]() {
        if (small) {
            assign_small(x_dev, n, d, cent.get(), k, P, asg.get(), st);
        } else {
            for (int p = 0; p < P; ++p)
                assign_nearest(x_dev + static_cast<size_t>(p) * n * d, n, cent.get() + p * kd, k, d,
                               asg.get() + static_cast<size_t>(p) * n, st);
        }
        d2h(out.assign.data(), asg.get(), out.assign.size(), st);
    };
    for (size_t it = 0; it < iters; ++it) {
        assign_all();
        for (int p = 0; p < P; ++p) {
            bucket(out.assign.data() + static_cast<size_t>(p) * n, n, k, order.data() + static_cast<size_t>(p) * n,
                   off.data() + static_cast<size_t>(p) * (k + 1), counts.data());
            for (int c = 0; c < k; ++c) sizes[static_cast<size_t>(p) * k + c] = counts[c];
        }
        h2d(dorder.get(), order.data(), order.size(), st);
        h2d(doff.get(), off.data(), off.size(), st);
        member_sums(x_dev, n, d, dorder.get(), doff.get(), k, P, sums.get(), st);
        d2h(nc.data(), sums.get(), nc.size(), st);
        // means (float division), unit length for spherical k-means
        for (int p = 0; p < P; ++p)
            for (int c = 0; c < k; ++c) {
                const size_t cnt = sizes[static_cast<size_t>(p) * k + c];
                if (cnt == 0) continue;
                float* s = nc.data() + p * kd + static_cast<size_t>(c) * d;
                const float fc = static_cast<float>(cnt);
                for (int l = 0; l < d; ++l) s[l] /= fc;
                if (spherical) {
                    double sq = 0;
                    for (int l = 0; l < d; ++l) sq += double(s[l]) * s[l];
                    if (sq > 0) {
                        const float scale = static_cast<float>(1.0 / std::sqrt(sq));
                        for (int l = 0; l < d; ++l) s[l] *= scale;
                    }
                }
            }
        // reseed empty clusters onto the points furthest from their centroid
        bool any_empty = false;
        for (size_t e = 0; e < sizes.size() && !any_empty; ++e) any_empty = sizes[e] == 0;
        if (any_empty) {
            h2d(sums.get(), nc.data(), nc.size(), st);
            dist.alloc(static_cast<size_t>(P) * n, st);
            own_dist(x_dev, n, d, sums.get(), k, asg.get(), P, dist.get(), st);
            std::vector<float> hd(static_cast<size_t>(P) * n);
            d2h(hd.data(), dist.get(), hd.size(), st);
            for (int p = 0; p < P; ++p) {
                size_t* sz = sizes.data() + static_cast<size_t>(p) * k;
                float* cp = nc.data() + p * kd;
                std::vector<size_t> empty;
                for (int c = 0; c < k; ++c)
                    if (sz[c] == 0) empty.push_back(c);
                if (empty.empty()) continue;
                const size_t E = empty.size();
                std::priority_queue<std::pair<float, size_t>, std::vector<std::pair<float, size_t>>,
                                    std::greater<std::pair<float, size_t>>>
                    heap;
                const float* pd = hd.data() + static_cast<size_t>(p) * n;
                for (size_t i = 0; i < n; ++i) {
                    const float dd = pd[i];
                    if (dd < 1e-6f) continue;
                    if (heap.size() < E) heap.emplace(dd, i);
                    else if (dd > heap.top().first) {
                        heap.pop();
                        heap.emplace(dd, i);
                    }
                }
                for (size_t e = 0; e < E; ++e) {
                    if (!heap.empty()) {
                        const size_t index = heap.top().second;
                        heap.pop();
                        QG_CUDA(cudaMemcpyAsync(cp + empty[e] * d, x_dev + (static_cast<size_t>(p) * n + index) * d,
                                                d * sizeof(float), cudaMemcpyDeviceToHost, st));
                        QG_CUDA(cudaStreamSynchronize(st));
                    } else {
                        const size_t largest = static_cast<size_t>(std::max_element(sz, sz + k) - sz);
                        const float eps = 1.0f / 1024.0f;
                        float* src = cp + largest * d;
                        float* dst = cp + empty[e] * d;
                        for (int l = 0; l < d; ++l) {
                            dst[l] = src[l] * (1.0f + eps);
                            src[l] *= (1.0f - eps);
                        }
                        sz[empty[e]] = sz[largest] / 2;
                        sz[largest] -= sz[empty[e]];
                    }
                }
            }
        }
        h2d(cent.get(), nc.data(), nc.size(), st);
    }
    assign_all();
    d2h(out.centroids.data(), cent.get(), out.centroids.size(), st);
    return out;
}

// ---------------------------------------------------------------------------
// e-means
// ---------------------------------------------------------------------------
KMeansOut emeans(const float* x_dev, size_t n, int d, int k, size_t passes, std::optional<uint32_t> seed,
                 bool spherical, cudaStream_t st) {
    if (n < static_cast<size_t>(k)) throw Error(kInvalidArgument, "emeans: need at least k points");
    if (passes == 0) throw Error(kInvalidArgument, "emeans: need at least one pass");
    std::mt19937 rng(seed_or_random(seed));
    const double T = double(passes), nd = double(n), kd = double(k);
    const bool quality = d <= 16;
    size_t batch = round_power_of_two((quality ? 0.00439175 : 0.035134) * std::pow(kd, 0.134749) *
                                      std::pow(nd, 0.876473) * std::pow(T, 0.813344));
    batch = quality ? std::min(batch, n / 2) : std::min(batch, round_power_of_two(nd / 2));
    batch = std::max<size_t>(1, std::min(batch, n));
    const double alpha0 = std::clamp(0.8244 * std::pow(kd, -0.4617) * std::pow(double(batch), 0.9003) *
                                         std::pow(nd, -0.4498) * std::pow(T, -0.1057),
                                     1e-4, 1.0);
    const size_t steps_per_pass = (n + batch - 1) / batch, total_steps = passes * steps_per_pass;
    const float tau = d <= 2 ? 0.0f : 0.1f;
    const size_t K = static_cast<size_t>(k), D = static_cast<size_t>(d);

    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    for (size_t i = 0; i < K; ++i) {
        std::uniform_int_distribution<size_t> pick(i, n - 1);
        std::swap(order[i], order[pick(rng)]);
    }
    std::vector<float> pos(K * D);
    {
        std::vector<uint32_t> idx(order.begin(), order.begin() + K);
        DevBuf<uint32_t> di(K, st);
        DevBuf<float> rows(K * D, st);
        h2d(di.get(), idx.data(), K, st);
        gather_rows(x_dev, di.get(), K, d, rows.get(), st);
        d2h(pos.data(), rows.get(), K * D, st);
    }
    if (spherical) unit_rows(pos.data(), K, D, pos.data());
    std::vector<float> mass(K, 1.0f / 65536.0f);
    std::vector<float> readout(spherical ? K * D : 0), sums(K * D), pass_sums(K * D, 0.0f);
    std::vector<double> pass_counts(K, 0.0);
    std::vector<uint32_t> counts(K), labels(batch), border(batch), boff(K + 1), bidx(batch);
    std::uniform_real_distribution<double> unif(0.0, 1.0);

    DevBuf<uint32_t> d_idx(batch, st), d_lab(batch, st), d_order(batch, st), d_off(K + 1, st);
    DevBuf<float> d_rows(batch * D, st), d_cent(K * D, st), d_sums(K * D, st);

    size_t step = 0;
    for (size_t pass = 0; pass < passes; ++pass) {
        std::shuffle(order.begin(), order.end(), rng);
        const bool last = pass + 1 == passes;
        for (size_t start = 0; start < n; start += batch, ++step) {
            const size_t b = std::min(batch, n - start);
            for (size_t r = 0; r < b; ++r) bidx[r] = static_cast<uint32_t>(order[start + r]);
            h2d(d_idx.get(), bidx.data(), b, st);
            gather_rows(x_dev, d_idx.get(), b, d, d_rows.get(), st);
            const float* cent = pos.data();
            if (spherical) {
                unit_rows(pos.data(), K, D, readout.data());
                cent = readout.data();
            }
            h2d(d_cent.get(), cent, K * D, st);
            assign_nearest(d_rows.get(), b, d_cent.get(), K, d, d_lab.get(), st);
            d2h(labels.data(), d_lab.get(), b, st);
            bucket(labels.data(), b, k, border.data(), boff.data(), counts.data());
            h2d(d_order.get(), border.data(), b, st);
            h2d(d_off.get(), boff.data(), K + 1, st);
            member_sums(d_rows.get(), b, d, d_order.get(), d_off.get(), k, 1, d_sums.get(), st);
            d2h(sums.data(), d_sums.get(), K * D, st);
            if (last) {
                for (size_t j = 0; j < K; ++j) pass_counts[j] += counts[j];
                for (size_t i = 0; i < K * D; ++i) pass_sums[i] += sums[i];
            }

            const double frac = double(std::min(step, total_steps)) / double(std::max<size_t>(1, total_steps));
            // 0.1 + 0.9 * 0.5 * (1 + cos(pi * frac)), the release build fusing the multiply-add
            const double alpha = alpha0 * std::fma(1.0 + std::cos(std::numbers::pi * frac), 0.9 * 0.5, 0.1);
            const bool replace = alpha == 1.0;
            if (!replace)
                for (float& m : mass) m = static_cast<float>(m * (1.0 - alpha));
            const float af = static_cast<float>(alpha);
            for (size_t j = 0; j < K; ++j) {
                if (counts[j] == 0) continue;
                const float nj = static_cast<float>(counts[j]);
                const float new_mass = std::fma(af, nj, replace ? 0.0f : mass[j]);
                const float w = (af * nj) / new_mass;
                float* c = pos.data() + j * D;
                const float* s = sums.data() + j * D;
                for (size_t l = 0; l < D; ++l) {
                    const float mean = s[l] / nj;
                    c[l] = w == 1.0f ? mean : std::fma(w, mean - c[l], c[l]);
                }
                mass[j] = new_mass;
            }

            // revival: split heavy donors into clusters that lost their mass
            if (tau > 0 && (step + 1) % 5 == 0) {
                float total = 0;
                for (float m : mass) total += m;
                const float threshold = total * tau / static_cast<float>(k);
                std::vector<size_t> unused;
                std::vector<std::pair<double, size_t>> donors;
                for (size_t j = 0; j < K; ++j) {
                    if (mass[j] < threshold) unused.push_back(j);
                    else if (mass[j] > 0) donors.emplace_back(0.0, j);
                }
                const size_t nsplit = std::min(unused.size(), donors.size());
                if (nsplit > 0) {
                    for (auto& [key, j] : donors)
                        key = std::log(double(mass[j])) - std::log(-std::log(std::max(unif(rng), 1e-300)));
                    std::partial_sort(donors.begin(), donors.begin() + nsplit, donors.end(), std::greater<>());
                    for (size_t t = 0; t < nsplit; ++t) {
                        const size_t src = donors[t].second, dst = unused[t];
                        float* a = pos.data() + src * D;
                        float* c = pos.data() + dst * D;
                        bool same = true;
                        for (size_t l = 0; l < D; ++l) {
                            const float off = (l % 2 == 0 ? 1e-4f : -1e-4f);
                            const float v = a[l];
                            a[l] = v * (1.0f - off);
                            c[l] = v * (1.0f + off);
                            same = same && a[l] == c[l];
                        }
                        if (same) c[0] = std::nextafter(c[0], std::numeric_limits<float>::infinity());
                        mass[src] = mass[dst] = mass[src] / 2.0f;
                    }
                }
            }
        }
    }
    // closing: means of the last pass's assignments; unassigned clusters keep their position
    for (size_t j = 0; j < K; ++j) {
        if (pass_counts[j] <= 0) continue;
        const float cnt = static_cast<float>(pass_counts[j]);
        for (size_t l = 0; l < D; ++l) pos[j * D + l] = pass_sums[j * D + l] / cnt;
    }
    if (spherical) unit_rows(pos.data(), K, D, pos.data());

    KMeansOut out;
    out.centroids = pos;
    out.assign.resize(n);
    h2d(d_cent.get(), pos.data(), K * D, st);
    DevBuf<uint32_t> tmp;
    assign_dev(x_dev, n, d, d_cent.get(), k, out.assign.data(), tmp, st);
    return out;
}

// ---------------------------------------------------------------------------
// Host restatements used by pick_cosine_inner_product (a training-time
// decision over 200 sample queries), in the same arithmetic as the kernels.
// ---------------------------------------------------------------------------
namespace {

float ip_avx2(const float* a, const float* b, size_t n) {
    float acc[4][8] = {};
    size_t i = 0;
    for (; i + 32 <= n; i += 32)
        for (int j = 0; j < 4; ++j)
            for (int L = 0; L < 8; ++L) acc[j][L] = std::fma(a[i + 8 * j + L], b[i + 8 * j + L], acc[j][L]);
    for (; i + 8 <= n; i += 8)
        for (int L = 0; L < 8; ++L) acc[0][L] = std::fma(a[i + L], b[i + L], acc[0][L]);
    float s[8];
    for (int L = 0; L < 8; ++L) s[L] = (acc[0][L] + acc[1][L]) + (acc[2][L] + acc[3][L]);
    float r = ((s[0] + s[4]) + (s[1] + s[5])) + ((s[2] + s[6]) + (s[3] + s[7]));
    if (n - i >= 4) {
        for (size_t e = i; e < i + 4; ++e) {
            const float p = a[e] * b[e];
            r = r + p;
        }
        i += 4;
    }
    for (; i < n; ++i) r = std::fma(a[i], b[i], r);
    return r;
}

void inner_table_h(const float* q, const float* yt, size_t m, size_t sd, float* out) {
    for (size_t s = 0; s < m; ++s)
        for (int k = 0; k < 16; ++k) {
            float o = 0.0f;
            for (size_t j = 0; j < sd; ++j) o = std::fma(-2.0f * q[s * sd + j], yt[(s * sd + j) * 16 + k], o);
            out[s * 16 + k] = o;
        }
}

void adc_table_h(const float* r, const float* yt, size_t m, size_t sd, float* out) {
    for (size_t s = 0; s < m; ++s)
        for (int k = 0; k < 16; ++k) {
            float o = 0.0f;
            for (size_t j = 0; j < sd; ++j) {
                const float d = r[s * sd + j] - yt[(s * sd + j) * 16 + k];
                o = std::fma(d, d, o);
            }
            out[s * 16 + k] = o;
        }
}

void quantize_h(const float* table, size_t m, uint8_t* lut, float& scale, float& offset) {
    std::vector<float> mins(m);
    float widest = 0.0f, part[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < m; ++i) {
        const float* row = table + i * 16;
        float lo = row[0], hi = row[0];
        for (int j = 1; j < 16; ++j) {
            lo = std::min(lo, row[j]);
            hi = std::max(hi, row[j]);
        }
        mins[i] = lo;
        part[i % 4] += lo;
        widest = std::max(widest, hi - lo);
    }
    offset = (part[0] + part[1]) + (part[2] + part[3]);
    scale = widest > 0.0f ? 63.0f / widest : 1.0f;
    for (size_t i = 0; i < m; ++i)
        for (int j = 0; j < 16; ++j)
            lut[i * 16 + j] = static_cast<uint8_t>(std::nearbyint((table[i * 16 + j] - mins[i]) * scale));
}

// Whether cosine PQ ranks the sample better by inner product (true) or by
// per-list L2 tables: rows [0, nd) are scored, rows [n - 200, n) query them.
bool pick_cosine_inner_product(const IVFModel& M, const float* x_dev, size_t n, const std::vector<uint32_t>& assign,
                               const std::vector<float>& centers, cudaStream_t st) {
    constexpr size_t kQueries = 200, kRows = 20000, kCandidates = 2000, kTop = 10, kKept = 20;
    if (n < kQueries + kCandidates) return true;
    const size_t nq = kQueries, nd = std::min(kRows, n - nq);
    const size_t m = M.pq.m, K = M.pq.K, T = m * K, dim = M.dim, sd = M.pq.sub_dim, nlist = M.nlist;
    const std::vector<float> yt = M.pq.transposed();

    // codes of the scored rows and the query rows on the host
    std::vector<uint8_t> codes(nd * m);
    std::vector<float> rows(nd * dim), queries(nq * dim);
    {
        DevBuf<float> dc(centers.size(), st), dyt(yt.size(), st);
        DevBuf<uint32_t> da(nd, st);
        DevBuf<uint8_t> dcodes(nd * m, st);
        h2d(dc.get(), centers.data(), centers.size(), st);
        h2d(dyt.get(), yt.data(), yt.size(), st);
        h2d(da.get(), assign.data(), nd, st);
        encode16(x_dev, nd, static_cast<int>(dim), dc.get(), da.get(), dyt.get(), static_cast<int>(m),
                 static_cast<int>(sd), dcodes.get(), st);
        d2h(codes.data(), dcodes.get(), codes.size(), st);
        d2h(rows.data(), x_dev, rows.size(), st);
        d2h(queries.data(), x_dev + (n - nq) * dim, queries.size(), st);
    }
    std::vector<std::vector<uint32_t>> by_list(nlist);
    for (size_t i = 0; i < nd; ++i) by_list[assign[i]].push_back(static_cast<uint32_t>(i));

    size_t total_ip = 0, total_l2 = 0;
    std::vector<float> table(T), resid(dim);
    std::vector<uint8_t> lut(T), list_lut(T);
    for (size_t qi = 0; qi < nq; ++qi) {
        const float* q = queries.data() + qi * dim;
        std::vector<std::pair<float, uint32_t>> lists(nlist);
        for (size_t l = 0; l < nlist; ++l)
            lists[l] = {-ip_avx2(q, M.centroids.data() + l * dim, dim), static_cast<uint32_t>(l)};
        std::sort(lists.begin(), lists.end());
        std::vector<uint32_t> probed;
        size_t nrows = 0;
        for (size_t p = 0; p < nlist && nrows < kCandidates; ++p) {
            if (by_list[lists[p].second].empty()) continue;
            probed.push_back(lists[p].second);
            nrows += by_list[lists[p].second].size();
        }
        std::vector<std::pair<float, uint32_t>> exact, ip, l2;
        inner_table_h(q, yt.data(), m, sd, table.data());
        float ip_scale = 1.0f, ip_offset = 0.0f;
        quantize_h(table.data(), m, lut.data(), ip_scale, ip_offset);
        for (uint32_t l : probed) {
            const float* c = centers.data() + static_cast<size_t>(l) * dim;
            const float base = std::fma(-2.0f, ip_avx2(q, c, dim), 2.0f);
            for (size_t dd = 0; dd < dim; ++dd) resid[dd] = q[dd] - c[dd];
            adc_table_h(resid.data(), yt.data(), m, sd, table.data());
            float l2_scale = 1.0f, l2_offset = 0.0f;
            quantize_h(table.data(), m, list_lut.data(), l2_scale, l2_offset);
            for (uint32_t i : by_list[l]) {
                const uint8_t* code = codes.data() + static_cast<size_t>(i) * m;
                uint32_t a = 0, b = 0;
                for (size_t s = 0; s < m; ++s) {
                    a += lut[s * K + code[s]];
                    b += list_lut[s * K + code[s]];
                }
                const float s_ip = static_cast<float>(a) / ip_scale + ip_offset;
                const float s_l2 = static_cast<float>(b) / l2_scale + l2_offset;
                exact.emplace_back(-ip_avx2(q, rows.data() + static_cast<size_t>(i) * dim, dim), i);
                ip.emplace_back(base + s_ip, i);
                l2.emplace_back(s_l2, i);
            }
        }
        const size_t top = std::min(kTop, exact.size()), kept = std::min(kKept, exact.size());
        std::partial_sort(exact.begin(), exact.begin() + top, exact.end());
        std::partial_sort(ip.begin(), ip.begin() + kept, ip.end());
        std::partial_sort(l2.begin(), l2.begin() + kept, l2.end());
        for (size_t t = 0; t < top; ++t) {
            const uint32_t want = exact[t].second;
            for (size_t j = 0; j < kept; ++j) total_ip += ip[j].second == want;
            for (size_t j = 0; j < kept; ++j) total_l2 += l2[j].second == want;
        }
    }
    return total_ip >= total_l2;
}

} // namespace

// ---------------------------------------------------------------------------
// IVFIndex::train
// ---------------------------------------------------------------------------
void train(IVFObj& o, const float* x, size_t n, size_t max_iters, int64_t seed_in, int clustering, size_t passes,
           cudaStream_t st) {
    IVFModel& M = o.model;
    if (M.idmap.slots() > 0) throw Error(kLogicError, "train() cannot be called after add()");
    if (M.trained) throw Error(kLogicError, "train() has already been called");
    if (n < M.nlist) throw Error(kInvalidArgument, "training set must have at least nlist vectors");
    require(M.sq_bits == 0, "SQ lists are not on the GPU path", kUnsupported);
    require(!M.has_pq || M.pq.K <= 256, "PQ needs at most 256 centroids per subspace");
    const std::optional<uint32_t> seed = seed_in >= 0 ? std::optional<uint32_t>(static_cast<uint32_t>(seed_in))
                                                      : std::nullopt;
    const size_t dim = M.dim;
    const bool cosine = M.metric == Metric::Cosine;
    DevBuf<float> xd(n * dim, st);
    {
        DevBuf<float> raw(n * dim, st);
        h2d(raw.get(), x, n * dim, st);
        if (cosine) {
            DevBuf<int> zero(1, st);
            QG_CUDA(cudaMemsetAsync(zero.get(), 0, sizeof(int), st));
            normalize_rows(raw.get(), xd.get(), static_cast<int>(n), static_cast<int>(dim), zero.get(), st);
            int z = 0;
            d2h(&z, zero.get(), 1, st);
            if (z) throw Error(kInvalidArgument, "cosine metric needs non-zero vectors");
        } else {
            xd = std::move(raw);
        }
    }
    const int k = static_cast<int>(M.nlist), d = static_cast<int>(dim);
    // learn the rotation, then cluster and train the codebook on the rotated
    // rows (reference src/ivf_index.cpp:738-745, src/rotation.cpp:71-130)
    std::vector<float> rotation;
    if (M.rotate) {
        if (M.pq.m == 0 || dim % M.pq.m != 0) throw Error(kInvalidArgument, "dim must be divisible by num_subspaces");
        rotation = balanced_rotation(covariance(xd.get(), n, d, st), dim, M.pq.m);
        DevBuf<float> R(rotation.size(), st), xr(n * dim, st);
        h2d(R.get(), rotation.data(), rotation.size(), st);
        rotate_rows(R.get(), xd.get(), n, d, xr.get(), st);
        QG_CUDA(cudaStreamSynchronize(st));
        xd = std::move(xr);
    }
    KMeansOut res = clustering == 0 ? emeans(xd.get(), n, d, k, passes, seed, cosine, st)
                                    : kmeans_lloyd(xd.get(), n, d, k, max_iters, {seed}, cosine, 1, st);
    std::vector<float> centroids = std::move(res.centroids);
    const std::vector<uint32_t>& assign = res.assign;

    std::vector<float> residual_centers;
    if (M.has_pq && cosine) {
        // each list's mean of its training vectors, summed in point order
        std::vector<uint32_t> order(n), off(M.nlist + 1), counts(M.nlist);
        bucket(assign.data(), n, k, order.data(), off.data(), counts.data());
        DevBuf<uint32_t> dorder(n, st), doff(M.nlist + 1, st);
        DevBuf<float> dsums(M.nlist * dim, st);
        h2d(dorder.get(), order.data(), n, st);
        h2d(doff.get(), off.data(), off.size(), st);
        member_sums(xd.get(), n, d, dorder.get(), doff.get(), k, 1, dsums.get(), st);
        residual_centers.resize(M.nlist * dim);
        d2h(residual_centers.data(), dsums.get(), residual_centers.size(), st);
        for (size_t l = 0; l < M.nlist; ++l) {
            float* e = residual_centers.data() + l * dim;
            if (counts[l] == 0) std::copy_n(centroids.data() + l * dim, dim, e);
            else
                for (size_t j = 0; j < dim; ++j) e[j] /= static_cast<float>(counts[l]);
        }
    }
    bool cosine_ip = M.cosine_ip;
    std::vector<float> pq_centroids;
    if (M.has_pq) {
        const std::vector<float>& centers = residual_centers.empty() ? centroids : residual_centers;
        DevBuf<float> dcent(centers.size(), st), resid(n * dim, st);
        DevBuf<uint32_t> dasg(n, st);
        h2d(dcent.get(), centers.data(), centers.size(), st);
        h2d(dasg.get(), assign.data(), n, st);
        residuals(xd.get(), n, d, dcent.get(), dasg.get(), resid.get(), st);
        // PQCodebook::train(residuals, n, 25, seed + 1)
        const size_t K = M.pq.K, m = M.pq.m, sd = M.pq.sub_dim;
        if (n < K) throw Error(kInvalidArgument, "training set must have at least centroids_per_subspace_ vectors");
        const std::optional<uint32_t> pq_seed = seed ? std::optional<uint32_t>(*seed + 1) : std::nullopt;
        const size_t cap = 256 * K;
        size_t nn = n;
        DevBuf<float> subset;
        const float* src = resid.get();
        if (n > cap) {
            std::mt19937 rng(seed_or_random(pq_seed));
            std::vector<size_t> rows(n);
            std::iota(rows.begin(), rows.end(), 0);
            std::vector<uint32_t> pick_rows(cap);
            for (size_t i = 0; i < cap; ++i) {
                std::uniform_int_distribution<size_t> pick(i, n - 1);
                std::swap(rows[i], rows[pick(rng)]);
                pick_rows[i] = static_cast<uint32_t>(rows[i]);
            }
            DevBuf<uint32_t> di(cap, st);
            h2d(di.get(), pick_rows.data(), cap, st);
            subset.alloc(cap * dim, st);
            gather_rows(resid.get(), di.get(), cap, d, subset.get(), st);
            src = subset.get();
            nn = cap;
        }
        DevBuf<float> cols(nn * dim, st);
        split_columns(src, nn, d, static_cast<int>(sd), static_cast<int>(m), cols.get(), st);
        std::vector<std::optional<uint32_t>> seeds(m);
        for (size_t i = 0; i < m; ++i)
            seeds[i] = pq_seed ? std::optional<uint32_t>(*pq_seed + static_cast<uint32_t>(i)) : std::nullopt;
        KMeansOut pq = kmeans_lloyd(cols.get(), nn, static_cast<int>(sd), static_cast<int>(K), 25, seeds, false,
                                    static_cast<int>(m), st);
        pq_centroids = std::move(pq.centroids);   // m * K * sd: the codebook layout
        M.pq.centroids = pq_centroids;
        if (cosine && M.pq_distance == 0) {
            require(M.fast_scan && K == 16,
                    "cosine IVF-PQ training on the GPU path needs fast-scan codes (enable_pq(m, fast_scan=True))",
                    kUnsupported);
            IVFModel probe = M;   // the decision reads centroids and the new codebook
            probe.centroids = centroids;
            cosine_ip = pick_cosine_inner_product(probe, xd.get(), n, assign, centers, st);
        }
    }
    M.centroids = std::move(centroids);
    M.rotation = std::move(rotation);
    M.residual_centers = std::move(residual_centers);
    M.cosine_ip = cosine_ip;
    M.trained = true;
    o.dev_dirty = true;
}

} // namespace qg
