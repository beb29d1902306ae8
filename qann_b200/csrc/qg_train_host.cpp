// Training on the GPU: the host side. Only the random draws stay here:
// libstdc++'s mt19937 and its distributions replay the reference's choices
// (initial rows, the per-pass shuffles of e-means, the donor draws of its
// revival step, the PQ subsample), in the reference's call order, so a GPU
// train writes the same index bytes. Every step that touches the data runs
// on the device (qg_cluster.cu, qg_train.cu, qg_build.cu, qg_search.cu): a
// k-means iteration or an e-means batch is a chain of kernels on one stream,
// and the host reads back only what a draw depends on (the masses before a
// revival, a flag for empty clusters) and the final centroids.
//
//   kmeans_lloyd    Lloyd iterations for P problems at once
//                   (reference src/kmeans.cpp:174-252, reseed :117-172)
//   emeans          mini-batch EMA k-means (reference src/kmeans.cpp:254-414)
//   train           IVFIndex::train (reference src/ivf_index.cpp:725-806)
//
// Host float arithmetic here (the e-means schedule, the revival threshold)
// is built with -ffp-contract=off and writes std::fma where the reference's
// GCC build fuses a multiply into an add.
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

// The first `count` places of a partial Fisher-Yates shuffle of 0..n-1 drawn
// from rng: place i swaps with a uniform pick from [i, n). `perm` keeps the
// whole permutation state (e-means goes on shuffling it).
void fisher_yates_prefix(std::vector<size_t>& perm, size_t count, std::mt19937& rng) {
    std::iota(perm.begin(), perm.end(), size_t{0});
    for (size_t i = 0; i < count; ++i) {
        std::uniform_int_distribution<size_t> pick(i, perm.size() - 1);
        std::swap(perm[i], perm[pick(rng)]);
    }
}

// ---- Lloyd: empty clusters --------------------------------------------------
// The E clusters left without points take points far from their own
// centroids (own distance >= 1e-6): E (distance, point) pairs are kept in a
// min-heap that admits a point only when its distance beats the heap's
// smallest, and the heap is drained smallest first into the empty clusters in
// cluster order. With no such point left, the largest cluster is split in
// two. Rare, so this runs on the host from the device's distances.
void refill_empty_clusters(const float* x_dev, size_t n, int d, int k, int P, float* next_dev, const uint32_t* labels,
                           const uint32_t* off_dev, cudaStream_t st) {
    const size_t kd = static_cast<size_t>(k) * d;
    std::vector<float> cent(P * kd);
    std::vector<uint32_t> off(static_cast<size_t>(P) * (k + 1));
    std::vector<float> dist(static_cast<size_t>(P) * n);
    {
        DevBuf<float> dd(dist.size(), st);
        own_dist(x_dev, n, d, next_dev, k, labels, P, dd.get(), st);
        d2h(dist.data(), dd.get(), dist.size(), st);
    }
    d2h(cent.data(), next_dev, cent.size(), st);
    d2h(off.data(), off_dev, off.size(), st);
    using Far = std::pair<float, size_t>;
    for (int p = 0; p < P; ++p) {
        std::vector<size_t> size(k);
        for (int c = 0; c < k; ++c) size[c] = off[p * (k + 1) + c + 1] - off[p * (k + 1) + c];
        std::vector<int> holes;
        for (int c = 0; c < k; ++c)
            if (size[c] == 0) holes.push_back(c);
        if (holes.empty()) continue;
        std::priority_queue<Far, std::vector<Far>, std::greater<Far>> far;
        const float* pd = dist.data() + static_cast<size_t>(p) * n;
        for (size_t i = 0; i < n; ++i) {
            if (pd[i] < 1e-6f) continue;
            if (far.size() < holes.size()) far.emplace(pd[i], i);
            else if (pd[i] > far.top().first) {
                far.pop();
                far.emplace(pd[i], i);
            }
        }
        float* cp = cent.data() + p * kd;
        for (int hole : holes) {
            if (!far.empty()) {
                const size_t i = far.top().second;
                far.pop();
                QG_CUDA(cudaMemcpyAsync(cp + static_cast<size_t>(hole) * d, x_dev + (static_cast<size_t>(p) * n + i) * d,
                                        d * sizeof(float), cudaMemcpyDeviceToHost, st));
                QG_CUDA(cudaStreamSynchronize(st));
                continue;
            }
            const size_t big = static_cast<size_t>(std::max_element(size.begin(), size.end()) - size.begin());
            constexpr float kApart = 1.0f / 1024.0f;
            float* keep = cp + big * d;
            float* fill = cp + static_cast<size_t>(hole) * d;
            for (int l = 0; l < d; ++l) {
                fill[l] = keep[l] * (1.0f + kApart);
                keep[l] *= (1.0f - kApart);
            }
            size[hole] = size[big] / 2;
            size[big] -= size[hole];
        }
    }
    h2d(next_dev, cent.data(), cent.size(), st);
}

} // namespace

// ---------------------------------------------------------------------------
// Lloyd
// ---------------------------------------------------------------------------
KMeansOut kmeans_lloyd(const float* x_dev, size_t n, int d, int k, size_t iters,
                       const std::vector<std::optional<uint32_t>>& seeds, bool spherical, int P, cudaStream_t st) {
    if (n < static_cast<size_t>(k)) throw Error(kInvalidArgument, "kmeans: need at least k points");
    const size_t kd = static_cast<size_t>(k) * d, pn = static_cast<size_t>(P) * n;
    // starting centroids: k distinct rows per problem
    std::vector<uint32_t> start(static_cast<size_t>(P) * k);
    {
        std::vector<size_t> perm(n);
        for (int p = 0; p < P; ++p) {
            std::mt19937 rng(seed_or_random(seeds[p]));
            fisher_yates_prefix(perm, k, rng);
            for (int i = 0; i < k; ++i) start[static_cast<size_t>(p) * k + i] = static_cast<uint32_t>(p * n + perm[i]);
        }
    }
    DevBuf<float> cent(P * kd, st), next(P * kd, st), sums(P * kd, st);
    {
        DevBuf<uint32_t> rows(start.size(), st);
        h2d(rows.get(), start.data(), start.size(), st);
        gather_rows(x_dev, rows.get(), start.size(), d, cent.get(), st);
    }
    KMeansOut out;
    out.assign.alloc(pn, st);
    DevBuf<uint32_t> order(pn, st), off(static_cast<size_t>(P) * (k + 1), st);
    DevBuf<int> empty(1, st);
    auto assign_all = [&]() {
        if (k <= 64) {
            assign_small(x_dev, n, d, cent.get(), k, P, out.assign.get(), st);
            return;
        }
        for (int p = 0; p < P; ++p)
            assign_nearest(x_dev + static_cast<size_t>(p) * n * d, n, cent.get() + p * kd, k, d,
                           out.assign.get() + static_cast<size_t>(p) * n, st);
    };
    for (size_t it = 0; it < iters; ++it) {
        assign_all();
        group_by_label(out.assign.get(), n, k, P, order.get(), off.get(), st);
        member_sums(x_dev, n, d, order.get(), off.get(), k, P, sums.get(), st);
        QG_CUDA(cudaMemsetAsync(empty.get(), 0, sizeof(int), st));
        cluster_means(sums.get(), off.get(), k, d, P, spherical, nullptr, next.get(), empty.get(), st);
        int any_empty = 0;
        d2h(&any_empty, empty.get(), 1, st);
        if (any_empty)
            refill_empty_clusters(x_dev, n, d, k, P, next.get(), out.assign.get(), off.get(), st);
        std::swap(cent, next);
    }
    assign_all();
    out.centroids.resize(P * kd);
    d2h(out.centroids.data(), cent.get(), out.centroids.size(), st);
    out.centroids_dev = std::move(cent);
    return out;
}

// ---------------------------------------------------------------------------
// e-means
// ---------------------------------------------------------------------------
namespace {

size_t nearest_power_of_two(double v) {
    if (v <= 1) return 1;
    const size_t below = size_t{1} << static_cast<int>(std::floor(std::log2(v)));
    return v / double(below) < double(2 * below) / v ? below : 2 * below;
}

// The schedule of faiss's e-means (contrib/e_means, NumpyEmeans), which the
// reference adopts: a batch-size law (the throughput law above 16 dimensions,
// the quality law at or below), a base step alpha0 from a second law, a
// cosine-annealed step down to 0.1 alpha0, and revival every 5 steps of the
// clusters under tau = 0.1 of the mean mass (none at d <= 2).
struct EMeansPlan {
    size_t batch = 1, steps = 1;
    double alpha0 = 1.0;
    float tau = 0.0f;

    EMeansPlan(size_t n, int d, int k, size_t passes) {
        const double T = double(passes), N = double(n), K = double(k);
        const bool small_d = d <= 16;
        const double law = (small_d ? 0.00439175 : 0.035134) * std::pow(K, 0.134749) * std::pow(N, 0.876473) *
                           std::pow(T, 0.813344);
        size_t b = nearest_power_of_two(law);
        b = small_d ? std::min(b, n / 2) : std::min(b, nearest_power_of_two(N / 2));
        batch = std::max<size_t>(1, std::min(b, n));
        alpha0 = std::clamp(0.8244 * std::pow(K, -0.4617) * std::pow(double(batch), 0.9003) * std::pow(N, -0.4498) *
                                std::pow(T, -0.1057),
                            1e-4, 1.0);
        steps = passes * ((n + batch - 1) / batch);
        tau = d <= 2 ? 0.0f : 0.1f;
    }

    // step size of step s: alpha0 * (0.1 + 0.45 * (1 + cos(pi * s / steps))),
    // the multiply-add fused as the reference's build fuses it
    double alpha(size_t s) const {
        const double frac = double(std::min(s, steps)) / double(std::max<size_t>(1, steps));
        return alpha0 * std::fma(1.0 + std::cos(std::numbers::pi * frac), 0.9 * 0.5, 0.1);
    }
};

// Revival plan from the masses after a step: clusters whose mass fell under
// tau times the mean (the total summed in cluster order) are refilled from
// donors with positive mass at or above it, drawn without replacement in
// proportion to mass by Gumbel keys log(mass) - log(-log(u)), one u per donor
// in cluster order; the i-th largest (key, donor) refills the i-th starved
// cluster. Returns (donor, starved) pairs.
std::vector<uint32_t> plan_revival(const std::vector<float>& mass, float tau, std::mt19937& rng,
                                   std::uniform_real_distribution<double>& u01) {
    const size_t k = mass.size();
    float total = 0.0f;
    for (size_t j = 0; j < k; ++j) total += mass[j];
    const float floor_mass = total * tau / static_cast<float>(k);
    std::vector<uint32_t> starved;
    std::vector<std::pair<double, uint32_t>> donor;
    for (size_t j = 0; j < k; ++j) {
        if (mass[j] < floor_mass) starved.push_back(static_cast<uint32_t>(j));
        else if (mass[j] > 0) donor.emplace_back(0.0, static_cast<uint32_t>(j));
    }
    const size_t pairs = std::min(starved.size(), donor.size());
    std::vector<uint32_t> out;
    if (pairs == 0) return out;
    for (auto& [key, j] : donor) {
        const double u = std::max(u01(rng), 1e-300);
        key = std::log(double(mass[j])) - std::log(-std::log(u));
    }
    std::partial_sort(donor.begin(), donor.begin() + pairs, donor.end(), std::greater<>());
    out.reserve(2 * pairs);
    for (size_t t = 0; t < pairs; ++t) {
        out.push_back(donor[t].second);
        out.push_back(starved[t]);
    }
    return out;
}

} // namespace

KMeansOut emeans(const float* x_dev, size_t n, int d, int k, size_t passes, std::optional<uint32_t> seed,
                 bool spherical, cudaStream_t st) {
    if (n < static_cast<size_t>(k)) throw Error(kInvalidArgument, "emeans: need at least k points");
    if (passes == 0) throw Error(kInvalidArgument, "emeans: need at least one pass");
    const EMeansPlan plan(n, d, k, passes);
    const size_t K = static_cast<size_t>(k), B = plan.batch;
    std::mt19937 rng(seed_or_random(seed));
    std::uniform_real_distribution<double> u01(0.0, 1.0);

    // starting positions: the rows at the first k places of a partial shuffle,
    // which the passes then keep shuffling
    std::vector<size_t> perm(n);
    fisher_yates_prefix(perm, K, rng);
    std::vector<uint32_t> perm32(n);
    DevBuf<uint32_t> perm_dev(n, st);
    for (size_t i = 0; i < K; ++i) perm32[i] = static_cast<uint32_t>(perm[i]);
    h2d(perm_dev.get(), perm32.data(), K, st);
    EMeansState S;
    S.init(k, d, st);
    gather_rows(x_dev, perm_dev.get(), K, d, S.pos.get(), st);
    if (spherical) unit_rows_dev(S.pos.get(), K, d, S.pos.get(), st);

    DevBuf<float> rows(B * d, st), readout(spherical ? K * d : 0, st), sums(K * d, st);
    DevBuf<uint32_t> labels(B, st), members(B, st), off(K + 1, st);
    std::vector<float> mass(K);
    size_t step = 0;
    for (size_t pass = 0; pass < passes; ++pass) {
        std::shuffle(perm.begin(), perm.end(), rng);
        for (size_t i = 0; i < n; ++i) perm32[i] = static_cast<uint32_t>(perm[i]);
        h2d(perm_dev.get(), perm32.data(), n, st);
        const bool closing_pass = pass + 1 == passes;
        for (size_t at = 0; at < n; at += B, ++step) {
            const size_t b = std::min(B, n - at);
            gather_rows(x_dev, perm_dev.get() + at, b, d, rows.get(), st);
            const float* cent = S.pos.get();
            if (spherical) {
                unit_rows_dev(S.pos.get(), K, d, readout.get(), st);
                cent = readout.get();
            }
            assign_nearest(rows.get(), b, cent, K, d, labels.get(), st);
            group_by_label(labels.get(), b, k, 1, members.get(), off.get(), st);
            member_sums(rows.get(), b, d, members.get(), off.get(), k, 1, sums.get(), st);
            S.step(sums.get(), off.get(), plan.alpha(step), closing_pass, st);
            if (plan.tau > 0 && (step + 1) % 5 == 0) {
                d2h(mass.data(), S.mass.get(), K, st);
                S.split(plan_revival(mass, plan.tau, rng, u01), st);
            }
        }
        // the host copy of the permutation must not change under a pending upload
        QG_CUDA(cudaStreamSynchronize(st));
    }
    S.close(st);
    if (spherical) unit_rows_dev(S.pos.get(), K, d, S.pos.get(), st);

    KMeansOut out;
    out.assign.alloc(n, st);
    assign_nearest(x_dev, n, S.pos.get(), K, d, out.assign.get(), st);
    out.centroids.resize(K * d);
    d2h(out.centroids.data(), S.pos.get(), K * d, st);
    out.centroids_dev = std::move(S.pos);
    return out;
}

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
    const uint32_t* assign = res.assign.get();   // on the device

    // cosine with PQ: each list's plain mean of its training vectors (summed
    // in point order), or its centroid when it has none
    std::vector<float> residual_centers;
    DevBuf<float> centers_dev;
    if (M.has_pq && cosine) {
        DevBuf<uint32_t> order(n, st), off(M.nlist + 1, st);
        DevBuf<float> sums(M.nlist * dim, st);
        group_by_label(assign, n, k, 1, order.get(), off.get(), st);
        member_sums(xd.get(), n, d, order.get(), off.get(), k, 1, sums.get(), st);
        centers_dev.alloc(M.nlist * dim, st);
        cluster_means(sums.get(), off.get(), k, d, 1, false, res.centroids_dev.get(), centers_dev.get(), nullptr, st);
        residual_centers.resize(M.nlist * dim);
        d2h(residual_centers.data(), centers_dev.get(), residual_centers.size(), st);
    }
    bool cosine_ip = M.cosine_ip;
    std::vector<float> pq_centroids;
    if (M.has_pq) {
        const float* centers = residual_centers.empty() ? res.centroids_dev.get() : centers_dev.get();
        DevBuf<float> resid(n * dim, st);
        residuals(xd.get(), n, d, centers, assign, resid.get(), st);
        // PQCodebook::train(residuals, n, 25, seed + 1)
        const size_t K = M.pq.K, m = M.pq.m, sd = M.pq.sub_dim;
        if (n < K) throw Error(kInvalidArgument, "training set must have at least centroids_per_subspace_ vectors");
        const std::optional<uint32_t> pq_seed = seed ? std::optional<uint32_t>(*seed + 1) : std::nullopt;
        const size_t cap = 256 * K;
        size_t nn = n;
        DevBuf<float> subset;
        const float* src = resid.get();
        if (n > cap) {   // a random subsample of 256 K rows: a partial shuffle's first places
            std::mt19937 rng(seed_or_random(pq_seed));
            std::vector<size_t> perm(n);
            fisher_yates_prefix(perm, cap, rng);
            std::vector<uint32_t> pick_rows(perm.begin(), perm.begin() + cap);
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
            // the decision scores with the new codebook (transposed, m x sd x 16)
            const std::vector<float> yt = M.pq.transposed();
            DevBuf<float> yt_dev(yt.size(), st);
            h2d(yt_dev.get(), yt.data(), yt.size(), st);
            cosine_ip = cosine_ip_wins(xd.get(), n, d, assign, res.centroids_dev.get(), centers, k, yt_dev.get(),
                                       static_cast<int>(m), static_cast<int>(sd), st);
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
