// Test infrastructure only: a C shim over the reference qann C++ library so the
// oracle can drive the reference's own code from Python (ctypes). It is
// compiled, together with the reference sources, into oracle/_ref/libqann_ref.so
// by oracle/build_ref.sh. Only tests/, __graft_entry__.smoke() and bench.py's
// CPU baseline load it; nothing on the product path does.
//
// Every entry point returns 0 on success or a status code (1 = invalid
// argument, 2 = logic error, 3 = runtime error, 4 = other) and leaves the
// exception text in ref_last_error(), mirroring how the reference's Python
// bindings map std::invalid_argument / std::logic_error / std::runtime_error.

#include "vecengine/flat_index.hpp"
#include "vecengine/index.hpp"
#include "vecengine/index_factory.hpp"
#include "vecengine/ivf_index.hpp"
#include "vecengine/pq.hpp"
#include "vecengine/refine_index.hpp"
#include "vecengine/threads.hpp"
#include "vecengine/distance.hpp"

#include "fast_scan.hpp"
#include "kmeans.hpp"
#include "topk.hpp"
#include "rotation.hpp"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <sstream>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace vecengine;

namespace {

thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return 1;
    } catch (const std::logic_error& e) {
        g_err = e.what();
        return 2;
    } catch (const std::runtime_error& e) {
        g_err = e.what();
        return 3;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 4;
    }
}

// An index handle: the shim owns every index it creates or loads. A
// RefineIndex built over a shim-owned IVF/Flat base keeps that base alive
// through `base_owner`.
struct Handle {
    std::shared_ptr<IndexBase> base_owner;   // declared first, so destroyed after `index`
    std::shared_ptr<IndexBase> index;
};

DenseIndex* dense(void* h) { return dynamic_cast<DenseIndex*>(static_cast<Handle*>(h)->index.get()); }

IVFIndex* ivf_of(void* h) {
    IndexBase* b = static_cast<Handle*>(h)->index.get();
    if (auto* ivf = dynamic_cast<IVFIndex*>(b)) return ivf;
    if (auto* r = dynamic_cast<RefineIndex*>(b)) return dynamic_cast<IVFIndex*>(&r->base());
    return nullptr;
}

} // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_num_threads(size_t n) { set_num_threads(n); }

int ref_ivf_create(size_t dim, size_t nlist, size_t nprobe, int metric, int custom_ids, void** out) {
    return guarded([&] {
        auto* h = new Handle;
        h->index = std::make_shared<IVFIndex>(dim, nlist, nprobe, custom_ids != 0, static_cast<Metric>(metric));
        *out = h;
    });
}

int ref_flat_create(size_t dim, int metric, int custom_ids, void** out) {
    return guarded([&] {
        auto* h = new Handle;
        h->index = std::make_shared<FlatIndex>(dim, 1024, custom_ids != 0, static_cast<Metric>(metric));
        *out = h;
    });
}

// The returned handle shares ownership of `base`, so freeing the base handle
// first is safe.
int ref_refine_create(void* base, size_t k_factor, int custom_ids, void** out) {
    return guarded([&] {
        auto* b = static_cast<Handle*>(base);
        auto* bd = dynamic_cast<DenseIndex*>(b->index.get());
        if (!bd) throw std::invalid_argument("base is not a dense index");
        auto* h = new Handle;
        h->base_owner = b->index;
        h->index = std::make_shared<RefineIndex>(*bd, k_factor, custom_ids != 0);
        *out = h;
    });
}

void ref_free(void* h) { delete static_cast<Handle*>(h); }

int ref_ivf_enable_pq(void* h, size_t m, size_t K, int fast_scan, int rotate) {
    return guarded([&] { ivf_of(h)->enable_pq(m, K, fast_scan != 0, rotate != 0); });
}

// seed < 0 means no seed
int ref_ivf_train(void* h, const float* x, size_t n, size_t max_iters, int64_t seed, int clustering, size_t passes) {
    return guarded([&] {
        IVFIndex* ivf = ivf_of(h);
        std::optional<uint32_t> s;
        if (seed >= 0) s = static_cast<uint32_t>(seed);
        ivf->train({x, n * ivf->dim()}, n, max_iters, s, static_cast<Clustering>(clustering), passes);
    });
}

int ref_add(void* h, const float* x, size_t n, const int64_t* ids, int64_t* out_ids) {
    return guarded([&] {
        DenseIndex* d = dense(h);
        auto added = d->add_batch({x, n * d->dim()}, n, ids);
        if (out_ids) std::memcpy(out_ids, added.data(), n * sizeof(int64_t));
    });
}

int ref_remove(void* h, const int64_t* ids, size_t n, size_t* removed) {
    return guarded([&] { *removed = static_cast<Handle*>(h)->index->remove({ids, n}); });
}

int ref_compact(void* h, size_t* reclaimed) {
    return guarded([&] { *reclaimed = static_cast<Handle*>(h)->index->compact(); });
}

// Results padded with -1 / +inf to k columns, as the reference's Python
// batch_query does. allowed may be null (no filter).
int ref_query_batch(void* h, const float* q, size_t nq, size_t k, const int64_t* allowed, size_t n_allowed,
                    int64_t* out_ids, float* out_dists) {
    return guarded([&] {
        DenseIndex* d = dense(h);
        const size_t dim = d->dim();
        std::vector<std::vector<Neighbor>> res =
            allowed ? d->query_batch({q, nq * dim}, nq, k, std::span<const int64_t>(allowed, n_allowed))
                    : d->query_batch({q, nq * dim}, nq, k);
        for (size_t i = 0; i < nq; ++i) {
            for (size_t j = 0; j < k; ++j) {
                if (j < res[i].size()) {
                    out_ids[i * k + j] = static_cast<int64_t>(res[i][j].index);
                    out_dists[i * k + j] = res[i][j].distance;
                } else {
                    out_ids[i * k + j] = -1;
                    out_dists[i * k + j] = std::numeric_limits<float>::infinity();
                }
            }
        }
    });
}

int ref_save(void* h, const char* path) {
    return guarded([&] { save_index(*static_cast<Handle*>(h)->index, path); });
}

// kind: 1 flat, 2 ivf, 3 refine (the file format's tags)
int ref_load(const char* path, void** out, int* kind) {
    return guarded([&] {
        auto* h = new Handle;
        h->index = load_index(std::filesystem::path(path), false);
        if (dynamic_cast<FlatIndex*>(h->index.get())) *kind = 1;
        else if (dynamic_cast<IVFIndex*>(h->index.get())) *kind = 2;
        else if (dynamic_cast<RefineIndex*>(h->index.get())) *kind = 3;
        else *kind = 0;
        *out = h;
    });
}

size_t ref_size(void* h) { return static_cast<Handle*>(h)->index->size(); }

int ref_ivf_set_nprobe(void* h, size_t nprobe) { return guarded([&] { ivf_of(h)->set_nprobe(nprobe); }); }
size_t ref_ivf_nprobe(void* h) { return ivf_of(h)->nprobe(); }
int ref_ivf_cosine_ip(void* h) { return ivf_of(h)->cosine_inner_product() ? 1 : 0; }
int ref_ivf_set_cosine_ip(void* h, int v) { return guarded([&] { ivf_of(h)->set_cosine_inner_product(v != 0); }); }
int ref_ivf_precomputed(void* h) { return ivf_of(h)->precomputed_tables() ? 1 : 0; }
int ref_ivf_set_precomputed(void* h, int v) { return guarded([&] { ivf_of(h)->set_precomputed_tables(v != 0); }); }
void ref_ivf_set_filter_probe_scaling(void* h, int v) { ivf_of(h)->set_filter_probe_scaling(v != 0); }

int ref_refine_set_k_factor(void* h, size_t kf) {
    return guarded([&] {
        auto* r = dynamic_cast<RefineIndex*>(static_cast<Handle*>(h)->index.get());
        if (!r) throw std::invalid_argument("not a RefineIndex");
        r->set_k_factor(kf);
    });
}

// ---- kernels of the path, called directly ---------------------------------

void ref_quantize_lut(const float* table, size_t m, uint8_t* lut, float* scale, float* offset) {
    detail::quantize_lut(table, m, lut, *scale, *offset);
}

void ref_quantize_lut_scalar(const float* table, size_t m, uint8_t* lut, float* scale, float* offset) {
    detail::quantize_lut_scalar(table, m, lut, *scale, *offset);
}

void ref_build_quantize_lut(const float* B, const float* C, float A, size_t m, float* table, uint8_t* lut, float* scale,
                            float* offset) {
    detail::build_quantize_lut(B, C, A, m, table, lut, *scale, *offset);
}

uint32_t ref_fast_scan_block_mask(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t limit, uint16_t* out) {
    return detail::fast_scan_block_mask(lut, block, m, limit, out);
}

uint32_t ref_fast_scan_block_mask_scalar(const uint8_t* lut, const uint8_t* block, size_t m, uint16_t limit,
                                         uint16_t* out) {
    return detail::fast_scan_block_mask_scalar(lut, block, m, limit, out);
}

float ref_l2_distance(const float* a, const float* b, size_t n) { return l2_distance(a, b, n); }
float ref_inner_product(const float* a, const float* b, size_t n) { return inner_product(a, b, n); }

// Pushes n (dist, id) pairs through the reference TopK with its threshold
// test, then writes take_sorted()'s result (count returned in *out_n).
void ref_topk_run(const float* dist, const uint64_t* ids, size_t n, size_t k, uint64_t* out_ids, float* out_dist,
                  size_t* out_n) {
    detail::TopK top(k);
    for (size_t i = 0; i < n; ++i)
        if (dist[i] < top.threshold()) top.push(dist[i], ids[i]);
    auto res = top.take_sorted();
    *out_n = res.size();
    for (size_t i = 0; i < res.size(); ++i) {
        out_ids[i] = res[i].index;
        out_dist[i] = res[i].distance;
    }
}

// Lloyd / e-means over packed rows (stride d); seed < 0 means no seed.
int ref_kmeans(const float* x, size_t n, size_t stride, size_t d, size_t k, size_t iters, int64_t seed, int spherical,
               int emeans, float* centroids, uint32_t* assign) {
    return guarded([&] {
        std::optional<uint32_t> s;
        if (seed >= 0) s = static_cast<uint32_t>(seed);
        auto res = emeans ? detail::emeans(x, n, stride, d, k, iters, s, spherical != 0)
                          : detail::kmeans(x, n, stride, d, k, iters, s, spherical != 0);
        std::memcpy(centroids, res.centroids.data(), res.centroids.size() * sizeof(float));
        std::memcpy(assign, res.assignments.data(), res.assignments.size() * sizeof(uint32_t));
    });
}

void ref_assign_nearest(const float* x, size_t n, size_t stride, const float* c, size_t k, size_t d, uint32_t* out) {
    detail::assign_nearest(x, n, stride, c, k, d, out);
}

// PQ codebook pieces: a codebook loaded from m*K*sub_dim centroids.
int ref_pq_tables(const float* centroids, size_t dim, size_t m, size_t K, const float* q, const float* coarse,
                  float* inner, float* list_term, float* adc) {
    return guarded([&] {
        // round-trip through the reference's own load path so build_tables() runs
        std::stringstream ss;
        auto w64 = [&](uint64_t v) { ss.write(reinterpret_cast<const char*>(&v), 8); };
        w64(dim);
        w64(m);
        w64(K);
        w64(m * K * (dim / m));
        ss.write(reinterpret_cast<const char*>(centroids), static_cast<std::streamsize>(m * K * (dim / m) * 4));
        PQCodebook cb = PQCodebook::load(ss);
        if (inner) cb.compute_inner_table({q, dim}, {inner, m * K});
        if (list_term) cb.compute_list_term({coarse, dim}, {list_term, m * K});
        if (adc) cb.compute_adc_table({q, dim}, {adc, m * K});
    });
}

int ref_pq_encode(const float* centroids, size_t dim, size_t m, size_t K, const float* x, size_t n, uint8_t* codes) {
    return guarded([&] {
        std::stringstream ss;
        auto w64 = [&](uint64_t v) { ss.write(reinterpret_cast<const char*>(&v), 8); };
        w64(dim);
        w64(m);
        w64(K);
        w64(m * K * (dim / m));
        ss.write(reinterpret_cast<const char*>(centroids), static_cast<std::streamsize>(m * K * (dim / m) * 4));
        PQCodebook cb = PQCodebook::load(ss);
        for (size_t i = 0; i < n; ++i) cb.encode({x + i * dim, dim}, codes + i * m);
    });
}

// PCA-balanced rotation (d x d, row-major) and the symmetric eigen-solver it uses.
int ref_pca_rotation(const float* x, size_t n, size_t d, size_t m, float* out) {
    return guarded([&] {
        auto r = detail::balanced_pca_rotation({x, n * d}, n, d, m);
        std::memcpy(out, r.data(), r.size() * sizeof(float));
    });
}

int ref_symmetric_eigen(const double* a, size_t d, double* values, double* vectors) {
    return guarded([&] {
        std::vector<double> v, w;
        detail::symmetric_eigen(std::vector<double>(a, a + d * d), d, v, w);
        std::memcpy(values, v.data(), d * sizeof(double));
        std::memcpy(vectors, w.data(), d * d * sizeof(double));
    });
}

} // extern "C"
