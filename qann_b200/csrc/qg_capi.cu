// The C ABI (include/qann_gpu.h): handles, status codes, argument checks with
// the reference's messages, locking, and per-thread streams.
#include "../../include/qann_gpu.h"

#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_search.h"
#include "qg_train.h"

#include <limits>
#include <string>

using namespace qg;

// (struct qg_index is defined in qg_ops.h)

namespace {

thread_local std::string t_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return QG_OK;
    } catch (const Error& e) {
        t_err = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        t_err = "out of host memory";
        return QG_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        t_err = e.what();
        return QG_RUNTIME_ERROR;
    }
}

} // namespace

// The stream-ordered allocator's default pool hands memory back to the driver
// at every synchronisation (release threshold 0), so each search would pay for
// fresh allocations; keep freed blocks cached in the pool instead.
void qg::keep_pool_memory() {
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    });
}

namespace {

// One non-blocking stream per host thread, so concurrent searches overlap.
cudaStream_t thread_stream() {
    thread_local cudaStream_t s = nullptr;
    if (!s) QG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    keep_pool_memory();
    return s;
}

IndexObj& obj(qg_index* h) {
    require(h && h->obj, "null index handle");
    return *h->obj;
}

IVFObj& ivf_of(qg_index* h) {
    IndexObj& o = obj(h);
    if (o.kind == Kind::IVF) return static_cast<IVFObj&>(o);
    if (o.kind == Kind::Refine) {
        auto& r = static_cast<RefineObj&>(o);
        if (r.base->kind == Kind::IVF) return static_cast<IVFObj&>(*r.base);
    }
    throw Error(kInvalidArgument, "not an IVFIndex");
}

qg_index* wrap(std::shared_ptr<IndexObj> o) {
    auto* h = new qg_index;
    h->obj = std::move(o);
    return h;
}

} // namespace

namespace qg {
// lets other translation units' entry points report through qg_last_error
void set_last_error(const std::string& msg) { t_err = msg; }
} // namespace qg

extern "C" {

const char* qg_last_error(void) { return t_err.c_str(); }

const char* qg_version(void) { return "qann-b200 0.1.0 (sm_100a)"; }

int qg_create_ivf(size_t dim, size_t nlist, size_t nprobe, int metric, int custom_ids, qg_index** out) {
    return guarded([&] {
        require(nlist >= 100 && nlist <= 65535, "nlist must be in [100, 65535]");
        require(dim >= 1, "dim must be >= 1");
        require(nprobe >= 1 && nprobe <= nlist, "nprobe must be in [1, nlist]");
        require(metric >= 0 && metric <= 2, "unknown metric");
        auto o = std::make_shared<IVFObj>();
        o->model.dim = dim;
        o->model.nlist = nlist;
        o->model.nprobe = nprobe;
        o->model.metric = static_cast<Metric>(metric);
        o->model.idmap = IdMap(custom_ids != 0);
        o->model.list_ids.resize(nlist);
        o->model.list_codes.resize(nlist);
        o->model.list_vecs.resize(nlist);
        *out = wrap(o);
    });
}

int qg_enable_pq(qg_index* h, size_t m, size_t K, int fast_scan, int rotate) {
    return guarded([&] {
        IVFObj& o = ivf_of(h);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        IVFModel& M = o.model;
        if (M.idmap.slots() > 0 || M.trained)
            throw Error(kLogicError, "enable_pq must be called before train()/add()");
        if (M.sq_bits) throw Error(kLogicError, "enable_pq cannot be combined with enable_sq");
        if (fast_scan && (K != 16 || m % 2 != 0 || m > kFsMaxSubspaces))
            throw Error(kInvalidArgument, "fast_scan needs 16 centroids per subspace and an even num_subspaces <= 1024");
        if (fast_scan && M.pq_distance == 1) throw Error(kInvalidArgument, "cannot use SDC with fast-scan");
        require(M.dim >= 1 && m >= 1, "dim and num_subspaces must be >= 1");
        require(M.dim % m == 0, "dim must be divisible by num_subspaces");
        require(K >= 1 && K <= 256, "centroids_per_subspace must be in [1, 256]");
        M.has_pq = true;
        M.fast_scan = fast_scan != 0;
        M.rotate = rotate != 0;
        M.pq = PQCodebook{};
        M.pq.dim = M.dim;
        M.pq.m = m;
        M.pq.K = K;
        M.pq.sub_dim = M.dim / m;
        M.pq.centroids.assign(m * K * M.pq.sub_dim, 0.0f);
        o.dev_dirty = true;
    });
}

int qg_create_flat(size_t dim, int metric, int custom_ids, qg_index** out) {
    return guarded([&] {
        require(dim >= 1, "dim must be >= 1");
        require(metric >= 0 && metric <= 2, "unknown metric");
        auto o = std::make_shared<FlatObj>();
        o->model.dim = dim;
        o->model.metric = static_cast<Metric>(metric);
        o->model.idmap = IdMap(custom_ids != 0);
        *out = wrap(o);
    });
}

int qg_create_refine(qg_index* base, size_t k_factor, int custom_ids, qg_index** out) {
    return guarded([&] {
        IndexObj& b = obj(base);
        std::unique_lock<std::shared_mutex> lk(b.mu);
        if (b.kind == Kind::Refine)
            throw Error(kInvalidArgument,
                        "a RefineIndex's base must not be a RefineIndex; wrap the approximate index directly");
        if (b.idmap().slots() != 0) throw Error(kInvalidArgument, "base index must be empty");
        if (k_factor == 0) throw Error(kInvalidArgument, "k_factor must be >= 1");
        if (!b.idmap().ids_are_slots())
            throw Error(kInvalidArgument, "base index must not use custom ids or have been compacted");
        if (b.wrapped) throw Error(kInvalidArgument, "base index is already wrapped by another index");
        auto o = std::make_shared<RefineObj>();
        o->base = base->obj;
        o->k_factor = k_factor;
        o->map = IdMap(custom_ids != 0);
        b.wrapped = true;
        *out = wrap(o);
    });
}

int qg_refine_base(qg_index* refine, qg_index** out) {
    return guarded([&] {
        IndexObj& o = obj(refine);
        require(o.kind == Kind::Refine, "not a RefineIndex");
        *out = wrap(static_cast<RefineObj&>(o).base);
    });
}

void qg_free(qg_index* h) { delete h; }

int qg_train(qg_index* h, const float* x, size_t n, size_t max_iters, int64_t seed, int clustering, size_t passes) {
    return guarded([&] {
        IndexObj& o0 = obj(h);
        require(o0.kind == Kind::IVF, "train() is an IVFIndex method");
        auto& o = static_cast<IVFObj&>(o0);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        train(o, x, n, max_iters, seed, clustering, passes, thread_stream());
    });
}

int qg_add(qg_index* h, const float* x, size_t n, const int64_t* ids, int64_t* out_ids) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        if (o.wrapped)
            throw Error(kInvalidArgument, "cannot add on an index wrapped by a RefineIndex or HybridIndex; add through "
                                          "the wrapper instead");
        std::unique_lock<std::shared_mutex> lb;
        if (o.kind == Kind::Refine) lb = std::unique_lock<std::shared_mutex>(static_cast<RefineObj&>(o).base->mu);
        validate_add(o, n, ids);
        if (n == 0) return;
        add(o, x, n, ids, out_ids, thread_stream());
    });
}

int qg_remove(qg_index* h, const int64_t* ids, size_t n, size_t* removed) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        if (o.wrapped)
            throw Error(kInvalidArgument, "cannot remove on an index wrapped by a RefineIndex or HybridIndex; remove "
                                          "through the wrapper instead");
        std::vector<uint32_t> slots;
        *removed = o.idmap().remove({ids, n}, &slots);
        o.dev_dirty = true;
        if (o.kind == Kind::Refine) {
            auto& r = static_cast<RefineObj&>(o);
            std::unique_lock<std::shared_mutex> lb(r.base->mu);
            std::vector<int64_t> base_ids(slots.begin(), slots.end());
            r.base->idmap().remove(base_ids);
            r.base->dev_dirty = true;
        }
    });
}

int qg_compact(qg_index* h, size_t* reclaimed) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        compact(o, reclaimed);
    });
}

static int search_common(qg_index* h, const float* q, size_t nq, size_t k, const SlotBits* filter, int64_t* out_ids,
                         float* out_d, IoSpace io, cudaStream_t st) {
    IndexObj& o = obj(h);
    std::shared_lock<std::shared_mutex> lk(o.mu);
    std::shared_lock<std::shared_mutex> lb;
    if (o.kind == Kind::Refine) lb = std::shared_lock<std::shared_mutex>(static_cast<RefineObj&>(o).base->mu);
    SearchRequest r;
    r.q = q;
    r.nq = nq;
    r.k = k;
    r.filter = filter;
    r.out_ids = out_ids;
    r.out_d = out_d;
    r.io = io;
    if (!search_graph(o, r, st)) search(o, r, st);
    return QG_OK;
}

int qg_search(qg_index* h, const float* q, size_t nq, size_t k, const int64_t* allowed, size_t n_allowed,
              int64_t* out_ids, float* out_dists) {
    return guarded([&] {
        IndexObj& o = obj(h);
        SlotBits f;
        if (allowed) {
            std::shared_lock<std::shared_mutex> lk(o.mu);
            f = o.idmap().filter({allowed, n_allowed});
        }
        search_common(h, q, nq, k, allowed ? &f : nullptr, out_ids, out_dists, IoSpace::Host, thread_stream());
    });
}

int qg_search_bitmap(qg_index* h, const float* q, size_t nq, size_t k, const uint64_t* words, size_t nwords,
                     int64_t* out_ids, float* out_dists) {
    return guarded([&] {
        IndexObj& o = obj(h);
        SlotBits f;
        {
            std::shared_lock<std::shared_mutex> lk(o.mu);
            require(nwords * 64 >= o.idmap().slots(), "the bitmap must cover every slot of the index");
            f = o.idmap().live(std::vector<uint64_t>(words, words + nwords));
        }
        search_common(h, q, nq, k, &f, out_ids, out_dists, IoSpace::Host, thread_stream());
    });
}

int qg_search_device(qg_index* h, const float* q_dev, size_t nq, size_t k, int64_t* out_ids_dev, float* out_dists_dev,
                     void* stream) {
    return guarded([&] {
        keep_pool_memory();
        search_common(h, q_dev, nq, k, nullptr, out_ids_dev, out_dists_dev, IoSpace::Device,
                      static_cast<cudaStream_t>(stream));
    });
}

int qg_candidate_count(qg_index* h, size_t k, size_t* kp) {
    return guarded([&] {
        require(kp != nullptr, "null argument");
        IndexObj& o = obj(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        *kp = candidate_count(o, k);
    });
}

int qg_search_candidates_device(qg_index* h, const float* q_dev, size_t nq, size_t k, uint64_t* key_dev,
                                uint32_t* slot_dev, void* stream) {
    return guarded([&] {
        keep_pool_memory();
        IndexObj& o = obj(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        std::shared_lock<std::shared_mutex> lb;
        if (o.kind == Kind::Refine) lb = std::shared_lock<std::shared_mutex>(static_cast<RefineObj&>(o).base->mu);
        search_candidates(o, q_dev, nq, k, key_dev, slot_dev, static_cast<cudaStream_t>(stream));
    });
}

int qg_merge_candidates_device(const uint64_t* key_dev, const uint32_t* slot_dev, size_t nq, size_t nparts, size_t kp,
                               uint64_t* out_key_dev, uint32_t* out_slot_dev, void* stream) {
    return guarded([&] {
        require(nparts >= 1 && kp >= 1 && kp <= 3072, "nparts must be >= 1 and kp in [1, 3072]");
        keep_pool_memory();
        merge_candidates(key_dev, slot_dev, static_cast<int>(nq), static_cast<int>(nparts), static_cast<int>(kp),
                         out_key_dev, out_slot_dev, static_cast<cudaStream_t>(stream));
        QG_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    });
}

int qg_finish_candidates_device(qg_index* h, const float* q_dev, size_t nq, size_t k, const uint64_t* key_dev,
                                const uint32_t* slot_dev, int64_t* out_ids_dev, float* out_dists_dev, void* stream) {
    return guarded([&] {
        keep_pool_memory();
        IndexObj& o = obj(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        std::shared_lock<std::shared_mutex> lb;
        if (o.kind == Kind::Refine) lb = std::shared_lock<std::shared_mutex>(static_cast<RefineObj&>(o).base->mu);
        finish_candidates(o, q_dev, nq, k, key_dev, slot_dev, out_ids_dev, out_dists_dev,
                          static_cast<cudaStream_t>(stream));
    });
}

int qg_get(qg_index* h, const char* key, int64_t* value) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        const std::string k(key);
        if (k == "dim") *value = static_cast<int64_t>(o.dim());
        else if (k == "kind") *value = static_cast<int64_t>(o.kind);
        else if (k == "metric") *value = static_cast<int64_t>(o.metric());
        else if (k == "size") *value = static_cast<int64_t>(o.idmap().live_count());
        else if (k == "slots") *value = static_cast<int64_t>(o.idmap().slots());
        else if (k == "custom_ids") *value = o.idmap().custom();
        else if (k == "wrapped") *value = o.wrapped;
        else if (k == "k_factor") {
            require(o.kind == Kind::Refine, "not a RefineIndex");
            *value = static_cast<int64_t>(static_cast<RefineObj&>(o).k_factor);
        } else if (k == "base_kind") {
            require(o.kind == Kind::Refine, "not a RefineIndex");
            *value = static_cast<int64_t>(static_cast<RefineObj&>(o).base->kind);
        } else if (k == "rows_mapped") {
            // 1: the raw rows are read in place from the mapped file (load with
            // mmap); 2: and the re-rank reads them there through host-mapped
            // memory rather than from a copy in HBM
            if (o.kind != Kind::Refine) {
                *value = 0;
            } else {
                const auto& r = static_cast<RefineObj&>(o);
                *value = r.mapped ? (r.dev.ext ? 2 : 1) : 0;
            }
        } else {
            require(o.kind == Kind::IVF, "unknown property '" + k + "' for this index");
            const IVFObj& v = static_cast<IVFObj&>(o);
            const IVFModel& M = v.model;
            if (k == "nprobe") *value = static_cast<int64_t>(M.nprobe);
            else if (k == "nlist") *value = static_cast<int64_t>(M.nlist);
            else if (k == "precomputed_tables") *value = v.precomputed_available();
            else if (k == "cosine_inner_product") *value = M.cosine_ip;
            else if (k == "filter_probe_scaling") *value = M.filter_probe_scaling;
            else if (k == "shard") *value = v.shard;
            else if (k == "shards") *value = v.shards;
            else if (k == "fast_scan") *value = M.fast_scan;
            else if (k == "pq_m") *value = static_cast<int64_t>(M.has_pq ? M.pq.m : 0);
            else if (k == "pq_k") *value = static_cast<int64_t>(M.has_pq ? M.pq.K : 0);
            else if (k == "trained") *value = M.trained;
            else if (k == "rotate") *value = M.rotate;
            else if (k == "sq_bits") *value = M.sq_bits;
            else if (k == "pq_distance") *value = M.pq_distance;
            else throw Error(kInvalidArgument, "unknown property '" + k + "'");
        }
    });
}

int qg_set(qg_index* h, const char* key, int64_t value) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::unique_lock<std::shared_mutex> lk(o.mu);
        const std::string k(key);
        if (k == "k_factor") {
            require(o.kind == Kind::Refine, "not a RefineIndex");
            require(value >= 1, "k_factor must be >= 1");
            static_cast<RefineObj&>(o).k_factor = static_cast<uint64_t>(value);
            return;
        }
        require(o.kind == Kind::IVF, "unknown property '" + k + "' for this index");
        IVFObj& v = static_cast<IVFObj&>(o);
        IVFModel& M = v.model;
        if (k == "nprobe") {
            require(value >= 1 && static_cast<uint64_t>(value) <= M.nlist, "nprobe must be in [1, nlist]");
            M.nprobe = static_cast<uint64_t>(value);
        } else if (k == "precomputed_tables") {
            M.use_precomputed = value != 0;
            v.dev_dirty = true;
        } else if (k == "cosine_inner_product") {
            M.cosine_ip = value != 0;
            v.dev_dirty = true;
        } else if (k == "filter_probe_scaling") {
            M.filter_probe_scaling = value != 0;
        } else if (k == "shards") {
            require(value >= 1 && value <= 4096, "shards must be in [1, 4096]");
            v.shards = static_cast<int>(value);
            if (v.shard >= v.shards) v.shard = 0;
            v.dev_dirty = true;
        } else if (k == "shard") {
            require(value >= 0 && value < v.shards, "shard must be in [0, shards)");
            v.shard = static_cast<int>(value);
            v.dev_dirty = true;
        } else if (k == "pq_distance") {
            if (M.fast_scan && value == 1) throw Error(kInvalidArgument, "cannot use SDC with fast-scan");
            if (M.metric == Metric::InnerProduct && value == 1)
                throw Error(kInvalidArgument, "cannot use SDC with Metric::InnerProduct");
            require(value == 0 || value == 1, "pq_distance must be ADC (0) or SDC (1)");
            M.pq_distance = static_cast<uint8_t>(value);
        } else {
            throw Error(kInvalidArgument, "unknown or read-only property '" + k + "'");
        }
    });
}

int qg_ivf_list_sizes(qg_index* h, uint32_t* out_sizes) {
    return guarded([&] {
        IVFObj& o = ivf_of(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        for (size_t l = 0; l < o.model.nlist; ++l) out_sizes[l] = static_cast<uint32_t>(o.model.list_ids[l].size());
    });
}

int qg_ivf_centroids(qg_index* h, float* out_centroids) {
    return guarded([&] {
        IVFObj& o = ivf_of(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        require(o.model.trained, "train() has not be run yet", kLogicError);
        std::copy(o.model.centroids.begin(), o.model.centroids.end(), out_centroids);
    });
}

int qg_save(qg_index* h, const char* path) {
    return guarded([&] {
        IndexObj& o = obj(h);
        std::shared_lock<std::shared_mutex> lk(o.mu);
        Writer w;
        if (o.kind == Kind::IVF) {
            write_header(w, Kind::IVF);
            static_cast<IVFObj&>(o).model.save_body(w);
        } else if (o.kind == Kind::Flat) {
            write_header(w, Kind::Flat);
            static_cast<FlatObj&>(o).model.save_body(w);
        } else {
            auto& r = static_cast<RefineObj&>(o);
            std::shared_lock<std::shared_mutex> lb(r.base->mu);
            write_header(w, Kind::Refine);
            w.pod<uint64_t>(r.k_factor);
            w.pod<uint64_t>(r.map.slots());
            if (r.base->kind == Kind::IVF) {
                write_header(w, Kind::IVF);
                static_cast<IVFObj&>(*r.base).model.save_body(w);
            } else {
                write_header(w, Kind::Flat);
                static_cast<FlatObj&>(*r.base).model.save_body(w);
            }
            w.pod<uint64_t>(r.map.slots() * r.dim());
            w.pad(64 * 1024);
            w.bytes(r.rows_host(), r.rows_len() * sizeof(float));
            r.map.save(w);
            r.meta.write(w);
        }
        write_file_atomic(path, w.buf);
    });
}

namespace {

// Reads an index from `bytes` (the whole file); with `file`, a RefineIndex
// keeps its raw rows inside that mapping.
void load_from(const char* data, size_t size, std::shared_ptr<const MappedFile> file, qg_index** out, int* kind) {
        Reader r{data, size};
        uint32_t version = 0;
        const Kind k = read_header(r, &version);
        std::shared_ptr<IndexObj> o;
        if (k == Kind::IVF) {
            auto v = std::make_shared<IVFObj>();
            v->model = std::move(*IVFModel::load_body(r, version));
            o = v;
        } else if (k == Kind::Flat) {
            auto f = std::make_shared<FlatObj>();
            f->model = std::move(*FlatModel::load_body(r, version));
            o = f;
        } else {
            auto m = RefineModel::load_body(r, version, file != nullptr);
            auto ro = std::make_shared<RefineObj>();
            if (m->base_kind == Kind::IVF) {
                auto v = std::make_shared<IVFObj>();
                v->model = std::move(*m->ivf);
                ro->base = v;
            } else {
                auto f = std::make_shared<FlatObj>();
                f->model = std::move(*m->flat);
                ro->base = f;
            }
            ro->base->wrapped = true;
            ro->k_factor = m->k_factor;
            ro->data = std::move(m->data);
            ro->map = std::move(m->idmap);
            ro->meta = std::move(m->meta);
            if (m->mapped) {
                ro->mapped = m->mapped;
                ro->file = file;
            }
            o = ro;
        }
        if (r.pos != r.size) throw Error(kRuntimeError, "corrupt file: unexpected data after the index");
        *kind = static_cast<int>(k);
        *out = wrap(o);
}

} // namespace

int qg_load(const char* path, qg_index** out, int* kind) {
    return guarded([&] {
        require(path && out && kind, "null argument");
        const std::vector<char> bytes = read_file(path);
        load_from(bytes.data(), bytes.size(), nullptr, out, kind);
    });
}

int qg_load_mapped(const char* path, qg_index** out, int* kind) {
    return guarded([&] {
        require(path && out && kind, "null argument");
        std::shared_ptr<const MappedFile> f = MappedFile::open(path);
        load_from(f->data, f->size, f, out, kind);
    });
}

// ---- profiling ------------------------------------------------------------------

int qg_profile_enable(int on) {
    profiler().on.store(on != 0);
    return QG_OK;
}

int qg_profile_reset(void) {
    return guarded([&] {
        std::lock_guard<std::mutex> g(profiler().mu);
        profiler().settle();
        profiler().totals.clear();
    });
}

int qg_profile_get(const char* kernel, double* total_ms, int64_t* launches) {
    return guarded([&] {
        std::lock_guard<std::mutex> g(profiler().mu);
        profiler().settle();
        auto it = profiler().totals.find(kernel);
        *total_ms = it == profiler().totals.end() ? 0.0 : it->second.first;
        *launches = it == profiler().totals.end() ? 0 : it->second.second;
    });
}

int64_t qg_launch_count(void) { return profiler().launches.load(); }

// ---- kernels on device memory ----------------------------------------------------

int qg_quantize_lut_dev(const float* tables_dev, size_t n, size_t m, uint8_t* lut_dev, float* scale_dev,
                        float* offset_dev, void* stream) {
    return guarded([&] { quantize_luts(tables_dev, nullptr, nullptr, n, m, lut_dev, scale_dev, offset_dev,
                                        static_cast<cudaStream_t>(stream)); });
}

int qg_build_quantize_lut_dev(const float* B_dev, const float* C_dev, const float* A_dev, size_t n, size_t m,
                              uint8_t* lut_dev, float* scale_dev, float* offset_dev, void* stream) {
    return guarded([&] { quantize_luts(B_dev, C_dev, A_dev, n, m, lut_dev, scale_dev, offset_dev,
                                        static_cast<cudaStream_t>(stream)); });
}

int qg_fast_scan_dev(const uint8_t* lut_dev, size_t nluts, size_t m, const uint8_t* codes_dev,
                     const uint32_t* lut_of_dev, size_t n, uint16_t* sums_dev, void* stream) {
    return guarded([&] { fast_scan_sums(lut_dev, nluts, m, codes_dev, lut_of_dev, n, sums_dev,
                                         static_cast<cudaStream_t>(stream)); });
}

int qg_exact_scores_dev(const float* a_dev, size_t na, const float* b_dev, size_t nb, size_t dim, int ip,
                        float* out_dev, void* stream) {
    return guarded([&] {
        pair_scores(a_dev, static_cast<int>(na), b_dev, static_cast<int>(nb), static_cast<int>(dim), ip != 0, out_dev,
                    nb, static_cast<cudaStream_t>(stream));
    });
}

int qg_set_option(const char* key, int64_t value) {
    return guarded([&] {
        require(key != nullptr, "null key");
        const std::string k(key);
        if (k == "tensor_filter") {
            require(value >= 0 && value <= 2, "tensor_filter must be 0, 1 or 2");
            set_tensor_filter(static_cast<int>(value));
        } else if (k == "search_graphs") {
            require(value == 0 || value == 1, "search_graphs must be 0 or 1");
            set_search_graphs(static_cast<int>(value));
        } else if (k == "scan_autotune") {
            require(value == 0 || value == 1, "scan_autotune must be 0 or 1");
            set_scan_autotune(static_cast<int>(value));
        } else if (k == "scan_variant") {
            require(value >= -1 && value <= 2, "scan_variant must be -1, 0, 1 or 2");
            set_scan_variant(static_cast<int>(value));
        } else if (k == "tensor_scan") {
            require(value >= 0 && value <= 2, "tensor_scan must be 0, 1 or 2");
            set_tensor_scan(static_cast<int>(value));
        } else if (k == "filter_autotune") {
            require(value == 0 || value == 1, "filter_autotune must be 0 or 1");
            set_filter_autotune(static_cast<int>(value));
        } else if (k == "filter_epilogue_warps") {
            require(value == 0 || value == 8 || value == 16, "filter_epilogue_warps must be 0, 8 or 16");
            set_filter_epilogue_warps(static_cast<int>(value));
        } else {
            throw Error(kInvalidArgument, "unknown option: " + k);
        }
    });
}

int qg_get_option(const char* key, int64_t* value) {
    return guarded([&] {
        require(key != nullptr && value != nullptr, "null argument");
        const std::string k(key);
        int64_t queries = 0, redone = 0;
        tensor_filter_counts(&queries, &redone);
        if (k == "tensor_filter") *value = tensor_filter();
        else if (k == "tensor_filter_queries") *value = queries;
        else if (k == "tensor_filter_redone") *value = redone;
        else if (k == "tensor_coarse_queries" || k == "tensor_coarse_redone") {
            int64_t cq = 0, cr = 0;
            tensor_coarse_counts(&cq, &cr);
            *value = k == "tensor_coarse_queries" ? cq : cr;
        }
        else if (k == "tensor_coarse_candidates") *value = tensor_coarse_candidates();
        else if (k == "filtered_batches" || k == "filtered_deep_walks") {
            int64_t b = 0, dw = 0;
            filtered_rank_counts(&b, &dw);
            *value = k == "filtered_batches" ? b : dw;
        }
        else if (k == "search_graphs") *value = search_graphs();
        else if (k == "search_graph_replays" || k == "search_graph_captures") {
            int64_t rp = 0, cp = 0;
            search_graph_counts(&rp, &cp);
            *value = k == "search_graph_replays" ? rp : cp;
        }
        else if (k == "scan_autotune") *value = scan_autotune();
        else if (k == "scan_variant") *value = scan_variant();
        else if (k == "scan_tuned_shapes") *value = scan_tuned_shapes();
        else if (k == "scan_last_shape") *value = scan_last_shape();
        else if (k == "tensor_scan") *value = tensor_scan();
        else if (k == "filter_autotune") *value = filter_autotune();
        else if (k == "filter_tuned_problems") *value = filter_tuned_problems();
        else if (k == "filter_last_epilogue_warps") *value = filter_last_epilogue_warps();
        else if (k == "filter_epilogue_warps") *value = filter_epilogue_warps();
        else if (k == "mapped_rows_error") *value = mapped_rows_error();
        else if (k.rfind("tensor_scan_stat_", 0) == 0) {
            require(tensor_scan_stat(k.substr(17), value), "unknown option: " + k);
        }
        else if (k == "tensor_scan_calls" || k == "tensor_scan_redone") {
            int64_t c = 0, r = 0;
            tensor_scan_counts(&c, &r);
            *value = k == "tensor_scan_calls" ? c : r;
        }
        else throw Error(kInvalidArgument, "unknown option: " + k);
    });
}

int qg_symmetric_eigen(const double* a, size_t d, double* values, double* vectors) {
    return guarded([&] {
        require(a && values && vectors, "null buffer");
        std::vector<double> v, w;
        symmetric_eigen(std::vector<double>(a, a + d * d), d, v, w);
        std::copy(v.begin(), v.end(), values);
        std::copy(w.begin(), w.end(), vectors);
    });
}

int qg_balanced_rotation(const double* cov, size_t d, size_t m, float* rotation) {
    return guarded([&] {
        require(cov && rotation, "null buffer");
        require(m > 0 && d % m == 0, "dim must be divisible by num_subspaces");
        const std::vector<float> r = balanced_rotation(std::vector<double>(cov, cov + d * d), d, m);
        std::copy(r.begin(), r.end(), rotation);
    });
}

} // extern "C"
