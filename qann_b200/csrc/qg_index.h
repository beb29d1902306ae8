// Index objects behind the C ABI: the host model (canonical, what save()
// writes) plus its device copy, rebuilt lazily after writes.
#pragma once

#include "qg_cuda.h"
#include "qg_host.h"
#include "qg_search.h"

#include <memory>
#include <mutex>
#include <shared_mutex>
#include <vector>

namespace qg {

// Device copy of an IVF fast-scan index.
struct DeviceIVF {
    IvfView view;
    DevBuf<float> centroids, resid, sqnorm, pq_t, B;
    DevBuf<float> rot;        // dim x dim PCA rotation, when the index rotates
    DevBuf<uint32_t> sb_off, list_size, ids;
    DevBuf<uint4> codes;
    DevBuf<uint64_t> deleted;
    DevBuf<int64_t> labels;   // slot -> id when the ids are not the slots
    DevBuf<uint16_t> cent_f16;   // scaled f16 centroids for the tensor-core coarse step
    DevBuf<float> cent_sq;
    DevBuf<int> cent_exp;
    size_t total_sb = 0;
};

// Device rows of a FlatIndex or of a RefineIndex's raw vectors.
struct DeviceRows {
    DevBuf<float> rows;
    const float* ext = nullptr;        // rows read in place from host memory (a mapped file), or null
    DevBuf<int64_t> labels;
    DevBuf<uint64_t> deleted;
    const float* ptr() const { return ext ? ext : rows.get(); }
};

// A captured device-resident search (search_graph).
struct SearchGraph {
    size_t nq = 0, k = 0, k_factor = 0;
    int nprobe = 0;
    const float* q = nullptr;
    int64_t* ids = nullptr;
    float* d = nullptr;
    cudaStream_t st = nullptr;
    uint64_t gen = 0;                 // device generation of the index (and its base) at capture
    cudaGraphExec_t exec = nullptr;
    int* err = nullptr;               // the search's error flags, read after each replay
    int64_t launches = 0;             // kernels in the graph
    bool failed = false;              // not capturable: the plain path serves this key
    ~SearchGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (err) cudaFree(err);
    }
};

struct IndexObj {
    Kind kind;
    mutable std::shared_mutex mu;     // shared for queries, exclusive for writes
    std::mutex dev_mu;                // guards (re)building the device copy
    bool dev_dirty = true;
    uint64_t dev_gen = 0;             // bumped on every rebuild of the device copy
    std::mutex graph_mu;              // guards `graphs`
    std::vector<std::unique_ptr<SearchGraph>> graphs;
    bool wrapped = false;             // a RefineIndex wraps this index
    int device = 0;
    explicit IndexObj(Kind k) : kind(k) {}
    virtual ~IndexObj() = default;
    virtual size_t dim() const = 0;
    virtual Metric metric() const = 0;
    virtual IdMap& idmap() = 0;
    virtual const IdMap& idmap() const = 0;
};

struct IVFObj : IndexObj {
    IVFModel model;
    DeviceIVF dev;
    // List sharding: the device copy holds the lists l with l % shards == shard
    // (codes and slots); list sizes stay global, so push indices (and so
    // candidate keys) agree across shards. Not saved.
    int shard = 0, shards = 1;
    IVFObj() : IndexObj(Kind::IVF) {}
    size_t dim() const override { return model.dim; }
    Metric metric() const override { return model.metric; }
    IdMap& idmap() override { return model.idmap; }
    const IdMap& idmap() const override { return model.idmap; }
    bool precomputed_available() const;
    int scan_mode() const;
};

struct FlatObj : IndexObj {
    FlatModel model;
    DeviceRows dev;
    FlatObj() : IndexObj(Kind::Flat) {}
    size_t dim() const override { return model.dim; }
    Metric metric() const override { return model.metric; }
    IdMap& idmap() override { return model.idmap; }
    const IdMap& idmap() const override { return model.idmap; }
};

struct RefineObj : IndexObj {
    std::shared_ptr<IndexObj> base;
    uint64_t k_factor = 10;
    std::vector<float> data;   // slots * dim raw rows (empty while mapped)
    // load(mmap=True) (reference include/vecengine/vector_store.hpp:50-110):
    // the rows stay in the mapped file, and the re-rank reads them there
    // through host-mapped memory instead of from an HBM copy, until the index
    // changes (add, compact), which copies them into `data` first.
    std::shared_ptr<const MappedFile> file;
    const float* mapped = nullptr;
    void* registered = nullptr;   // the page range registered with CUDA for mapped reads
    void* priv = nullptr;         // a private view of the rows' pages, when the shared one cannot be registered
    size_t priv_len = 0;
    const float* dev_src = nullptr;   // the registered copy of the rows' first element
    IdMap map;
    MetaBlob meta;
    DeviceRows dev;
    RefineObj() : IndexObj(Kind::Refine) {}
    ~RefineObj() override {
        release_mapping();
        if (base) base->wrapped = false;
    }
    const float* rows_host() const { return mapped ? mapped : data.data(); }
    size_t rows_len() const { return mapped ? map.slots() * dim() : data.size(); }
    void materialize();      // mapped rows into `data`, the mapping released
    void release_mapping();
    size_t dim() const override { return base->dim(); }
    Metric metric() const override { return base->metric(); }
    IdMap& idmap() override { return map; }
    const IdMap& idmap() const override { return map; }
};

// The last refused registration of mapped rows (two cudaError_t codes:
// read-only shared view * 1000 + private view), 0 if none.
int mapped_rows_error();

// The library's own stream on the current device (never destroyed).
cudaStream_t resident_stream();

// Builds / refreshes the device copy (callers hold the object's lock). The
// arrays are made on resident_stream() and ready when this returns.
void ensure_device(IVFObj& o, cudaStream_t st);
void ensure_device(FlatObj& o, cudaStream_t st);
void ensure_device(RefineObj& o, cudaStream_t st);

// Packs plain codes (n x m bytes, lists concatenated in order) into the
// device superblock layout. sb_list: the list of each superblock; voff: the
// first vector of each list in `codes`; sb_off: first superblock of each list.
void pack_superblocks(const uint8_t* codes_dev, const uint32_t* ids_dev, const uint32_t* voff_dev,
                      const uint32_t* sb_off_dev, const uint32_t* list_size_dev, const uint32_t* sb_list_dev,
                      size_t total_sb, int m, int m_pad, uint4* out_codes, uint32_t* out_ids, cudaStream_t st);

} // namespace qg
