// Operations on index objects: search, add, train. Callers hold the object's
// lock (shared for search, exclusive for the rest).
#pragma once

#include "qg_index.h"

namespace qg {

// Keeps freed device memory cached in the default pool (once per process).
void keep_pool_memory();
// Sets the calling thread's qg_last_error() message.
void set_last_error(const std::string& msg);

// Where the query and result buffers live.
enum class IoSpace { Host, Device };

struct SearchRequest {
    const float* q = nullptr;        // nq * dim
    size_t nq = 0, k = 0;
    const SlotBits* filter = nullptr;   // host bitmap of allowed slots, or null
    int64_t* out_ids = nullptr;      // nq * k
    float* out_d = nullptr;
    IoSpace io = IoSpace::Host;
    int nprobe = 0;                  // > 0: probes instead of the IVF index's nprobe
    bool capture = false;            // being captured into a CUDA graph: no host reads or waits
    int* err_dev = nullptr;          // caller-owned error flags (3 ints), read by the caller, or null
    // the filter's allowed slots in ascending order on the device (filter->count
    // of them), or null: RefineIndex direct scans then list them from the bitmap
    const uint32_t* filter_slots_dev = nullptr;
};

// Runs a batch query on `st` and, for host I/O, waits for it.
void search(IndexObj& idx, const SearchRequest& r, cudaStream_t st);

// Sharded search of an IVF index (or a RefineIndex over one) whose device
// copy holds one shard of the lists: the k' candidates per query from this
// device's lists (sorted (key64, slot) lists, keys comparable across shards),
// and the results from the merged candidates of every shard. Device buffers;
// unfiltered queries.
size_t candidate_count(IndexObj& idx, size_t k);
void search_candidates(IndexObj& idx, const float* q_dev, size_t nq, size_t k, uint64_t* key, uint32_t* slot,
                       cudaStream_t st);
void finish_candidates(IndexObj& idx, const float* q_dev, size_t nq, size_t k, const uint64_t* key, const uint32_t* slot,
                       int64_t* out_ids, float* out_d, cudaStream_t st);

// A device-resident, unfiltered search of an IVF index (or a RefineIndex over
// one) replayed as a CUDA graph: the first call with a given batch size, k,
// nprobe, k_factor, buffers and stream runs the search and captures it; later
// calls launch the graph. Returns false when the request does not qualify
// (the caller runs search()). Off unless set_search_graphs(1).
bool search_graph(IndexObj& idx, const SearchRequest& r, cudaStream_t st);
void set_search_graphs(int on);
int search_graphs();
// Graph replays and captures so far.
void search_graph_counts(int64_t* replays, int64_t* captures);

// One query of a mixed batch: a served request with its own settings.
struct MixedQuery {
    int k = 10;                      // results wanted, >= 1
    int nprobe = 0;                  // <= 0: the index's nprobe
    const SlotBits* filter = nullptr;   // allowed slots, or null
    const uint64_t* filter_dev = nullptr;   // the same bitmap already on the device (a server's
                                            // registered filter), or null: uploaded per batch
    const uint32_t* filter_slots_dev = nullptr;   // its allowed slots, ascending, on the device, or null
};

// A batch of queries that differ in k, nprobe and filter (host rows q, nq x
// dim). IVF indexes and RefineIndexes over IVF run the batch as one coarse
// step, one scan and one re-rank; each query's results are the ones it gets
// searched alone with its settings. Results are nq x kmax (host), query i's
// first qs[i].k valid and the rest padded with -1 / +inf. With a second
// stream st2, a batch holding both classes of k' (up to 256 and above) runs
// the larger class on st2 from a second host thread, at the same time.
void search_mixed(IndexObj& idx, const float* q, size_t nq, const MixedQuery* qs, size_t kmax, int64_t* out_ids,
                  float* out_d, cudaStream_t st, cudaStream_t st2 = nullptr);

// add()'s argument checks alone, so they fail before any CUDA work.
void validate_add(const IndexObj& idx, size_t n, const int64_t* ids);

// Adds n vectors (host rows); returns their ids in out_ids (may be null).
void add(IndexObj& idx, const float* x, size_t n, const int64_t* ids, int64_t* out_ids, cudaStream_t st);

// IVFIndex::train on the GPU.
void train(IVFObj& o, const float* x, size_t n, size_t max_iters, int64_t seed, int clustering, size_t passes,
           cudaStream_t st);

// A row set's bf16 copy for the tensor-core filter (rows zero-padded to dpad,
// a multiple of 8) and each row's squared norm.
struct MmRows {
    size_t n = 0;
    int dim = 0, dpad = 0;
    DevBuf<uint16_t> bf16;
    DevBuf<float> sq;
};
bool mm_supported(int dim);
// The filter's epilogue-warp autotuner (qg_mm.cu): on or off, problems tuned, the last launch's pick.
void set_filter_autotune(int on);
int filter_autotune();
int64_t filter_tuned_problems();
int filter_last_epilogue_warps();
// 0: the autotuner's pick; 8 or 16: that epilogue on every filter launch.
void set_filter_epilogue_warps(int warps);
int filter_epilogue_warps();
void mm_prepare(const float* rows, size_t n, int dim, MmRows& out, cudaStream_t st);
// The exact top-k by the BF16 tensor-core filter and FP32 recheck (qg_mm.cu);
// queries whose candidate lists overflowed are listed in overflow_q and must
// be redone exactly.
void mm_topk(const float* q, size_t nq, const float* rows, const MmRows& base, bool ip, size_t k, const uint64_t* allow,
             const uint64_t* deny, uint64_t* out_key, uint32_t* out_slot, std::vector<int>& overflow_q,
             cudaStream_t st);
// 0: never use the tensor-core filter; 1: when the work pays for it; 2: whenever supported.
void set_tensor_filter(int mode);
int tensor_filter();
// Queries answered through the filter so far, and those of them redone exactly
// because their candidate lists overflowed.
void tensor_filter_counts(int64_t* queries, int64_t* redone);
// Whether an exact top-k of nq queries over n rows goes through the filter.
bool use_tensor_filter(size_t nq, size_t n, int dim, size_t k);

// Flat exact search over device rows: the k smallest by (score, slot) per
// query, as (key64 = key_eq0(score) << 32 | slot) sorted lists of length k.
// Large problems go through the tensor-core filter (identical results) unless
// allow_mm is false; pre is the rows' prepared bf16 copy, if the caller keeps one.
void flat_candidates(const float* q_dev, size_t nq, const float* rows_dev, size_t n, int dim, bool ip, size_t k,
                     const uint64_t* allow_dev, const uint64_t* deny_dev, uint64_t* out_key, uint32_t* out_slot,
                     cudaStream_t st, bool allow_mm = true, const MmRows* pre = nullptr);

// Nearest centroid (squared L2, first index on ties) of each row, as the
// reference's assign_nearest without BLAS (reference src/kmeans.cpp:34-115).
void assign_nearest(const float* x_dev, size_t n, const float* c_dev, size_t k, int dim, uint32_t* out_dev,
                    cudaStream_t st);

// Drops deleted slots (IndexBase::compact); *reclaimed = slots freed.
void compact(IndexObj& idx, size_t* reclaimed);

// Kernel-level entry points (qg_tools.cu): n tables rounded to uint8 LUTs
// (C == null: the tables are B; else B + C, plus A on row 0 when A != null),
// and fast-scan sums of plain codes with one LUT per 64 vectors.
void quantize_luts(const float* B, const float* C, const float* A, size_t n, size_t m, uint8_t* lut, float* scale,
                   float* offset, cudaStream_t st);
void fast_scan_sums(const uint8_t* lut, size_t nluts, size_t m, const uint8_t* codes, const uint32_t* lut_of, size_t n,
                    uint16_t* sums, cudaStream_t st);

} // namespace qg

// A C-ABI handle: one reference to an index object.
struct qg_index {
    std::shared_ptr<qg::IndexObj> obj;
};
