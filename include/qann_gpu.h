/*
 * qann_gpu — C ABI of the B200 search path for qann's dense indexes.
 *
 * Every function returns 0 (QG_OK) or a status code; qg_last_error() gives the
 * message of the calling thread's last failure. Buffers passed in are HOST
 * memory owned by the caller unless a name says _dev. Status codes map onto
 * the exceptions qann's Python layer raises (reference
 * bindings/python_bindings.cpp): QG_INVALID_ARGUMENT -> ValueError,
 * QG_LOGIC_ERROR / QG_RUNTIME_ERROR -> RuntimeError.
 *
 * Handles are reference-counted views of an index; a RefineIndex keeps its
 * base alive. Concurrent qg_search calls on one handle are safe (readers
 * share the index; writers — add, remove, train, setters — are exclusive),
 * as the reference's bindings lock (reference bindings/python_bindings.cpp:97-131).
 */
#ifndef QANN_GPU_H
#define QANN_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qg_index qg_index;

enum {
    QG_OK = 0,
    QG_INVALID_ARGUMENT = 1,
    QG_LOGIC_ERROR = 2,
    QG_RUNTIME_ERROR = 3,
    QG_CUDA_ERROR = 4,
    QG_OUT_OF_MEMORY = 5,
    QG_UNSUPPORTED = 6,
};

/* Index kinds: the .qann file format's tags (reference src/serialize.hpp:29-38). */
enum { QG_KIND_FLAT = 1, QG_KIND_IVF = 2, QG_KIND_REFINE = 3 };
/* Metrics (reference include/vecengine/index.hpp:57-62). */
enum { QG_METRIC_L2 = 0, QG_METRIC_COSINE = 1, QG_METRIC_INNER_PRODUCT = 2 };
/* Coarse clustering (reference include/vecengine/ivf_index.hpp:27-30). */
enum { QG_CLUSTERING_EMEANS = 0, QG_CLUSTERING_LLOYD = 1 };

/* The calling thread's last error message ("" when none). */
const char* qg_last_error(void);

/* Version string of the library build. */
const char* qg_version(void);

/* --- construction ------------------------------------------------------------
 * qg_create_ivf   replaces IVFIndex::IVFIndex(dim, nlist, nprobe, custom_ids, metric)
 *                 (reference include/vecengine/ivf_index.hpp:62)
 * qg_enable_pq    replaces IVFIndex::enable_pq(m, K, fast_scan, rotate) (ivf_index.hpp:69-70)
 * qg_create_flat  replaces FlatIndex::FlatIndex(dim, capacity, custom_ids, metric)
 *                 (reference include/vecengine/flat_index.hpp:25)
 * qg_create_refine replaces RefineIndex::RefineIndex(base, k_factor, custom_ids)
 *                 (reference include/vecengine/refine_index.hpp:37)
 */
int qg_create_ivf(size_t dim, size_t nlist, size_t nprobe, int metric, int custom_ids, qg_index** out);
int qg_enable_pq(qg_index* h, size_t m, size_t centroids_per_subspace, int fast_scan, int rotate);
int qg_create_flat(size_t dim, int metric, int custom_ids, qg_index** out);
int qg_create_refine(qg_index* base, size_t k_factor, int custom_ids, qg_index** out);
/* A new handle to a RefineIndex's base (reference refine_index.hpp:88-89 base()). */
int qg_refine_base(qg_index* refine, qg_index** out);
void qg_free(qg_index* h);

/* --- training and adding --------------------------------------------------------
 * qg_train replaces IVFIndex::train(vectors, n, max_iters, seed, clustering, passes)
 *          (reference include/vecengine/ivf_index.hpp:143-145); seed < 0 = unseeded.
 * qg_add   replaces DenseIndex::add_batch(vecs, n, ids) (reference index.hpp:185);
 *          ids is NULL unless the index has custom ids; out_ids (n) may be NULL.
 */
int qg_train(qg_index* h, const float* x, size_t n, size_t max_iters, int64_t seed, int clustering, size_t passes);
int qg_add(qg_index* h, const float* x, size_t n, const int64_t* ids, int64_t* out_ids);
/* replaces IndexBase::remove / compact (reference index.hpp:122-128) */
int qg_remove(qg_index* h, const int64_t* ids, size_t n, size_t* removed);
int qg_compact(qg_index* h, size_t* reclaimed);

/* --- search ------------------------------------------------------------------------
 * Replaces DenseIndex::query_batch(queries, nq, k[, allowed]) (reference
 * include/vecengine/index.hpp:197-209) as the Python batch_query presents it
 * (reference bindings/python_bindings.cpp:582-648): out_ids / out_dists are
 * nq * k, padded with -1 / +inf. allowed: NULL for no filter, else n_allowed
 * ids (unknown / deleted / repeated ids are ignored).
 * Host buffers; the copies to and from the device are part of the call.
 */
int qg_search(qg_index* h, const float* q, size_t nq, size_t k, const int64_t* allowed, size_t n_allowed,
              int64_t* out_ids, float* out_dists);
/* The same with the filter as a slot bitmap (bit s of words[s / 64]: slot s
 * may be returned), the form a host-side where= evaluation produces
 * (reference src/index.cpp:156-163). nwords must cover the index's slots. */
int qg_search_bitmap(qg_index* h, const float* q, size_t nq, size_t k, const uint64_t* words, size_t nwords,
                     int64_t* out_ids, float* out_dists);
/* Device-resident variant: q_dev, out_ids_dev, out_dists_dev are device
 * pointers and the work runs on `stream` (a cudaStream_t, NULL = the legacy
 * default stream); the call returns when the results are written. */
int qg_search_device(qg_index* h, const float* q_dev, size_t nq, size_t k, int64_t* out_ids_dev, float* out_dists_dev,
                     void* stream);

/* --- sharded search (no counterpart in the reference, which searches one
 * in-process index) -------------------------------------------------------------------
 * Spreads an IVF index's lists over several devices or processes. qg_set(h,
 * "shards", n) and qg_set(h, "shard", s) on an IVF handle make its device copy
 * hold only the lists l with l % n == s. The sizes of all lists stay known, so
 * every shard numbers the probed vectors alike and candidate keys compare
 * across shards. Each shard computes its candidates:
 *   qg_candidate_count(h, k, &kp);      k' per query (k, or min(k * k_factor, size))
 *   qg_search_candidates_device(h, q_dev, nq, k, key_dev, slot_dev, stream);   nq x kp sorted
 * The shards exchange candidates (an all-gather into [nq][nparts][kp]). Each
 * then merges and finishes, with the same results as one unsharded search:
 *   qg_merge_candidates_device(keys, slots, nq, nparts, kp, key_out, slot_out, stream);
 *   qg_finish_candidates_device(h, q_dev, nq, k, key_out, slot_out, ids_dev, dists_dev, stream);
 * h may be the IVF handle or a RefineIndex over it (whose raw rows every shard keeps).
 * Unfiltered queries. A sharded handle refuses qg_search and the server. */
int qg_candidate_count(qg_index* h, size_t k, size_t* kp);
int qg_search_candidates_device(qg_index* h, const float* q_dev, size_t nq, size_t k, uint64_t* key_dev,
                                uint32_t* slot_dev, void* stream);
int qg_merge_candidates_device(const uint64_t* key_dev, const uint32_t* slot_dev, size_t nq, size_t nparts, size_t kp,
                               uint64_t* out_key_dev, uint32_t* out_slot_dev, void* stream);
int qg_finish_candidates_device(qg_index* h, const float* q_dev, size_t nq, size_t k, const uint64_t* key_dev,
                                const uint32_t* slot_dev, int64_t* out_ids_dev, float* out_dists_dev, void* stream);

/* --- properties ------------------------------------------------------------------
 * keys: "nprobe", "k_factor", "precomputed_tables", "cosine_inner_product",
 * "filter_probe_scaling" (settable; reference ivf_index.hpp:83-118,
 * refine_index.hpp:91-93) and the read-only "dim", "kind", "metric", "nlist",
 * "size", "slots", "custom_ids", "fast_scan", "pq_m", "pq_k", "trained",
 * "rotate", "sq_bits", "wrapped". Also settable, with no reference
 * counterpart: "shard" / "shards", the sharded search's list partition.
 */
int qg_get(qg_index* h, const char* key, int64_t* value);
int qg_set(qg_index* h, const char* key, int64_t value);
/* IVF inspection (for sizing and accounting; the reference keeps these
 * private, reference include/vecengine/ivf_index.hpp:251-283): the vector
 * count of each of the nlist lists, and the nlist x dim coarse centroids. */
int qg_ivf_list_sizes(qg_index* h, uint32_t* out_sizes);
int qg_ivf_centroids(qg_index* h, float* out_centroids);

/* --- files ------------------------------------------------------------------------
 * .qann format 13, interchangeable with qann (reference src/index_factory.cpp:94-141).
 * qg_load: *kind receives QG_KIND_*.
 */
int qg_save(qg_index* h, const char* path);
int qg_load(const char* path, qg_index** out, int* kind);
/* qg_load_mapped replaces qann.load(path, mmap=True) (reference
 * src/index_factory.cpp:120-141, include/vecengine/vector_store.hpp:21-110):
 * the file is mapped read-only and a RefineIndex's raw rows (format 10 and
 * later, 64 KB aligned in the file) stay in the mapping, read in place by the
 * re-rank through host-mapped memory rather than copied into HBM, so rows
 * larger than the GPU's memory can be served. An add or compact copies them
 * into memory first; qg_get(h, "rows_mapped") reads 2 while the re-rank reads
 * the mapping, 1 while the rows are mapped but copied to HBM (the driver
 * refused the registration), 0 otherwise. Results are the same either way. */
int qg_load_mapped(const char* path, qg_index** out, int* kind);

/* --- profiling (no counterpart in the reference, which times sections with
 * compile-time timers, reference src/profile.hpp) --------------------------------
 * qg_profile_enable(1) brackets each launch of the named kernels ("scan",
 * "pair_scores", "select_rows", "query_tables", "merge", "refine") with CUDA
 * events on its stream; qg_profile_get folds finished timings in and returns
 * the total milliseconds and launch count for one name; qg_launch_count is
 * the number of this library's kernel launches since the library loaded. */
int qg_profile_enable(int on);
int qg_profile_reset(void);
int qg_profile_get(const char* kernel, double* total_ms, int64_t* launches);
int64_t qg_launch_count(void);

/* --- kernels of the path on device memory (parity tests and tools) ----------------
 * qg_quantize_lut_dev: n tables of m x 16 floats -> n LUTs of m x 16 bytes plus
 *   scale / offset each; bit-exact with quantize_lut (reference src/fast_scan.cpp:22-46).
 * qg_build_quantize_lut_dev: n tables B_i + C_i (+ A_i on row 0) rounded the same
 *   way (reference src/fast_scan.cpp:243-254 build_quantize_lut).
 * qg_fast_scan_dev: sums[v] = sum_s lut[lut_of[v / 64]][s][code(v, s)] for n
 *   vectors with plain codes (n x m bytes, one code per byte) and one LUT index
 *   per group of 64 vectors; the same values fast_scan_block computes
 *   (reference src/fast_scan.cpp:256-262). LUTs are nluts x m x 16 bytes,
 *   16-byte aligned. Waits for its work; a LUT index lut_of[i] >= nluts is
 *   caught on the device and returned as QG_INVALID_ARGUMENT.
 * qg_exact_scores_dev: out[i * nb + j] = squared L2 (ip = 0) or -(a . b) (ip = 1)
 *   in the reference's AVX2 accumulation order (reference src/distance.cpp:66-96, :138-151).
 */
int qg_quantize_lut_dev(const float* tables_dev, size_t n, size_t m, uint8_t* lut_dev, float* scale_dev,
                        float* offset_dev, void* stream);
int qg_build_quantize_lut_dev(const float* B_dev, const float* C_dev, const float* A_dev, size_t n, size_t m,
                              uint8_t* lut_dev, float* scale_dev, float* offset_dev, void* stream);
int qg_fast_scan_dev(const uint8_t* lut_dev, size_t nluts, size_t m, const uint8_t* codes_dev,
                     const uint32_t* lut_of_dev, size_t n, uint16_t* sums_dev, void* stream);
int qg_exact_scores_dev(const float* a_dev, size_t na, const float* b_dev, size_t nb, size_t dim, int ip,
                        float* out_dev, void* stream);

/* qg_fast_scan_noalloc_dev: qg_fast_scan_dev (same arguments, same sums) for
 * callers that cannot let the library allocate device memory — processes that
 * reserve all GPU memory for their own pool, frameworks whose allocator must
 * be the only one, latency-critical loops where cudaMalloc's device
 * synchronisation or failure under memory pressure is not acceptable. It
 * allocates nothing: its scratch is one 32 MiB device array built into the
 * library (held on every GPU that loads it), which bounds n to what fits
 * (about 1 million vectors at m = 64; larger n returns QG_INVALID_ARGUMENT).
 * The first call on a device looks the array up (cudaGetSymbolAddress): make
 * it before any stream capture. Calls share the array, so calls that overlap
 * on the GPU race. Like qg_fast_scan_dev, the call waits for its work on
 * `stream`: a LUT index lut_of[i] >= nluts is caught on the device and
 * returned as QG_INVALID_ARGUMENT.
 * No counterpart in the reference, which runs on the CPU only. */
int qg_fast_scan_noalloc_dev(const uint8_t* lut_dev, size_t nluts, size_t m, const uint8_t* codes_dev,
                             const uint32_t* lut_of_dev, size_t n, uint16_t* sums_dev, void* stream);

/* --- process-wide options ---------------------------------------------------------
 * "tensor_filter": exact top-k searches over many rows (flat search, RefineIndex
 *   direct scans, nearest-centroid assignment in add and k-means) first filter
 *   candidates with a BF16 tcgen05 GEMM and a rigorous error bound, then rescore
 *   them exactly; the results are those of the exact path either way.
 *   0 = never, 1 = when the work is large enough to pay (default), 2 = whenever
 *   the dimension is supported (<= 128). qg_get_option also reads
 *   "tensor_filter_queries" (queries answered through the filter so far) and
 *   "tensor_filter_redone" (those redone exactly after a candidate overflow). The same mode sends an IVF search's
 *   coarse step (the nprobe nearest lists, reference src/ivf_index.cpp:305-419) through BF16 estimates with an
 *   error bound and an exact FP32 recheck of the lists that can still be among the nearest; qg_get_option reads
 *   "tensor_coarse_queries", "tensor_coarse_redone" (queries sent back to the exact path after too many
 *   near-ties) and "tensor_coarse_candidates" (lists rescored exactly). No counterpart in the reference, whose
 *   exact scores always come from its CPU distance kernels (reference src/flat_index.cpp:33-64).
 *   Filtered IVF searches rank only the nearest lists their probe walk is expected to need, through the same
 *   coarse step; "filtered_batches" counts filtered batches and "filtered_deep_walks" those of them whose walk
 *   went past the ranked lists, so that every list was ranked (reference src/ivf_index.cpp:501-521 ranks every
 *   list of every filtered query).
 * "scan_autotune": 1 (default) times the fast-scan kernel's candidate shapes
 *   (warps per block, lists per LUT group, codes read from global memory or
 *   staged through shared memory by bulk copies) on the first large search of
 *   each problem (scoring mode, m, k', and nprobe and batch size by their power
 *   of two) and keeps the
 *   fastest; 0 uses the first shape. "scan_variant": -1 (default) any shape,
 *   0 only unstaged shapes sized for two blocks per SM, 1 only staged, 2 only
 *   the dense unstaged shapes (registers sized for 3 blocks of 8 warps or 5
 *   of 4). qg_get_option also reads "scan_tuned_shapes" (problems tuned so
 *   far) and "scan_last_shape" (the last scan's shape: warps * 1000 + lists
 *   per group * 10 + 1 staged / 2 dense). Results are the same under
 *   every shape. No counterpart in the reference, whose scan kernel is fixed
 *   (reference src/fast_scan.cpp:306-338).
 * "tensor_scan": the fast-scan of large unfiltered IVF batches with per-list
 *   L2 tables on the tensor cores, list-major: each list's vectors as one-hot
 *   rows times the rounded LUTs of every query probing it, a tcgen05 int8 GEMM
 *   whose integer sums equal the lookups' (reference src/fast_scan.cpp:306-338
 *   computes them one query and block at a time). 0 = never, 1 = when it
 *   pays (default; on the workloads measured so far it is slower than the
 *   query-major kernel, so 1 does not pick it), 2 = whenever it applies.
 *   Results are the same in every mode. qg_get_option also reads
 *   "tensor_scan_calls" and "tensor_scan_redone" (queries whose candidates
 *   overflowed and were rescanned query-major).
 * "search_graphs": 1 makes qg_search_device replay device-resident, unfiltered
 *   searches of an IVF index (or a RefineIndex over one) as CUDA graphs. The
 *   first call with a given batch size, k, nprobe, k_factor, buffers and stream
 *   (a non-default stream) runs the search and captures it; later calls launch
 *   the graph and read its error flags. A change to the index invalidates its
 *   graphs. 0 (default) runs every search directly. qg_get_option also reads
 *   "search_graph_replays" and "search_graph_captures". No counterpart in the
 *   reference, which has no GPU path. */
int qg_set_option(const char* key, int64_t value);
int qg_get_option(const char* key, int64_t* value);

/* --- serving (no counterpart in the reference, whose query_batch answers one
 * call on the calling threads, reference bindings/python_bindings.cpp:600-648) ----
 * A server keeps the index on the device and runs requests with continuous
 * batching: `slots` worker threads, each with its own CUDA stream, take the
 * oldest waiting requests as soon as they are free (at most max_batch at a
 * time, and only while the estimated device memory of all batches in flight
 * stays within mem_budget_bytes; 0 = 2 GiB) and search them as one mixed batch.
 * Each request has its own k, nprobe (<= 0: the index's) and filter, and gets
 * the results it gets searched alone (qg_search with that nprobe set). Over a
 * RefineIndex, requests whose filter allows at most 6 * nlist slots (those the
 * RefineIndex answers by its exact direct scan) queue apart and run on one
 * extra worker thread, so that they never hold up the approximate batches.
 *
 * qg_server_add_filter registers a slot bitmap (deleted slots are masked out)
 *   that requests then name by filter_id.
 * qg_server_submit queues one query (dim floats); its filter is `allowed`
 *   (n_allowed ids, as qg_search) when non-NULL, else filter_id (-1 = none).
 * qg_server_wait blocks for a ticket's k results and its latency (submission
 *   to completion, microseconds); each ticket is waited for once.
 * qg_server_replay runs an open-loop arrival trace: request i is submitted at
 *   arrival_us[i] after the call starts, whatever the state of the others, with
 *   k[i], nprobe[i] (NULL = the index's) and filter_id[i] (NULL or -1 = none);
 *   results are nq x kmax (padded), latency_us[i] from its arrival time.
 * qg_server_free stops the workers (requests still queued fail); no other call
 *   on the server may be in progress. The server keeps its index alive. */
typedef struct qg_server qg_server;
int qg_server_create(qg_index* h, int slots, int max_batch, size_t mem_budget_bytes, qg_server** out);
int qg_server_add_filter(qg_server* s, const uint64_t* words, size_t nwords, int* filter_id);
int qg_server_submit(qg_server* s, const float* q, size_t k, int nprobe, const int64_t* allowed, size_t n_allowed,
                     int filter_id, uint64_t* ticket);
int qg_server_wait(qg_server* s, uint64_t ticket, int64_t* out_ids, float* out_dists, double* latency_us);
int qg_server_replay(qg_server* s, const float* q, size_t nq, const int32_t* k, const int32_t* nprobe,
                     const int32_t* filter_id, const double* arrival_us, size_t kmax, int64_t* out_ids,
                     float* out_dists, double* latency_us);
int qg_server_stats(qg_server* s, int64_t* completed, int64_t* batches, int64_t* peak_bytes);
void qg_server_free(qg_server* s);

/* --- host-side pieces of training (parity tests; no GPU needed) ------------------
 * qg_symmetric_eigen: eigenvalues (d) and eigenvectors (d x d, as columns) of a
 *   symmetric d x d matrix by cyclic Jacobi sweeps, bit-identical with the
 *   reference's symmetric_eigen (reference src/rotation.cpp:20-69).
 * qg_balanced_rotation: the PCA-balanced rotation (d x d, row-major) for m PQ
 *   subspaces from a d x d covariance, as balanced_pca_rotation derives it
 *   after its covariance step (reference src/rotation.cpp:106-130). */
int qg_symmetric_eigen(const double* a, size_t d, double* values, double* vectors);
int qg_balanced_rotation(const double* cov, size_t d, size_t m, float* rotation);

#ifdef __cplusplus
}
#endif

#endif /* QANN_GPU_H */
