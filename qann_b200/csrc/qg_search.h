// Device views of an index and the launchers of the search kernels.
#pragma once

#include <cuda_runtime.h>

#include "qg_cuda.h"

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace qg {

// How an IVF fast-scan index scores codes (reference src/ivf_index.cpp:436-456):
enum ScanMode : int {
    kModeL2 = 0,      // per-list LUT from the precomputed tables: B[list] + C[query] + A on row 0
    kModeL2Adc = 1,   // per-list LUT from the ADC table of (query - list center), no precomputed tables
    kModeIP = 2,      // one LUT per query from half the inner table; the list adds -(q . c)
    kModeCosIP = 3,   // cosine scored by inner product: one LUT per query; the list adds (A + 1) - |e|^2
};

// Device arrays of an IVF fast-scan index (all owned by the index object).
struct IvfView {
    int dim = 0, nlist = 0, m = 0, m_pad = 0, sd = 0;
    int mode = kModeL2;
    bool ip_metric = false;   // coarse ranks by -(q . c)
    bool has_resid = false;   // cosine: A is measured against each list's residual center
    const float* centroids = nullptr;   // nlist * dim
    const float* resid = nullptr;       // nlist * dim: residual centers, or the centroids
    const float* sqnorm = nullptr;      // nlist: |resid center|^2 (cosine-IP base)
    const float* pq_t = nullptr;        // m * sd * 16, transposed codebook
    const float* B = nullptr;           // nlist * m * 16 precomputed list terms (mode L2)
    const uint32_t* sb_off = nullptr;   // nlist + 1 superblock offsets
    const uint32_t* list_size = nullptr;
    const uint4* codes = nullptr;       // superblocks, 2 * m_pad uint4 each
    const uint32_t* ids = nullptr;      // 64 slots per superblock, kRemoved for padding
    const uint64_t* deleted = nullptr;  // slot bitmap of deleted vectors, or null
    const uint16_t* cent_f16 = nullptr;    // f16 copy of the centroids, each row scaled by 2^cent_exp
                                           // (cent_dpad per row), or null
    const float* cent_sq = nullptr;        // |centroid|^2 in float
    const int* cent_exp = nullptr;
    int cent_dpad = 0;
};

// Per-query settings of a mixed batch: served requests that each carry their
// own k, nprobe and filter. Device arrays of nq entries; a null array means
// the batch-wide value for every query.
struct PerQuery {
    const int* k = nullptr;            // results wanted
    const int* kp = nullptr;           // candidates kept (k, or min(k * k_factor, live))
    const int* nprobe = nullptr;       // probes of an unfiltered query
    const uint64_t* const* filter = nullptr;   // allowed-slot bitmap of each query (null entry: none)
    const int* min_probes = nullptr;   // filtered queries: probe at least this many lists,
    const int* wanted = nullptr;       // then on until this many allowed vectors were seen
};

struct ScanArgs {
    IvfView v;
    const float* q;          // nq * dim prepared queries
    const uint32_t* probe;   // nq * P lists, nearest first
    const float* pterm;      // nq * P per-probe terms
    const float* qC;         // mode L2: nq * m * 16
    const uint4* qlut;       // modes IP / cosine-IP: nq * m_pad rows
    const float* qscale;
    const float* qoffset;
    const uint64_t* filter;  // allowed-slot bitmap of every query, or null
    const uint64_t* const* filters;   // per-query bitmaps (overrides filter), or null
    const int* nprobe_q;     // per-query probe count, or null for P each
    int P, pch, nchunks, kp;
    int nunits;              // nq * nchunks work units (query, chunk of pch probes)
    int lc;                  // lists per LUT group
    int* work;               // next unit to take (zero at launch)
    // per query, shared by its chunks (nchunks > 1; else null): a bound on the
    // query's k'-th key, all ones at launch; every chunk lowers it and prunes by it
    unsigned long long* qthr;
    uint64_t* out_key;       // (nq * nchunks) * kp
    uint32_t* out_slot;
    int* err;
};

struct IvfSearchArgs {
    const float* q = nullptr;   // nq * dim, prepared (normalised for cosine)
    int nq = 0, k = 0, kp = 0, nprobe = 0;
    const uint64_t* filter = nullptr;
    // filtered probing (reference src/ivf_index.cpp:501-521): probes run past
    // nprobe to at least min_probes, then until `wanted` allowed vectors were seen
    int min_probes = 0, wanted = 0;
    // filtered batches: the nearest lists ranked per query before the walk
    // (0 = every list); a walk that runs past them ranks every list instead
    int rank_depth = 0;
    PerQuery pq;                // mixed batches; nprobe above is then the largest nprobe
    bool any_filter = false;    // some query of a mixed batch has a filter
    int sm_count = 0;
    int* d_err = nullptr;       // [0] scan overflow, [2] tensor-core pipeline timeout
    bool capture = false;       // being captured into a CUDA graph: no host reads, waits or tuning
};

void normalize_rows(const float* x, float* y, int n, int d, int* d_zero, cudaStream_t st);
// out = x R for n rows of d (R: d x d row-major), in the reference's FMA order.
void rotate_rows(const float* R, const float* x, size_t n, int d, float* out, cudaStream_t st);
void pair_scores(const float* A, int na, const float* B, int nb, int d, bool ip, float* out, size_t ld_out,
                 cudaStream_t st);
// The P smallest scores of each row by (key, column), sorted; refused columns
// (allow / deny bitmaps over col_base + column) come out as 0xFFFFFFFF / +inf.
// eq0 compares -0 and +0 as equal (float operator< semantics).
void select_rows(const float* scores, size_t ld, int nrows, int ncols, int P, uint32_t* out_col, float* out_score,
                 cudaStream_t st, const uint64_t* allow = nullptr, const uint64_t* deny = nullptr, size_t col_base = 0,
                 bool eq0 = false);
// Per-probe terms (A, or the cosine-IP base) and per-query tables (C, or the
// query's uint8 LUT with its scale / offset).
void probe_terms(const IvfView& v, const float* q, int nq, int P, const uint32_t* probe, const float* pdist, float* term,
                 cudaStream_t st);
void query_tables(const IvfView& v, const float* q, int nq, float* qC, uint4* qlut, float* qscale, float* qoffset,
                  cudaStream_t st);
// Probe lists of filtered queries: the s.rank_depth nearest lists (or every
// list) ranked by (score, list), each query's probe count (nprobe_q) from the
// filter's per-list allowed counts; probe / pdist are nq x Pmax, and Pmax is
// returned.
int filtered_probes(const IvfView& v, const IvfSearchArgs& s, DevBuf<uint32_t>& probe, DevBuf<float>& pdist,
                    DevBuf<int>& nprobe_q, cudaStream_t st);
// Filtered batches ranked so far, and how many of them ranked every list
// because a walk went past their rank_depth nearest lists.
void filtered_rank_counts(int64_t* batches, int64_t* deep);
// The P nearest lists of each query by (exact score, list), -0 == +0, nearest
// first, with their scores (reference src/ivf_index.cpp:305-419): the tensor
// cores' estimates and exact recheck, or exact tiles and a row select.
void nearest_lists(const IvfView& v, const IvfSearchArgs& s, int nq, int P, uint32_t* probe, float* pdist,
                   cudaStream_t st);
// The k' = s.kp best candidates of each query, as sorted (key64, slot) lists
// (key64 = key(dist) << 32 | push index; 0xFFFF... marks an empty entry).
void ivf_candidates(const IvfView& v, const IvfSearchArgs& s, uint64_t* out_key, uint32_t* out_slot, cudaStream_t st);
// Coarse assignment through the tensor cores (qg_mm.cu): the P nearest lists
// of each query by exact score, ties by list, from BF16 estimates with an
// error bound and an exact recheck; queries with too many near-ties are
// listed in redo_q for the exact path. use_tensor_coarse: whether the batch
// goes this way (the process-wide tensor-filter mode and the work's size).
bool coarse_mm_supported(int nlist, int dim, int P, bool cent_prepared, bool no_readback = false);
bool use_tensor_coarse(size_t nq, int nlist, int dim);
// Queries whose coarse step went through the tensor cores, and those of them redone exactly.
void count_tensor_coarse(int64_t queries, int64_t redone);
void tensor_coarse_counts(int64_t* queries, int64_t* redone);
// Lists rescored exactly by the tensor-core coarse step so far (its candidates).
void count_tensor_coarse_candidates(int64_t n);
int64_t tensor_coarse_candidates();
// With err_dev (under graph capture, and for batches of at most one query per
// SM) nothing is read back and redo_q stays empty: every list fits the
// recheck, queries with extreme norms rescore every list, and a pipeline
// timeout is flagged in *err_dev for the caller to read with the results.
void coarse_probes_mm(const IvfView& v, const float* q, int nq, int P, uint32_t* probe, float* pdist,
                      std::vector<int>& redo_q, cudaStream_t st, int* err_dev = nullptr);
// Rows scaled by powers of two (2^exps) and rounded to f16 (zero-padded to
// dpad, a multiple of 8), with their float squared norms (unscaled).
void prepare_f16_rows(const float* rows, size_t n, int dim, DevBuf<uint16_t>& f16, DevBuf<float>& sq,
                      DevBuf<int>& exps, int& dpad, cudaStream_t st);

// The scan's shape autotuner: on (1, the default) it times the candidate
// shapes on the first large search of each problem key; off (0) every search
// uses the first candidate. The variant restricts the candidates: -1 any, 0
// codes read from global memory, 1 codes staged through shared memory.
void set_scan_autotune(int on);
int scan_autotune();
void set_scan_variant(int v);
int scan_variant();
int scan_tuned_shapes();
// The last scan's shape: warps * 1000 + lists per LUT group * 10 + staged.
int scan_last_shape();
// The kp smallest key64 over nchunks sorted lists per query.
void merge_candidates(const uint64_t* in_key, const uint32_t* in_slot, int nq, int nchunks, int kp, uint64_t* out_key,
                      uint32_t* out_slot, cudaStream_t st);
// IVF results from candidates: the first k, sorted by (distance, id). With
// k_q, query i takes its first k_q[i] candidates and pads the rest of its k.
void finalize_ivf(const uint64_t* key, const uint32_t* slot, int nq, int kp, int k, const int64_t* labels, bool cosine,
                  int64_t* out_ids, float* out_d, cudaStream_t st, const int* k_q = nullptr);
// Exact re-rank of candidates from raw rows: the k best by (score, slot).
// With kp_q / k_q, query i re-ranks its first kp_q[i] candidates into k_q[i] results.
void refine_candidates(const float* q, int nq, int dim, const float* rows, const uint64_t* key, const uint32_t* slot,
                       int kp, int k, bool ip, const int64_t* labels, bool cosine, int64_t* out_ids, float* out_d,
                       cudaStream_t st, const int* kp_q = nullptr, const int* k_q = nullptr);
// The fast-scan on the tensor cores (qg_tscan.cu), list-major, for large
// unfiltered batches of per-list L2 tables. Mode 0 never, 1 when the batch
// is large enough to pay (default), 2 whenever it applies.
void set_tensor_scan(int mode);
int tensor_scan();
void tensor_scan_counts(int64_t* calls, int64_t* redone);
// work counters: "units", "tiles", "luts_live", "luts_hopeless", "candidates", "pairs", "pairs_kept"
bool tensor_scan_stat(const std::string& name, int64_t* value);
bool tensor_scan_applies(const IvfView& v, const IvfSearchArgs& s, int P, bool per_query);
int tensor_scan_first(int P);   // probes per query that wave 0 scans query-major
void fill_i32(int* a, int n, int value, cudaStream_t st);
// Wave 1 and the final cut: key0 holds wave 0's k' best keys per query
// (sorted, from its first tensor_scan_first(P) probes). Fills out_key /
// out_slot except for the queries listed in redo_q, whose candidates
// overflowed (the caller redoes them).
void tensor_scan_candidates(const IvfView& v, int nq, int P, int kp, const uint32_t* probe, const float* pterm,
                            const float* qC, const uint64_t* key0, uint64_t* out_key, uint32_t* out_slot,
                            std::vector<int>& redo_q, int* d_err, cudaStream_t st);
} // namespace qg
