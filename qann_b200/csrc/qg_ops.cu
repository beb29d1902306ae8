// Search dispatch over the index kinds, flat exact search, and the pieces of
// add (nearest-centroid assignment, PQ encoding) that run on the GPU.
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_train.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <numeric>
#include <thread>

namespace qg {

// ---------------------------------------------------------------------------
// Flat exact search: tiles of rows scored for a block of queries, each tile's
// k best per query (by (score, slot), -0 == +0 as the reference's heap of
// (float, slot) pairs compares; reference src/flat_index.cpp:33-64) merged
// into the running k best.
// ---------------------------------------------------------------------------
__global__ void k_cols_to_keys(const uint32_t* __restrict__ col, const float* __restrict__ score, size_t n, int P,
                               int k, size_t col_base, uint64_t* __restrict__ key, uint32_t* __restrict__ slot) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * k) return;
    const size_t row = t / k;
    const int j = static_cast<int>(t % k);
    if (j < P && col[row * P + j] != 0xFFFFFFFFu) {
        const uint64_t s = col_base + col[row * P + j];
        key[t] = (static_cast<uint64_t>(float_key_eq0(score[row * P + j])) << 32) | s;
        slot[t] = static_cast<uint32_t>(s);
    } else {
        key[t] = ~0ull;
        slot[t] = 0xFFFFFFFFu;
    }
}

// merges running (a) and tile (b) lists of k into a, per query
__global__ void __launch_bounds__(256) k_merge2(uint64_t* __restrict__ akey, uint32_t* __restrict__ aslot,
                                                const uint64_t* __restrict__ bkey, const uint32_t* __restrict__ bslot,
                                                int k) {
    extern __shared__ uint8_t sm_raw[];
    const int n = next_pow2(2 * k);
    uint64_t* key = reinterpret_cast<uint64_t*>(sm_raw);
    int64_t* val = reinterpret_cast<int64_t*>(key + n);
    const size_t base = static_cast<size_t>(blockIdx.x) * k;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (i < k) {
            key[i] = akey[base + i];
            val[i] = aslot[base + i];
        } else if (i < 2 * k) {
            key[i] = bkey[base + i - k];
            val[i] = bslot[base + i - k];
        } else {
            key[i] = ~0ull;
            val[i] = INT64_MAX;
        }
    }
    bitonic_sort(key, val, n);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        akey[base + i] = key[i];
        aslot[base + i] = key[i] == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(val[i]);
    }
}

static void flat_candidates_fp32(const float* q_dev, size_t nq, const float* rows_dev, size_t n, int dim, bool ip,
                                 size_t k, const uint64_t* allow_dev, const uint64_t* deny_dev, uint64_t* out_key,
                                 uint32_t* out_slot, cudaStream_t st) {
    if (nq == 0 || k == 0) return;
    require(k <= 4096, "k above 4096 is not supported by the GPU flat search", kUnsupported);
    QG_CUDA(cudaMemsetAsync(out_key, 0xFF, nq * k * sizeof(uint64_t), st));
    QG_CUDA(cudaMemsetAsync(out_slot, 0xFF, nq * k * sizeof(uint32_t), st));
    if (n == 0) return;
    size_t QB = std::min<size_t>(nq, 4096);
    const size_t T = std::min<size_t>(n, std::max<size_t>(k, (size_t{256} << 20) / (QB * sizeof(float))));
    // a short row range (a seed of a few hundred rows) takes larger query
    // blocks in the same 256 MB of scores and of per-query keys (at most
    // 65,536 queries: 4,096 tile rows)
    const size_t big = std::min<size_t>({size_t{65536}, (size_t{256} << 20) / (T * sizeof(float)),
                                         (size_t{256} << 20) / (k * 16)});
    QB = std::min<size_t>(nq, std::max<size_t>(QB, big));
    DevBuf<float> scores(QB * T, st);
    DevBuf<uint32_t> col(QB * std::min(k, T), st);
    DevBuf<float> sc(QB * std::min(k, T), st);
    DevBuf<uint64_t> tkey(QB * k, st);
    DevBuf<uint32_t> tslot(QB * k, st);
    const int msm_n = next_pow2(static_cast<int>(2 * k));
    const size_t msm = static_cast<size_t>(msm_n) * 16;
    if (msm > 48 * 1024)
        allow_large_smem<k_merge2>();
    for (size_t q0 = 0; q0 < nq; q0 += QB) {
        const size_t nb = std::min(QB, nq - q0);
        for (size_t r0 = 0; r0 < n; r0 += T) {
            const size_t nr = std::min(T, n - r0);
            const int P = static_cast<int>(std::min(k, nr));
            pair_scores(q_dev + q0 * dim, static_cast<int>(nb), rows_dev + r0 * dim, static_cast<int>(nr), dim, ip,
                        scores.get(), nr, st);
            select_rows(scores.get(), nr, static_cast<int>(nb), static_cast<int>(nr), P, col.get(), sc.get(), st,
                        allow_dev, deny_dev, r0, true);
            k_cols_to_keys<<<static_cast<unsigned>(ceil_div(nb * k, 256)), 256, 0, st>>>(col.get(), sc.get(), nb, P,
                                                                                        static_cast<int>(k), r0,
                                                                                        tkey.get(), tslot.get());
            QG_LAUNCH_CHECK();
            k_merge2<<<static_cast<unsigned>(nb), 256, msm, st>>>(out_key + q0 * k, out_slot + q0 * k, tkey.get(),
                                                                   tslot.get(), static_cast<int>(k));
            QG_LAUNCH_CHECK();
        }
    }
}

namespace {
std::atomic<int> g_tensor_filter{1};
std::atomic<int64_t> g_filter_queries{0}, g_filter_redone{0};
}

void tensor_filter_counts(int64_t* queries, int64_t* redone) {
    *queries = g_filter_queries.load();
    *redone = g_filter_redone.load();
}

void set_tensor_filter(int mode) { g_tensor_filter.store(mode); }
int tensor_filter() { return g_tensor_filter.load(); }

// The exact top-k either way; the tensor-core filter when the work is large
// enough to pay for its bf16 copies (or always, in mode 2), the FP32 tiles
// otherwise.
bool use_tensor_filter(size_t nq, size_t n, int dim, size_t k) {
    const int mode = g_tensor_filter.load();
    const size_t seed = std::max<size_t>(4096, 4 * k);
    return mode > 0 && mm_supported(dim) && k <= 1024 && n > 2 * seed &&
           (mode == 2 || (nq >= 64 && static_cast<double>(nq) * double(n) * dim >= 2e10));
}

namespace {
std::atomic<int64_t> g_coarse_queries{0}, g_coarse_redone{0}, g_coarse_candidates{0};
}

void count_tensor_coarse_candidates(int64_t n) { g_coarse_candidates += n; }
int64_t tensor_coarse_candidates() { return g_coarse_candidates.load(); }

void count_tensor_coarse(int64_t queries, int64_t redone) {
    g_coarse_queries += queries;
    g_coarse_redone += redone;
}

void tensor_coarse_counts(int64_t* queries, int64_t* redone) {
    *queries = g_coarse_queries.load();
    *redone = g_coarse_redone.load();
}

// The coarse step on the tensor cores once the exact tiles' work passes
// 2.5e7 multiply-adds (about 12 queries against 16,384 lists of 128
// dimensions): there the exact scores and row select of a batch took 66 us
// at 16 queries and 310 us at 256, the F16 GEMM and recheck 47 and 56 us.
// Coarse tables of at least 2^21 values (16,384 lists of 128 dimensions)
// take the tensor cores at every batch size: for a single query there the
// exact path took 92 us and the F16 GEMM and recheck 66 us.
bool use_tensor_coarse(size_t nq, int nlist, int dim) {
    const int mode = g_tensor_filter.load();
    return mode > 0 && mm_supported(dim) &&
           (mode == 2 || static_cast<double>(nq) * nlist * dim >= 2.5e7 ||
            static_cast<double>(nlist) * dim >= 2097152.0);
}

void flat_candidates(const float* q_dev, size_t nq, const float* rows_dev, size_t n, int dim, bool ip, size_t k,
                     const uint64_t* allow_dev, const uint64_t* deny_dev, uint64_t* out_key, uint32_t* out_slot,
                     cudaStream_t st, bool allow_mm, const MmRows* pre) {
    if (!allow_mm || !use_tensor_filter(nq, n, dim, k)) {
        flat_candidates_fp32(q_dev, nq, rows_dev, n, dim, ip, k, allow_dev, deny_dev, out_key, out_slot, st);
        return;
    }
    MmRows tmp;
    const MmRows* base = pre;
    if (!base) {
        mm_prepare(rows_dev, n, dim, tmp, st);
        base = &tmp;
    }
    std::vector<int> ovf;
    mm_topk(q_dev, nq, rows_dev, *base, ip, k, allow_dev, deny_dev, out_key, out_slot, ovf, st);
    g_filter_queries += static_cast<int64_t>(nq);
    g_filter_redone += static_cast<int64_t>(ovf.size());
    if (ovf.empty()) return;
    // queries whose candidate list overflowed: the exact FP32 tiles over every row
    const size_t m = ovf.size();
    DevBuf<uint32_t> idx(m, st);
    std::vector<uint32_t> hidx(ovf.begin(), ovf.end());
    QG_CUDA(cudaMemcpyAsync(idx.get(), hidx.data(), m * 4, cudaMemcpyHostToDevice, st));
    DevBuf<float> qs(m * dim, st);
    gather_rows(q_dev, idx.get(), m, dim, qs.get(), st);
    DevBuf<uint64_t> sk(m * k, st);
    DevBuf<uint32_t> ss(m * k, st);
    flat_candidates_fp32(qs.get(), m, rows_dev, n, dim, ip, k, allow_dev, deny_dev, sk.get(), ss.get(), st);
    for (size_t j = 0; j < m; ++j) {
        QG_CUDA(cudaMemcpyAsync(out_key + static_cast<size_t>(ovf[j]) * k, sk.get() + j * k, k * 8,
                                cudaMemcpyDeviceToDevice, st));
        QG_CUDA(cudaMemcpyAsync(out_slot + static_cast<size_t>(ovf[j]) * k, ss.get() + j * k, k * 4,
                                cudaMemcpyDeviceToDevice, st));
    }
    QG_CUDA(cudaStreamSynchronize(st));
}

// Flat results in (score, slot) order with ids and the exact score.
__global__ void k_finalize_flat(const float* __restrict__ q, int dim, const float* __restrict__ rows,
                                const uint32_t* __restrict__ slot, int k, bool ip, const int64_t* __restrict__ labels,
                                bool cosine, int64_t* __restrict__ out_ids, float* __restrict__ out_d, size_t nq) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= nq * k) return;
    const size_t qi = t / k;
    const uint32_t s = slot[t];
    if (s == 0xFFFFFFFFu) {
        out_ids[t] = -1;
        out_d[t] = __int_as_float(0x7f800000);
        return;
    }
    const float d = exact_score(rows + static_cast<size_t>(s) * dim, q + qi * dim, dim, ip);
    out_ids[t] = labels ? labels[s] : static_cast<int64_t>(s);
    out_d[t] = cosine ? __fmul_rn(d, 0.5f) : d;
}

// ---------------------------------------------------------------------------
// Search dispatch
// ---------------------------------------------------------------------------
static int sm_count_cached() {
    static int n = 0;
    if (!n) n = sm_count();
    return n;
}

namespace {
struct Prepared {
    DevBuf<float> q;     // prepared queries (normalised for cosine)
    DevBuf<uint64_t> filter;
    DevBuf<int> err_own;
    int* err = nullptr;  // [0] scan overflow, [1] zero cosine row, [2] tensor-core pipeline timeout
};
} // namespace

static void prepare(IndexObj& idx, const SearchRequest& r, Prepared& p, cudaStream_t st, bool upload_filter = true) {
    const size_t dim = idx.dim();
    const size_t n = r.nq * dim;
    if (r.err_dev) {
        p.err = r.err_dev;
    } else {
        p.err_own.alloc(3, st);
        p.err = p.err_own.get();
    }
    QG_CUDA(cudaMemsetAsync(p.err, 0, 3 * sizeof(int), st));
    DevBuf<float> raw;
    const float* src = r.q;
    if (r.io == IoSpace::Host) {
        raw.alloc(n, st);
        QG_CUDA(cudaMemcpyAsync(raw.get(), r.q, n * sizeof(float), cudaMemcpyHostToDevice, st));
        src = raw.get();
    }
    p.q.alloc(n, st);
    if (idx.metric() == Metric::Cosine) {
        normalize_rows(src, p.q.get(), static_cast<int>(r.nq), static_cast<int>(dim), p.err + 1, st);
    } else {
        QG_CUDA(cudaMemcpyAsync(p.q.get(), src, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    if (r.filter && upload_filter) {
        p.filter.alloc(r.filter->words.size(), st);
        QG_CUDA(cudaMemcpyAsync(p.filter.get(), r.filter->words.data(), r.filter->words.size() * 8,
                                cudaMemcpyHostToDevice, st));
    }
}

// IVF stages see rotated queries when the index rotates (reference
// src/ivf_index.cpp:196-204); a RefineIndex re-ranks with the unrotated ones.
static const float* ivf_queries(const IVFObj& o, const Prepared& p, size_t nq, DevBuf<float>& rot, cudaStream_t st) {
    if (!o.model.rotate) return p.q.get();
    const int dim = static_cast<int>(o.model.dim);
    rot.alloc(nq * dim, st);
    rotate_rows(o.dev.rot.get(), p.q.get(), nq, dim, rot.get(), st);
    return rot.get();
}

static void fill_empty(const SearchRequest& r, cudaStream_t st) {
    const size_t n = r.nq * r.k;
    if (!n) return;
    std::vector<int64_t> ids(n, -1);
    std::vector<float> d(n, std::numeric_limits<float>::infinity());
    if (r.io == IoSpace::Host) {
        std::copy(ids.begin(), ids.end(), r.out_ids);
        std::copy(d.begin(), d.end(), r.out_d);
    } else {
        QG_CUDA(cudaMemcpyAsync(r.out_ids, ids.data(), n * 8, cudaMemcpyHostToDevice, st));
        QG_CUDA(cudaMemcpyAsync(r.out_d, d.data(), n * 4, cudaMemcpyHostToDevice, st));
        QG_CUDA(cudaStreamSynchronize(st));
    }
}

static void check_err(const int* err, cudaStream_t st) {
    int h[3] = {0, 0, 0};
    QG_CUDA(cudaMemcpyAsync(h, err, sizeof(h), cudaMemcpyDeviceToHost, st));
    QG_CUDA(cudaStreamSynchronize(st));
    if (h[1]) throw Error(kInvalidArgument, "cosine metric needs non-zero vectors");
    if (h[0]) throw Error(kRuntimeError, "fast-scan candidate buffer overflowed (internal error)");
    if (h[2]) throw Error(kRuntimeError, "tensor-core coarse step: a pipeline wait timed out");
}

// Filtered probing of an IVF index (reference src/ivf_index.cpp:501-521): at
// least min_probes lists, then on until `wanted` allowed vectors were seen.
static size_t min_probes_for(const IVFModel& M, size_t nprobe, size_t count) {
    if (!M.filter_probe_scaling || count == 0) return nprobe;
    const double want = std::ceil(0.75 * double(nprobe) * std::cbrt(double(M.idmap.live_count()) / double(count)));
    return std::clamp<size_t>(static_cast<size_t>(std::min(want, double(M.nlist))), nprobe, M.nlist);
}

// Lists a filtered query's probe walk is expected to need, to be ranked before
// it: its min_probes, or twice as many lists as hold `wanted` allowed vectors
// at the filter's mean density, plus 16; 0 (rank every list) from half of
// them. A walk that goes further ranks every list, so this sets only the cost.
static int rank_depth_for(const IVFModel& M, size_t min_probes, size_t wanted, size_t count) {
    const double per_list = double(count) / double(M.nlist);
    const double need = per_list > 0.0 ? 2.0 * double(wanted) / per_list : double(M.nlist);
    const double r = std::max(double(min_probes), std::ceil(need)) + 16.0;
    return 2.0 * r >= double(M.nlist) ? 0 : static_cast<int>(r);
}

static void filter_probing(IvfSearchArgs& a, const IVFModel& M, const SlotBits* f, const uint64_t* f_dev, size_t k) {
    if (!f) return;
    a.filter = f_dev;
    a.wanted = static_cast<int>(std::min(k, f->count));
    a.min_probes = static_cast<int>(min_probes_for(M, static_cast<size_t>(a.nprobe), f->count));
    a.rank_depth = rank_depth_for(M, static_cast<size_t>(a.min_probes), static_cast<size_t>(a.wanted), f->count);
}

__global__ void k_cols_to_slots(uint32_t* __restrict__ cs, size_t n, const uint32_t* __restrict__ slots) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n && cs[t] != 0xFFFFFFFFu) cs[t] = slots[cs[t]];
}

// RefineIndex::direct_scan on the GPU: the k best allowed rows by exact score,
// first pushed (lowest slot) among ties, then sorted by (distance, id).
static void refine_direct(RefineObj& o, const Prepared& p, const SearchRequest& r, int dim, bool ip, bool cosine,
                          int64_t* out_ids, float* out_d, cudaStream_t st) {
    // the allowed slots in ascending order: a server's registered filter keeps
    // them on the device; otherwise they are listed from the bitmap here
    DevBuf<uint32_t> ds;
    const uint32_t* slots_dev = r.filter_slots_dev;
    size_t n = r.filter->count;
    if (!slots_dev) {
        std::vector<uint32_t> slots;
        slots.reserve(r.filter->count);
        for (size_t w = 0; w < r.filter->words.size(); ++w)
            for (uint64_t bits = r.filter->words[w]; bits; bits &= bits - 1)
                slots.push_back(static_cast<uint32_t>(w * 64 + __builtin_ctzll(bits)));
        n = slots.size();
        ds.alloc(n, st);
        QG_CUDA(cudaMemcpyAsync(ds.get(), slots.data(), n * 4, cudaMemcpyHostToDevice, st));
        slots_dev = ds.get();
    }
    DevBuf<float> rows(n * dim, st);
    gather_rows(o.dev.ptr(), slots_dev, n, dim, rows.get(), st);
    DevBuf<uint64_t> ck(r.nq * r.k, st);
    DevBuf<uint32_t> cs(r.nq * r.k, st);
    flat_candidates(p.q.get(), r.nq, rows.get(), n, dim, ip, r.k, nullptr, nullptr, ck.get(), cs.get(), st);
    k_cols_to_slots<<<static_cast<unsigned>(ceil_div(r.nq * r.k, 256)), 256, 0, st>>>(cs.get(), r.nq * r.k, slots_dev);
    QG_LAUNCH_CHECK();
    finalize_ivf(ck.get(), cs.get(), static_cast<int>(r.nq), static_cast<int>(r.k), static_cast<int>(r.k),
                 o.dev.labels.get(), cosine, out_ids, out_d, st);
}

// A list-sharded IVF device copy holds only some lists: it answers through
// search_candidates / merge / finish_candidates alone.
static void require_unsharded(const IndexObj& idx) {
    const IndexObj* b = idx.kind == Kind::Refine ? static_cast<const RefineObj&>(idx).base.get() : &idx;
    require(b->kind != Kind::IVF || static_cast<const IVFObj&>(*b).shards == 1,
            "this index holds one shard of its lists: search it through the sharded search", kLogicError);
}

void search(IndexObj& idx, const SearchRequest& r, cudaStream_t st) {
    if (r.nq == 0) return;
    require_unsharded(idx);
    const bool empty_filter = r.filter && r.filter->count == 0;
    if (r.k == 0) return;
    const int dim = static_cast<int>(idx.dim());
    const bool cosine = idx.metric() == Metric::Cosine;
    const bool ip = idx.metric() == Metric::InnerProduct;
    // output staging
    DevBuf<int64_t> o_ids;
    DevBuf<float> o_d;
    int64_t* out_ids = r.out_ids;
    float* out_d = r.out_d;
    if (r.io == IoSpace::Host) {
        o_ids.alloc(r.nq * r.k, st);
        o_d.alloc(r.nq * r.k, st);
        out_ids = o_ids.get();
        out_d = o_d.get();
    }
    auto finish = [&](const Prepared& p) {
        if (r.io == IoSpace::Host) {
            QG_CUDA(cudaMemcpyAsync(r.out_ids, out_ids, r.nq * r.k * 8, cudaMemcpyDeviceToHost, st));
            QG_CUDA(cudaMemcpyAsync(r.out_d, out_d, r.nq * r.k * 4, cudaMemcpyDeviceToHost, st));
        }
        if (!r.capture) check_err(p.err, st);   // a captured search's caller reads the flags after each replay
    };

    if (idx.kind == Kind::IVF) {
        auto& o = static_cast<IVFObj&>(idx);
        if (empty_filter || o.model.idmap.live_count() == 0) {
            fill_empty(r, st);
            return;
        }
        ensure_device(o, st);
        Prepared p;
        prepare(idx, r, p, st);
        const int kp = static_cast<int>(r.k);
        require(kp <= 3072, "k above 3072 is not supported by the GPU fast-scan", kUnsupported);
        DevBuf<uint64_t> ck(r.nq * kp, st);
        DevBuf<uint32_t> cs(r.nq * kp, st);
        DevBuf<float> qrot;
        IvfSearchArgs a;
        a.q = ivf_queries(o, p, r.nq, qrot, st);
        a.nq = static_cast<int>(r.nq);
        a.k = static_cast<int>(r.k);
        a.kp = kp;
        a.nprobe = r.nprobe > 0 ? r.nprobe : static_cast<int>(o.model.nprobe);
        filter_probing(a, o.model, r.filter, p.filter.get(), r.k);
        a.capture = r.capture;
        a.sm_count = sm_count_cached();
        a.d_err = p.err;
        ivf_candidates(o.dev.view, a, ck.get(), cs.get(), st);
        finalize_ivf(ck.get(), cs.get(), a.nq, kp, a.k, o.dev.labels.get(), cosine, out_ids, out_d, st);
        finish(p);
        return;
    }

    if (idx.kind == Kind::Flat) {
        auto& o = static_cast<FlatObj&>(idx);
        if (empty_filter || o.model.idmap.live_count() == 0) {
            fill_empty(r, st);
            return;
        }
        ensure_device(o, st);
        Prepared p;
        prepare(idx, r, p, st);
        DevBuf<uint64_t> ck(r.nq * r.k, st);
        DevBuf<uint32_t> cs(r.nq * r.k, st);
        flat_candidates(p.q.get(), r.nq, o.dev.rows.get(), o.model.idmap.slots(), dim, ip, r.k, p.filter.get(),
                        r.filter ? nullptr : o.dev.deleted.get(), ck.get(), cs.get(), st);
        k_finalize_flat<<<static_cast<unsigned>(ceil_div(r.nq * r.k, 256)), 256, 0, st>>>(
            p.q.get(), dim, o.dev.rows.get(), cs.get(), static_cast<int>(r.k), ip, o.dev.labels.get(), cosine, out_ids,
            out_d, r.nq);
        QG_LAUNCH_CHECK();
        finish(p);
        return;
    }

    // RefineIndex
    auto& o = static_cast<RefineObj&>(idx);
    const size_t live = r.filter ? r.filter->count : o.map.live_count();
    if (empty_filter || o.map.live_count() == 0) {
        fill_empty(r, st);
        return;
    }
    ensure_device(o, st);
    // narrow filters through an IVF base: exact scores of the allowed rows
    // (RefineIndex::use_direct / direct_scan, reference src/refine_index.cpp:59-82)
    const bool direct =
        r.filter && o.base->kind == Kind::IVF && r.filter->count <= 6 * static_cast<IVFObj&>(*o.base).model.nlist;
    Prepared p;
    prepare(idx, r, p, st, !direct);   // (the direct scan lists the allowed slots on the host)
    if (direct) {
        refine_direct(o, p, r, dim, ip, cosine, out_ids, out_d, st);
        finish(p);
        return;
    }
    const size_t kp = std::min(r.k * o.k_factor, live);
    require(kp <= 3072, "k * k_factor above 3072 is not supported by the GPU path", kUnsupported);
    DevBuf<uint64_t> ck(r.nq * kp, st);
    DevBuf<uint32_t> cs(r.nq * kp, st);
    if (o.base->kind == Kind::IVF) {
        auto& b = static_cast<IVFObj&>(*o.base);
        DevBuf<float> qrot;
        IvfSearchArgs a;
        a.q = ivf_queries(b, p, r.nq, qrot, st);
        a.nq = static_cast<int>(r.nq);
        a.k = static_cast<int>(r.k);
        a.kp = static_cast<int>(kp);
        a.nprobe = r.nprobe > 0 ? r.nprobe : static_cast<int>(b.model.nprobe);
        filter_probing(a, b.model, r.filter, p.filter.get(), kp);
        a.capture = r.capture;
        a.sm_count = sm_count_cached();
        a.d_err = p.err;
        ivf_candidates(b.dev.view, a, ck.get(), cs.get(), st);
    } else {
        auto& b = static_cast<FlatObj&>(*o.base);
        flat_candidates(p.q.get(), r.nq, b.dev.rows.get(), b.model.idmap.slots(), dim, ip, kp, p.filter.get(),
                        r.filter ? nullptr : b.dev.deleted.get(), ck.get(), cs.get(), st);
    }
    refine_candidates(p.q.get(), static_cast<int>(r.nq), dim, o.dev.ptr(), ck.get(), cs.get(), static_cast<int>(kp),
                      static_cast<int>(r.k), ip, o.dev.labels.get(), cosine, out_ids, out_d, st);
    finish(p);
}

// ---------------------------------------------------------------------------
// Sharded search: candidates from this device's lists, merge, finish
// ---------------------------------------------------------------------------
static IVFObj& ivf_of(IndexObj& idx) {
    IndexObj* b = idx.kind == Kind::Refine ? static_cast<RefineObj&>(idx).base.get() : &idx;
    require(b->kind == Kind::IVF, "the sharded search serves IVF indexes and RefineIndexes over them", kUnsupported);
    return static_cast<IVFObj&>(*b);
}

size_t candidate_count(IndexObj& idx, size_t k) {
    IVFObj& ivf = ivf_of(idx);
    if (idx.kind != Kind::Refine) return k;
    auto& o = static_cast<RefineObj&>(idx);
    (void)ivf;
    return std::min(k * o.k_factor, o.map.live_count());
}

void search_candidates(IndexObj& idx, const float* q_dev, size_t nq, size_t k, uint64_t* key, uint32_t* slot,
                       cudaStream_t st) {
    if (nq == 0 || k == 0) return;
    IVFObj& b = ivf_of(idx);
    const size_t kp = candidate_count(idx, k);
    require(kp >= 1 && kp <= 3072, "k * k_factor must be in [1, 3072] for the GPU fast-scan", kUnsupported);
    if (idx.kind == Kind::Refine) ensure_device(static_cast<RefineObj&>(idx), st);
    else ensure_device(b, st);
    SearchRequest r;
    r.q = q_dev;
    r.nq = nq;
    r.k = k;
    r.io = IoSpace::Device;
    Prepared p;
    prepare(idx, r, p, st);
    DevBuf<float> qrot;
    IvfSearchArgs a;
    a.q = ivf_queries(b, p, nq, qrot, st);
    a.nq = static_cast<int>(nq);
    a.k = static_cast<int>(k);
    a.kp = static_cast<int>(kp);
    a.nprobe = static_cast<int>(b.model.nprobe);
    a.sm_count = sm_count_cached();
    a.d_err = p.err;
    ivf_candidates(b.dev.view, a, key, slot, st);
    check_err(p.err, st);
}

void finish_candidates(IndexObj& idx, const float* q_dev, size_t nq, size_t k, const uint64_t* key, const uint32_t* slot,
                       int64_t* out_ids, float* out_d, cudaStream_t st) {
    if (nq == 0 || k == 0) return;
    IVFObj& b = ivf_of(idx);
    const size_t kp = candidate_count(idx, k);
    const bool cosine = idx.metric() == Metric::Cosine, ip = idx.metric() == Metric::InnerProduct;
    if (idx.kind == Kind::Refine) ensure_device(static_cast<RefineObj&>(idx), st);
    else ensure_device(b, st);
    SearchRequest r;
    r.q = q_dev;
    r.nq = nq;
    r.k = k;
    r.io = IoSpace::Device;
    Prepared p;
    prepare(idx, r, p, st);
    if (idx.kind == Kind::Refine) {
        auto& o = static_cast<RefineObj&>(idx);
        refine_candidates(p.q.get(), static_cast<int>(nq), static_cast<int>(idx.dim()), o.dev.ptr(), key, slot,
                          static_cast<int>(kp), static_cast<int>(k), ip, o.dev.labels.get(), cosine, out_ids, out_d, st);
    } else {
        finalize_ivf(key, slot, static_cast<int>(nq), static_cast<int>(kp), static_cast<int>(k), b.dev.labels.get(),
                     cosine, out_ids, out_d, st);
    }
    check_err(p.err, st);
}

// ---------------------------------------------------------------------------
// Device-resident searches replayed as CUDA graphs
// ---------------------------------------------------------------------------
namespace {
std::atomic<int> g_graphs{0};
std::atomic<int64_t> g_graph_replays{0}, g_graph_captures{0};
}

void set_search_graphs(int on) { g_graphs.store(on); }
int search_graphs() { return g_graphs.load(); }
void search_graph_counts(int64_t* replays, int64_t* captures) {
    *replays = g_graph_replays.load();
    *captures = g_graph_captures.load();
}

bool search_graph(IndexObj& idx, const SearchRequest& r, cudaStream_t st) {
    if (!g_graphs.load() || r.io != IoSpace::Device || r.filter || st == nullptr || r.nq == 0 || r.k == 0) return false;
    const bool refine = idx.kind == Kind::Refine;
    IndexObj* base = refine ? static_cast<RefineObj&>(idx).base.get() : &idx;
    if (base->kind != Kind::IVF) return false;
    auto& ivf = static_cast<IVFObj&>(*base);
    if (refine) ensure_device(static_cast<RefineObj&>(idx), st);
    else ensure_device(ivf, st);
    if (ivf.model.idmap.live_count() == 0 || (refine && static_cast<RefineObj&>(idx).map.live_count() == 0)) return false;
    const int nprobe = r.nprobe > 0 ? r.nprobe : static_cast<int>(ivf.model.nprobe);
    const size_t kf = refine ? static_cast<RefineObj&>(idx).k_factor : 0;
    const uint64_t gen = idx.dev_gen * 1000003u + (refine ? ivf.dev_gen : 0);
    std::lock_guard<std::mutex> g(idx.graph_mu);
    SearchGraph* e = nullptr;
    for (auto it = idx.graphs.begin(); it != idx.graphs.end();) {
        SearchGraph& x = **it;
        if (x.nq == r.nq && x.k == r.k && x.nprobe == nprobe && x.k_factor == kf && x.q == r.q && x.ids == r.out_ids &&
            x.d == r.out_d && x.st == st) {
            if (x.gen != gen) {   // the index was rebuilt since the capture
                it = idx.graphs.erase(it);
                continue;
            }
            e = &x;
        }
        ++it;
    }
    if (e) {
        if (e->failed) return false;
        QG_CUDA(cudaGraphLaunch(e->exec, st));
        profiler().launches.fetch_add(e->launches, std::memory_order_relaxed);
        g_graph_replays += 1;
        int h[3] = {0, 0, 0};
        QG_CUDA(cudaMemcpyAsync(h, e->err, sizeof(h), cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        if (h[1]) throw Error(kInvalidArgument, "cosine metric needs non-zero vectors");
        if (h[0]) throw Error(kRuntimeError, "fast-scan candidate buffer overflowed (internal error)");
        if (h[2]) throw Error(kRuntimeError, "tensor-core coarse step: a pipeline wait timed out");
        return true;
    }
    // first call with this key: the search itself (results, tuning, one-time setup), then its capture
    search(idx, r, st);
    auto ent = std::make_unique<SearchGraph>();
    ent->nq = r.nq;
    ent->k = r.k;
    ent->k_factor = kf;
    ent->nprobe = nprobe;
    ent->q = r.q;
    ent->ids = r.out_ids;
    ent->d = r.out_d;
    ent->st = st;
    ent->gen = gen;
    QG_CUDA(cudaMalloc(reinterpret_cast<void**>(&ent->err), 3 * sizeof(int)));
    SearchRequest rc = r;
    rc.capture = true;
    rc.err_dev = ent->err;
    const int64_t launches0 = profiler().launches.load();
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        try {
            search(idx, rc, st);
        } catch (...) {
            ok = false;
        }
        ok = cudaStreamEndCapture(st, &graph) == cudaSuccess && ok && graph != nullptr;
    }
    if (ok) ok = cudaGraphInstantiate(&ent->exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    // captured launches did not run: they count once per replay instead
    const int64_t captured = profiler().launches.load() - launches0;
    profiler().launches.fetch_sub(captured, std::memory_order_relaxed);
    if (!ok) {
        (void)cudaGetLastError();   // a capture that failed leaves no sticky error; this key runs uncaptured
        ent->failed = true;
    } else {
        ent->launches = captured;
        g_graph_captures += 1;
    }
    idx.graphs.push_back(std::move(ent));
    return true;
}

// ---------------------------------------------------------------------------
// Mixed batches (served requests with their own k, nprobe and filter)
// ---------------------------------------------------------------------------
void search_mixed(IndexObj& idx, const float* q, size_t nq, const MixedQuery* qs, size_t kmax, int64_t* out_ids,
                  float* out_d, cudaStream_t st, cudaStream_t st2) {
    require_unsharded(idx);
    std::fill(out_ids, out_ids + nq * kmax, int64_t{-1});
    std::fill(out_d, out_d + nq * kmax, std::numeric_limits<float>::infinity());
    if (nq == 0 || kmax == 0) return;
    const size_t dim = idx.dim();
    for (size_t i = 0; i < nq; ++i) require(qs[i].k >= 1 && static_cast<size_t>(qs[i].k) <= kmax, "k out of range");

    // one request on its own (indexes without an IVF, and RefineIndex direct scans)
    std::vector<int64_t> one_ids(kmax);
    std::vector<float> one_d(kmax);
    auto alone = [&](size_t i) {
        SearchRequest r;
        r.q = q + i * dim;
        r.nq = 1;
        r.k = static_cast<size_t>(qs[i].k);
        r.filter = qs[i].filter;
        r.out_ids = one_ids.data();
        r.out_d = one_d.data();
        r.nprobe = qs[i].nprobe;
        search(idx, r, st);
        std::copy_n(one_ids.data(), r.k, out_ids + i * kmax);
        std::copy_n(one_d.data(), r.k, out_d + i * kmax);
    };
    IVFObj* ivf = nullptr;
    RefineObj* ref = nullptr;
    if (idx.kind == Kind::IVF) {
        ivf = static_cast<IVFObj*>(&idx);
    } else if (idx.kind == Kind::Refine && static_cast<RefineObj&>(idx).base->kind == Kind::IVF) {
        ref = static_cast<RefineObj*>(&idx);
        ivf = static_cast<IVFObj*>(ref->base.get());
    }
    if (!ivf) {
        for (size_t i = 0; i < nq; ++i) alone(i);
        return;
    }
    const IVFModel& M = ivf->model;
    const size_t live = idx.idmap().live_count();
    std::vector<size_t> batch;
    // narrow filters of a RefineIndex (RefineIndex::use_direct): exact scans of
    // the allowed rows, one per (filter, k) among the batch's requests
    std::vector<std::pair<std::pair<const SlotBits*, int>, std::vector<size_t>>> direct;
    std::vector<const uint32_t*> direct_slots;   // each group's filter's device slot list, or null
    for (size_t i = 0; i < nq; ++i) {
        const SlotBits* f = qs[i].filter;
        if (live == 0 || (f && f->count == 0)) continue;                      // nothing to return
        if (ref && f && f->count <= 6 * M.nlist) {
            const auto key = std::make_pair(f, qs[i].k);
            auto it = std::find_if(direct.begin(), direct.end(), [&](const auto& g) { return g.first == key; });
            if (it == direct.end()) {
                direct.push_back({key, {i}});
                direct_slots.push_back(qs[i].filter_slots_dev);
            } else {
                it->second.push_back(i);
            }
            continue;
        }
        batch.push_back(i);
    }
    for (size_t gi = 0; gi < direct.size(); ++gi) {
        const auto& g = direct[gi];
        const size_t n = g.second.size(), k = static_cast<size_t>(g.first.second);
        std::vector<float> qh(n * dim);
        for (size_t j = 0; j < n; ++j) std::copy_n(q + g.second[j] * dim, dim, qh.data() + j * dim);
        std::vector<int64_t> hi(n * k);
        std::vector<float> hd(n * k);
        SearchRequest r;
        r.q = qh.data();
        r.nq = n;
        r.k = k;
        r.filter = g.first.first;
        r.filter_slots_dev = direct_slots[gi];
        r.out_ids = hi.data();
        r.out_d = hd.data();
        search(idx, r, st);
        for (size_t j = 0; j < n; ++j) {
            std::copy_n(hi.data() + j * k, k, out_ids + g.second[j] * kmax);
            std::copy_n(hd.data() + j * k, k, out_d + g.second[j] * kmax);
        }
    }
    if (batch.empty()) return;
    if (ref) ensure_device(*ref, st);
    ensure_device(*ivf, st);
    auto kp_of = [&](size_t i) {
        const MixedQuery& m = qs[i];
        const size_t lv = m.filter ? m.filter->count : live;
        return ref ? std::min(static_cast<size_t>(m.k) * ref->k_factor, lv) : static_cast<size_t>(m.k);
    };
    // One batched search per class of k' (up to 256, above): a few requests
    // with a large k' would otherwise size every query's candidate lists and
    // scan trims by theirs.
    auto run = [&](const std::vector<size_t>& batch, cudaStream_t st) {
        const size_t nb = batch.size();
        size_t kmax_g = 1;
        for (size_t i : batch) kmax_g = std::max(kmax_g, static_cast<size_t>(qs[i].k));
        std::vector<float> qh(nb * dim);
        for (size_t j = 0; j < nb; ++j) std::copy_n(q + batch[j] * dim, dim, qh.data() + j * dim);
        SearchRequest pr;
        pr.q = qh.data();
        pr.nq = nb;
        Prepared p;
        prepare(idx, pr, p, st);

        // per-query settings, and each distinct filter uploaded once
        enum { kK, kKp, kNprobe, kMin, kWanted, kFields };
        std::vector<int> h(kFields * nb);
        std::vector<const SlotBits*> distinct;
        std::vector<size_t> which(nb, SIZE_MAX);
        int npmax = 1, kpmax = 1, depth = 1;
        bool any_filter = false, deep = false;
        for (size_t j = 0; j < nb; ++j) {
            const MixedQuery& m = qs[batch[j]];
            const size_t np = std::min<size_t>(m.nprobe > 0 ? static_cast<size_t>(m.nprobe) : M.nprobe, M.nlist);
            const size_t lv = m.filter ? m.filter->count : live;
            const size_t kp = ref ? std::min(static_cast<size_t>(m.k) * ref->k_factor, lv) : static_cast<size_t>(m.k);
            h[kK * nb + j] = m.k;
            h[kKp * nb + j] = static_cast<int>(kp);
            h[kNprobe * nb + j] = static_cast<int>(np);
            if (m.filter) {
                any_filter = true;
                h[kMin * nb + j] = static_cast<int>(min_probes_for(M, np, m.filter->count));
                h[kWanted * nb + j] = static_cast<int>(std::min(kp, m.filter->count));
                const int dj = rank_depth_for(M, static_cast<size_t>(h[kMin * nb + j]),
                                              static_cast<size_t>(h[kWanted * nb + j]), m.filter->count);
                deep = deep || dj == 0;
                depth = std::max(depth, dj);
                if (!m.filter_dev) {   // (registered filters are on the device already)
                    auto it = std::find(distinct.begin(), distinct.end(), m.filter);
                    which[j] = static_cast<size_t>(it - distinct.begin());
                    if (it == distinct.end()) distinct.push_back(m.filter);
                }
            }
            npmax = std::max(npmax, static_cast<int>(np));
            kpmax = std::max(kpmax, static_cast<int>(kp));
        }
        require(kpmax <= 3072, "k * k_factor above 3072 is not supported by the GPU path", kUnsupported);
        DevBuf<int> dh(h.size(), st);
        QG_CUDA(cudaMemcpyAsync(dh.get(), h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        DevBuf<uint64_t> fwords;
        DevBuf<const uint64_t*> fptr;
        if (any_filter) {
            const size_t words = (idx.idmap().slots() + 63) / 64;
            for (size_t j = 0; j < nb; ++j)   // (a filter registered before the index grew no longer covers it)
                if (const SlotBits* f = qs[batch[j]].filter)
                    require(f->words.size() == words, "a filter does not cover the index's slots");
            if (!distinct.empty()) fwords.alloc(words * distinct.size(), st);
            for (size_t d = 0; d < distinct.size(); ++d)
                QG_CUDA(cudaMemcpyAsync(fwords.get() + d * words, distinct[d]->words.data(), words * 8,
                                        cudaMemcpyHostToDevice, st));
            std::vector<const uint64_t*> ptr(nb, nullptr);
            for (size_t j = 0; j < nb; ++j) {
                if (which[j] != SIZE_MAX) ptr[j] = fwords.get() + which[j] * words;
                else if (qs[batch[j]].filter) ptr[j] = qs[batch[j]].filter_dev;
            }
            fptr.alloc(nb, st);
            QG_CUDA(cudaMemcpyAsync(fptr.get(), ptr.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, st));
        }
        DevBuf<float> qrot;
        IvfSearchArgs a;
        a.q = ivf_queries(*ivf, p, nb, qrot, st);
        a.nq = static_cast<int>(nb);
        a.k = static_cast<int>(kmax_g);
        a.kp = kpmax;
        a.nprobe = npmax;
        a.pq.k = dh.get() + kK * nb;
        a.pq.kp = dh.get() + kKp * nb;
        a.pq.nprobe = dh.get() + kNprobe * nb;
        a.pq.filter = any_filter ? fptr.get() : nullptr;
        a.pq.min_probes = dh.get() + kMin * nb;
        a.pq.wanted = dh.get() + kWanted * nb;
        a.any_filter = any_filter;
        a.rank_depth = deep ? 0 : std::max(depth, npmax);
        a.sm_count = sm_count_cached();
        a.d_err = p.err;
        DevBuf<uint64_t> ck(nb * kpmax, st);
        DevBuf<uint32_t> cs(nb * kpmax, st);
        ivf_candidates(ivf->dev.view, a, ck.get(), cs.get(), st);
        DevBuf<int64_t> oid(nb * kmax_g, st);
        DevBuf<float> od(nb * kmax_g, st);
        const bool cosine = idx.metric() == Metric::Cosine, ip = idx.metric() == Metric::InnerProduct;
        if (ref)
            refine_candidates(p.q.get(), static_cast<int>(nb), static_cast<int>(dim), ref->dev.ptr(), ck.get(), cs.get(),
                              kpmax, static_cast<int>(kmax_g), ip, ref->dev.labels.get(), cosine, oid.get(), od.get(), st,
                              a.pq.kp, a.pq.k);
        else
            finalize_ivf(ck.get(), cs.get(), static_cast<int>(nb), kpmax, static_cast<int>(kmax_g), ivf->dev.labels.get(), cosine,
                         oid.get(), od.get(), st, a.pq.k);
        std::vector<int64_t> hid(nb * kmax_g);
        std::vector<float> hd(nb * kmax_g);
        QG_CUDA(cudaMemcpyAsync(hid.data(), oid.get(), hid.size() * 8, cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaMemcpyAsync(hd.data(), od.get(), hd.size() * 4, cudaMemcpyDeviceToHost, st));
        check_err(p.err, st);
        for (size_t j = 0; j < nb; ++j) {
            std::copy_n(hid.data() + j * kmax_g, kmax_g, out_ids + batch[j] * kmax);
            std::copy_n(hd.data() + j * kmax_g, kmax_g, out_d + batch[j] * kmax);
        }
    };
    std::vector<size_t> small, large;
    for (size_t i : batch) (kp_of(i) <= 256 ? small : large).push_back(i);
    if (st2 && !small.empty() && !large.empty()) {
        // both classes at once: the larger k' on st2 from a second thread (the
        // two write disjoint requests' results); its error, if any, rethrown here
        // st2 starts after what st holds so far (device copies of the index)
        cudaEvent_t ready;
        QG_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        QG_CUDA(cudaEventRecord(ready, st));
        QG_CUDA(cudaStreamWaitEvent(st2, ready, 0));
        QG_CUDA(cudaEventDestroy(ready));
        std::exception_ptr err2;
        std::thread t2([&] {
            try {
                QG_CUDA(cudaSetDevice(idx.device));
                run(large, st2);
            } catch (...) {
                err2 = std::current_exception();
            }
        });
        try {
            run(small, st);
        } catch (...) {
            t2.join();
            throw;
        }
        t2.join();
        if (err2) std::rethrow_exception(err2);
        return;
    }
    if (!small.empty()) run(small, st);
    if (!large.empty()) run(large, st);
}

} // namespace qg
