// Adding vectors (assignment, residual PQ encoding, list append) and
// compaction. The arithmetic that decides list membership and codes runs on
// the GPU and matches the reference's no-BLAS build exactly: nearest centroid
// by the AVX2-order squared L2 with the first index winning ties (reference
// src/kmeans.cpp:102-115), and the AVX2+FMA 16-centroid encoder (reference
// src/pq.cpp:88-116).
#include "qg_device.cuh"
#include "qg_ops.h"
#include "qg_train.h"

#include <algorithm>
#include <numeric>

namespace qg {

// Warp per row: the column with the smallest key, first column on ties.
__global__ void k_row_argmin(const float* __restrict__ scores, size_t ld, int nrows, int ncols, uint32_t* __restrict__ out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nrows) return;
    const float* row = scores + static_cast<size_t>(warp) * ld;
    uint64_t best = ~0ull;
    for (int c = lane; c < ncols; c += 32) {
        const uint64_t k = (static_cast<uint64_t>(float_key(row[c])) << 32) | static_cast<uint32_t>(c);
        best = k < best ? k : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other < best ? other : best;
    }
    if (lane == 0) out[warp] = static_cast<uint32_t>(best);
}

void assign_nearest(const float* x_dev, size_t n, const float* c_dev, size_t k, int dim, uint32_t* out_dev,
                    cudaStream_t st) {
    if (n == 0) return;
    if (use_tensor_filter(n, k, dim, 1)) {
        // the smallest (score, centroid): the same first-index-on-ties rule
        DevBuf<uint64_t> key(n, st);
        flat_candidates(x_dev, n, c_dev, k, dim, false, 1, nullptr, nullptr, key.get(), out_dev, st);
        return;
    }
    const size_t T = std::max<size_t>(1, std::min<size_t>(n, (size_t{512} << 20) / (k * sizeof(float))));
    DevBuf<float> scores(T * k, st);
    for (size_t r0 = 0; r0 < n; r0 += T) {
        const size_t nr = std::min(T, n - r0);
        pair_scores(x_dev + r0 * dim, static_cast<int>(nr), c_dev, static_cast<int>(k), dim, false, scores.get(), k, st);
        k_row_argmin<<<static_cast<unsigned>(ceil_div(nr * 32, 256)), 256, 0, st>>>(scores.get(), k, static_cast<int>(nr),
                                                                                    static_cast<int>(k), out_dev + r0);
        QG_LAUNCH_CHECK();
    }
}

// PQ codes of residuals x - center[assign], K = 16, thread per (row, subspace):
// lo/hi halves start with a rounded product, then FMA over the remaining
// sub-dimensions; the code is the first index of the minimum.
__global__ void k_encode16(const float* __restrict__ x, size_t n, int dim, const float* __restrict__ centers,
                           const uint32_t* __restrict__ assign, const float* __restrict__ yt, int m, int sd,
                           uint8_t* __restrict__ codes) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * m) return;
    const size_t i = t / m;
    const int s = static_cast<int>(t % m);
    const float* xr = x + i * dim + s * sd;
    const float* cr = centers + static_cast<size_t>(assign[i]) * dim + s * sd;
    float acc[16];
    {
        const float q = __fsub_rn(xr[0], cr[0]);
        const float* y = yt + static_cast<size_t>(s * sd) * 16;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float d = __fsub_rn(q, y[k]);
            acc[k] = __fmul_rn(d, d);
        }
    }
    for (int j = 1; j < sd; ++j) {
        const float q = __fsub_rn(xr[j], cr[j]);
        const float* y = yt + static_cast<size_t>(s * sd + j) * 16;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float d = __fsub_rn(q, y[k]);
            acc[k] = __fmaf_rn(d, d, acc[k]);
        }
    }
    float mn = acc[0];
#pragma unroll
    for (int k = 1; k < 16; ++k) mn = fminf(mn, acc[k]);
    int best = 0;
#pragma unroll
    for (int k = 15; k >= 0; --k)
        if (acc[k] == mn) best = k;
    codes[t] = static_cast<uint8_t>(best);
}

void encode16(const float* x, size_t n, int dim, const float* centers, const uint32_t* assign, const float* yt, int m,
              int sd, uint8_t* codes, cudaStream_t st) {
    if (n == 0) return;
    k_encode16<<<static_cast<unsigned>(ceil_div(n * m, 256)), 256, 0, st>>>(x, n, dim, centers, assign, yt, m, sd, codes);
    QG_LAUNCH_CHECK();
}

// Rows prepared for the metric: cosine rows scaled to unit length on the GPU
// (reference src/index.cpp:193-218); a zero row refuses the whole call.
static std::vector<float> prepare_rows(Metric metric, const float* x, size_t n, size_t dim, DevBuf<float>& dev,
                                       cudaStream_t st) {
    DevBuf<float> raw(n * dim, st);
    QG_CUDA(cudaMemcpyAsync(raw.get(), x, n * dim * 4, cudaMemcpyHostToDevice, st));
    std::vector<float> out(n * dim);
    if (metric == Metric::Cosine) {
        dev.alloc(n * dim, st);
        DevBuf<int> zero(1, st);
        QG_CUDA(cudaMemsetAsync(zero.get(), 0, 4, st));
        normalize_rows(raw.get(), dev.get(), static_cast<int>(n), static_cast<int>(dim), zero.get(), st);
        int z = 0;
        QG_CUDA(cudaMemcpyAsync(&z, zero.get(), 4, cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaMemcpyAsync(out.data(), dev.get(), n * dim * 4, cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
        if (z) throw Error(kInvalidArgument, "cosine metric needs non-zero vectors");
    } else {
        dev = std::move(raw);
        std::copy(x, x + n * dim, out.begin());
    }
    return out;
}

// IVFIndex::add_batch_impl on prepared rows (reference src/ivf_index.cpp:111-195).
static void ivf_add_impl(IVFObj& o, const float* x_dev, size_t n, const int64_t* ids, cudaStream_t st) {
    IVFModel& M = o.model;
    if (!M.trained) throw Error(kLogicError, "train() has not be run yet");
    require(M.has_pq && M.fast_scan, "the GPU build adds to IVF indexes with fast-scan PQ", kUnsupported);
    M.idmap.check(n, ids);
    const uint32_t first = static_cast<uint32_t>(M.idmap.slots());
    const int dim = static_cast<int>(M.dim), m = static_cast<int>(M.pq.m), sd = static_cast<int>(M.pq.sub_dim);
    std::vector<uint32_t> assign(n);
    std::vector<uint8_t> codes(n * m);
    if (n) {
        DevBuf<float> cent(M.centroids.size(), st);
        QG_CUDA(cudaMemcpyAsync(cent.get(), M.centroids.data(), cent.bytes(), cudaMemcpyHostToDevice, st));
        DevBuf<float> resid;
        const float* centers = cent.get();
        if (!M.residual_centers.empty()) {
            resid.alloc(M.residual_centers.size(), st);
            QG_CUDA(cudaMemcpyAsync(resid.get(), M.residual_centers.data(), resid.bytes(), cudaMemcpyHostToDevice, st));
            centers = resid.get();
        }
        const std::vector<float> yt = M.pq.transposed();
        DevBuf<float> dyt(yt.size(), st);
        QG_CUDA(cudaMemcpyAsync(dyt.get(), yt.data(), dyt.bytes(), cudaMemcpyHostToDevice, st));
        // a rotating index assigns and encodes the rotated rows (reference src/ivf_index.cpp:111-120)
        DevBuf<float> xr;
        if (M.rotate) {
            DevBuf<float> R(M.rotation.size(), st);
            QG_CUDA(cudaMemcpyAsync(R.get(), M.rotation.data(), R.bytes(), cudaMemcpyHostToDevice, st));
            xr.alloc(n * dim, st);
            rotate_rows(R.get(), x_dev, n, dim, xr.get(), st);
            x_dev = xr.get();
        }
        DevBuf<uint32_t> da(n, st);
        assign_nearest(x_dev, n, cent.get(), M.nlist, dim, da.get(), st);
        DevBuf<uint8_t> dc(n * m, st);
        k_encode16<<<static_cast<unsigned>(ceil_div(n * m, 256)), 256, 0, st>>>(x_dev, n, dim, centers, da.get(), dyt.get(),
                                                                                 m, sd, dc.get());
        QG_LAUNCH_CHECK();
        QG_CUDA(cudaMemcpyAsync(assign.data(), da.get(), n * 4, cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaMemcpyAsync(codes.data(), dc.get(), n * m, cudaMemcpyDeviceToHost, st));
        QG_CUDA(cudaStreamSynchronize(st));
    }
    M.idmap.add(n, ids);
    // append in input order within each list
    for (size_t i = 0; i < n; ++i) {
        const uint32_t l = assign[i];
        M.list_ids[l].push_back(first + static_cast<uint32_t>(i));
        M.list_codes[l].insert(M.list_codes[l].end(), codes.begin() + i * m, codes.begin() + (i + 1) * m);
    }
    o.dev_dirty = true;
}

void validate_add(const IndexObj& idx, size_t n, const int64_t* ids) {
    if (idx.kind == Kind::IVF) {
        const auto& o = static_cast<const IVFObj&>(idx);
        if (!o.model.trained) throw Error(kLogicError, "train() has not be run yet");
        o.model.idmap.check(n, ids);
    } else if (idx.kind == Kind::Flat) {
        static_cast<const FlatObj&>(idx).model.idmap.check(n, ids);
    } else {
        const auto& o = static_cast<const RefineObj&>(idx);
        o.map.check(n, ids);
        if (o.base->kind == Kind::IVF && !static_cast<const IVFObj&>(*o.base).model.trained)
            throw Error(kLogicError, "train() has not be run yet");
    }
}

void add(IndexObj& idx, const float* x, size_t n, const int64_t* ids, int64_t* out_ids, cudaStream_t st) {
    const size_t dim = idx.dim();
    const size_t first = idx.idmap().slots();
    if (idx.kind == Kind::IVF) {
        auto& o = static_cast<IVFObj&>(idx);
        if (!o.model.trained) throw Error(kLogicError, "train() has not be run yet");
        o.model.idmap.check(n, ids);
        DevBuf<float> dev;
        prepare_rows(o.model.metric, x, n, dim, dev, st);
        ivf_add_impl(o, dev.get(), n, ids, st);
    } else if (idx.kind == Kind::Flat) {
        auto& o = static_cast<FlatObj&>(idx);
        o.model.idmap.check(n, ids);
        DevBuf<float> dev;
        std::vector<float> rows = prepare_rows(o.model.metric, x, n, dim, dev, st);
        o.model.idmap.add(n, ids);
        o.model.data.insert(o.model.data.end(), rows.begin(), rows.end());
        o.dev_dirty = true;
    } else {
        auto& o = static_cast<RefineObj&>(idx);
        o.map.check(n, ids);
        o.materialize();   // rows of a mapped file move to memory before they change
        DevBuf<float> dev;
        std::vector<float> rows = prepare_rows(o.metric(), x, n, dim, dev, st);
        if (o.base->kind == Kind::IVF) {
            ivf_add_impl(static_cast<IVFObj&>(*o.base), dev.get(), n, nullptr, st);
        } else {
            auto& b = static_cast<FlatObj&>(*o.base);
            b.model.idmap.add(n, nullptr);
            b.model.data.insert(b.model.data.end(), rows.begin(), rows.end());
            b.dev_dirty = true;
        }
        o.map.add(n, ids);
        o.data.insert(o.data.end(), rows.begin(), rows.end());
        o.dev_dirty = true;
    }
    if (out_ids)
        for (size_t i = 0; i < n; ++i) out_ids[i] = idx.idmap().label(static_cast<uint32_t>(first + i));
}

// ---- compaction (reference src/ivf_index.cpp:656-720, src/flat_index.cpp:69-99,
// src/refine_index.cpp:147-160) ---------------------------------------------------

static void compact_rows(std::vector<float>& data, const std::vector<uint32_t>& remap, size_t dim, size_t live) {
    for (size_t s = 0; s < remap.size(); ++s)
        if (remap[s] != kRemoved && remap[s] != s)
            std::copy_n(data.data() + s * dim, dim, data.data() + static_cast<size_t>(remap[s]) * dim);
    data.resize(live * dim);
}

static void compact_ivf_storage(IVFModel& M, const std::vector<uint32_t>& remap) {
    const size_t m = M.m();
    for (size_t l = 0; l < M.nlist; ++l) {
        auto& ids = M.list_ids[l];
        auto& codes = M.list_codes[l];
        size_t w = 0;
        for (size_t j = 0; j < ids.size(); ++j) {
            const uint32_t ns = remap[ids[j]];
            if (ns == kRemoved) continue;
            ids[w] = ns;
            if (w != j) std::copy_n(codes.data() + j * m, m, codes.data() + w * m);
            ++w;
        }
        ids.resize(w);
        codes.resize(w * m);
    }
}

static size_t compact_obj(IndexObj& idx, bool keep_ids) {
    if (idx.kind == Kind::Flat) {
        auto& o = static_cast<FlatObj&>(idx);
        if (o.model.idmap.deleted_count() && !o.model.meta.empty())
            throw Error(kUnsupported, "compacting an index with metadata columns is not supported by this library");
        auto remap = o.model.idmap.compact(keep_ids);
        if (remap.empty()) return 0;
        compact_rows(o.model.data, remap, o.model.dim, o.model.idmap.slots());
        o.dev_dirty = true;
        return remap.size() - o.model.idmap.slots();
    }
    if (idx.kind == Kind::IVF) {
        auto& o = static_cast<IVFObj&>(idx);
        if (o.model.idmap.deleted_count() && !o.model.meta.empty())
            throw Error(kUnsupported, "compacting an index with metadata columns is not supported by this library");
        auto remap = o.model.idmap.compact(keep_ids);
        if (remap.empty()) return 0;
        compact_ivf_storage(o.model, remap);
        o.dev_dirty = true;
        return remap.size() - o.model.idmap.slots();
    }
    auto& o = static_cast<RefineObj&>(idx);
    if (o.map.deleted_count() && !o.meta.empty())
        throw Error(kUnsupported, "compacting an index with metadata columns is not supported by this library");
    if (o.map.deleted_count()) o.materialize();   // (before the slot count changes)
    auto remap = o.map.compact(keep_ids);
    if (remap.empty()) return 0;
    {
        std::unique_lock<std::shared_mutex> lb(o.base->mu);
        compact_obj(*o.base, false);
    }
    compact_rows(o.data, remap, o.dim(), o.map.slots());
    o.dev_dirty = true;
    return remap.size() - o.map.slots();
}

void compact(IndexObj& idx, size_t* reclaimed) {
    if (idx.wrapped)
        throw Error(kInvalidArgument, "cannot compact on an index wrapped by a RefineIndex or HybridIndex; compact "
                                      "through the wrapper instead");
    *reclaimed = compact_obj(idx, true);
}

} // namespace qg
