// Device copies of the indexes and the search entry points.
#include "qg_device.cuh"
#include "qg_index.h"
#include "qg_ops.h"

#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>

#include <fcntl.h>
#include <sys/mman.h>
#include <unistd.h>

namespace qg {

// ---------------------------------------------------------------------------
// Superblock packing (layout: qg_device.cuh, kSuperBlock). One thread per
// (superblock, octet lane): builds the lane's m words from 8 vectors' codes.
// ---------------------------------------------------------------------------
__global__ void k_pack_codes(const uint8_t* __restrict__ codes, const uint32_t* __restrict__ voff,
                             const uint32_t* __restrict__ sb_off, const uint32_t* __restrict__ list_size,
                             const uint32_t* __restrict__ sb_list, size_t total_sb, int m, int m_pad,
                             uint32_t* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= total_sb * 8) return;
    const size_t sb = t >> 3;
    const int r = static_cast<int>(t & 7);
    const uint32_t l = sb_list[sb];
    const uint32_t sbl = static_cast<uint32_t>(sb - sb_off[l]);
    const uint32_t size = list_size[l];
    uint32_t* o = out + sb * static_cast<size_t>(8 * m_pad);
    for (int s = 0; s < m_pad; ++s) {
        uint32_t w = 0;
        if (s < m) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t pos = sbl * kSuperBlock + 8 * r + i;
                if (pos < size) w |= static_cast<uint32_t>(codes[(static_cast<size_t>(voff[l]) + pos) * m + s] & 15) << (4 * i);
            }
        }
        o[((s >> 2) * 8 + r) * 4 + (s & 3)] = w;
    }
}

__global__ void k_pack_ids(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ voff,
                           const uint32_t* __restrict__ sb_off, const uint32_t* __restrict__ list_size,
                           const uint32_t* __restrict__ sb_list, size_t total_sb, uint32_t* __restrict__ out) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= total_sb * kSuperBlock) return;
    const size_t sb = t / kSuperBlock;
    const uint32_t pos_in_sb = static_cast<uint32_t>(t % kSuperBlock);
    const uint32_t l = sb_list[sb];
    const uint32_t pos = static_cast<uint32_t>(sb - sb_off[l]) * kSuperBlock + pos_in_sb;
    out[t] = pos < list_size[l] ? ids[voff[l] + pos] : kRemoved;
}

void pack_superblocks(const uint8_t* codes_dev, const uint32_t* ids_dev, const uint32_t* voff_dev,
                      const uint32_t* sb_off_dev, const uint32_t* list_size_dev, const uint32_t* sb_list_dev,
                      size_t total_sb, int m, int m_pad, uint4* out_codes, uint32_t* out_ids, cudaStream_t st) {
    if (total_sb == 0) return;
    k_pack_codes<<<static_cast<unsigned>(ceil_div(total_sb * 8, 256)), 256, 0, st>>>(
        codes_dev, voff_dev, sb_off_dev, list_size_dev, sb_list_dev, total_sb, m, m_pad,
        reinterpret_cast<uint32_t*>(out_codes));
    QG_LAUNCH_CHECK();
    if (out_ids) {
        k_pack_ids<<<static_cast<unsigned>(ceil_div(total_sb * kSuperBlock, 256)), 256, 0, st>>>(
            ids_dev, voff_dev, sb_off_dev, list_size_dev, sb_list_dev, total_sb, out_ids);
        QG_LAUNCH_CHECK();
    }
}

// ---------------------------------------------------------------------------
// Per-list tables built once per upload.
// ---------------------------------------------------------------------------
__global__ void k_sqnorms(const float* __restrict__ c, int n, int d, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = c + static_cast<size_t>(i) * d;
    out[i] = exact_avx2<false>(r, r, d);
}

// B[l][s][k] = compute_list_term(center_l) (reference src/pq.cpp:206-223)
__global__ void k_list_terms(const float* __restrict__ centers, int nlist, int dim, const float* __restrict__ pq_t, int m,
                             int sd, float* __restrict__ B) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t per = static_cast<size_t>(m) * 16;
    if (t >= per * nlist) return;
    const size_t l = t / per;
    const int e = static_cast<int>(t % per);
    B[t] = list_term(centers + l * dim, pq_t, e >> 4, sd, 16, e & 15);
}

static std::vector<uint64_t> deleted_words(const IdMap& map) {
    std::vector<uint64_t> w((map.slots() + 63) / 64, 0);
    if (map.deleted_count() == 0) return w;
    const auto& del = map.deleted();
    for (size_t s = 0; s < map.slots(); ++s)
        if (del[s]) w[s >> 6] |= uint64_t{1} << (s & 63);
    return w;
}

template <class T>
static void upload(DevBuf<T>& b, const T* src, size_t n, cudaStream_t st) {
    b.alloc(n, st);
    if (n) QG_CUDA(cudaMemcpyAsync(b.get(), src, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

template <class T>
static void upload(DevBuf<T>& b, const std::vector<T>& v, cudaStream_t st) {
    upload(b, v.data(), v.size(), st);
}

bool IVFObj::precomputed_available() const {
    const IVFModel& m = model;
    if (!m.use_precomputed || !m.trained || !m.has_pq || m.metric == Metric::InnerProduct ||
        (m.metric == Metric::Cosine && m.cosine_ip))
        return false;
    return m.nlist * m.pq.m * m.pq.K * sizeof(float) <= (size_t{256} << 20);
}

int IVFObj::scan_mode() const {
    if (model.metric == Metric::InnerProduct) return kModeIP;
    if (model.metric == Metric::Cosine && model.cosine_ip) return kModeCosIP;
    return precomputed_available() ? kModeL2 : kModeL2Adc;
}

// Index-resident arrays are built (and later freed) on a stream the library
// never destroys: a DevBuf is freed on the stream it was made on, and the
// caller's stream (a server worker's, say) may be gone by the time the index
// is rebuilt or dropped. Builds finish before they return, so the caller's
// stream sees the arrays; they are dropped only when no search is in flight.
cudaStream_t resident_stream() {
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    int dev = 0;
    QG_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, "device ordinal out of range", kCudaError);
    std::lock_guard<std::mutex> g(mu);
    if (!streams[dev]) QG_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
    return streams[dev];
}

void ensure_device(IVFObj& o, cudaStream_t) {
    const cudaStream_t st = resident_stream();
    std::lock_guard<std::mutex> g(o.dev_mu);
    if (!o.dev_dirty) return;
    const IVFModel& M = o.model;
    require(M.trained, "train() has not be run yet", kLogicError);
    require(M.has_pq && M.fast_scan, "the GPU search path serves IVF indexes with fast-scan PQ (enable_pq(m, fast_scan=True))",
            kUnsupported);
    DeviceIVF& D = o.dev;
    D = DeviceIVF{};
    if (M.rotate) upload(D.rot, M.rotation, st);
    const int nlist = static_cast<int>(M.nlist), dim = static_cast<int>(M.dim), m = static_cast<int>(M.pq.m);
    const int m_pad = (m + 3) & ~3;
    upload(D.centroids, M.centroids, st);
    if (!M.residual_centers.empty()) upload(D.resid, M.residual_centers, st);
    const float* centers = M.residual_centers.empty() ? D.centroids.get() : D.resid.get();
    D.sqnorm.alloc(nlist, st);
    k_sqnorms<<<static_cast<unsigned>(ceil_div(nlist, 128)), 128, 0, st>>>(centers, nlist, dim, D.sqnorm.get());
    QG_LAUNCH_CHECK();
    upload(D.pq_t, M.pq.transposed(), st);
    const int mode = o.scan_mode();
    if (mode == kModeL2) {
        const size_t nB = static_cast<size_t>(nlist) * m * 16;
        D.B.alloc(nB, st);
        k_list_terms<<<static_cast<unsigned>(ceil_div(nB, 256)), 256, 0, st>>>(centers, nlist, dim, D.pq_t.get(), m,
                                                                                 static_cast<int>(M.pq.sub_dim), D.B.get());
        QG_LAUNCH_CHECK();
    }
    // lists -> superblocks (a shard keeps only its own lists' codes; the sizes stay global)
    std::vector<uint32_t> sizes(nlist), voff(nlist + 1, 0), sb_off(nlist + 1, 0);
    auto own = [&](int l) { return l % o.shards == o.shard; };
    for (int l = 0; l < nlist; ++l) {
        sizes[l] = static_cast<uint32_t>(M.list_ids[l].size());
        const uint32_t held = own(l) ? sizes[l] : 0;
        voff[l + 1] = voff[l] + held;
        sb_off[l + 1] = sb_off[l] + static_cast<uint32_t>(ceil_div(held, kSuperBlock));
    }
    const size_t n = voff[nlist], total_sb = sb_off[nlist];
    std::vector<uint8_t> codes(n * m);
    std::vector<uint32_t> ids(n);
    std::vector<uint32_t> sb_list(total_sb);
    for (int l = 0; l < nlist; ++l) {
        if (sizes[l] && own(l)) {
            std::memcpy(codes.data() + static_cast<size_t>(voff[l]) * m, M.list_codes[l].data(), static_cast<size_t>(sizes[l]) * m);
            std::memcpy(ids.data() + voff[l], M.list_ids[l].data(), sizes[l] * sizeof(uint32_t));
        }
        for (uint32_t b = sb_off[l]; b < sb_off[l + 1]; ++b) sb_list[b] = static_cast<uint32_t>(l);
    }
    DevBuf<uint8_t> dcodes;
    DevBuf<uint32_t> dids, dvoff, dsbl;
    upload(dcodes, codes, st);
    upload(dids, ids, st);
    upload(dvoff, voff, st);
    upload(dsbl, sb_list, st);
    upload(D.sb_off, sb_off, st);
    upload(D.list_size, sizes, st);
    D.total_sb = total_sb;
    D.codes.alloc(total_sb * 2 * m_pad + kCodePad, st);   // (the scan reads up to kCodePad uint4 past the end)
    D.ids.alloc(std::max<size_t>(1, total_sb * kSuperBlock), st);
    pack_superblocks(dcodes.get(), dids.get(), dvoff.get(), D.sb_off.get(), D.list_size.get(), dsbl.get(), total_sb, m,
                     m_pad, D.codes.get(), D.ids.get(), st);
    if (M.idmap.deleted_count()) upload(D.deleted, deleted_words(M.idmap), st);
    if (!M.idmap.labels().empty()) upload(D.labels, M.idmap.labels(), st);
    QG_CUDA(cudaStreamSynchronize(st));

    IvfView& v = D.view;
    v.dim = dim;
    v.nlist = nlist;
    v.m = m;
    v.m_pad = m_pad;
    v.sd = static_cast<int>(M.pq.sub_dim);
    v.mode = mode;
    v.ip_metric = M.metric == Metric::InnerProduct;
    v.has_resid = !M.residual_centers.empty();
    v.centroids = D.centroids.get();
    v.resid = centers;
    v.sqnorm = D.sqnorm.get();
    v.pq_t = D.pq_t.get();
    v.B = D.B.get();
    v.sb_off = D.sb_off.get();
    v.list_size = D.list_size.get();
    v.codes = D.codes.get();
    v.ids = D.ids.get();
    v.deleted = M.idmap.deleted_count() ? D.deleted.get() : nullptr;
    if (mm_supported(dim)) {
        prepare_f16_rows(D.centroids.get(), nlist, dim, D.cent_f16, D.cent_sq, D.cent_exp, v.cent_dpad, st);
        QG_CUDA(cudaStreamSynchronize(st));
        v.cent_f16 = D.cent_f16.get();
        v.cent_sq = D.cent_sq.get();
        v.cent_exp = D.cent_exp.get();
    }
    o.dev_dirty = false;
    ++o.dev_gen;
}

static void upload_rows(DeviceRows& D, const std::vector<float>& rows, const IdMap& map, cudaStream_t st) {
    D = DeviceRows{};
    upload(D.rows, rows, st);
    if (!map.labels().empty()) upload(D.labels, map.labels(), st);
    if (map.deleted_count()) upload(D.deleted, deleted_words(map), st);
    QG_CUDA(cudaStreamSynchronize(st));
}

void ensure_device(FlatObj& o, cudaStream_t) {
    std::lock_guard<std::mutex> g(o.dev_mu);
    if (!o.dev_dirty) return;
    upload_rows(o.dev, o.model.data, o.model.idmap, resident_stream());
    o.dev_dirty = false;
    ++o.dev_gen;
}

void RefineObj::release_mapping() {
    if (registered) {
        cudaHostUnregister(registered);
        (void)cudaGetLastError();
        registered = nullptr;
    }
    if (priv) {
        ::munmap(priv, priv_len);
        priv = nullptr;
        priv_len = 0;
    }
    dev_src = nullptr;
    dev.ext = nullptr;
    mapped = nullptr;
    file.reset();
}

void RefineObj::materialize() {
    if (!mapped) return;
    data.assign(mapped, mapped + rows_len());
    release_mapping();
    dev_dirty = true;
}

// Mapped rows read in place: the file's pages holding them registered with
// CUDA as mapped host memory, so device loads reach them over the host link.
// First the shared read-only mapping itself (read-only registration); where
// the platform refuses that, a private writable view of the same file pages
// (never written; pinning it copies the pages into host memory, still not
// GPU memory). Returns the device address of the rows, or null when both are
// refused (the rows are then copied into HBM as usual; the refusals are kept
// in g_mapped_rows_error).
static std::atomic<int> g_mapped_rows_error{0};
int mapped_rows_error() { return g_mapped_rows_error.load(); }

static const float* map_rows_for_device(RefineObj& o) {
    const size_t page = static_cast<size_t>(sysconf(_SC_PAGESIZE));
    const uintptr_t b = reinterpret_cast<uintptr_t>(o.mapped) & ~(page - 1);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(o.mapped + o.rows_len()) + page - 1) & ~(page - 1);
    if (e <= b || !o.file) return nullptr;
    if (!o.registered) {
        const cudaError_t e1 = cudaHostRegister(reinterpret_cast<void*>(b), e - b,
                                                cudaHostRegisterMapped | cudaHostRegisterPortable |
                                                    cudaHostRegisterReadOnly);
        if (e1 == cudaSuccess) {
            o.registered = reinterpret_cast<void*>(b);
            o.dev_src = o.mapped;
        } else {
            (void)cudaGetLastError();
            const size_t off = b - reinterpret_cast<uintptr_t>(o.file->data);   // page aligned: the map starts the file
            const int fd = ::open(o.file->path.c_str(), O_RDONLY | O_CLOEXEC);
            void* p = fd >= 0 ? ::mmap(nullptr, e - b, PROT_READ | PROT_WRITE, MAP_PRIVATE, fd, static_cast<off_t>(off))
                              : MAP_FAILED;
            if (fd >= 0) ::close(fd);
            cudaError_t e2 = cudaErrorUnknown;
            if (p != MAP_FAILED) {
                e2 = cudaHostRegister(p, e - b, cudaHostRegisterMapped | cudaHostRegisterPortable);
                if (e2 == cudaSuccess) {
                    o.priv = p;
                    o.priv_len = e - b;
                    o.registered = p;
                    o.dev_src = reinterpret_cast<const float*>(static_cast<char*>(p) +
                                                               (reinterpret_cast<uintptr_t>(o.mapped) - b));
                } else {
                    (void)cudaGetLastError();
                    ::munmap(p, e - b);
                }
            }
            if (!o.registered) {
                g_mapped_rows_error.store(static_cast<int>(e1) * 1000 + static_cast<int>(e2));
                return nullptr;
            }
        }
    }
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, const_cast<float*>(o.dev_src), 0) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return static_cast<const float*>(d);
}

void ensure_device(RefineObj& o, cudaStream_t st) {
    {
        std::lock_guard<std::mutex> g(o.dev_mu);
        if (o.dev_dirty) {
            const float* ext = o.mapped && o.rows_len() ? map_rows_for_device(o) : nullptr;
            if (ext) {
                upload_rows(o.dev, {}, o.map, resident_stream());
                o.dev.ext = ext;
            } else if (o.mapped) {
                upload_rows(o.dev, std::vector<float>(o.mapped, o.mapped + o.rows_len()), o.map, resident_stream());
            } else {
                upload_rows(o.dev, o.data, o.map, resident_stream());
            }
            o.dev_dirty = false;
            ++o.dev_gen;
        }
    }
    if (o.base->kind == Kind::IVF) ensure_device(static_cast<IVFObj&>(*o.base), st);
    else ensure_device(static_cast<FlatObj&>(*o.base), st);
}

} // namespace qg
