// `.qann` reader/writer and the slot<->id map for the host-side models.
//
// Field order per body follows the reference file format (format version
// 13), so files move between qann and this library in both directions:
//   IVF    reference src/ivf_index.cpp:904-974 (save), :976-1122 (load)
//   Refine reference src/refine_index.cpp:158-213
//   Flat   reference src/flat_index.cpp:101-133
//   IdMap  reference src/id_map.cpp:187-241
#include "qg_host.h"
#include "qg_error.h"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <numeric>
#include <unordered_set>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace qg {

[[noreturn]] void Reader::throw_corrupt(const std::string& what) { throw Error(kRuntimeError, "corrupt file: " + what); }

void Reader::need(size_t n) const {
    if (n > size - pos) throw Error(kRuntimeError, "truncated file");
}

void Reader::pad(uint64_t align) {
    const uint32_t n = pod<uint32_t>();
    if (n >= align) throw_corrupt("invalid padding");
    need(n);
    pos += n;
}

// ---- IdMap -----------------------------------------------------------------

void IdMap::check(size_t n, const int64_t* ids) const {
    if (n > UINT32_MAX - slots_) throw Error(kInvalidArgument, "an index holds at most 2^32 - 1 vectors");
    if (custom_ && ids == nullptr) throw Error(kInvalidArgument, "ids are required: this index was created with custom ids");
    if (!custom_ && ids != nullptr)
        throw Error(kInvalidArgument, "ids are not accepted: this index was created without custom ids");
    if (!custom_) return;
    std::unordered_set<int64_t> seen;
    seen.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        const int64_t id = ids[i];
        if (id < 0) throw Error(kInvalidArgument, "ids must be >= 0, got " + std::to_string(id));
        if (!seen.insert(id).second) throw Error(kInvalidArgument, "duplicate id " + std::to_string(id) + " in this batch");
        if (slot_of_.count(id)) throw Error(kInvalidArgument, "id " + std::to_string(id) + " is already in the index");
    }
}

void IdMap::add(size_t n, const int64_t* ids) {
    check(n, ids);
    if (!custom_) {
        if (labels_.empty() && static_cast<size_t>(next_id_) == slots_) {
            slots_ += n;
            next_id_ += static_cast<int64_t>(n);
        } else {
            for (size_t i = 0; i < n; ++i) labels_.push_back(next_id_++);
            slots_ += n;
        }
        deleted_.resize(slots_, 0);
        return;
    }
    for (size_t i = 0; i < n; ++i) {
        labels_.push_back(ids[i]);
        slot_of_[ids[i]] = static_cast<uint32_t>(slots_);
        ++slots_;
    }
    deleted_.resize(slots_, 0);
}

// slot of an id, or -1 when unknown (deleted slots are reported; callers check)
static int64_t find_slot(bool custom, const std::vector<int64_t>& labels,
                         const std::unordered_map<int64_t, uint32_t>& slot_of, size_t slots, int64_t id) {
    if (custom) {
        auto it = slot_of.find(id);
        return it == slot_of.end() ? int64_t{-1} : static_cast<int64_t>(it->second);
    }
    if (labels.empty()) return (id < 0 || static_cast<uint64_t>(id) >= slots) ? -1 : id;
    auto it = std::lower_bound(labels.begin(), labels.end(), id);
    if (it == labels.end() || *it != id) return -1;
    return it - labels.begin();
}

size_t IdMap::remove(std::span<const int64_t> ids, std::vector<uint32_t>* removed) {
    size_t n = 0;
    for (int64_t id : ids) {
        const int64_t s = find_slot(custom_, labels_, slot_of_, slots_, id);
        if (s < 0 || deleted_[s]) continue;
        if (custom_) slot_of_.erase(id);
        deleted_[s] = 1;
        ++deleted_count_;
        ++n;
        if (removed) removed->push_back(static_cast<uint32_t>(s));
    }
    return n;
}

SlotBits IdMap::filter(std::span<const int64_t> ids) const {
    SlotBits f;
    f.words.assign((slots_ + 63) / 64, 0);
    for (int64_t id : ids) {
        const int64_t s = find_slot(custom_, labels_, slot_of_, slots_, id);
        if (s < 0 || deleted_[s]) continue;
        uint64_t& w = f.words[s >> 6];
        const uint64_t bit = uint64_t{1} << (s & 63);
        if (!(w & bit)) {
            w |= bit;
            ++f.count;
        }
    }
    return f;
}

SlotBits IdMap::live(std::vector<uint64_t> words) const {
    SlotBits f;
    f.words = std::move(words);
    f.words.resize((slots_ + 63) / 64, 0);
    if (slots_ % 64) f.words.back() &= (uint64_t{1} << (slots_ % 64)) - 1;
    if (deleted_count_)
        for (size_t s = 0; s < slots_; ++s)
            if (deleted_[s]) f.words[s >> 6] &= ~(uint64_t{1} << (s & 63));
    for (uint64_t w : f.words) f.count += static_cast<size_t>(__builtin_popcountll(w));
    return f;
}

std::vector<uint32_t> IdMap::compact(bool keep_ids) {
    if (deleted_count_ == 0) return {};
    std::vector<uint32_t> remap(slots_, kRemoved);
    uint32_t next = 0;
    for (size_t s = 0; s < slots_; ++s)
        if (!deleted_[s]) remap[s] = next++;
    if (keep_ids && !custom_ && labels_.empty()) {
        labels_.resize(slots_);
        std::iota(labels_.begin(), labels_.end(), int64_t{0});
    }
    if (!labels_.empty()) {
        for (size_t s = 0; s < slots_; ++s)
            if (remap[s] != kRemoved) labels_[remap[s]] = labels_[s];
        labels_.resize(next);
    }
    for (auto& kv : slot_of_) kv.second = remap[kv.second];
    if (!keep_ids) next_id_ = next;
    deleted_.assign(next, 0);
    slots_ = next;
    deleted_count_ = 0;
    return remap;
}

void IdMap::save(Writer& w) const {
    w.pod<uint8_t>(custom_ ? 1 : 0);
    w.pod<uint64_t>(slots_);
    w.pod<int64_t>(next_id_);
    w.vec(labels_);
    w.vec(deleted_);
}

IdMap IdMap::load(Reader& r, uint64_t slots, uint32_t version) {
    const auto custom = r.pod<uint8_t>();
    const auto slot_num = r.pod<uint64_t>();
    const int64_t next_id = version >= 3 ? r.pod<int64_t>() : static_cast<int64_t>(slot_num);
    auto labels = r.vec<int64_t>(slot_num);
    if (slots != slot_num || slots > UINT32_MAX) Reader::throw_corrupt("id map slot count mismatch");
    if (custom > 1 || next_id < 0) Reader::throw_corrupt("invalid id map shape");
    if (custom) {
        if (labels.size() != slots) Reader::throw_corrupt("invalid id map shape");
    } else if (labels.empty()) {
        if (next_id != static_cast<int64_t>(slots) && slots != 0) Reader::throw_corrupt("invalid id map shape");
    } else {
        if (version < 3 || labels.size() != slots || labels[0] < 0 || labels.back() >= next_id)
            Reader::throw_corrupt("invalid id map shape");
        for (size_t i = 1; i < labels.size(); ++i)
            if (labels[i] <= labels[i - 1]) Reader::throw_corrupt("auto ids out of order");
    }
    auto deleted = r.vec<uint8_t>(slot_num);
    if (deleted.size() != slots) Reader::throw_corrupt("invalid deleted flags length");
    IdMap m(custom == 1);
    m.slots_ = slots;
    m.next_id_ = next_id;
    m.labels_ = std::move(labels);
    m.deleted_ = std::move(deleted);
    for (uint64_t s = 0; s < slots; ++s) {
        if (m.deleted_[s] > 1) Reader::throw_corrupt("invalid deleted flag value");
        if (m.deleted_[s]) {
            ++m.deleted_count_;
            continue;
        }
        if (custom && !m.slot_of_.emplace(m.labels_[s], static_cast<uint32_t>(s)).second)
            Reader::throw_corrupt("duplicate live id");
    }
    return m;
}

// ---- metadata passthrough ----------------------------------------------------

MetaBlob MetaBlob::read(Reader& r, uint64_t slots) {
    const size_t start = r.pos;
    const auto ncols = r.pod<uint64_t>();
    if (ncols > (uint64_t{1} << 16)) Reader::throw_corrupt("too many metadata columns");
    auto skip_vec = [&](size_t elem, uint64_t max_len) {
        const uint64_t n = r.pod<uint64_t>();
        if (n > max_len) Reader::throw_corrupt("vector length exceeds expected size");
        r.need(n * elem);
        r.pos += n * elem;
        return n;
    };
    for (uint64_t c = 0; c < ncols; ++c) {
        skip_vec(1, uint64_t{1} << 24);   // name
        const auto type = r.pod<uint8_t>();
        if (type > 2) Reader::throw_corrupt("invalid metadata column type");
        if (skip_vec(1, slots) != slots) Reader::throw_corrupt("metadata column length mismatch");
        if (type == 0 || type == 1) {
            if (skip_vec(8, slots) != slots) Reader::throw_corrupt("metadata column length mismatch");
        } else {
            if (skip_vec(4, slots) != slots) Reader::throw_corrupt("metadata column length mismatch");
            const auto dict = r.pod<uint64_t>();
            if (dict > UINT32_MAX) Reader::throw_corrupt("metadata dictionary too large");
            for (uint64_t d = 0; d < dict; ++d) skip_vec(1, uint64_t{1} << 24);
        }
    }
    MetaBlob b;
    if (ncols) b.bytes.assign(r.data + start, r.data + r.pos);
    return b;
}

void MetaBlob::write(Writer& w) const {
    if (bytes.empty()) w.pod<uint64_t>(0);
    else w.bytes(bytes.data(), bytes.size());
}

// ---- fast-scan block layout ----------------------------------------------------

std::vector<uint8_t> fs_pack(const std::vector<uint8_t>& codes, size_t n, size_t m) {
    const size_t blocks = (n + kFsBlock - 1) / kFsBlock;
    std::vector<uint8_t> out(blocks * m * 16, 0);
    for (size_t v = 0; v < n; ++v) {
        uint8_t* blk = out.data() + (v / kFsBlock) * m * 16;
        const size_t pos = v % kFsBlock;
        for (size_t s = 0; s < m; ++s) {
            uint8_t& b = blk[s * 16 + (pos % 16)];
            const uint8_t c = codes[v * m + s] & 15;
            b = pos < 16 ? static_cast<uint8_t>((b & 0xF0) | c) : static_cast<uint8_t>((b & 0x0F) | (c << 4));
        }
    }
    return out;
}

std::vector<uint8_t> fs_unpack(const std::vector<uint8_t>& blocks, size_t n, size_t m) {
    std::vector<uint8_t> out(n * m);
    for (size_t v = 0; v < n; ++v) {
        const uint8_t* blk = blocks.data() + (v / kFsBlock) * m * 16;
        const size_t pos = v % kFsBlock;
        for (size_t s = 0; s < m; ++s) {
            const uint8_t b = blk[s * 16 + (pos % 16)];
            out[v * m + s] = pos < 16 ? (b & 15) : (b >> 4);
        }
    }
    return out;
}

// ---- headers / files -------------------------------------------------------------

void write_header(Writer& w, Kind kind) {
    w.pod<uint32_t>(kMagic);
    w.pod<uint32_t>(kFormatVersion);
    w.pod<uint8_t>(static_cast<uint8_t>(kind));
}

Kind read_header(Reader& r, uint32_t* version) {
    if (r.pod<uint32_t>() != kMagic) throw Error(kRuntimeError, "not a qann index file");
    const uint32_t v = r.pod<uint32_t>();
    if (v < 1 || v > kFormatVersion) throw Error(kRuntimeError, "unsupported format version");
    const uint8_t k = r.pod<uint8_t>();
    if (k < 1 || k > 8) throw Error(kRuntimeError, "unknown index kind");
    if (k > 3)
        throw Error(kUnsupported, "index kind " + std::to_string(k) +
                                      " (HNSW, sparse, hybrid or codebook) is not on the GPU search path");
    *version = v;
    return static_cast<Kind>(k);
}

std::shared_ptr<const MappedFile> MappedFile::open(const std::string& path) {
    const int fd = ::open(path.c_str(), O_RDONLY | O_CLOEXEC);
    if (fd < 0) throw Error(kRuntimeError, "cannot open " + path + " for reading");
    struct stat sb {};
    if (::fstat(fd, &sb) != 0) {
        ::close(fd);
        throw Error(kRuntimeError, "cannot stat " + path);
    }
    auto f = std::make_shared<MappedFile>();
    f->path = path;
    f->size = static_cast<size_t>(sb.st_size);
    if (f->size) {
        void* p = ::mmap(nullptr, f->size, PROT_READ, MAP_SHARED, fd, 0);
        if (p == MAP_FAILED) {
            ::close(fd);
            throw Error(kRuntimeError, "cannot map " + path);
        }
        f->data = static_cast<const char*>(p);
    }
    ::close(fd);   // the mapping keeps the file
    return f;
}

MappedFile::~MappedFile() {
    if (data) ::munmap(const_cast<char*>(data), size);
}

std::vector<char> read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) throw Error(kRuntimeError, "cannot open " + path + " for reading");
    const auto n = static_cast<size_t>(in.tellg());
    in.seekg(0);
    std::vector<char> buf(n);
    if (n && !in.read(buf.data(), static_cast<std::streamsize>(n))) throw Error(kRuntimeError, "truncated file");
    return buf;
}

void write_file_atomic(const std::string& path, const std::vector<char>& bytes) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::binary | std::ios::trunc);
        if (!out) throw Error(kRuntimeError, "cannot open " + tmp + " for writing");
        out.write(bytes.data(), static_cast<std::streamsize>(bytes.size()));
        out.close();
        if (!out) {
            std::remove(tmp.c_str());
            throw Error(kRuntimeError, "failed to write " + tmp);
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw Error(kRuntimeError, "cannot rename " + tmp + " to " + path);
    }
}

// ---- PQ ----------------------------------------------------------------------------

std::vector<float> PQCodebook::transposed() const {
    std::vector<float> t(m * sub_dim * K);
    for (size_t i = 0; i < m; ++i)
        for (size_t j = 0; j < sub_dim; ++j)
            for (size_t k = 0; k < K; ++k) t[(i * sub_dim + j) * K + k] = centroids[(i * K + k) * sub_dim + j];
    return t;
}

// Columns of R (d x d, row-major) orthonormal within 1e-3, dots in double
// (reference src/rotation.cpp:132-143, the check load() makes).
static bool rotation_orthonormal(const std::vector<float>& R, size_t d) {
    for (size_t a = 0; a < d; ++a)
        for (size_t b = a; b < d; ++b) {
            double dot = 0.0;
            for (size_t k = 0; k < d; ++k) dot += double(R[k * d + a]) * double(R[k * d + b]);
            if (std::abs(dot - (a == b ? 1.0 : 0.0)) > 1e-3) return false;
        }
    return true;
}

static Metric read_metric(Reader& r) {
    const auto m = r.pod<uint8_t>();
    if (m > 2) Reader::throw_corrupt("unknown metric");
    return static_cast<Metric>(m);
}

// ---- IVF -----------------------------------------------------------------------------

static constexpr uint64_t kListAlign = 64;        // float / SQ rows in IVF lists (format 11)
static constexpr uint64_t kRowAlign = 64 * 1024;  // RefineIndex raw rows (format 10)

void IVFModel::save_body(Writer& w) const {
    w.pod<uint64_t>(dim);
    w.pod<uint64_t>(nlist);
    w.pod<uint64_t>(nprobe);
    w.pod<uint64_t>(idmap.slots());
    w.pod<uint8_t>(trained ? 1 : 0);
    w.pod<uint8_t>(pq_distance);
    w.vec(centroids);
    w.pod<uint8_t>(has_pq ? 1 : 0);
    if (has_pq) {
        w.pod<uint64_t>(pq.dim);
        w.pod<uint64_t>(pq.m);
        w.pod<uint64_t>(pq.K);
        w.vec(pq.centroids);
        w.pod<uint8_t>(fast_scan ? 1 : 0);
        w.pod<uint8_t>(rotate ? 1 : 0);
        w.vec(rotation);
    }
    w.pod<uint8_t>(sq_bits);
    if (sq_bits) {
        w.vec(sq_vmin);
        w.vec(sq_step);
    }
    const size_t row_bytes = sq_bits ? (sq_bits == 8 ? dim : (dim + 1) / 2) : dim * sizeof(float);
    for (size_t l = 0; l < nlist; ++l) {
        const auto& ids = list_ids[l];
        w.vec(ids);
        if (has_pq) {
            const size_t n = ids.size();
            if (fast_scan) w.vec(fs_pack(list_codes[l], n, pq.m));
            else w.vec(list_codes[l]);
            continue;
        }
        const size_t per_row = sq_bits ? row_bytes : dim;
        w.pod<uint64_t>(ids.size() * per_row);
        w.pad(kListAlign);
        if (sq_bits) w.bytes(list_codes[l].data(), ids.size() * row_bytes);
        else w.bytes(list_vecs[l].data(), ids.size() * row_bytes);
    }
    idmap.save(w);
    w.pod<uint8_t>(use_precomputed ? 1 : 0);
    w.pod<uint8_t>(static_cast<uint8_t>(metric));
    meta.write(w);
    w.pod<uint8_t>(cosine_ip ? 1 : 0);
    w.vec(residual_centers);
}

std::unique_ptr<IVFModel> IVFModel::load_body(Reader& r, uint32_t version) {
    auto m = std::make_unique<IVFModel>();
    m->dim = r.pod<uint64_t>();
    m->nlist = r.pod<uint64_t>();
    m->nprobe = r.pod<uint64_t>();
    const auto n_total = r.pod<uint64_t>();
    const auto trained = r.pod<uint8_t>();
    const auto pq_distance = r.pod<uint8_t>();
    if (m->dim == 0 || n_total > UINT32_MAX || trained > 1) Reader::throw_corrupt("invalid IVFIndex shape");
    if (m->nlist < 100 || m->nlist > 65535) Reader::throw_corrupt("nlist must be in [100, 65535]");
    if (m->nprobe == 0 || m->nprobe > m->nlist) Reader::throw_corrupt("nprobe must be in [1, nlist]");
    if (m->dim > UINT64_MAX / m->nlist) Reader::throw_corrupt("invalid IVFIndex shape");
    m->centroids = r.vec<float>(m->nlist * m->dim);
    if (pq_distance > 1) Reader::throw_corrupt("invalid IVFIndex shape");
    if (!trained && n_total > 0) Reader::throw_corrupt("invalid IVFIndex shape");
    if ((trained && m->centroids.size() != m->nlist * m->dim) || (!trained && !m->centroids.empty()))
        Reader::throw_corrupt("invalid IVFIndex shape");
    m->trained = trained;
    m->pq_distance = pq_distance;

    if (r.pod<uint8_t>()) {
        m->has_pq = true;
        PQCodebook& pq = m->pq;
        pq.dim = r.pod<uint64_t>();
        pq.m = r.pod<uint64_t>();
        pq.K = r.pod<uint64_t>();
        if (pq.dim == 0 || pq.m == 0 || pq.dim % pq.m != 0 || pq.K == 0 || pq.K > 256)
            Reader::throw_corrupt("invalid PQ codebook shape");
        pq.sub_dim = pq.dim / pq.m;
        const uint64_t expect = pq.m * pq.K * pq.sub_dim;
        pq.centroids = r.vec<float>(expect);
        if (pq.centroids.size() != expect) Reader::throw_corrupt("unexpected number of centroids");
        if (pq.dim != m->dim) Reader::throw_corrupt("invalid IVFIndex shape");
        if (version >= 4) {
            const auto fs = r.pod<uint8_t>();
            if (fs > 1 || (fs && (pq.K != 16 || pq.m % 2 != 0 || pq.m > kFsMaxSubspaces || pq_distance != 0)))
                Reader::throw_corrupt("invalid IVFIndex fast-scan settings");
            m->fast_scan = fs;
        }
        if (version >= 8) {
            const auto rot = r.pod<uint8_t>();
            if (rot > 1) Reader::throw_corrupt("invalid IVFIndex rotation");
            m->rotate = rot;
            m->rotation = r.vec<float>(m->dim * m->dim);
            if (m->rotation.size() != (rot && trained ? m->dim * m->dim : 0))
                Reader::throw_corrupt("IVFIndex rotation length mismatch");
            if (!m->rotation.empty() && !rotation_orthonormal(m->rotation, m->dim))
                Reader::throw_corrupt("IVFIndex rotation is not orthogonal");
        }
    }
    if (version >= 7) {
        const auto bits = r.pod<uint8_t>();
        if ((bits != 0 && bits != 4 && bits != 8) || (bits && m->has_pq)) Reader::throw_corrupt("invalid IVFIndex SQ settings");
        m->sq_bits = bits;
        if (bits) {
            m->sq_vmin = r.vec<float>(m->dim);
            m->sq_step = r.vec<float>(m->dim);
            const size_t ranges = trained ? m->dim : 0;
            if (m->sq_vmin.size() != ranges || m->sq_step.size() != ranges) Reader::throw_corrupt("IVF SQ range length mismatch");
        }
    }

    const size_t pm = m->m();
    const size_t sq_row = m->sq_bits == 8 ? m->dim : (m->dim + 1) / 2;
    m->list_ids.resize(m->nlist);
    m->list_codes.resize(m->nlist);
    m->list_vecs.resize(m->nlist);
    uint64_t seen = 0;
    for (size_t l = 0; l < m->nlist; ++l) {
        auto& ids = m->list_ids[l];
        ids = r.vec<uint32_t>(n_total);
        const size_t n = ids.size();
        if (!m->has_pq && version >= 11) {
            const size_t row_bytes = m->sq_bits ? sq_row : m->dim * sizeof(float);
            const uint64_t expected = n * (m->sq_bits ? row_bytes : m->dim);
            if (r.pod<uint64_t>() != expected) Reader::throw_corrupt("IVF list length mismatch");
            r.pad(kListAlign);
            if (m->sq_bits) {
                m->list_codes[l].resize(n * row_bytes);
                r.bytes(m->list_codes[l].data(), n * row_bytes);
            } else {
                m->list_vecs[l].resize(n * m->dim);
                r.bytes(m->list_vecs[l].data(), n * row_bytes);
            }
        } else if (m->sq_bits) {
            m->list_codes[l] = r.vec<uint8_t>(n * sq_row);
            if (m->list_codes[l].size() != n * sq_row) Reader::throw_corrupt("IVF code length mismatch");
        } else if (m->has_pq) {
            const uint64_t blocks = (n + kFsBlock - 1) / kFsBlock;
            const uint64_t expected = m->fast_scan ? blocks * pm * 16 : n * pm;
            auto codes = r.vec<uint8_t>(expected);
            if (codes.size() != expected) Reader::throw_corrupt("IVF code length mismatch");
            m->list_codes[l] = m->fast_scan ? fs_unpack(codes, n, pm) : std::move(codes);
        } else {
            m->list_vecs[l] = r.vec<float>(n * m->dim);
            if (m->list_vecs[l].size() != n * m->dim) Reader::throw_corrupt("IVF vector length mismatch");
        }
        for (uint32_t id : ids)
            if (id >= n_total) Reader::throw_corrupt("IVF id out of range");
        seen += n;
    }
    if (seen != n_total) Reader::throw_corrupt("invalid IVFIndex shape");

    if (version >= 2) m->idmap = IdMap::load(r, n_total, version);
    else m->idmap.add(n_total, nullptr);
    if (version >= 3) {
        const auto up = r.pod<uint8_t>();
        if (up > 1) Reader::throw_corrupt("invalid IVFIndex shape");
        m->use_precomputed = up;
    }
    if (version >= 5) m->metric = read_metric(r);
    if (version >= 9) m->meta = MetaBlob::read(r, n_total);
    if (version >= 12) {
        const auto c = r.pod<uint8_t>();
        if (c > 1) Reader::throw_corrupt("invalid IVFIndex shape");
        m->cosine_ip = c;
    }
    if (version >= 13) {
        m->residual_centers = r.vec<float>(m->nlist * m->dim);
        const bool expected = trained && m->has_pq && m->metric == Metric::Cosine;
        if (m->residual_centers.size() != (expected ? m->nlist * m->dim : 0))
            Reader::throw_corrupt("IVFIndex residual centers length mismatch");
    }
    return m;
}

// ---- Flat ------------------------------------------------------------------------------

void FlatModel::save_body(Writer& w) const {
    w.pod<uint64_t>(dim);
    w.pod<uint64_t>(idmap.slots());
    w.vec(data);
    idmap.save(w);
    w.pod<uint8_t>(static_cast<uint8_t>(metric));
    meta.write(w);
}

std::unique_ptr<FlatModel> FlatModel::load_body(Reader& r, uint32_t version) {
    auto m = std::make_unique<FlatModel>();
    m->dim = r.pod<uint64_t>();
    const auto count = r.pod<uint64_t>();
    if (m->dim == 0 || count > UINT64_MAX / m->dim) Reader::throw_corrupt("invalid FlatIndex shape");
    m->data = r.vec<float>(count * m->dim);
    if (m->data.size() != count * m->dim) Reader::throw_corrupt("FlatIndex data length mismatch");
    if (version >= 2) m->idmap = IdMap::load(r, count, version);
    else m->idmap.add(count, nullptr);
    if (version >= 5) m->metric = read_metric(r);
    if (version >= 9) m->meta = MetaBlob::read(r, count);
    return m;
}

// ---- Refine ----------------------------------------------------------------------------

void RefineModel::save_body(Writer& w) const {
    w.pod<uint64_t>(k_factor);
    w.pod<uint64_t>(idmap.slots());
    write_header(w, base_kind);
    if (base_kind == Kind::IVF) ivf->save_body(w);
    else flat->save_body(w);
    const uint64_t dim = base_kind == Kind::IVF ? ivf->dim : flat->dim;
    w.pod<uint64_t>(idmap.slots() * dim);
    w.pad(kRowAlign);
    w.bytes(data.data(), data.size() * sizeof(float));
    idmap.save(w);
    meta.write(w);
}

std::unique_ptr<RefineModel> RefineModel::load_body(Reader& r, uint32_t version, bool map_rows) {
    auto m = std::make_unique<RefineModel>();
    m->k_factor = r.pod<uint64_t>();
    const auto count = r.pod<uint64_t>();
    if (m->k_factor == 0) Reader::throw_corrupt("invalid RefineIndex shape");
    uint32_t bv = 0;
    const Kind bk = read_header(r, &bv);
    if (bv != version) Reader::throw_corrupt("RefineIndex base has a different format version");
    m->base_kind = bk;
    uint64_t dim = 0, base_slots = 0;
    bool ids_are_slots = false;
    if (bk == Kind::IVF) {
        m->ivf = IVFModel::load_body(r, bv);
        dim = m->ivf->dim;
        base_slots = m->ivf->idmap.slots();
        ids_are_slots = m->ivf->idmap.ids_are_slots();
    } else if (bk == Kind::Flat) {
        m->flat = FlatModel::load_body(r, bv);
        dim = m->flat->dim;
        base_slots = m->flat->idmap.slots();
        ids_are_slots = m->flat->idmap.ids_are_slots();
    } else {
        Reader::throw_corrupt("RefineIndex base must be Flat, IVF or HNSW");
    }
    if (!ids_are_slots) Reader::throw_corrupt("RefineIndex base ids must equal its slots");
    if (count != base_slots || count > UINT64_MAX / dim) Reader::throw_corrupt("invalid RefineIndex shape");
    const auto len = r.pod<uint64_t>();
    if (len != count * dim) Reader::throw_corrupt("unexpected number of vectors");
    if (version >= 10) r.pad(kRowAlign);
    if (map_rows && version >= 10 && reinterpret_cast<uintptr_t>(r.data + r.pos) % 16 == 0) {
        r.need(len * sizeof(float));
        m->mapped = reinterpret_cast<const float*>(r.data + r.pos);
        r.pos += len * sizeof(float);
    } else {
        m->data.resize(len);
        r.bytes(m->data.data(), len * sizeof(float));
    }
    if (version >= 2) m->idmap = IdMap::load(r, count, version);
    else m->idmap.add(count, nullptr);
    if (version >= 9) m->meta = MetaBlob::read(r, count);
    return m;
}

} // namespace qg
