// Host-side model of the indexes on the search path and the `.qann` file
// format they round-trip through.
//
// The format is the reference's (header `QANN`, version 1..13, kind tags
// 1 Flat / 2 IVF / 3 Refine; reference src/serialize.hpp:20-39), so files
// saved by qann load here and files saved here load in qann. The host copy is
// canonical (it is what save() writes); device copies are built from it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <unordered_map>
#include <vector>

namespace qg {

enum class Metric : uint8_t { L2 = 0, Cosine = 1, InnerProduct = 2 };
enum class Kind : uint8_t { Flat = 1, IVF = 2, Refine = 3 };

inline constexpr uint32_t kMagic = 0x4E4E4151;      // "QANN" little-endian
inline constexpr uint32_t kFormatVersion = 13;
inline constexpr size_t kFsBlock = 32;               // fast-scan block (vectors)
inline constexpr size_t kFsMaxSubspaces = 1024;
inline constexpr uint32_t kRemoved = UINT32_MAX;

// ---- byte streams ----------------------------------------------------------

struct Writer {
    std::vector<char> buf;   // starts at file offset 0, so buf.size() is the offset
    template <class T>
    void pod(const T& v) {
        const char* p = reinterpret_cast<const char*>(&v);
        buf.insert(buf.end(), p, p + sizeof(T));
    }
    void bytes(const void* p, size_t n) {
        const char* c = static_cast<const char*>(p);
        buf.insert(buf.end(), c, c + n);
    }
    template <class T>
    void vec(const std::vector<T>& v) {
        pod<uint64_t>(v.size());
        bytes(v.data(), v.size() * sizeof(T));
    }
    // u32 pad length then zeros, so the data after it starts at a multiple of align
    // (reference src/vector_store.cpp:59-72).
    void pad(uint64_t align) {
        const uint64_t after = buf.size() + sizeof(uint32_t);
        const uint32_t n = static_cast<uint32_t>((align - after % align) % align);
        pod(n);
        buf.insert(buf.end(), n, 0);
    }
};

struct Reader {
    const char* data;
    size_t size;
    size_t pos = 0;
    void need(size_t n) const;
    template <class T>
    T pod() {
        need(sizeof(T));
        T v;
        std::memcpy(&v, data + pos, sizeof(T));
        pos += sizeof(T);
        return v;
    }
    void bytes(void* out, size_t n) {
        need(n);
        std::memcpy(out, data + pos, n);
        pos += n;
    }
    template <class T>
    std::vector<T> vec(uint64_t max_len) {
        const uint64_t n = pod<uint64_t>();
        if (n > max_len) throw_corrupt("vector length exceeds expected size");
        std::vector<T> v(n);
        if (n) bytes(v.data(), n * sizeof(T));
        return v;
    }
    void pad(uint64_t align);
    [[noreturn]] static void throw_corrupt(const std::string& what);
};

// ---- slot <-> id map (reference include/vecengine/id_map.hpp:42-131) --------

struct SlotBits {
    std::vector<uint64_t> words;   // bit s of the filter: slot s may be returned
    size_t count = 0;
    bool test(uint32_t s) const { return (words[s >> 6] >> (s & 63)) & 1; }
};

class IdMap {
public:
    explicit IdMap(bool custom = false) : custom_(custom) {}
    void check(size_t n, const int64_t* ids) const;
    void add(size_t n, const int64_t* ids);
    size_t remove(std::span<const int64_t> ids, std::vector<uint32_t>* removed = nullptr);
    SlotBits filter(std::span<const int64_t> ids) const;
    SlotBits live(std::vector<uint64_t> words) const;
    std::vector<uint32_t> compact(bool keep_ids);
    int64_t label(uint32_t s) const { return labels_.empty() ? static_cast<int64_t>(s) : labels_[s]; }
    bool is_deleted(uint32_t s) const { return deleted_[s] != 0; }
    bool ids_are_slots() const { return !custom_ && labels_.empty() && static_cast<size_t>(next_id_) == slots_; }
    bool custom() const { return custom_; }
    size_t slots() const { return slots_; }
    size_t live_count() const { return slots_ - deleted_count_; }
    size_t deleted_count() const { return deleted_count_; }
    const std::vector<int64_t>& labels() const { return labels_; }
    const std::vector<uint8_t>& deleted() const { return deleted_; }
    void save(Writer& w) const;
    static IdMap load(Reader& r, uint64_t slots, uint32_t version);

private:
    bool custom_;
    size_t slots_ = 0;
    int64_t next_id_ = 0;
    size_t deleted_count_ = 0;
    std::vector<int64_t> labels_;
    std::unordered_map<int64_t, uint32_t> slot_of_;
    std::vector<uint8_t> deleted_;
};

// Metadata columns ride along unchanged: the search path only consumes the
// slot bitmaps a where= filter evaluates to. The store is kept as its saved
// bytes (reference src/metadata.cpp:1542-1610 writes/reads them).
struct MetaBlob {
    std::vector<char> bytes;       // empty = a store with no columns
    static MetaBlob read(Reader& r, uint64_t slots);
    void write(Writer& w) const;
    bool empty() const { return bytes.empty(); }
};

// ---- models ------------------------------------------------------------------

struct PQCodebook {
    uint64_t dim = 0, m = 0, K = 0, sub_dim = 0;
    std::vector<float> centroids;   // m * K * sub_dim, centroid-major per subspace
    // m * sub_dim * K: the layout the reference's table loops read (reference src/pq.cpp:260-268)
    std::vector<float> transposed() const;
};

struct IVFModel {
    uint64_t dim = 0, nlist = 0, nprobe = 10;
    bool trained = false;
    uint8_t pq_distance = 0;   // 0 ADC, 1 SDC
    std::vector<float> centroids;   // nlist * dim
    bool has_pq = false;
    PQCodebook pq;
    bool fast_scan = false, rotate = false;
    std::vector<float> rotation;    // dim * dim row-major, when rotate and trained
    uint8_t sq_bits = 0;
    std::vector<float> sq_vmin, sq_step;
    std::vector<std::vector<uint32_t>> list_ids;   // nlist lists of slots
    std::vector<std::vector<uint8_t>> list_codes;  // PQ: m code bytes per vector (one code per byte)
    std::vector<std::vector<float>> list_vecs;     // plain IVF: dim floats per vector
    IdMap idmap;
    bool use_precomputed = true;
    Metric metric = Metric::L2;
    MetaBlob meta;
    bool cosine_ip = true;
    std::vector<float> residual_centers;            // cosine + PQ (format 13), else empty
    bool filter_probe_scaling = true;               // not saved (reference ivf_index.hpp:117-118)

    size_t m() const { return has_pq ? pq.m : 0; }
    void save_body(Writer& w) const;
    static std::unique_ptr<IVFModel> load_body(Reader& r, uint32_t version);
};

struct FlatModel {
    uint64_t dim = 0;
    std::vector<float> data;   // slots * dim
    IdMap idmap;
    Metric metric = Metric::L2;
    MetaBlob meta;
    void save_body(Writer& w) const;
    static std::unique_ptr<FlatModel> load_body(Reader& r, uint32_t version);
};

// A whole file mapped read-only (reference include/vecengine/vector_store.hpp:21-49),
// unmapped when the last owner lets go.
struct MappedFile {
    const char* data = nullptr;
    size_t size = 0;
    std::string path;
    static std::shared_ptr<const MappedFile> open(const std::string& path);
    ~MappedFile();
};

struct RefineModel {
    uint64_t k_factor = 10;
    Kind base_kind = Kind::IVF;
    std::shared_ptr<IVFModel> ivf;     // one of ivf / flat is the base
    std::shared_ptr<FlatModel> flat;
    std::vector<float> data;           // raw rows, slots * dim
    const float* mapped = nullptr;     // load_body(map_rows): the rows inside the reader's buffer instead of `data`
    IdMap idmap;
    MetaBlob meta;
    void save_body(Writer& w) const;
    // map_rows: leave the raw rows in the reader's buffer (format 10 and
    // later keep them 64 KB aligned there) and point `mapped` at them
    static std::unique_ptr<RefineModel> load_body(Reader& r, uint32_t version, bool map_rows = false);
};

void write_header(Writer& w, Kind kind);
// Returns the kind; throws on a bad magic / version / kind.
Kind read_header(Reader& r, uint32_t* version);

std::vector<char> read_file(const std::string& path);
// Writes path.tmp then renames it over path (reference src/index_factory.cpp:94-118).
void write_file_atomic(const std::string& path, const std::vector<char>& bytes);

// Fast-scan block layout of the file format (reference src/fast_scan.hpp:6-34):
// block b of a list is m * 16 bytes; byte s * 16 + j holds vector j's code of
// subspace s in its low nibble and vector j + 16's in its high nibble.
std::vector<uint8_t> fs_pack(const std::vector<uint8_t>& codes, size_t n, size_t m);
std::vector<uint8_t> fs_unpack(const std::vector<uint8_t>& blocks, size_t n, size_t m);

} // namespace qg
