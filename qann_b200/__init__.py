"""qann_b200 — qann's dense-vector search path on NVIDIA B200.

A drop-in for the part of qann (https://github.com/maxtmiller/qann) that
searches dense vectors: ``IVFIndex`` with 4-bit PQ fast-scan, ``RefineIndex``
re-ranking, ``FlatIndex``, their ``train`` / ``add`` / ``batch_query`` /
``save`` / ``load``, ``nprobe``, ``k_factor`` and ``allowed`` filters, with
the same signatures, defaults, errors and ``.qann`` files. Behind it, C++ host
code drives hand-written sm_100a CUDA kernels through the C ABI in
``include/qann_gpu.h``; results match the reference's CPU build: the same
ids, bit-identical distances and byte-identical ``.qann`` files after
training and adding.

Differences from qann: ``where=`` metadata filters are evaluated by the
caller (pass the matching ids as ``allowed``); HNSW, SQ, sparse, hybrid and
journal indexes are not part of this package.
"""
from __future__ import annotations

import ctypes as C
import enum
import os

import numpy as np

from . import _lib
from ._lib import CudaError, check

__all__ = [
    "Metric", "Clustering", "PQDistance", "DenseIndex", "FlatIndex", "IVFIndex", "RefineIndex", "load",
    "set_num_threads", "CudaError", "version",
]


class Metric(enum.IntEnum):
    """How an index compares vectors (reference include/vecengine/index.hpp:57-62)."""
    L2 = 0
    Cosine = 1
    InnerProduct = 2


class Clustering(enum.IntEnum):
    """How IVFIndex.train learns the coarse centroids."""
    EMeans = 0
    Lloyd = 1


class PQDistance(enum.IntEnum):
    ADC = 0
    SDC = 1


def version() -> str:
    return _lib.lib.qg_version().decode()


_threads = os.cpu_count() or 1


def set_num_threads(n: int) -> None:
    """Accepted for API compatibility: the search path runs on the GPU, so the
    host thread count has no effect on it."""
    global _threads
    if n < 1:
        raise ValueError("num_threads must be >= 1")
    _threads = int(n)


def _f32_rows(data, dim: int, what: str = "data") -> np.ndarray:
    a = np.asarray(data, dtype=np.float32)
    if a.ndim != 2:
        raise ValueError(f"{what} must be a 2D array of shape (n, dim)")
    if a.shape[1] != dim:
        raise ValueError(f"{what} dimension does not match index dimension")
    return np.ascontiguousarray(a)


def _ids(ids) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(list(ids) if not hasattr(ids, "__len__") else ids, dtype=np.int64).ravel())


def set_tensor_filter(mode: int) -> None:
    """Exact top-k over many rows through the BF16 tensor-core filter and FP32
    recheck: 0 never, 1 when it pays (default), 2 whenever supported. Results
    are identical in every mode."""
    check(_lib.lib.qg_set_option(b"tensor_filter", int(mode)))


def tensor_filter() -> int:
    v = C.c_int64()
    check(_lib.lib.qg_get_option(b"tensor_filter", C.byref(v)))
    return v.value


def tensor_filter_counts() -> dict:
    """Queries answered through the tensor-core filter so far, and how many of
    them were redone exactly because their candidate lists overflowed; the
    same for the coarse step; filtered batches, and how many of them ranked
    every list because a probe walk went past the lists ranked first."""
    out = {}
    for key in ("queries", "redone"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"tensor_filter_{key}".encode(), C.byref(v)))
        out[key] = v.value
    for key in ("queries", "redone", "candidates"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"tensor_coarse_{key}".encode(), C.byref(v)))
        out[f"coarse_{key}"] = v.value
    for key in ("batches", "deep_walks"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"filtered_{key}".encode(), C.byref(v)))
        out[f"filtered_{key}"] = v.value
    return out


def set_scan_options(autotune: bool | None = None, variant: int | None = None) -> None:
    """Fast-scan kernel shapes. autotune: time the candidate shapes on the
    first large search of each problem and keep the fastest (default on).
    variant: -1 any shape, 0 codes read from global memory (registers sized
    for two blocks per SM), 1 codes staged through shared memory by bulk
    copies, 2 codes from global memory with registers sized for more resident
    warps (3 blocks of 8 warps or 5 of 4). Results are identical under every shape."""
    if autotune is not None:
        check(_lib.lib.qg_set_option(b"scan_autotune", int(bool(autotune))))
    if variant is not None:
        check(_lib.lib.qg_set_option(b"scan_variant", int(variant)))


def merge_candidates_device(key_ptr: int, slot_ptr: int, nq: int, nparts: int, kp: int, out_key_ptr: int,
                            out_slot_ptr: int, stream: int = 0) -> None:
    """The k' smallest keys per query over nparts sorted candidate lists laid
    out [nq][nparts][kp] (uint64 keys, uint32 slots), sorted."""
    check(_lib.lib.qg_merge_candidates_device(key_ptr, slot_ptr, nq, nparts, kp, out_key_ptr, out_slot_ptr,
                                              stream or None))


def set_search_graphs(on: bool) -> None:
    """search_device replays fixed-shape, unfiltered IVF searches as CUDA
    graphs (captured on the first call with each batch size, k, nprobe and
    buffers). Off by default; results are identical either way."""
    check(_lib.lib.qg_set_option(b"search_graphs", int(bool(on))))


def search_graph_counts() -> dict:
    out = {}
    for key in ("replays", "captures"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"search_graph_{key}".encode(), C.byref(v)))
        out[key] = v.value
    return out


def set_tensor_scan(mode: int) -> None:
    """The fast-scan on the tensor cores (list-major, int8 MMA over one-hot
    codes and rounded LUTs) for large unfiltered batches with per-list L2
    tables: 0 never, 1 when it pays (default; slower than the query-major
    kernel on the workloads measured so far, so not picked), 2 whenever it
    applies. Results are identical in every mode."""
    check(_lib.lib.qg_set_option(b"tensor_scan", int(mode)))


def tensor_scan_counts() -> dict:
    """Searches that went through the tensor-core scan, and queries of them
    redone by the query-major scan because their candidates overflowed."""
    out = {}
    for key in ("calls", "redone"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"tensor_scan_{key}".encode(), C.byref(v)))
        out[key] = v.value
    for key in ("units", "tiles", "luts_live", "luts_hopeless", "candidates", "pairs", "pairs_kept"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"tensor_scan_stat_{key}".encode(), C.byref(v)))
        out[key] = v.value
    return out


def scan_options() -> dict:
    out = {}
    for key in ("autotune", "variant", "tuned_shapes", "last_shape"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"scan_{key}".encode(), C.byref(v)))
        out[key] = v.value
    return out


def set_filter_options(autotune: bool | None = None, epilogue_warps: int | None = None) -> None:
    """The tensor-core filter's schedule (flat search, direct scans,
    nearest-centroid assignment, the coarse step). autotune: time its 8- and
    16-warp epilogues on the first large launch of each problem and keep the
    faster (default on); off, the 8-warp one. epilogue_warps: 8 or 16 forces
    that epilogue on every launch, 0 leaves the pick to the autotuner. Results
    are identical under every setting."""
    if autotune is not None:
        check(_lib.lib.qg_set_option(b"filter_autotune", int(bool(autotune))))
    if epilogue_warps is not None:
        check(_lib.lib.qg_set_option(b"filter_epilogue_warps", int(epilogue_warps)))


def filter_options() -> dict:
    """autotune (on or off), tuned_problems (problems timed so far),
    last_epilogue_warps (8 or 16, the last filter launch's schedule) and
    epilogue_warps (the forced schedule, 0 for none)."""
    out = {}
    for key in ("autotune", "tuned_problems", "last_epilogue_warps", "epilogue_warps"):
        v = C.c_int64()
        check(_lib.lib.qg_get_option(f"filter_{key}".encode(), C.byref(v)))
        out[key] = v.value
    return out


class DenseIndex:
    """An index of dense float32 vectors. Not constructed directly."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        self._parent = None

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_lib, "lib", None) if _lib is not None else None
        if h is not None and h.value and lib is not None:   # (module globals may be gone at interpreter exit)
            lib.qg_free(h)
            self._h = None

    # -- properties -----------------------------------------------------------------
    def _get(self, key: str) -> int:
        v = C.c_int64()
        check(_lib.lib.qg_get(self._h, key.encode(), C.byref(v)))
        return v.value

    def _set(self, key: str, value) -> None:
        check(_lib.lib.qg_set(self._h, key.encode(), int(value)))

    def dim(self) -> int:
        return self._get("dim")

    def size(self) -> int:
        """Number of live (not deleted) vectors."""
        return self._get("size")

    @property
    def metric(self) -> Metric:
        return Metric(self._get("metric"))

    @property
    def custom_ids(self) -> bool:
        return bool(self._get("custom_ids"))

    @property
    def stores_vectors(self) -> bool:
        return isinstance(self, (FlatIndex, RefineIndex))

    # -- writes -----------------------------------------------------------------------
    def add(self, data, ids=None, *, metadata=None):
        """Adds an (n, dim) array; returns the vectors' int64 ids."""
        if metadata is not None:
            raise NotImplementedError(
                "metadata columns are not kept by qann_b200: keep them beside the index, evaluate filters on the "
                "host into a slot bitmap and query with batch_query_bitmap(query, k, words), or pass allowed= ids")
        x = _f32_rows(data, self.dim())
        n = x.shape[0]
        idarr = None if ids is None else _ids(ids)
        if idarr is not None and idarr.size != n:
            raise ValueError("ids must have one id per row")
        out = np.empty(n, np.int64)
        check(_lib.lib.qg_add(self._h, x.ctypes.data, n, None if idarr is None else idarr.ctypes.data,
                              out.ctypes.data))
        return out

    def remove(self, ids) -> int:
        a = _ids(ids)
        r = C.c_size_t()
        check(_lib.lib.qg_remove(self._h, a.ctypes.data, a.size, C.byref(r)))
        return r.value

    def compact(self) -> int:
        r = C.c_size_t()
        check(_lib.lib.qg_compact(self._h, C.byref(r)))
        return r.value

    # -- queries ----------------------------------------------------------------------
    def batch_query(self, query, k, *, allowed=None, where=None):
        """k nearest neighbours of each row: (ids int64 (nq, k), distances
        float32 (nq, k)), padded with -1 / inf."""
        if where is not None:
            raise NotImplementedError(
                "where= needs the metadata store, which qann_b200 does not keep: evaluate the expression on the "
                "host into a slot bitmap (uint64 words, bit s allows slot s) and call batch_query_bitmap(query, k, "
                "words), or pass the matching ids as allowed=")
        q = _f32_rows(query, self.dim(), "query")
        k = int(k)
        if k < 0:
            raise ValueError("k must be >= 0")
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int64)
        d = np.empty((nq, k), np.float32)
        if allowed is None:
            check(_lib.lib.qg_search(self._h, q.ctypes.data, nq, k, None, 0, ids.ctypes.data, d.ctypes.data))
        else:
            al = _ids(allowed)
            check(_lib.lib.qg_search(self._h, q.ctypes.data, nq, k, al.ctypes.data, al.size, ids.ctypes.data,
                                     d.ctypes.data))
        return ids, d

    def batch_query_bitmap(self, query, k, words):
        """batch_query with the filter given as a slot bitmap (uint64 words,
        bit s of words[s // 64] allows slot s), as a where= evaluation yields."""
        q = _f32_rows(query, self.dim(), "query")
        w = np.ascontiguousarray(words, dtype=np.uint64)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int64)
        d = np.empty((nq, k), np.float32)
        check(_lib.lib.qg_search_bitmap(self._h, q.ctypes.data, nq, k, w.ctypes.data, w.size, ids.ctypes.data,
                                        d.ctypes.data))
        return ids, d

    def query(self, query, k, *, allowed=None, where=None):
        """k nearest neighbours of one (dim,) vector: 1D (ids, distances), one
        entry per result found."""
        q = np.asarray(query, dtype=np.float32)
        if q.ndim != 1:
            raise ValueError("query must be a 1D array of shape (dim,)")
        ids, d = self.batch_query(q[None], k, allowed=allowed, where=where)
        keep = ids[0] >= 0
        return ids[0][keep], d[0][keep]

    def search_device(self, q_ptr: int, nq: int, k: int, out_ids_ptr: int, out_d_ptr: int, stream: int = 0) -> None:
        """batch_query on device memory (raw CUDA pointers, e.g. torch
        ``tensor.data_ptr()``): q (nq, dim) float32 in, ids (nq, k) int64 and
        distances (nq, k) float32 out, on ``stream``."""
        check(_lib.lib.qg_search_device(self._h, q_ptr, nq, k, out_ids_ptr, out_d_ptr, stream or None))

    # -- sharded search (the lists of an IVF index spread over devices) --------------
    def candidate_count(self, k: int) -> int:
        """k' candidates per query that search_candidates_device returns."""
        v = C.c_size_t()
        check(_lib.lib.qg_candidate_count(self._h, int(k), C.byref(v)))
        return v.value

    def search_candidates_device(self, q_ptr: int, nq: int, k: int, key_ptr: int, slot_ptr: int,
                                 stream: int = 0) -> None:
        """The k' best candidates of each query from this handle's shard of
        the lists: (nq, k') uint64 keys and uint32 slots, sorted."""
        check(_lib.lib.qg_search_candidates_device(self._h, q_ptr, nq, k, key_ptr, slot_ptr, stream or None))

    def finish_candidates_device(self, q_ptr: int, nq: int, k: int, key_ptr: int, slot_ptr: int, out_ids_ptr: int,
                                 out_d_ptr: int, stream: int = 0) -> None:
        """Results from merged candidates (re-ranked for a RefineIndex)."""
        check(_lib.lib.qg_finish_candidates_device(self._h, q_ptr, nq, k, key_ptr, slot_ptr, out_ids_ptr, out_d_ptr,
                                                   stream or None))

    def save(self, path) -> None:
        check(_lib.lib.qg_save(self._h, os.fspath(path).encode()))

    def __len__(self):
        return self.size()


class FlatIndex(DenseIndex):
    """Exact search over every stored vector (reference include/vecengine/flat_index.hpp)."""

    def __init__(self, dim, *, custom_ids=False, metric=Metric.L2, _handle=None):
        if _handle is None:
            h = C.c_void_p()
            check(_lib.lib.qg_create_flat(int(dim), int(metric), int(bool(custom_ids)), C.byref(h)))
            _handle = h.value
        super().__init__(_handle)


class IVFIndex(DenseIndex):
    """Inverted-file index with residual PQ (4-bit fast-scan on the GPU path)
    (reference include/vecengine/ivf_index.hpp)."""

    def __init__(self, dim, nlist, nprobe=10, *, custom_ids=False, metric=Metric.L2, _handle=None):
        if _handle is None:
            h = C.c_void_p()
            check(_lib.lib.qg_create_ivf(int(dim), int(nlist), int(nprobe), int(metric), int(bool(custom_ids)),
                                         C.byref(h)))
            _handle = h.value
        super().__init__(_handle)

    def train(self, data, max_iters=10, seed=None, *, clustering=Clustering.EMeans, passes=2):
        x = _f32_rows(data, self.dim())
        check(_lib.lib.qg_train(self._h, x.ctypes.data, x.shape[0], int(max_iters), -1 if seed is None else int(seed),
                                int(clustering), int(passes)))

    def enable_pq(self, num_subspaces, centroids_per_subspace=None, *, fast_scan=False, rotate=False):
        K = centroids_per_subspace if centroids_per_subspace is not None else (16 if fast_scan else 256)
        check(_lib.lib.qg_enable_pq(self._h, int(num_subspaces), int(K), int(bool(fast_scan)), int(bool(rotate))))

    nlist = property(lambda self: self._get("nlist"))
    nprobe = property(lambda self: self._get("nprobe"), lambda self, v: self._set("nprobe", v))
    precomputed_tables = property(lambda self: bool(self._get("precomputed_tables")),
                                  lambda self, v: self._set("precomputed_tables", bool(v)))
    cosine_inner_product = property(lambda self: bool(self._get("cosine_inner_product")),
                                    lambda self, v: self._set("cosine_inner_product", bool(v)))
    filter_probe_scaling = property(lambda self: bool(self._get("filter_probe_scaling")),
                                    lambda self, v: self._set("filter_probe_scaling", bool(v)))
    pq_distance = property(lambda self: PQDistance(self._get("pq_distance")),
                           lambda self, v: self._set("pq_distance", int(v)))
    def list_sizes(self) -> np.ndarray:
        """Vectors per inverted list (nlist,), uint32."""
        out = np.empty(self.nlist, np.uint32)
        check(_lib.lib.qg_ivf_list_sizes(self._h, out.ctypes.data))
        return out

    def centroids(self) -> np.ndarray:
        """The (nlist, dim) coarse centroids."""
        out = np.empty((self.nlist, self.dim()), np.float32)
        check(_lib.lib.qg_ivf_centroids(self._h, out.ctypes.data))
        return out

    fast_scan = property(lambda self: bool(self._get("fast_scan")))
    pq_rotate = property(lambda self: bool(self._get("rotate")))
    sq_bits = property(lambda self: self._get("sq_bits"))
    mapped = property(lambda self: False)

    def set_shard(self, shard: int, shards: int) -> None:
        """Keep on the device only the lists l with l % shards == shard, for
        the sharded search (qann_b200.sharded); shards=1 holds every list."""
        self._set("shards", shards)
        self._set("shard", shard)


class RefineIndex(DenseIndex):
    """Re-ranks an approximate base's k * k_factor candidates with exact
    distances (reference include/vecengine/refine_index.hpp)."""

    def __init__(self, base=None, k_factor=10, *, custom_ids=False, _handle=None):
        if _handle is None:
            if not isinstance(base, DenseIndex):
                raise TypeError("base must be a qann_b200 index")
            h = C.c_void_p()
            check(_lib.lib.qg_create_refine(base._h, int(k_factor), int(bool(custom_ids)), C.byref(h)))
            _handle = h.value
        super().__init__(_handle)
        self._base = base

    k_factor = property(lambda self: self._get("k_factor"), lambda self, v: self._set("k_factor", v))
    # 2: raw rows read in place from the mapped file by the re-rank; 1: mapped
    # but copied to GPU memory; 0: in memory (see load(mmap=True))
    rows_mapped = property(lambda self: self._get("rows_mapped"))
    mapped = property(lambda self: False)

    @property
    def base(self):
        if self._base is None:
            h = C.c_void_p()
            check(_lib.lib.qg_refine_base(self._h, C.byref(h)))
            kind = self._get("base_kind")
            self._base = (IVFIndex if kind == 2 else FlatIndex)(0, 0, _handle=h.value) if kind == 2 else \
                FlatIndex(0, _handle=h.value)
        return self._base


def load(path, *, mmap=False):
    """Loads an index saved by qann or by this package (.qann format 1..13);
    returns FlatIndex, IVFIndex or RefineIndex. With mmap=True the file is
    mapped read-only and a RefineIndex's raw rows stay in it: the re-rank
    reads them in place over the host link instead of from a copy in GPU
    memory, so rows larger than the GPU's memory can be served (an add or
    compact copies them into memory first). Results are the same either way."""
    h = C.c_void_p()
    kind = C.c_int()
    fn = _lib.lib.qg_load_mapped if mmap else _lib.lib.qg_load
    check(fn(os.fspath(path).encode(), C.byref(h), C.byref(kind)))
    if kind.value == 1:
        return FlatIndex(0, _handle=h.value)
    if kind.value == 2:
        return IVFIndex(0, 0, _handle=h.value)
    return RefineIndex(_handle=h.value)


Index = DenseIndex


class Server:
    """Continuous-batching server over one device-resident index.

    Requests carry their own k, nprobe and filter; worker slots (one CUDA
    stream each) take the oldest waiting requests as soon as they are free,
    up to max_batch at a time while the estimated device memory of all
    batches in flight fits mem_budget bytes, and search each batch as one
    mixed batch. Every request gets the results it gets searched alone. Over
    a RefineIndex, requests with a filter narrow enough for its exact direct
    scan (at most 6 * nlist allowed ids) run on one extra worker of their own.
    """

    def __init__(self, index: DenseIndex, *, slots: int = 4, max_batch: int = 512, mem_budget: int = 2 << 30):
        self._index = index
        self._dim = index.dim()
        h = C.c_void_p()
        check(_lib.lib.qg_server_create(index._h, int(slots), int(max_batch), int(mem_budget), C.byref(h)))
        self._s = h
        self._k = {}

    def close(self) -> None:
        s = getattr(self, "_s", None)
        if s is not None and s.value:
            _lib.lib.qg_server_free(s)
            self._s = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_filter(self, words) -> int:
        """Registers an allowed-slot bitmap (uint64 words); returns its filter id."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        fid = C.c_int()
        check(_lib.lib.qg_server_add_filter(self._s, w.ctypes.data, w.size, C.byref(fid)))
        return fid.value

    def submit(self, query, k: int, *, nprobe: int | None = None, allowed=None, filter_id: int = -1) -> int:
        """Queues one query; returns a ticket for result()."""
        q = _f32_rows(np.asarray(query, np.float32).reshape(1, -1), self._dim, "query")
        t = C.c_uint64()
        np_ = 0 if nprobe is None else int(nprobe)
        if allowed is not None:
            al = _ids(allowed)
            check(_lib.lib.qg_server_submit(self._s, q.ctypes.data, int(k), np_, al.ctypes.data, al.size, -1,
                                            C.byref(t)))
        else:
            check(_lib.lib.qg_server_submit(self._s, q.ctypes.data, int(k), np_, None, 0, int(filter_id), C.byref(t)))
        self._k[t.value] = int(k)
        return t.value

    def result(self, ticket: int):
        """(ids int64 (k,), distances float32 (k,), latency in seconds) of a ticket."""
        k = self._k.pop(ticket)
        ids = np.empty(k, np.int64)
        d = np.empty(k, np.float32)
        lat = C.c_double()
        check(_lib.lib.qg_server_wait(self._s, C.c_uint64(ticket), ids.ctypes.data, d.ctypes.data, C.byref(lat)))
        return ids, d, lat.value * 1e-6

    def replay(self, queries, ks, arrivals_s, *, nprobes=None, filter_ids=None):
        """Open-loop trace: request i arrives arrivals_s[i] seconds after the
        start with k = ks[i]. Returns (ids (nq, max k), distances, latencies s)."""
        q = _f32_rows(queries, self._dim, "query")
        nq = q.shape[0]
        ks = np.ascontiguousarray(ks, dtype=np.int32)
        kmax = int(ks.max()) if nq else 1
        arr = np.ascontiguousarray(np.asarray(arrivals_s, np.float64) * 1e6)
        npb = None if nprobes is None else np.ascontiguousarray(nprobes, dtype=np.int32)
        fid = None if filter_ids is None else np.ascontiguousarray(filter_ids, dtype=np.int32)
        ids = np.empty((nq, kmax), np.int64)
        d = np.empty((nq, kmax), np.float32)
        lat = np.empty(nq, np.float64)
        check(_lib.lib.qg_server_replay(self._s, q.ctypes.data, nq, ks.ctypes.data,
                                        None if npb is None else npb.ctypes.data,
                                        None if fid is None else fid.ctypes.data, arr.ctypes.data, kmax,
                                        ids.ctypes.data, d.ctypes.data, lat.ctypes.data))
        return ids, d, lat * 1e-6

    def stats(self) -> dict:
        c, b, p = C.c_int64(), C.c_int64(), C.c_int64()
        check(_lib.lib.qg_server_stats(self._s, C.byref(c), C.byref(b), C.byref(p)))
        return {"completed": c.value, "batches": b.value, "peak_in_flight_bytes": p.value}
