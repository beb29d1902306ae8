"""Test infrastructure: ctypes driver for the reference qann C++ core.

``oracle/_ref/libqann_ref.so`` is the reference's own C++ sources compiled by
``oracle/Makefile`` (no BLAS, AVX2+FMA) plus ``oracle/ref_shim.cpp``. This
module exposes it with the reference's Python API shape (``IVFIndex``,
``RefineIndex``, ``FlatIndex``, ``load``) so tests can run the reference and
this project's CUDA path on the same inputs.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
import this module; the product package never does.

Import this module before the first GPU call in a process; it sets
``QANN_DISABLE_AVX512=1`` (read once, when the library loads) unless the
caller set it already, pinning the reference's AVX2 distance kernels
(reference ``src/distance.cpp:180-185``) whose accumulation order the CUDA
kernels reproduce.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "_ref" / "libqann_ref.so"

_lib = None


class RefError(Exception):
    pass


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        os.environ.setdefault("QANN_DISABLE_AVX512", "1")
        if not LIB_PATH.exists():
            raise RefError(f"{LIB_PATH} is missing: run `make -C oracle` where the reference sources exist")
        L = C.CDLL(str(LIB_PATH))
        vp, sz, i64p, f32p = C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p
        L.ref_last_error.restype = C.c_char_p
        L.ref_set_num_threads.argtypes = [sz]
        L.ref_ivf_create.argtypes = [sz, sz, sz, C.c_int, C.c_int, C.POINTER(vp)]
        L.ref_flat_create.argtypes = [sz, C.c_int, C.c_int, C.POINTER(vp)]
        L.ref_refine_create.argtypes = [vp, sz, C.c_int, C.POINTER(vp)]
        L.ref_free.argtypes = [vp]
        L.ref_ivf_enable_pq.argtypes = [vp, sz, sz, C.c_int, C.c_int]
        L.ref_ivf_train.argtypes = [vp, f32p, sz, sz, C.c_int64, C.c_int, sz]
        L.ref_add.argtypes = [vp, f32p, sz, i64p, i64p]
        L.ref_remove.argtypes = [vp, i64p, sz, C.POINTER(sz)]
        L.ref_compact.argtypes = [vp, C.POINTER(sz)]
        L.ref_query_batch.argtypes = [vp, f32p, sz, sz, i64p, sz, i64p, f32p]
        L.ref_save.argtypes = [vp, C.c_char_p]
        L.ref_load.argtypes = [C.c_char_p, C.POINTER(vp), C.POINTER(C.c_int)]
        L.ref_size.argtypes = [vp]
        L.ref_size.restype = sz
        L.ref_ivf_set_nprobe.argtypes = [vp, sz]
        L.ref_ivf_nprobe.argtypes = [vp]
        L.ref_ivf_nprobe.restype = sz
        L.ref_ivf_cosine_ip.argtypes = [vp]
        L.ref_ivf_set_cosine_ip.argtypes = [vp, C.c_int]
        L.ref_ivf_precomputed.argtypes = [vp]
        L.ref_ivf_set_precomputed.argtypes = [vp, C.c_int]
        L.ref_ivf_set_filter_probe_scaling.argtypes = [vp, C.c_int]
        L.ref_refine_set_k_factor.argtypes = [vp, sz]
        L.ref_quantize_lut.argtypes = [f32p, sz, vp, f32p, f32p]
        L.ref_quantize_lut_scalar.argtypes = [f32p, sz, vp, f32p, f32p]
        L.ref_build_quantize_lut.argtypes = [f32p, f32p, C.c_float, sz, f32p, vp, f32p, f32p]
        L.ref_fast_scan_block_mask.argtypes = [vp, vp, sz, C.c_uint16, vp]
        L.ref_fast_scan_block_mask.restype = C.c_uint32
        L.ref_fast_scan_block_mask_scalar.argtypes = [vp, vp, sz, C.c_uint16, vp]
        L.ref_fast_scan_block_mask_scalar.restype = C.c_uint32
        L.ref_l2_distance.argtypes = [f32p, f32p, sz]
        L.ref_l2_distance.restype = C.c_float
        L.ref_inner_product.argtypes = [f32p, f32p, sz]
        L.ref_inner_product.restype = C.c_float
        L.ref_topk_run.argtypes = [f32p, vp, sz, sz, vp, f32p, C.POINTER(sz)]
        L.ref_kmeans.argtypes = [f32p, sz, sz, sz, sz, sz, C.c_int64, C.c_int, C.c_int, f32p, vp]
        L.ref_assign_nearest.argtypes = [f32p, sz, sz, f32p, sz, sz, vp]
        L.ref_pq_tables.argtypes = [f32p, sz, sz, sz, f32p, f32p, f32p, f32p, f32p]
        L.ref_pq_encode.argtypes = [f32p, sz, sz, sz, f32p, sz, vp]
        L.ref_pca_rotation.argtypes = [f32p, sz, sz, sz, f32p]
        L.ref_symmetric_eigen.argtypes = [vp, sz, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _check(rc):
    if rc == 0:
        return
    msg = lib().ref_last_error().decode()
    if rc == 1:
        raise ValueError(msg)
    if rc == 2:
        raise RuntimeError(msg)
    raise RefError(msg)


def set_num_threads(n: int) -> None:
    lib().ref_set_num_threads(n)


L2, COSINE, INNER_PRODUCT = 0, 1, 2
EMEANS, LLOYD = 0, 1


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


class _Index:
    kind = 0

    def __init__(self, handle, dim, keep=None):
        self._h = C.c_void_p(handle)
        self._dim = dim
        self._keep = keep

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value and _lib is not None:
            _lib.ref_free(self._h)
            self._h = None

    def dim(self):
        return self._dim

    def size(self):
        return lib().ref_size(self._h)

    def add(self, data, ids=None):
        x = _f32(data)
        n = x.shape[0]
        out = np.empty(n, np.int64)
        idarr = None if ids is None else np.ascontiguousarray(ids, dtype=np.int64)
        _check(lib().ref_add(self._h, _ptr(x), n, _ptr(idarr), _ptr(out)))
        return out

    def remove(self, ids):
        a = np.ascontiguousarray(ids, dtype=np.int64)
        r = C.c_size_t()
        _check(lib().ref_remove(self._h, _ptr(a), a.size, C.byref(r)))
        return r.value

    def compact(self):
        r = C.c_size_t()
        _check(lib().ref_compact(self._h, C.byref(r)))
        return r.value

    def batch_query(self, q, k, *, allowed=None):
        q = _f32(q)
        if q.ndim == 1:
            q = q[None]
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int64)
        d = np.empty((nq, k), np.float32)
        al = None if allowed is None else np.ascontiguousarray(allowed, dtype=np.int64)
        _check(lib().ref_query_batch(self._h, _ptr(q), nq, k, _ptr(al), 0 if al is None else al.size,
                                     _ptr(ids), _ptr(d)))
        return ids, d

    def save(self, path):
        _check(lib().ref_save(self._h, str(path).encode()))


class IVFIndex(_Index):
    kind = 2

    def __init__(self, dim, nlist, nprobe=10, *, custom_ids=False, metric=L2, _handle=None):
        if _handle is None:
            h = C.c_void_p()
            _check(lib().ref_ivf_create(dim, nlist, nprobe, int(metric), int(custom_ids), C.byref(h)))
            _handle = h.value
        super().__init__(_handle, dim)

    def enable_pq(self, m, centroids_per_subspace=None, *, fast_scan=False, rotate=False):
        K = centroids_per_subspace or (16 if fast_scan else 256)
        _check(lib().ref_ivf_enable_pq(self._h, m, K, int(fast_scan), int(rotate)))

    def train(self, data, max_iters=10, seed=None, *, clustering=EMEANS, passes=2):
        x = _f32(data)
        _check(lib().ref_ivf_train(self._h, _ptr(x), x.shape[0], max_iters, -1 if seed is None else seed,
                                   int(clustering), passes))

    @property
    def nprobe(self):
        return lib().ref_ivf_nprobe(self._h)

    @nprobe.setter
    def nprobe(self, v):
        _check(lib().ref_ivf_set_nprobe(self._h, v))

    @property
    def cosine_inner_product(self):
        return bool(lib().ref_ivf_cosine_ip(self._h))

    @cosine_inner_product.setter
    def cosine_inner_product(self, v):
        _check(lib().ref_ivf_set_cosine_ip(self._h, int(v)))

    @property
    def precomputed_tables(self):
        return bool(lib().ref_ivf_precomputed(self._h))

    @precomputed_tables.setter
    def precomputed_tables(self, v):
        _check(lib().ref_ivf_set_precomputed(self._h, int(v)))

    @property
    def filter_probe_scaling(self):
        raise AttributeError("write-only in the shim")

    @filter_probe_scaling.setter
    def filter_probe_scaling(self, v):
        lib().ref_ivf_set_filter_probe_scaling(self._h, int(v))


class FlatIndex(_Index):
    kind = 1

    def __init__(self, dim, *, custom_ids=False, metric=L2, _handle=None):
        if _handle is None:
            h = C.c_void_p()
            _check(lib().ref_flat_create(dim, int(metric), int(custom_ids), C.byref(h)))
            _handle = h.value
        super().__init__(_handle, dim)


class RefineIndex(_Index):
    kind = 3

    def __init__(self, base=None, k_factor=10, *, custom_ids=False, _handle=None, _dim=None):
        if _handle is None:
            h = C.c_void_p()
            _check(lib().ref_refine_create(base._h, k_factor, int(custom_ids), C.byref(h)))
            _handle, _dim = h.value, base.dim()
        super().__init__(_handle, _dim, keep=base)
        self.base = base if base is not None else IVFIndexView(self)

    @property
    def k_factor(self):
        raise AttributeError("write-only in the shim")

    @k_factor.setter
    def k_factor(self, v):
        _check(lib().ref_refine_set_k_factor(self._h, v))


class IVFIndexView:
    """The IVF base of a loaded RefineIndex: the shim reaches it through the refine handle."""

    def __init__(self, owner):
        self._h = owner._h

    nprobe = IVFIndex.nprobe
    cosine_inner_product = IVFIndex.cosine_inner_product
    precomputed_tables = IVFIndex.precomputed_tables
    filter_probe_scaling = IVFIndex.filter_probe_scaling


def load(path, dim=None):
    """Loads a ``.qann`` file with the reference's own loader. ``dim`` is the
    vector dimension (the shim does not report it); batch_query infers it from
    the query array when omitted."""
    h = C.c_void_p()
    kind = C.c_int()
    _check(lib().ref_load(str(path).encode(), C.byref(h), C.byref(kind)))
    if kind.value == 1:
        return FlatIndex(dim, _handle=h.value)
    if kind.value == 2:
        return IVFIndex(dim, 0, _handle=h.value)
    if kind.value == 3:
        return RefineIndex(_handle=h.value, _dim=dim)
    lib().ref_free(h)
    raise RefError("unsupported index kind in this shim")


# ---- kernels of the path ------------------------------------------------------

def quantize_lut(table, scalar=False):
    t = _f32(table)
    m = t.size // 16
    lut = np.empty(m * 16, np.uint8)
    s, o = C.c_float(), C.c_float()
    fn = lib().ref_quantize_lut_scalar if scalar else lib().ref_quantize_lut
    fn(_ptr(t), m, _ptr(lut), C.byref(s), C.byref(o))
    return lut, np.float32(s.value), np.float32(o.value)


def build_quantize_lut(B, C_, A):
    B = _f32(B)
    C_ = _f32(C_)
    m = B.size // 16
    table = np.empty(m * 16, np.float32)
    lut = np.empty(m * 16, np.uint8)
    s, o = C.c_float(), C.c_float()
    lib().ref_build_quantize_lut(_ptr(B), _ptr(C_), C.c_float(A), m, _ptr(table), _ptr(lut), C.byref(s), C.byref(o))
    return table, lut, np.float32(s.value), np.float32(o.value)


def fast_scan_block_mask(lut, block, m, limit, scalar=False):
    lut = np.ascontiguousarray(lut, np.uint8)
    block = np.ascontiguousarray(block, np.uint8)
    out = np.empty(32, np.uint16)
    fn = lib().ref_fast_scan_block_mask_scalar if scalar else lib().ref_fast_scan_block_mask
    mask = fn(_ptr(lut), _ptr(block), m, limit, _ptr(out))
    return mask, out


def l2_distance(a, b):
    a, b = _f32(a), _f32(b)
    return np.float32(lib().ref_l2_distance(_ptr(a), _ptr(b), a.size))


def inner_product(a, b):
    a, b = _f32(a), _f32(b)
    return np.float32(lib().ref_inner_product(_ptr(a), _ptr(b), a.size))


def topk_run(dist, ids, k):
    dist = _f32(dist)
    ids = np.ascontiguousarray(ids, np.uint64)
    oi = np.empty(k, np.uint64)
    od = np.empty(k, np.float32)
    n = C.c_size_t()
    lib().ref_topk_run(_ptr(dist), _ptr(ids), dist.size, k, _ptr(oi), _ptr(od), C.byref(n))
    return oi[: n.value], od[: n.value]


def kmeans(x, k, iters, seed, *, spherical=False, emeans=False, stride=None, d=None):
    x = _f32(x)
    n = x.shape[0]
    d = d or x.shape[1]
    stride = stride or x.shape[1]
    cent = np.empty((k, d), np.float32)
    assign = np.empty(n, np.uint32)
    _check(lib().ref_kmeans(_ptr(x), n, stride, d, k, iters, -1 if seed is None else seed, int(spherical),
                            int(emeans), _ptr(cent), _ptr(assign)))
    return cent, assign


def assign_nearest(x, c):
    x, c = _f32(x), _f32(c)
    out = np.empty(x.shape[0], np.uint32)
    lib().ref_assign_nearest(_ptr(x), x.shape[0], x.shape[1], _ptr(c), c.shape[0], c.shape[1], _ptr(out))
    return out


def pq_tables(centroids, m, K, q=None, coarse=None, adc=False):
    """centroids: (m, K, sub_dim). Returns (inner C, list term B, adc table) for q / coarse."""
    cen = _f32(centroids)
    dim = m * cen.shape[-1]
    inner = np.empty(m * K, np.float32) if q is not None else None
    lt = np.empty(m * K, np.float32) if coarse is not None else None
    at = np.empty(m * K, np.float32) if (adc and q is not None) else None
    qq = _f32(q) if q is not None else np.zeros(dim, np.float32)
    cc = _f32(coarse) if coarse is not None else np.zeros(dim, np.float32)
    _check(lib().ref_pq_tables(_ptr(cen), dim, m, K, _ptr(qq), _ptr(cc), _ptr(inner), _ptr(lt), _ptr(at)))
    return inner, lt, at


def pq_encode(centroids, m, K, x):
    cen = _f32(centroids)
    x = _f32(x)
    codes = np.empty((x.shape[0], m), np.uint8)
    _check(lib().ref_pq_encode(_ptr(cen), x.shape[1], m, K, _ptr(x), x.shape[0], _ptr(codes)))
    return codes


def pca_rotation(x, m):
    """balanced_pca_rotation (reference src/rotation.cpp:71-130): d x d, row-major."""
    x = _f32(x)
    out = np.empty((x.shape[1], x.shape[1]), np.float32)
    _check(lib().ref_pca_rotation(_ptr(x), x.shape[0], x.shape[1], m, _ptr(out)))
    return out


def symmetric_eigen(a):
    """symmetric_eigen (reference src/rotation.cpp:20-69): (values, vectors as columns)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    d = a.shape[0]
    values, vectors = np.empty(d), np.empty((d, d))
    _check(lib().ref_symmetric_eigen(_ptr(a), d, _ptr(values), _ptr(vectors)))
    return values, vectors
