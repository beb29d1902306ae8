"""Test infrastructure: ctypes driver for oracle/liboracle.so, this project's
C restatement of the reference search path (oracle/qann_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it; it is
the checker, never the thing measured or shipped. Build it with
``make -C oracle liboracle.so``.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "liboracle.so"
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C oracle liboracle.so`")
        L = C.CDLL(str(LIB_PATH))
        vp, sz = C.c_void_p, C.c_size_t
        L.or_l2.argtypes = [vp, vp, sz]
        L.or_l2.restype = C.c_float
        L.or_ip.argtypes = [vp, vp, sz]
        L.or_ip.restype = C.c_float
        for f in ("or_inner_table", "or_list_term", "or_adc_table"):
            getattr(L, f).argtypes = [vp, vp, sz, sz, vp]
        L.or_quantize_lut.argtypes = [vp, sz, vp, vp, vp]
        L.or_build_quantize_lut.argtypes = [vp, vp, C.c_float, sz, vp, vp, vp, vp]
        L.or_fast_scan_block.argtypes = [vp, vp, sz, vp]
        L.or_fast_scan_block_mask.argtypes = [vp, vp, sz, C.c_uint16, vp]
        L.or_fast_scan_block_mask.restype = C.c_uint32
        L.or_encode16.argtypes = [vp, vp, sz, sz, vp]
        L.or_normalize_row.argtypes = [vp, sz, vp]
        L.or_normalize_row.restype = C.c_int
        L.or_ivf_fs_query.argtypes = [vp, sz, sz, C.c_int, vp, sz, vp, vp, vp, vp, vp, vp, vp, vp, sz, sz, vp, C.c_int,
                                      vp, vp]
        L.or_ivf_fs_query.restype = sz
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return None if a is None else a.ctypes.data


def l2(a, b):
    a, b = _f(a), _f(b)
    return np.float32(lib().or_l2(_p(a), _p(b), a.size))


def ip(a, b):
    a, b = _f(a), _f(b)
    return np.float32(lib().or_ip(_p(a), _p(b), a.size))


def _table(fn, v, yt, m, sd):
    v, yt = _f(v), _f(yt)
    out = np.empty(m * 16, np.float32)
    getattr(lib(), fn)(_p(v), _p(yt), m, sd, _p(out))
    return out


def inner_table(q, yt, m, sd):
    return _table("or_inner_table", q, yt, m, sd)


def list_term(c, yt, m, sd):
    return _table("or_list_term", c, yt, m, sd)


def adc_table(r, yt, m, sd):
    return _table("or_adc_table", r, yt, m, sd)


def quantize_lut(table):
    t = _f(table)
    m = t.size // 16
    lut = np.empty(m * 16, np.uint8)
    s, o = np.empty(1, np.float32), np.empty(1, np.float32)
    lib().or_quantize_lut(_p(t), m, _p(lut), _p(s), _p(o))
    return lut, s[0], o[0]


def build_quantize_lut(B, Cq, A):
    B, Cq = _f(B), _f(Cq)
    m = B.size // 16
    table = np.empty(m * 16, np.float32)
    lut = np.empty(m * 16, np.uint8)
    s, o = np.empty(1, np.float32), np.empty(1, np.float32)
    lib().or_build_quantize_lut(_p(B), _p(Cq), C.c_float(A), m, _p(table), _p(lut), _p(s), _p(o))
    return table, lut, s[0], o[0]


def fast_scan_block_mask(lut, block, m, limit):
    lut = np.ascontiguousarray(lut, np.uint8)
    block = np.ascontiguousarray(block, np.uint8)
    out = np.empty(32, np.uint16)
    mask = lib().or_fast_scan_block_mask(_p(lut), _p(block), m, limit, _p(out))
    return mask, out


def encode16(residual, yt, m, sd):
    r, yt = _f(residual), _f(yt)
    out = np.empty(m, np.uint8)
    lib().or_encode16(_p(r), _p(yt), m, sd, _p(out))
    return out


def normalize_row(x):
    x = _f(x)
    out = np.empty_like(x)
    if lib().or_normalize_row(_p(x), x.size, _p(out)):
        raise ValueError("cosine metric needs non-zero vectors")
    return out


class IVFArrays:
    """Plain-array view of an IVF fast-scan index for the oracle: built from a
    `.qann` file through this package's own reader (oracle/qann_file.py)."""

    def __init__(self, dim, m, sd, mode, yt, B, centers, codes, slots, offsets, sizes, deleted):
        self.dim, self.m, self.sd, self.mode = dim, m, sd, mode
        self.yt, self.B, self.centers = _f(yt), None if B is None else _f(B), _f(centers)
        self.codes = np.ascontiguousarray(codes, np.uint8)
        self.slots = np.ascontiguousarray(slots, np.uint32)
        self.offsets = np.ascontiguousarray(offsets, np.uint64)
        self.sizes = np.ascontiguousarray(sizes, np.uint32)
        self.deleted = None if deleted is None else np.ascontiguousarray(deleted, np.uint64)

    def query(self, q, probes, pterm, k, semantics=1):
        q = _f(q)
        probes = np.ascontiguousarray(probes, np.uint32)
        pterm = _f(pterm)
        d = np.empty(k, np.float32)
        s = np.empty(k, np.uint32)
        n = lib().or_ivf_fs_query(_p(q), self.dim, self.m, self.mode, _p(self.yt), self.sd, _p(self.B),
                                  _p(self.centers), _p(self.codes), _p(self.slots), _p(self.offsets), _p(self.sizes),
                                  _p(probes), _p(pterm), probes.size, k, _p(self.deleted), semantics, _p(d), _p(s))
        return d[:n], s[:n]
