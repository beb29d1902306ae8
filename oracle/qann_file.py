"""Test infrastructure: a numpy reader of `.qann` files for the oracle (IVF,
Flat and Refine bodies; reference src/ivf_index.cpp:976-1122,
src/flat_index.cpp:115-133, src/refine_index.cpp:168-213, src/id_map.cpp:207-241),
plus the oracle-side coarse step (reference src/ivf_index.cpp:305-356) and a
whole fast-scan query built on oracle/qann_oracle.c.
"""
from __future__ import annotations

import numpy as np

from . import oracle as orc

MAGIC = 0x4E4E4151


class _R:
    def __init__(self, b: bytes):
        self.b, self.p = b, 0

    def pod(self, dt):
        v = np.frombuffer(self.b, dtype=dt, count=1, offset=self.p)[0]
        self.p += np.dtype(dt).itemsize
        return v

    def vec(self, dt):
        n = int(self.pod(np.uint64))
        a = np.frombuffer(self.b, dtype=dt, count=n, offset=self.p).copy()
        self.p += n * np.dtype(dt).itemsize
        return a

    def pad(self):
        n = int(self.pod(np.uint32))
        self.p += n

    def header(self):
        assert int(self.pod(np.uint32)) == MAGIC
        ver = int(self.pod(np.uint32))
        kind = int(self.pod(np.uint8))
        return kind, ver


def _idmap(r, ver):
    custom = int(r.pod(np.uint8))
    slots = int(r.pod(np.uint64))
    if ver >= 3:
        r.pod(np.int64)
    labels = r.vec(np.int64)
    deleted = r.vec(np.uint8)
    return {"custom": custom, "slots": slots, "labels": labels, "deleted": deleted}


def _meta(r):
    ncols = int(r.pod(np.uint64))
    for _ in range(ncols):
        r.vec(np.uint8)
        t = int(r.pod(np.uint8))
        r.vec(np.uint8)
        if t in (0, 1):
            r.vec(np.int64)
        else:
            r.vec(np.uint32)
            nd = int(r.pod(np.uint64))
            for _ in range(nd):
                r.vec(np.uint8)


def _fs_unpack(blocks, n, m):
    blk = blocks.reshape(-1, m, 16)
    out = np.empty((n, m), np.uint8)
    for v in range(n):
        b, p = divmod(v, 32)
        row = blk[b, :, p % 16]
        out[v] = (row & 15) if p < 16 else (row >> 4)
    return out


def _ivf(r, ver):
    d = {}
    d["dim"], d["nlist"], d["nprobe"] = int(r.pod(np.uint64)), int(r.pod(np.uint64)), int(r.pod(np.uint64))
    n_total = int(r.pod(np.uint64))
    d["trained"], d["pq_distance"] = int(r.pod(np.uint8)), int(r.pod(np.uint8))
    d["centroids"] = r.vec(np.float32).reshape(-1, d["dim"]) if True else None
    assert int(r.pod(np.uint8)) == 1, "oracle reader handles PQ lists only"
    pdim, m, K = int(r.pod(np.uint64)), int(r.pod(np.uint64)), int(r.pod(np.uint64))
    d["pq"] = r.vec(np.float32).reshape(m, K, pdim // m)
    d["m"], d["K"] = m, K
    d["fast_scan"] = int(r.pod(np.uint8)) if ver >= 4 else 0
    if ver >= 8:
        d["rotate"] = int(r.pod(np.uint8))
        d["rotation"] = r.vec(np.float32)
    if ver >= 7:
        assert int(r.pod(np.uint8)) == 0
    ids, codes = [], []
    for _ in range(d["nlist"]):
        li = r.vec(np.uint32)
        c = r.vec(np.uint8)
        ids.append(li)
        codes.append(_fs_unpack(c, li.size, m) if d["fast_scan"] else c.reshape(li.size, m))
    d["ids"], d["codes"] = ids, codes
    d["idmap"] = _idmap(r, ver) if ver >= 2 else None
    d["use_precomputed"] = int(r.pod(np.uint8)) if ver >= 3 else 1
    d["metric"] = int(r.pod(np.uint8)) if ver >= 5 else 0
    if ver >= 9:
        _meta(r)
    d["cosine_ip"] = int(r.pod(np.uint8)) if ver >= 12 else 1
    d["resid"] = r.vec(np.float32).reshape(-1, d["dim"]) if ver >= 13 else np.zeros((0, d["dim"]), np.float32)
    return d


def read(path):
    """Returns {"kind": 2, "ivf": {...}} or {"kind": 3, "ivf": ..., "rows": ..., "idmap": ...}."""
    r = _R(open(path, "rb").read())
    kind, ver = r.header()
    if kind == 2:
        return {"kind": 2, "ivf": _ivf(r, ver)}
    assert kind == 3, "oracle reader handles IVF and Refine(IVF) files"
    kf = int(r.pod(np.uint64))
    count = int(r.pod(np.uint64))
    bk, bver = r.header()
    assert bk == 2
    ivf = _ivf(r, bver)
    n = int(r.pod(np.uint64))
    if ver >= 10:
        r.pad()
    rows = np.frombuffer(r.b, np.float32, count=n, offset=r.p).reshape(count, -1).copy()
    r.p += n * 4
    idmap = _idmap(r, ver) if ver >= 2 else None
    return {"kind": 3, "k_factor": kf, "ivf": ivf, "rows": rows, "idmap": idmap}


def scan_mode(ivf) -> int:
    """0 L2 precomputed, 1 L2 per-list ADC, 2 inner product, 3 cosine by inner
    product (reference src/ivf_index.cpp:66-81, :436-456)."""
    if ivf["metric"] == 2:
        return 2
    if ivf["metric"] == 1 and ivf["cosine_ip"]:
        return 3
    too_big = ivf["nlist"] * ivf["m"] * 16 * 4 > (256 << 20)
    return 1 if (not ivf["use_precomputed"] or too_big) else 0


def arrays(ivf):
    m, sd = ivf["m"], ivf["pq"].shape[2]
    yt = np.ascontiguousarray(ivf["pq"].transpose(0, 2, 1))   # m, sd, K
    centers = ivf["resid"] if ivf["resid"].size else ivf["centroids"]
    mode = scan_mode(ivf)
    B = None
    if mode == 0:
        B = np.stack([orc.list_term(c, yt, m, sd) for c in centers])
    sizes = np.array([a.size for a in ivf["ids"]], np.uint32)
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    codes = np.concatenate(ivf["codes"]) if sizes.sum() else np.zeros((0, m), np.uint8)
    slots = np.concatenate(ivf["ids"]) if sizes.sum() else np.zeros(0, np.uint32)
    deleted = None
    if ivf["idmap"] is not None and ivf["idmap"]["deleted"].any():
        dl = ivf["idmap"]["deleted"]
        words = np.zeros((dl.size + 63) // 64, np.uint64)
        for s in np.nonzero(dl)[0]:
            words[s >> 6] |= np.uint64(1) << np.uint64(s & 63)
        deleted = words
    return orc.IVFArrays(ivf["dim"], m, sd, mode, yt, B, centers, codes, slots, offsets, sizes, deleted)


def coarse(ivf, q, nprobe):
    """The nprobe lists nearest to q by (exact score, list), and each probe's
    term: A (L2 / IP) or the cosine base (A + 1) - |e|^2."""
    ip = ivf["metric"] == 2
    scores = np.array([-orc.ip(q, c) if ip else orc.l2(q, c) for c in ivf["centroids"]], np.float32)
    order = np.lexsort((np.arange(scores.size), scores))[:nprobe]
    pterm = scores[order].copy()
    centers = ivf["resid"] if ivf["resid"].size else None
    if centers is not None:
        pterm = np.array([orc.l2(q, centers[l]) for l in order], np.float32)
    if scan_mode(ivf) == 3:
        cen = centers if centers is not None else ivf["centroids"]
        sq = np.array([orc.ip(cen[l], cen[l]) for l in order], np.float32)
        pterm = ((pterm + np.float32(1.0)).astype(np.float32) - sq).astype(np.float32)
    return order.astype(np.uint32), pterm
