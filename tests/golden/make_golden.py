"""Writes the golden fixtures the parity tests read (run from the repo root:
``python tests/golden/make_golden.py``). Needs the reference sources (for the
copies) and ``oracle/_ref/libqann_ref.so`` (``make -C oracle``).

1. ``ref/``: the reference's own cross-version fixtures for the dense path,
   copied unchanged from its ``tests/data`` (index files saved by qann
   releases plus the query results those releases returned).
2. ``gen/``: indexes built by the reference library itself on seeded
   synthetic data, one per fast-scan scoring mode, with the reference's query
   results. These pin the CUDA path to the reference's current code.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402

HERE = pathlib.Path(__file__).resolve().parent
REF_DATA = pathlib.Path(os.environ.get("QANN_REFERENCE", "/root/reference")) / "tests" / "data"

# (index file, queries file) of the reference fixtures on the dense search path
REF_CASES = [
    ("v4_ivf_fs", "v4_queries"),
    ("v11_ivf_cos_fs", "v11_cos_queries"),
    ("v12_ivf_cos_l2", "v12_cos_queries"),
    ("v9_ip_refine_ivf_fs", "v9_ip_queries"),
    ("v1_flat", "v1_queries"),
    ("v2_flat", "v2_queries"),
    ("v3_flat", "v3_queries"),
    ("v4_flat", "v4_queries"),
    ("v5_flat", "v5_queries"),
    ("v9_ip_flat", "v9_ip_queries"),
    ("v1_refine", "v1_queries"),
    ("v2_refine", "v2_queries"),
    ("v3_refine", "v3_queries"),
    ("v10_refine", "v10_queries"),
]


def copy_reference():
    out = HERE / "ref"
    out.mkdir(exist_ok=True)
    for name, qn in REF_CASES:
        for f in (f"{name}.qann", f"{name}_ids.npy", f"{name}_dists.npy", f"{qn}.npy"):
            shutil.copy2(REF_DATA / f, out / f)


def clustered(rng, n, d, centres=40, sigma=0.15):
    c = rng.normal(size=(centres, d)).astype(np.float32)
    lab = rng.integers(0, centres, size=n)
    return (c[lab] + sigma * rng.normal(size=(n, d))).astype(np.float32)


# name -> (metric, cosine_inner_product override or None, precomputed_tables, custom_ids, deletions)
GEN_CASES = {
    "l2": (ref.L2, None, True, False, False),
    "l2_adc": (ref.L2, None, False, False, False),
    "ip": (ref.INNER_PRODUCT, None, True, False, False),
    "cos_ip": (ref.COSINE, True, True, False, False),
    "cos_l2": (ref.COSINE, False, True, False, False),
    "l2_custom_del": (ref.L2, None, True, True, True),
}


def generate():
    out = HERE / "gen"
    out.mkdir(exist_ok=True)
    ref.set_num_threads(1)
    rng = np.random.default_rng(7)
    d, n, nq = 32, 3000, 40
    x = clustered(rng, n, d)
    q = clustered(rng, nq, d)
    if True:
        q[:, :] = q * rng.uniform(0.5, 2.0, size=(nq, 1)).astype(np.float32)
    np.save(out / "queries.npy", q)
    for name, (metric, cos_ip, pre, custom, dele) in GEN_CASES.items():
        base = ref.IVFIndex(d, 100, 8, metric=metric)
        base.enable_pq(16, fast_scan=True)
        base.train(x, seed=3)
        if cos_ip is not None:
            base.cosine_inner_product = cos_ip
        base.precomputed_tables = pre
        ids = np.arange(5000, 5000 + n, dtype=np.int64) if custom else None
        # the bare IVF index (custom ids / deletions apply to it)
        ivf = ref.IVFIndex(d, 100, 8, metric=metric, custom_ids=custom)
        ivf.enable_pq(16, fast_scan=True)
        ivf.train(x, seed=3)
        if cos_ip is not None:
            ivf.cosine_inner_product = cos_ip
        ivf.precomputed_tables = pre
        ivf.add(x, ids=ids)
        if dele:
            ivf.remove(ids[::7] if custom else np.arange(0, n, 7))
        ivf.save(out / f"ivf_{name}.qann")
        i1, d1 = ivf.batch_query(q, 10)
        np.save(out / f"ivf_{name}_ids.npy", i1)
        np.save(out / f"ivf_{name}_dists.npy", d1)
        # RefineIndex over the same kind of base
        r = ref.RefineIndex(base, 5, custom_ids=custom)
        r.add(x, ids=ids)
        if dele:
            r.remove(ids[::7] if custom else np.arange(0, n, 7))
        r.save(out / f"refine_{name}.qann")
        i2, d2 = r.batch_query(q, 10)
        np.save(out / f"refine_{name}_ids.npy", i2)
        np.save(out / f"refine_{name}_dists.npy", d2)
        print(name, "ok")


if __name__ == "__main__":
    if REF_DATA.exists():
        copy_reference()
    generate()
