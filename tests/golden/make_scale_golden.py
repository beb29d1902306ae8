"""Writes the config-scale golden fixtures (run from the repo root:
``python tests/golden/make_scale_golden.py [angular|small]``). Needs
``oracle/_ref/libqann_ref.so`` (``make -C oracle``).

The reference library builds the benchmark's own indexes from the same
seeded generators ``bench.py`` uses, then answers a fixed sample of queries.
Saved under ``scale/``: the SHA-256 of the ``.qann`` file it wrote, the list
sizes, and its query results (ids and distances) at a few nprobe values. The
GPU parity tests rebuild the same index on the device and must reproduce
those bytes and results exactly; the reference's own build of the 1.2M-row
angular index takes minutes on one core, too long for every test run, so its
outputs are pinned here once.
"""
from __future__ import annotations

import hashlib
import json
import os
import pathlib
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
os.environ.setdefault("QANN_DISABLE_AVX512", "1")

import bench  # noqa: E402  (the workload generators)
from oracle import ref  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent / "scale"
SAMPLE = 300   # queries 0..299 of the workload's query set
NPROBES = (16, 64, 256)


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def angular():
    cfg = bench.FULL
    base = bench.mixture(cfg, 0, cfg["n"])
    queries = bench.mixture(cfg, 1, cfg["nq"])[:SAMPLE]
    ref.set_num_threads(os.cpu_count() or 1)
    t = time.time()
    ivf = ref.IVFIndex(cfg["d"], cfg["nlist"], 16, metric=ref.COSINE)
    ivf.enable_pq(cfg["m"], fast_scan=True)
    ivf.train(base, seed=cfg["train_seed"])
    t_train = time.time() - t
    r = ref.RefineIndex(ivf, cfg["kf"])
    r.add(base)
    t_add = time.time() - t - t_train
    with tempfile.TemporaryDirectory() as td:
        path = pathlib.Path(td) / "angular.qann"
        r.save(path)
        digest = sha256(path)
        size = path.stat().st_size
    meta = {"workload": bench.tag(cfg), "qann_sha256": digest, "qann_bytes": size, "sample_queries": SAMPLE,
            "k": cfg["k"], "k_factor": cfg["kf"], "nprobes": list(NPROBES),
            "cosine_inner_product": bool(ivf.cosine_inner_product),
            "reference_build_s": {"train": round(t_train, 1), "add": round(t_add, 1)}}
    for npb in NPROBES:
        ivf.nprobe = npb
        ids, d = r.batch_query(queries, cfg["k"])
        np.save(OUT / f"angular_ids_np{npb}.npy", ids)
        np.save(OUT / f"angular_dists_np{npb}.npy", d)
    (OUT / "angular.json").write_text(json.dumps(meta, indent=1) + "\n")
    print(json.dumps(meta))


if __name__ == "__main__":
    OUT.mkdir(exist_ok=True)
    which = sys.argv[1:] or ["angular"]
    if "angular" in which:
        angular()
