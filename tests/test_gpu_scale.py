"""Parity at the benchmark's own sizes, not only on small fixtures.

* The 100,000 x 128 uniform workload (IVF 256, PQ 64 x 4-bit fast-scan,
  RefineIndex k_factor 10, nprobe 16, 1,000 queries, k = 10): built by the
  reference library on the CPU and by this library on the GPU from the same
  seeded rows; the saved indexes must be byte-identical and every query must
  return the reference's ids and distance bits.
* The 1,200,000 x 100 angular workload (IVF 4096, PQ 50 x 4-bit, cosine,
  k_factor 10): rebuilt on the GPU and checked against the reference's own
  build of it, pinned in tests/golden/scale/ by make_scale_golden.py (the
  reference takes minutes on one core to train it): the same .qann bytes
  (SHA-256), and the reference's results for 300 queries at nprobe 16, 64 and
  256, ids identical and distances bit-identical.
"""
import hashlib
import json

import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


def _sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def test_small_workload_full_size_matches_reference(ref, tmp_path):
    n, d, nq, k = 100_000, 128, 1_000, 10
    x = np.random.default_rng(0).random((n, d), dtype=np.float32)
    q = np.random.default_rng(1).random((nq, d), dtype=np.float32)
    ref.set_num_threads(8)
    built = {}
    for name, lib in (("mine", qb), ("ref", ref)):
        ivf = lib.IVFIndex(d, 256, 16)
        ivf.enable_pq(64, fast_scan=True)
        ivf.train(x, seed=1)
        r = lib.RefineIndex(ivf, 10)
        r.add(x)
        path = tmp_path / f"{name}.qann"
        r.save(path)
        built[name] = (r, path)
    assert _sha256(built["mine"][1]) == _sha256(built["ref"][1]), "GPU-built index differs from the reference's"
    i_mine, d_mine = built["mine"][0].batch_query(q, k)
    i_ref, d_ref = built["ref"][0].batch_query(q, k)
    np.testing.assert_array_equal(i_mine, i_ref)
    assert d_mine.tobytes() == d_ref.tobytes()


@pytest.fixture(scope="module")
def angular_golden(golden):
    meta_path = golden / "scale" / "angular.json"
    if not meta_path.exists():
        pytest.skip("tests/golden/scale/angular.json not generated")
    return json.loads(meta_path.read_text())


def test_angular_workload_full_size_matches_reference(angular_golden, golden, tmp_path):
    import bench
    cfg = bench.FULL
    assert angular_golden["workload"] == bench.tag(cfg)
    base = bench.mixture(cfg, 0, cfg["n"])
    queries = bench.mixture(cfg, 1, cfg["nq"])[:angular_golden["sample_queries"]]
    ivf = qb.IVFIndex(cfg["d"], cfg["nlist"], 16, metric=qb.Metric.Cosine)
    ivf.enable_pq(cfg["m"], fast_scan=True)
    ivf.train(base, seed=cfg["train_seed"])
    r = qb.RefineIndex(ivf, cfg["kf"])
    r.add(base)
    path = tmp_path / "angular.qann"
    r.save(path)
    assert ivf.cosine_inner_product == angular_golden["cosine_inner_product"]
    assert path.stat().st_size == angular_golden["qann_bytes"]
    assert _sha256(path) == angular_golden["qann_sha256"], "GPU-built angular index differs from the reference's"
    for npb in angular_golden["nprobes"]:
        ivf.nprobe = npb
        ids, d = r.batch_query(queries, cfg["k"])
        want_ids = np.load(golden / "scale" / f"angular_ids_np{npb}.npy")
        want_d = np.load(golden / "scale" / f"angular_dists_np{npb}.npy")
        np.testing.assert_array_equal(ids, want_ids, err_msg=f"nprobe {npb}")
        assert d.tobytes() == want_d.tobytes(), f"nprobe {npb}"
