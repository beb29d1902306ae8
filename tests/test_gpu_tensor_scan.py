"""The fast-scan on the tensor cores (list-major int8 MMA over one-hot codes
and rounded LUTs) against the query-major kernel and the reference library:
the same ids and the same distance bits, on the reference-built indexes with
per-list L2 tables (plain, cosine, custom ids with deletions), at probe
counts past the first wave's 16, and on a clustered set whose lists are
probed by many queries at once (several units per list)."""
import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu

GEN_L2 = ["l2", "cos_l2", "l2_custom_del"]


@pytest.fixture
def tensor_scan_mode():
    yield
    qb.set_tensor_scan(1)


def _both(idx, q, k):
    qb.set_tensor_scan(0)
    base = idx.batch_query(q, k)
    before = qb.tensor_scan_counts()["calls"]
    qb.set_tensor_scan(2)
    got = idx.batch_query(q, k)
    used = qb.tensor_scan_counts()["calls"] - before
    return base, got, used


@pytest.mark.parametrize("nprobe", [17, 40, 100])
@pytest.mark.parametrize("kind", ["ivf", "refine"])
@pytest.mark.parametrize("name", GEN_L2)
def test_tensor_scan_equals_query_major_and_reference(golden, ref, tensor_scan_mode, kind, name, nprobe):
    path = golden / "gen" / f"{kind}_{name}.qann"
    idx = qb.load(path)
    ivf = idx.base if kind == "refine" else idx
    nprobe = min(nprobe, ivf.nlist)
    ivf.nprobe = nprobe
    q = np.load(golden / "gen" / "queries.npy")
    (i0, d0), (i1, d1), used = _both(idx, q, 10)
    assert used >= 1, "the tensor-core scan did not run"
    np.testing.assert_array_equal(i1, i0)
    assert d1.tobytes() == d0.tobytes()
    theirs = ref.load(path)
    theirs_ivf = theirs.base if kind == "refine" else theirs
    theirs_ivf.nprobe = nprobe
    ri, rd = theirs.batch_query(q, 10)
    np.testing.assert_array_equal(i1, ri)
    assert d1.tobytes() == rd.tobytes()


def test_tensor_scan_many_queries_per_list(ref, tmp_path, tensor_scan_mode):
    """4,000 queries over 120 lists: each list is probed by hundreds of
    queries, so it is cut into several units of the GEMM's query dimension,
    and its vectors span several 128-row tiles."""
    rng = np.random.default_rng(4)
    d, n = 48, 30_000
    c = rng.normal(size=(60, d)).astype(np.float32)
    x = (c[rng.integers(0, 60, n)] + 0.3 * rng.normal(size=(n, d))).astype(np.float32)
    q = (c[rng.integers(0, 60, 4000)] + 0.3 * rng.normal(size=(4000, d))).astype(np.float32)
    theirs = ref.IVFIndex(d, 120, 40)
    theirs.enable_pq(24, fast_scan=True)
    theirs.train(x, seed=3)
    r = ref.RefineIndex(theirs, 10)
    r.add(x)
    path = tmp_path / "many.qann"
    r.save(path)
    mine = qb.load(path)
    (i0, d0), (i1, d1), used = _both(mine, q, 10)
    assert used >= 1
    np.testing.assert_array_equal(i1, i0)
    assert d1.tobytes() == d0.tobytes()
    ri, rd = r.batch_query(q, 10)
    np.testing.assert_array_equal(i1, ri)
    assert d1.tobytes() == rd.tobytes()
