"""The BF16 tensor-core filter (tcgen05 GEMM + exact FP32 recheck) returns
exactly what the exact path returns: flat search in every metric, with
deletions and filters, on random and tie-heavy clustered data, and
nearest-centroid assignment inside IVF training and adding (byte-identical
files). Also checked against the reference library."""
import filecmp

import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def default_mode():
    yield
    qb.set_tensor_filter(1)


def lognormal_rows(seed, n, d):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, d)) * np.exp(rng.normal(0.0, 0.25, size=(n, 1)))
    return x.astype(np.float32)


def clustered(seed, n, d, centres=40, sigma=0.05):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(centres, d)).astype(np.float32)
    return (c[rng.integers(0, centres, size=n)] + sigma * rng.normal(size=(n, d))).astype(np.float32)


def both_modes(fn, max_redone=0.05):
    """fn's result on the exact path and through the filter; the filter must
    have answered the queries itself (few redone after an overflow)."""
    qb.set_tensor_filter(0)
    exact = fn()
    qb.set_tensor_filter(2)
    before = qb.tensor_filter_counts()
    fast = fn()
    after = qb.tensor_filter_counts()
    n = after["queries"] - before["queries"]
    assert n > 0, "the filter did not run"
    assert after["redone"] - before["redone"] <= max_redone * n
    return exact, fast


def assert_same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1].tobytes() == b[1].tobytes()


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("d", [16, 24, 96, 100, 128])
def test_flat_search_identical(metric, d):
    n = 30000
    x = lognormal_rows(d, n, d)
    q = lognormal_rows(d + 1, 300, d)
    idx = qb.FlatIndex(d, metric=qb.Metric(metric))
    idx.add(x)
    idx.remove(np.arange(0, n, 7))
    for k in (1, 10, 100):
        exact, fast = both_modes(lambda: idx.batch_query(q, k))
        assert_same(exact, fast)
    allowed = np.arange(0, n, 3)
    exact, fast = both_modes(lambda: idx.batch_query(q, 10, allowed=allowed))
    assert_same(exact, fast)


@pytest.mark.parametrize("metric", [0, 2])
def test_flat_search_near_ties(metric):
    d = 32
    x = clustered(3, 40000, d)
    q = clustered(4, 257, d)
    x[1000:1100] = x[2000:2100]          # exact duplicates: ties broken by slot
    idx = qb.FlatIndex(d, metric=qb.Metric(metric), custom_ids=True)
    idx.add(x, ids=np.arange(40000) * 3 + 11)
    for k in (1, 50, 200):
        exact, fast = both_modes(lambda: idx.batch_query(q, k))
        assert_same(exact, fast)


def test_flat_search_matches_reference(ref):
    d, n = 96, 20000
    x = lognormal_rows(7, n, d)
    q = lognormal_rows(8, 64, d)
    for metric in (0, 2):
        mine = qb.FlatIndex(d, metric=qb.Metric(metric))
        theirs = ref.FlatIndex(d, metric=metric)
        for idx in (mine, theirs):
            idx.add(x)
        qb.set_tensor_filter(2)
        i1, d1 = mine.batch_query(q, 100)
        i2, d2 = theirs.batch_query(q, 100)
        np.testing.assert_array_equal(i1, i2)
        assert d1.tobytes() == d2.tobytes()


def test_assignment_in_training_and_adding(tmp_path):
    """nlist large enough that assignment goes through the filter."""
    d, nlist = 16, 9000
    x = clustered(9, 30000, d, centres=3000, sigma=0.1)

    def build(path):
        idx = qb.IVFIndex(d, nlist, 8)
        idx.enable_pq(8, fast_scan=True)
        idx.train(x, max_iters=2, seed=3, clustering=qb.Clustering.Lloyd)
        idx.add(x)
        idx.save(path)
        return path

    a, b = both_modes(lambda: build(tmp_path / f"m{qb.tensor_filter()}.qann"))
    assert filecmp.cmp(a, b, shallow=False)
