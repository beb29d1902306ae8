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


def coarse_runs(fn):
    """fn on the exact coarse path and through the tensor cores; the tensor
    path must have answered the queries."""
    qb.set_tensor_filter(0)
    exact = fn()
    qb.set_tensor_filter(2)
    before = qb.tensor_filter_counts()
    fast = fn()
    after = qb.tensor_filter_counts()
    assert after["coarse_queries"] > before["coarse_queries"], "the tensor-core coarse step did not run"
    return exact, fast, after["coarse_redone"] - before["coarse_redone"]


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("d", [24, 100, 128])
def test_coarse_identical(metric, d):
    """IVF search with the coarse step on the tensor cores returns exactly the
    exact path's results, for nprobe from 1 to most of the lists, also for
    queries far from every list (their bounds overlap: many lists rescored)."""
    x = clustered(d, 20000, d, centres=300, sigma=0.2)
    ivf = qb.IVFIndex(d, 400, 8, metric=qb.Metric(metric))
    ivf.enable_pq({24: 12, 100: 50, 128: 32}[d], fast_scan=True)
    ivf.train(x, seed=5)
    idx = qb.RefineIndex(ivf, 4)
    idx.add(x)
    q = clustered(d + 7, 200, d, centres=300, sigma=0.25)
    far = np.full((3, d), 1000.0, dtype=np.float32)
    qs = np.vstack([q, far])
    for nprobe in (1, 16, 200):
        ivf.nprobe = nprobe
        for k in (1, 10):
            exact, fast, _ = coarse_runs(lambda: idx.batch_query(qs, k))
            assert_same(exact, fast)


def test_coarse_overflow_redone_exactly():
    """More lists within the error bound than the recheck holds (queries far
    from every list, 2048 lists). In a batch of more queries than SMs those
    queries go back to the exact path; in a smaller batch the recheck holds
    every list and rescores them all in place, with nothing redone."""
    d = 32
    x = clustered(11, 30000, d, centres=1000, sigma=0.2)
    ivf = qb.IVFIndex(d, 2048, 16)
    ivf.enable_pq(8, fast_scan=True)
    ivf.train(x, seed=5)
    ivf.add(x)
    far = np.full((4, d), 1000.0, dtype=np.float32)
    qs = np.vstack([clustered(12, 300, d, centres=1000, sigma=0.2), far])
    exact, fast, redone = coarse_runs(lambda: ivf.batch_query(qs, 10))
    assert_same(exact, fast)
    assert redone >= 4
    qs = np.vstack([clustered(13, 60, d, centres=1000, sigma=0.2), far])
    exact, fast, redone = coarse_runs(lambda: ivf.batch_query(qs, 10))
    assert_same(exact, fast)
    assert redone == 0


@pytest.mark.parametrize("name", ["l2", "l2_adc", "ip", "cos_ip", "cos_l2", "l2_custom_del"])
def test_coarse_matches_reference_files(golden, name):
    """Reference-built indexes and their saved results, coarse step on the tensor cores."""
    qb.set_tensor_filter(2)
    for kind in ("ivf", "refine"):
        idx = qb.load(golden / "gen" / f"{kind}_{name}.qann")
        q = np.load(golden / "gen" / "queries.npy")
        ids, d = idx.batch_query(q, 10)
        np.testing.assert_array_equal(ids, np.load(golden / "gen" / f"{kind}_{name}_ids.npy"))
        np.testing.assert_array_equal(d, np.load(golden / "gen" / f"{kind}_{name}_dists.npy"))


@pytest.fixture
def filter_schedule_reset():
    yield
    qb.set_filter_options(autotune=True, epilogue_warps=0)


def test_filter_epilogue_schedules_identical(filter_schedule_reset):
    """The filter's 8- and 16-warp epilogues, and the autotuner's pick, return
    exactly the exact path's flat-search results; the autotuner times a
    launch large enough to tune (at least 8 tiles per SM) and records it."""
    d, n = 96, 200_000
    x = lognormal_rows(21, n, d)
    q = lognormal_rows(22, 3000, d)
    idx = qb.FlatIndex(d, metric=qb.Metric(0))
    idx.add(x)
    qb.set_tensor_filter(0)
    exact = idx.batch_query(q, 10)
    qb.set_tensor_filter(2)
    for warps in (8, 16):
        qb.set_filter_options(epilogue_warps=warps)
        got = idx.batch_query(q, 10)
        assert_same(exact, got)
        assert qb.filter_options()["last_epilogue_warps"] == warps
    qb.set_filter_options(autotune=True, epilogue_warps=0)
    before = qb.filter_options()["tuned_problems"]
    assert_same(exact, idx.batch_query(q, 10))
    assert qb.filter_options()["tuned_problems"] > before
    assert_same(exact, idx.batch_query(q, 10))   # the kept pick


def test_coarse_step_epilogue_schedules_identical(filter_schedule_reset):
    """The tensor-core coarse step (store mode) under either epilogue returns
    the exact path's results."""
    d, nlist = 64, 1024
    x = clustered(31, 60_000, d, centres=200)
    q = clustered(32, 2000, d, centres=200)
    ivf = qb.IVFIndex(d, nlist, 8)
    ivf.enable_pq(16, fast_scan=True)
    ivf.train(x, seed=1)
    ivf.add(x)
    ivf.nprobe = 32
    qb.set_tensor_filter(0)
    exact = ivf.batch_query(q, 10)
    qb.set_tensor_filter(1)
    for warps in (8, 16):
        qb.set_filter_options(epilogue_warps=warps)
        before = qb.tensor_filter_counts()
        got = ivf.batch_query(q, 10)
        assert qb.tensor_filter_counts()["coarse_queries"] > before["coarse_queries"], "the coarse step was not on the tensor cores"
        assert_same(exact, got)
