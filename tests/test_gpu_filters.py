"""Filtered queries (allowed ids) on the GPU path against the reference
library on the same indexes: IVF filtered probing with probe scaling
(reference src/ivf_index.cpp:501-521), RefineIndex's exact direct scan for
narrow filters (reference src/refine_index.cpp:59-82), Flat filters, unknown
and deleted ids in the allowed set, and empty filters. Ids and distances
must be identical."""
import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


def clustered(seed, n, d, centres=25, sigma=0.25):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(centres, d)).astype(np.float32)
    lab = rng.integers(0, centres, size=n)
    return (c[lab] + sigma * rng.normal(size=(n, d))).astype(np.float32)


@pytest.fixture(scope="module")
def built(ref, tmp_path_factory):
    """A RefineIndex over IVF fast-scan and a bare IVF, built by the reference and loaded here."""
    x = clustered(1, 8000, 32)
    out = {}
    d = tmp_path_factory.mktemp("filt")
    for metric in (0, 1, 2):
        base = ref.IVFIndex(32, 100, 6, metric=metric)
        base.enable_pq(16, fast_scan=True)
        base.train(x, seed=4)
        r = ref.RefineIndex(base, 5)
        r.add(x)
        r.remove(np.arange(0, 8000, 11))
        r.save(d / f"r{metric}.qann")
        ivf = ref.IVFIndex(32, 100, 6, metric=metric)
        ivf.enable_pq(16, fast_scan=True)
        ivf.train(x, seed=4)
        ivf.add(x)
        ivf.remove(np.arange(3, 8000, 13))
        ivf.save(d / f"i{metric}.qann")
        out[metric] = (d / f"r{metric}.qann", d / f"i{metric}.qann")
    return out


SELECTIVITY = [0.5, 0.1, 0.02, 0.004, 0.0005]


def _allowed(seed, frac, n=8000):
    rng = np.random.default_rng(seed)
    ids = np.nonzero(rng.random(n) < frac)[0]
    # unknown and repeated ids are ignored by both implementations
    return np.concatenate([ids, ids[:3], [n + 5, n + 99]]).astype(np.int64)


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("frac", SELECTIVITY)
@pytest.mark.parametrize("kind", ["refine", "ivf"])
@pytest.mark.parametrize("scaling", [True, False])
def test_filtered_queries_match_reference(ref, built, metric, frac, kind, scaling):
    path = built[metric][0 if kind == "refine" else 1]
    mine, theirs = qb.load(path), ref.load(path)
    ivf_mine = mine.base if kind == "refine" else mine
    ivf_theirs = theirs.base if kind == "refine" else theirs
    ivf_mine.filter_probe_scaling = scaling
    ivf_theirs.filter_probe_scaling = scaling
    q = clustered(7, 30, 32)
    allowed = _allowed(int(frac * 1e5) + metric, frac)
    for k in (1, 10):
        i1, d1 = mine.batch_query(q, k, allowed=allowed)
        i2, d2 = theirs.batch_query(q, k, allowed=allowed)
        np.testing.assert_array_equal(i1, i2)
        assert d1.tobytes() == d2.tobytes()


def test_empty_and_all_deleted_filters(ref, built):
    path = built[0][0]
    mine = qb.load(path)
    q = clustered(8, 5, 32)
    ids, d = mine.batch_query(q, 10, allowed=[])
    assert (ids == -1).all() and np.isinf(d).all()
    ids, d = mine.batch_query(q, 10, allowed=[0, 11, 22])   # deleted slots only
    assert (ids == -1).all()


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_flat_filters(ref, tmp_path, metric):
    x = clustered(3, 3000, 24)
    f = ref.FlatIndex(24, metric=metric, custom_ids=True)
    f.add(x, ids=np.arange(100, 3100))
    f.remove(np.arange(100, 3100, 9))
    f.save(tmp_path / "f.qann")
    mine = qb.load(tmp_path / "f.qann")
    q = clustered(4, 20, 24)
    allowed = np.arange(100, 3100)[::3]
    i1, d1 = mine.batch_query(q, 10, allowed=allowed)
    i2, d2 = f.batch_query(q, 10, allowed=allowed)
    np.testing.assert_array_equal(i1, i2)
    assert d1.tobytes() == d2.tobytes()
