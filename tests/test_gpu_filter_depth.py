"""Filtered IVF probing that ranks only the nearest lists first: on an index
with 1,024 lists the probe walk of a filtered query (reference
src/ivf_index.cpp:501-521) normally stays inside the lists ranked before it,
and a filter whose allowed ids lie in far clusters makes it walk past them,
so that every list is ranked after all. Either way ids and distances must be
those of the reference library, alone and in served mixed batches. The walk
is exercised on a bare IVF index: a RefineIndex sends filters of up to
6 * nlist allowed ids to its exact direct scan (reference
src/refine_index.cpp:59-82) and walks only wider ones."""
import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu

N, D, NLIST, CENTRES = 60_000, 32, 1024, 400


def _data():
    rng = np.random.default_rng(21)
    c = rng.normal(size=(CENTRES, D)).astype(np.float32)
    lab = rng.integers(0, CENTRES, size=N)
    x = (c[lab] + 0.2 * rng.normal(size=(N, D))).astype(np.float32)
    return x, lab, c


@pytest.fixture(scope="module")
def deep(ref, tmp_path_factory):
    x, lab, c = _data()
    out = {}
    d = tmp_path_factory.mktemp("depth")
    for metric in (0, 2):
        ivf = ref.IVFIndex(D, NLIST, 8, metric=metric)
        ivf.enable_pq(16, fast_scan=True)
        ivf.train(x, seed=5)
        ivf.add(x)
        ivf.save(d / f"i{metric}.qann")
        out[metric] = d / f"i{metric}.qann"
    base = ref.IVFIndex(D, NLIST, 8)
    base.enable_pq(16, fast_scan=True)
    base.train(x, seed=5)
    r = ref.RefineIndex(base, 10)
    r.add(x)
    r.save(d / "r0.qann")
    out["refine"] = d / "r0.qann"
    return out, x, lab, c


def _queries(c, n, seed):
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, 40, size=n)   # near the first 40 centres
    return (c[pick] + 0.2 * rng.normal(size=(n, D))).astype(np.float32)


def _counts():
    return qb.tensor_filter_counts()


@pytest.mark.parametrize("metric", [0, 2])
def test_walk_inside_ranked_lists(ref, deep, metric):
    paths, x, lab, c = deep
    mine, theirs = qb.load(paths[metric]), ref.load(paths[metric])
    q = _queries(c, 64, 3)
    rng = np.random.default_rng(4)
    for frac in (0.3, 0.05, 0.01):
        allowed = np.nonzero(rng.random(N) < frac)[0].astype(np.int64)
        before = _counts()
        for k in (1, 10, 50):
            i1, d1 = mine.batch_query(q, k, allowed=allowed)
            i2, d2 = theirs.batch_query(q, k, allowed=allowed)
            np.testing.assert_array_equal(i1, i2)
            assert d1.tobytes() == d2.tobytes()
        after = _counts()
        assert after["filtered_batches"] > before["filtered_batches"]
        if frac >= 0.05:   # (at 1 % a walk may still outrun the mean-density estimate)
            assert after["filtered_deep_walks"] == before["filtered_deep_walks"], frac


def test_refine_wide_filter(ref, deep):
    paths, x, lab, c = deep
    mine, theirs = qb.load(paths["refine"]), ref.load(paths["refine"])
    q = _queries(c, 32, 8)
    allowed = np.nonzero(np.random.default_rng(9).random(N) < 0.3)[0].astype(np.int64)
    for k in (10, 30):
        i1, d1 = mine.batch_query(q, k, allowed=allowed)
        i2, d2 = theirs.batch_query(q, k, allowed=allowed)
        np.testing.assert_array_equal(i1, i2)
        assert d1.tobytes() == d2.tobytes()


@pytest.mark.parametrize("metric", [0, 2])
def test_walk_past_ranked_lists(ref, deep, metric):
    """Allowed ids only in clusters far from the queries: the walk runs past
    the lists ranked first and every list is ranked."""
    paths, x, lab, c = deep
    mine, theirs = qb.load(paths[metric]), ref.load(paths[metric])
    q = _queries(c, 16, 5)
    allowed = np.nonzero(lab >= CENTRES - 3)[0].astype(np.int64)   # about 450 rows in 3 far clusters
    before = _counts()
    i1, d1 = mine.batch_query(q, 10, allowed=allowed)
    i2, d2 = theirs.batch_query(q, 10, allowed=allowed)
    np.testing.assert_array_equal(i1, i2)
    assert d1.tobytes() == d2.tobytes()
    assert _counts()["filtered_deep_walks"] > before["filtered_deep_walks"]


def test_served_mixed_batches_with_depth(ref, deep):
    """A served mix of filtered and unfiltered requests, nprobe 4..64, k 10 and
    50: every result equals the reference's search of that request alone."""
    paths, x, lab, c = deep
    mine, theirs = qb.load(paths[0]), ref.load(paths[0])
    rng = np.random.default_rng(6)
    pool = [np.nonzero(rng.random(N) < f)[0].astype(np.int64) for f in (0.3, 0.05, 0.01)]
    pool.append(np.nonzero(lab >= CENTRES - 3)[0].astype(np.int64))
    nreq = 96
    q = _queries(c, nreq, 7)
    ks = rng.choice(np.array([10, 50], np.int32), size=nreq)
    npb = rng.choice(np.array([4, 8, 16, 64], np.int32), size=nreq)
    which = np.where(rng.random(nreq) < 0.6, rng.integers(0, len(pool), nreq), -1)
    with qb.Server(mine, slots=2, max_batch=64) as srv:
        fids = []
        for a in pool:
            bits = np.zeros(N, bool)
            bits[a] = True
            fids.append(srv.add_filter(np.packbits(np.concatenate([bits, np.zeros((-N) % 64, bool)]),
                                                   bitorder="little").view(np.uint64)))
        fid = np.array([fids[w] if w >= 0 else -1 for w in which], np.int32)
        ids, dist, _ = srv.replay(q, ks, np.zeros(nreq), nprobes=npb, filter_ids=fid)
    for i in range(nreq):
        theirs.nprobe = int(npb[i])
        k = int(ks[i])
        if which[i] >= 0:
            i2, d2 = theirs.batch_query(q[i:i + 1], k, allowed=pool[which[i]])
        else:
            i2, d2 = theirs.batch_query(q[i:i + 1], k)
        np.testing.assert_array_equal(ids[i, :k], i2[0])
        assert dist[i, :k].tobytes() == d2[0].tobytes(), i
