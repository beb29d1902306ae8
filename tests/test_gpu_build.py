"""Training and adding on the GPU against the reference library on the same
seeded inputs: the saved `.qann` files must be byte-identical (coarse
centroids, PQ codebook, cosine scoring choice, residual centers, lists, codes
and ids), and queries must return the reference's results exactly."""
import filecmp

import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


def clustered(seed, n, d, centres=30, sigma=0.2):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(centres, d)).astype(np.float32)
    lab = rng.integers(0, centres, size=n)
    return (c[lab] + sigma * rng.normal(size=(n, d))).astype(np.float32)


CASES = [
    # metric, clustering, d, m, nlist, PCA rotation
    (0, 0, 32, 16, 100, False),
    (0, 1, 32, 16, 100, False),
    (1, 0, 32, 16, 100, False),
    (1, 1, 24, 12, 120, False),
    (2, 0, 16, 8, 100, False),
    (0, 0, 100, 50, 128, False),
    (0, 0, 32, 16, 100, True),
    (1, 1, 24, 12, 120, True),
    (2, 0, 16, 8, 100, True),
    (1, 0, 100, 50, 128, True),
]


@pytest.mark.parametrize("metric,clustering,d,m,nlist,rotate", CASES)
def test_train_add_save_byte_identical(ref, tmp_path, metric, clustering, d, m, nlist, rotate):
    x = clustered(metric * 10 + clustering + d, 6000, d)
    mine = qb.IVFIndex(d, nlist, 8, metric=qb.Metric(metric))
    theirs = ref.IVFIndex(d, nlist, 8, metric=metric)
    for idx in (mine, theirs):
        idx.enable_pq(m, fast_scan=True, rotate=rotate)
        idx.train(x, max_iters=6, seed=11, clustering=clustering, passes=2)
    r_mine, r_theirs = qb.RefineIndex(mine, 4), ref.RefineIndex(theirs, 4)
    r_mine.add(x[:4000])
    r_theirs.add(x[:4000])
    r_mine.add(x[4000:])
    r_theirs.add(x[4000:])
    a, b = tmp_path / "mine.qann", tmp_path / "ref.qann"
    r_mine.save(a)
    r_theirs.save(b)
    assert filecmp.cmp(a, b, shallow=False), "trained / added index differs from the reference's"
    q = clustered(99, 50, d)
    i1, d1 = r_mine.batch_query(q, 10)
    i2, d2 = r_theirs.batch_query(q, 10)
    np.testing.assert_array_equal(i1, i2)
    assert d1.tobytes() == d2.tobytes()


def test_custom_ids_add_and_remove(ref, tmp_path):
    x = clustered(5, 3000, 32)
    ids = np.arange(10_000, 13_000)
    mine = qb.IVFIndex(32, 100, 10, custom_ids=True)
    theirs = ref.IVFIndex(32, 100, 10, custom_ids=True)
    for idx in (mine, theirs):
        idx.enable_pq(16, fast_scan=True)
        idx.train(x, seed=2)
        idx.add(x, ids=ids)
        idx.remove(ids[::5])
    q = clustered(6, 40, 32)
    i1, d1 = mine.batch_query(q, 10)
    i2, d2 = theirs.batch_query(q, 10)
    np.testing.assert_array_equal(i1, i2)
    assert d1.tobytes() == d2.tobytes()
    mine.save(tmp_path / "a.qann")
    theirs.save(tmp_path / "b.qann")
    assert filecmp.cmp(tmp_path / "a.qann", tmp_path / "b.qann", shallow=False)
