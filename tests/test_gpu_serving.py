"""The serving loop on the GPU: requests with their own k, nprobe and filter,
batched continuously, must each return exactly what they return searched
alone (the index's nprobe set to theirs), and what the reference library
returns for them. Covers IVF and RefineIndex over IVF in L2, cosine and
inner product, narrow filters (RefineIndex direct scan), empty filters,
open-loop arrivals, and several submitting threads."""
import threading

import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


def clustered(seed, n, d, centres=25, sigma=0.25):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(centres, d)).astype(np.float32)
    lab = rng.integers(0, centres, size=n)
    return (c[lab] + sigma * rng.normal(size=(n, d))).astype(np.float32)


N, D = 8000, 32


@pytest.fixture(scope="module")
def built(ref, tmp_path_factory):
    x = clustered(11, N, D)
    out = {}
    d = tmp_path_factory.mktemp("serve")
    for metric in (0, 1, 2):
        base = ref.IVFIndex(D, 100, 6, metric=metric)
        base.enable_pq(16, fast_scan=True)
        base.train(x, seed=5)
        r = ref.RefineIndex(base, 4)
        r.add(x)
        r.remove(np.arange(0, N, 17))
        r.save(d / f"r{metric}.qann")
        ivf = ref.IVFIndex(D, 100, 6, metric=metric)
        ivf.enable_pq(16, fast_scan=True)
        ivf.train(x, seed=5)
        ivf.add(x)
        ivf.save(d / f"i{metric}.qann")
        out[metric] = {"refine": d / f"r{metric}.qann", "ivf": d / f"i{metric}.qann"}
    return out


def _mix(seed, n):
    rng = np.random.default_rng(seed)
    q = clustered(seed + 100, n, D)
    ks = rng.choice([1, 3, 10, 25], size=n).astype(np.int32)
    nprobes = rng.choice([1, 3, 6, 20, 100], size=n).astype(np.int32)
    return q, ks, nprobes


def _bitmaps(seed):
    """Slot bitmaps of selectivity 0.4, 0.1, 0.01 (narrow: direct scan) and 0 (empty)."""
    rng = np.random.default_rng(seed)
    out = []
    for s in (0.4, 0.1, 0.01, 0.0):
        bits = rng.random(N) < s
        words = np.zeros((N + 63) // 64, np.uint64)
        for i in np.nonzero(bits)[0]:
            words[i >> 6] |= np.uint64(1) << np.uint64(i & 63)
        out.append((words, np.nonzero(bits)[0].astype(np.int64)))
    return out


def _alone(idx, ivf, q, k, nprobe, allowed):
    ivf.nprobe = int(nprobe)
    return idx.batch_query(q[None], int(k), allowed=allowed)


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("kind", ["refine", "ivf"])
@pytest.mark.parametrize("spread", [0.0, 0.02])
def test_replay_matches_alone(built, metric, kind, spread):
    idx = qb.load(built[metric][kind])
    ivf = idx.base if kind == "refine" else idx
    n = 120
    q, ks, nprobes = _mix(metric * 7 + (kind == "ivf") + int(spread * 100), n)
    maps = _bitmaps(metric)
    rng = np.random.default_rng(3)
    fids = np.where(rng.random(n) < 0.35, rng.integers(0, len(maps), size=n), -1).astype(np.int32)
    with qb.Server(idx, slots=3, max_batch=32) as srv:
        reg = [srv.add_filter(w) for w, _ in maps]
        arrivals = np.sort(rng.random(n)) * spread   # 0: one burst; else spread over 20 ms
        ids, d, lat = srv.replay(q, ks, arrivals, nprobes=nprobes,
                                 filter_ids=np.where(fids >= 0, np.take(reg, np.maximum(fids, 0)), -1))
        st = srv.stats()
    assert st["completed"] == n and st["batches"] >= 1
    assert (lat > 0).all()
    for i in range(n):
        allowed = maps[fids[i]][1] if fids[i] >= 0 else None
        ai, ad = _alone(idx, ivf, q[i], ks[i], nprobes[i], allowed)
        k = ks[i]
        np.testing.assert_array_equal(ids[i, :k], ai[0], err_msg=f"request {i}")
        assert d[i, :k].tobytes() == ad[0].tobytes(), f"request {i}"
        assert (ids[i, k:] == -1).all()


def test_served_results_match_reference(built, ref):
    path = built[1]["refine"]
    idx, theirs = qb.load(path), ref.load(path)
    n = 40
    q, ks, nprobes = _mix(77, n)
    with qb.Server(idx, slots=2, max_batch=16) as srv:
        ids, d, _ = srv.replay(q, ks, np.zeros(n), nprobes=nprobes)
    for i in range(n):
        theirs.base.nprobe = int(nprobes[i])
        ti, td = theirs.batch_query(q[i][None], int(ks[i]))
        np.testing.assert_array_equal(ids[i, :ks[i]], ti[0])
        assert d[i, :ks[i]].tobytes() == td[0].tobytes()


def test_submit_from_threads_with_allowed_ids(built):
    idx = qb.load(built[0]["refine"])
    ivf = idx.base
    q, ks, nprobes = _mix(5, 64)
    maps = _bitmaps(9)
    results = {}
    with qb.Server(idx, slots=4, max_batch=8) as srv:
        def client(part):
            for i in range(part, 64, 4):
                allowed = maps[i % 4][1] if i % 3 == 0 else None
                t = srv.submit(q[i], int(ks[i]), nprobe=int(nprobes[i]), allowed=allowed)
                results[i] = (srv.result(t), allowed)
        threads = [threading.Thread(target=client, args=(p,)) for p in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert len(results) == 64
    for i, ((ids, d, lat), allowed) in results.items():
        ai, ad = _alone(idx, ivf, q[i], ks[i], nprobes[i], allowed)
        np.testing.assert_array_equal(ids, ai[0])
        assert d.tobytes() == ad[0].tobytes()
        assert lat > 0


def test_memory_budget_limits_batches(built):
    idx = qb.load(built[2]["ivf"])
    q, ks, nprobes = _mix(8, 64)
    with qb.Server(idx, slots=2, max_batch=64, mem_budget=1) as srv:   # one request per batch
        ids, _, _ = srv.replay(q, ks, np.zeros(64), nprobes=nprobes)
        st = srv.stats()
    assert st["batches"] == 64
    for i in range(0, 64, 9):
        idx.nprobe = int(nprobes[i])
        ai, _ = idx.batch_query(q[i][None], int(ks[i]))
        np.testing.assert_array_equal(ids[i, :ks[i]], ai[0])


def test_index_first_searched_by_a_server_outlives_its_workers(built):
    """The first search of a fresh index builds its device arrays; when that
    search runs on a server worker, the arrays must outlive the worker."""
    import gc
    idx = qb.load(built[0]["ivf"])
    q = clustered(1, 4, D)
    with qb.Server(idx, slots=1) as srv:
        a, _, _ = srv.result(srv.submit(q[0], 5))
    b, _ = idx.batch_query(q[:1], 5)
    np.testing.assert_array_equal(a, b[0])
    del idx
    gc.collect()
    other = qb.load(built[1]["ivf"])
    ids, _ = other.batch_query(q, 5)
    assert (ids >= 0).all()


def test_many_threads_submit_while_others_wait(built):
    """Sixteen threads keep several tickets open each while the others
    submit, so the server's request map rehashes many times while threads
    sleep in result(); every result must still be the request's own."""
    idx = qb.load(built[0]["ivf"])
    ivf = idx
    n_threads, per_thread, window = 16, 96, 6
    q, ks, nprobes = _mix(21, n_threads * per_thread)
    results = {}
    errors = []
    with qb.Server(idx, slots=3, max_batch=16) as srv:
        def client(part):
            try:
                open_ = []
                for i in range(part, n_threads * per_thread, n_threads):
                    open_.append((i, srv.submit(q[i], int(ks[i]), nprobe=int(nprobes[i]))))
                    if len(open_) == window:
                        j, t = open_.pop(0)
                        results[j] = srv.result(t)
                for j, t in open_:
                    results[j] = srv.result(t)
            except Exception as e:   # reported below, on the main thread
                errors.append(e)
        threads = [threading.Thread(target=client, args=(p,)) for p in range(n_threads)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = srv.stats()
    assert not errors, errors[:3]
    assert len(results) == n_threads * per_thread and st["completed"] == len(results)
    for i in range(0, len(results), 37):
        ai, ad = _alone(idx, ivf, q[i], ks[i], nprobes[i], None)
        ids, d, _ = results[i]
        np.testing.assert_array_equal(ids, ai[0])
        assert d.tobytes() == ad[0].tobytes()
