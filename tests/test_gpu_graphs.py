"""Device-resident searches replayed as CUDA graphs return what the direct
path returns: the same buffers refilled with new queries between replays,
IVF and RefineIndex over IVF in several scoring modes, and a fresh capture
after the index changes."""
import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture
def graphs():
    qb.set_search_graphs(True)
    yield
    qb.set_search_graphs(False)


def run_device(idx, q_dev, ids, d, stream):
    with torch.cuda.stream(stream):
        idx.search_device(q_dev.data_ptr(), q_dev.shape[0], ids.shape[1], ids.data_ptr(), d.data_ptr(),
                          stream.cuda_stream)
    stream.synchronize()
    return ids.cpu().numpy(), d.cpu().numpy()


@pytest.mark.parametrize("kind", ["ivf", "refine"])
@pytest.mark.parametrize("name", ["l2", "ip", "cos_ip", "cos_l2"])
def test_replays_match_direct(golden, graphs, kind, name):
    idx = qb.load(golden / "gen" / f"{kind}_{name}.qann")
    q = np.load(golden / "gen" / "queries.npy")
    n, k = 16, 10
    stream = torch.cuda.Stream()
    q_dev = torch.empty((n, q.shape[1]), dtype=torch.float32, device="cuda")
    ids = torch.empty((n, k), dtype=torch.int64, device="cuda")
    d = torch.empty((n, k), dtype=torch.float32, device="cuda")
    before = qb.search_graph_counts()
    for rep in range(3):
        rows = q[(rep * n) % (q.shape[0] - n):][:n]
        q_dev.copy_(torch.from_numpy(np.ascontiguousarray(rows)))
        torch.cuda.synchronize()
        gi, gd = run_device(idx, q_dev, ids, d, stream)
        ei, ed = idx.batch_query(rows, k)
        np.testing.assert_array_equal(gi, ei)
        assert gd.tobytes() == ed.tobytes()
    after = qb.search_graph_counts()
    assert after["captures"] - before["captures"] == 1
    assert after["replays"] - before["replays"] == 2


def test_recaptured_after_add(graphs):
    rng = np.random.default_rng(4)
    d_ = 32
    x = rng.normal(size=(6000, d_)).astype(np.float32)
    ivf = qb.IVFIndex(d_, 128, 8)
    ivf.enable_pq(8, fast_scan=True)
    ivf.train(x, seed=2)
    ivf.add(x[:4000])
    q = rng.normal(size=(8, d_)).astype(np.float32)
    stream = torch.cuda.Stream()
    q_dev = torch.from_numpy(q).cuda()
    ids = torch.empty((8, 5), dtype=torch.int64, device="cuda")
    dist = torch.empty((8, 5), dtype=torch.float32, device="cuda")
    run_device(ivf, q_dev, ids, dist, stream)
    run_device(ivf, q_dev, ids, dist, stream)
    ivf.add(x[4000:])                       # the device copy is rebuilt: the old graph must not run
    before = qb.search_graph_counts()
    gi, gd = run_device(ivf, q_dev, ids, dist, stream)
    after = qb.search_graph_counts()
    ei, ed = ivf.batch_query(q, 5)
    np.testing.assert_array_equal(gi, ei)
    assert gd.tobytes() == ed.tobytes()
    assert after["captures"] - before["captures"] == 1


@pytest.mark.parametrize("name", ["l2", "cos_l2"])
def test_replays_with_tensor_coarse(golden, graphs, name):
    """The coarse step on the tensor cores inside a captured search (its
    recheck then holds every list) matches the direct exact path."""
    qb.set_tensor_filter(2)
    try:
        idx = qb.load(golden / "gen" / f"refine_{name}.qann")
        q = np.load(golden / "gen" / "queries.npy")
        n, k = 32, 10
        stream = torch.cuda.Stream()
        q_dev = torch.from_numpy(np.ascontiguousarray(q[:n])).cuda()
        ids = torch.empty((n, k), dtype=torch.int64, device="cuda")
        d = torch.empty((n, k), dtype=torch.float32, device="cuda")
        for _ in range(3):
            gi, gd = run_device(idx, q_dev, ids, d, stream)
        qb.set_tensor_filter(0)
        ei, ed = idx.batch_query(q[:n], k)
        np.testing.assert_array_equal(gi, ei)
        assert gd.tobytes() == ed.tobytes()
    finally:
        qb.set_tensor_filter(1)
