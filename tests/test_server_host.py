"""Host-side logic of the serving loop (no GPU needed): argument checks,
ticket and filter bookkeeping, error propagation from the workers, stats
and shutdown."""
import os

import numpy as np
import pytest

import qann_b200 as qb

NO_GPU = not os.path.exists("/dev/nvidia0")


@pytest.fixture
def index(golden):
    return qb.load(golden / "gen" / "refine_cos_ip.qann")


def test_rejects_bad_requests(index):
    dim = index.dim()
    with qb.Server(index, slots=1) as srv:
        with pytest.raises(ValueError, match="k must be at least 1"):
            srv.submit(np.ones(dim, np.float32), 0)
        with pytest.raises(ValueError, match="nprobe must be <= nlist"):
            srv.submit(np.ones(dim, np.float32), 5, nprobe=index.base.nlist + 1)
        with pytest.raises(ValueError, match="non-zero"):
            srv.submit(np.zeros(dim, np.float32), 5)
        with pytest.raises(ValueError, match="unknown filter id"):
            srv.submit(np.ones(dim, np.float32), 5, filter_id=3)
        with pytest.raises(ValueError, match="cover every slot"):
            srv.add_filter(np.zeros(1, np.uint64))
        assert srv.stats()["completed"] == 0


def test_server_arguments():
    with pytest.raises((ValueError, RuntimeError)):
        qb.Server(qb.FlatIndex(4), slots=0)
    with pytest.raises((ValueError, RuntimeError)):
        qb.Server(qb.FlatIndex(4), max_batch=0)


def test_filters_register_in_order(index):
    words = np.full((index._get("slots") + 63) // 64, ~np.uint64(0), np.uint64)
    with qb.Server(index, slots=1) as srv:
        assert [srv.add_filter(words) for _ in range(3)] == [0, 1, 2]


@pytest.mark.skipif(not NO_GPU, reason="checks the error path taken without a GPU")
def test_worker_errors_reach_each_ticket(index):
    dim = index.dim()
    rng = np.random.default_rng(0)
    with qb.Server(index, slots=2, max_batch=4) as srv:
        tickets = [srv.submit(rng.normal(size=dim).astype(np.float32), 3) for _ in range(9)]
        for t in tickets:
            with pytest.raises(qb.CudaError, match="CUDA stream"):
                srv.result(t)
        st = srv.stats()
        with pytest.raises(ValueError, match="unknown ticket"):   # each ticket is taken once
            qb.check(qb._lib.lib.qg_server_wait(srv._s, tickets[0], None, None, None))
    assert st["completed"] == 9 and 3 <= st["batches"] <= 9
    with pytest.raises(ValueError, match="null server handle"):
        qb.check(qb._lib.lib.qg_server_wait(None, 1, None, None, None))


def test_close_is_idempotent(index):
    srv = qb.Server(index, slots=2)
    srv.close()
    srv.close()
