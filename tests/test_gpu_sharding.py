"""List-sharded search on one GPU: the shards of an index (one handle each,
as the ranks of a sharded search hold them) produce candidates that, merged
and finished, give exactly the unsharded search's results."""
import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def sharded_results(path, q, k, shards):
    handles = [qb.load(path) for _ in range(shards)]
    for s, h in enumerate(handles):
        (h.base if isinstance(h, qb.RefineIndex) else h).set_shard(s, shards)
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    nq = q.shape[0]
    kp = handles[0].candidate_count(k)
    keys = torch.empty((nq, shards, kp), dtype=torch.int64, device="cuda")
    slots = torch.empty((nq, shards, kp), dtype=torch.int32, device="cuda")
    for s, h in enumerate(handles):
        key = torch.empty((nq, kp), dtype=torch.int64, device="cuda")
        slot = torch.empty((nq, kp), dtype=torch.int32, device="cuda")
        h.search_candidates_device(qd.data_ptr(), nq, k, key.data_ptr(), slot.data_ptr())
        keys[:, s] = key
        slots[:, s] = slot
    mk = torch.empty((nq, kp), dtype=torch.int64, device="cuda")
    ms = torch.empty((nq, kp), dtype=torch.int32, device="cuda")
    qb.merge_candidates_device(keys.data_ptr(), slots.data_ptr(), nq, shards, kp, mk.data_ptr(), ms.data_ptr())
    ids = torch.empty((nq, k), dtype=torch.int64, device="cuda")
    d = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    handles[0].finish_candidates_device(qd.data_ptr(), nq, k, mk.data_ptr(), ms.data_ptr(), ids.data_ptr(), d.data_ptr())
    torch.cuda.synchronize()
    return ids.cpu().numpy(), d.cpu().numpy(), handles[0]


@pytest.mark.parametrize("shards", [2, 3])
@pytest.mark.parametrize("kind", ["ivf", "refine"])
@pytest.mark.parametrize("name", ["l2", "ip", "cos_l2", "l2_custom_del"])
def test_sharded_equals_unsharded(golden, shards, kind, name):
    path = golden / "gen" / f"{kind}_{name}.qann"
    q = np.load(golden / "gen" / "queries.npy")
    ids, d, sharded = sharded_results(path, q, 10, shards)
    ei, ed = qb.load(path).batch_query(q, 10)
    np.testing.assert_array_equal(ids, ei)
    assert d.tobytes() == ed.tobytes()
    with pytest.raises(RuntimeError, match="shard"):
        sharded.batch_query(q[:2], 10)
