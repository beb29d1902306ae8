"""The host side of the sharded search with two gloo ranks on the CPU:
ShardedSearch gathers every rank's candidates in the layout the merge
expects and returns the global top-k on every rank. The device steps are
replaced by CPU stand-ins that keep the same contract (sorted candidate
lists of (key, slot), merge of [nq][nparts][kp])."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

N, NQ, K, KP = 500, 6, 5, 12


def keys_for(q):
    """Distinct uint63 keys of all N vectors for each query (a fixed problem)."""
    rng = np.random.default_rng(q)
    return (rng.permutation(N).astype(np.int64) << 20) | np.arange(N, dtype=np.int64)


class CpuOps:
    def __init__(self, rank, world):
        self.rank, self.world = rank, world

    def count(self, k):
        return KP

    def candidates(self, q, k, kp):
        key = np.empty((NQ, kp), np.int64)
        for i in range(NQ):
            mine = keys_for(i)[np.arange(N) % self.world == self.rank]   # this rank's "lists"
            key[i] = np.sort(mine)[:kp]
        return torch.from_numpy(key), torch.from_numpy((key & 0xFFFFF).astype(np.int32))

    def merge(self, keys, slots):
        assert keys.shape == (NQ, self.world, KP) and slots.shape == (NQ, self.world, KP)
        k = keys.numpy().reshape(NQ, -1)
        s = slots.numpy().reshape(NQ, -1)
        order = np.argsort(k, axis=1, kind="stable")[:, :KP]
        return torch.from_numpy(np.take_along_axis(k, order, 1)), torch.from_numpy(np.take_along_axis(s, order, 1))

    def finish(self, q, k, key, slot):
        return slot[:, :k].long(), (key[:, :k] >> 20).float()


def run_rank(rank, world, port, out):
    import torch.distributed as dist
    from qann_b200.sharded import ShardedSearch
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ss = ShardedSearch(None, rank, world, ops=CpuOps(rank, world))
        ids, d = ss.search(torch.zeros((NQ, 4)), K)
        np.save(os.path.join(out, f"ids{rank}.npy"), ids.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_return_the_global_top_k(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(run_rank, args=(2, free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    want = np.stack([np.sort(keys_for(i))[:K] & 0xFFFFF for i in range(NQ)])
    for r in range(2):
        np.testing.assert_array_equal(np.load(tmp_path / f"ids{r}.npy"), want)
