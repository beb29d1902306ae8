"""Sharded search: one process per GPU, each holding a shard of an IVF
index's lists. No counterpart in the reference, which searches one in-process
index.

Every rank loads the same index and keeps on its device only the lists
l with l % world == rank. List sizes stay known to every rank, so the
position of each probed vector in a query's probe sequence (the low half of
a candidate key) is the same on every rank. A search is:

1. each rank's k' best candidates from its own lists (device kernels);
2. one all-gather of the (key, slot) candidate lists over the process group;
3. on every rank, a merge of the gathered lists into the k' smallest keys,
   then the final k (re-ranked with the raw rows for a RefineIndex).

The merged candidates are the ones a single unsharded search keeps, so the
results are identical to it. Only the candidate exchange crosses devices.
Queries are unfiltered.
"""
from __future__ import annotations


class CandidateOps:
    """The device steps of a sharded search on one rank (the library's
    kernels). Tensors are torch CUDA tensors."""

    def __init__(self, index):
        self.index = index

    def count(self, k):
        return self.index.candidate_count(k)

    def candidates(self, q, k, kp):
        import torch
        key = torch.empty((q.shape[0], kp), dtype=torch.int64, device=q.device)
        slot = torch.empty((q.shape[0], kp), dtype=torch.int32, device=q.device)
        stream = torch.cuda.current_stream(q.device).cuda_stream
        self.index.search_candidates_device(q.data_ptr(), q.shape[0], k, key.data_ptr(), slot.data_ptr(), stream)
        return key, slot

    def merge(self, keys, slots):
        """keys / slots: (nq, nparts, kp) -> (nq, kp)."""
        import torch
        from . import merge_candidates_device
        nq, nparts, kp = keys.shape
        keys, slots = keys.contiguous(), slots.contiguous()
        out_k = torch.empty((nq, kp), dtype=torch.int64, device=keys.device)
        out_s = torch.empty((nq, kp), dtype=torch.int32, device=keys.device)
        stream = torch.cuda.current_stream(keys.device).cuda_stream
        merge_candidates_device(keys.data_ptr(), slots.data_ptr(), nq, nparts, kp, out_k.data_ptr(), out_s.data_ptr(),
                                stream)
        return out_k, out_s

    def finish(self, q, k, key, slot):
        import torch
        ids = torch.empty((q.shape[0], k), dtype=torch.int64, device=q.device)
        d = torch.empty((q.shape[0], k), dtype=torch.float32, device=q.device)
        stream = torch.cuda.current_stream(q.device).cuda_stream
        self.index.finish_candidates_device(q.data_ptr(), q.shape[0], k, key.data_ptr(), slot.data_ptr(),
                                            ids.data_ptr(), d.data_ptr(), stream)
        return ids, d


class ShardedSearch:
    """Search of an index whose lists are spread over the ranks of a process
    group. `index` is this rank's copy (an IVFIndex or a RefineIndex over
    one); the constructor makes it keep only this rank's lists on the device.
    `ops` replaces the device steps (tests run the host side with CPU ops)."""

    def __init__(self, index, rank: int, world: int, group=None, ops=None):
        import torch.distributed as dist
        self.rank, self.world, self.group, self.dist = rank, world, group, dist
        self.ops = ops if ops is not None else CandidateOps(index)
        if ops is None:
            ivf = index.base if hasattr(index, "base") else index
            ivf.set_shard(rank, world)

    def search(self, q, k: int):
        """(ids, distances) of the nq queries in q (a (nq, dim) float32
        tensor on this rank's device), the same on every rank."""
        import torch
        kp = self.ops.count(k)
        key, slot = self.ops.candidates(q, k, kp)
        keys = [torch.empty_like(key) for _ in range(self.world)]
        slots = [torch.empty_like(slot) for _ in range(self.world)]
        self.dist.all_gather(keys, key, group=self.group)
        self.dist.all_gather(slots, slot, group=self.group)
        mk, ms = self.ops.merge(torch.stack(keys, dim=1), torch.stack(slots, dim=1))   # (nq, world, kp)
        return self.ops.finish(q, k, mk, ms)
