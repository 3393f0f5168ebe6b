"""Multi-GPU sharding of the database scan: one process per GPU (torch.distributed), each holding
one shard of the database on its own device.

The scan shards with a single exchange step (no collective inside the scan): every rank scans its
shard, then the per-query best hits are all-gathered as small int64 rows and reduced with the
reference's tie-break across the database (src/database.rs:160-208, grouped scan: higher score,
then smaller GLOBAL index), and per-target scores are all-gathered and scattered back to global
order. With NCCL the rows stay on the device; with gloo (the CPU tests) they live on the host.

Shards are length-balanced: sequences sorted by length are dealt to ranks in snake order, so every
rank gets about the same residues and the same length distribution, and each shard keeps its
sequences in ascending global order. That last property makes a shard's own smallest-index
tie-break agree with the global one.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

HIT_COLUMNS = 4  # score, global db index, query end, target end (-1: None)


def shard_indices(lengths: Sequence[int], world: int) -> List[np.ndarray]:
    """Global indices of each rank's shard: longest first, dealt 0..W-1, W-1..0, ... Each array is
    in ascending global order."""
    lengths = np.asarray(lengths, dtype=np.int64)
    order = np.argsort(-lengths, kind="stable")
    pos = np.arange(len(order))
    cyc = pos % (2 * world)
    rank = np.where(cyc < world, cyc, 2 * world - 1 - cyc)
    return [np.sort(order[rank == r]) for r in range(world)]


def hit_rows(hits, local_to_global):
    """Rows (score, global index, query end, target end) for a list of BestHit of one shard."""
    import torch

    g = np.asarray(local_to_global, dtype=np.int64)
    rows = [[h.score, int(g[h.db_index]), -1 if h.query_end is None else h.query_end,
             -1 if h.target_end is None else h.target_end] for h in hits]
    return torch.tensor(rows, dtype=torch.int64).reshape(-1, HIT_COLUMNS)


def device_hit_rows(hits_u8, local_to_global):
    """The same rows from a device tensor of hy_hit records ([Q, 32] uint8, as written by
    hy_scan_device) and a device int64 tensor mapping local to global indices."""
    import torch

    words = hits_u8.view(torch.int64).reshape(-1, 4)
    score = (words[:, 0] & 0xFFFFFFFF).to(torch.int32).to(torch.int64)  # low half: int32 score
    gidx = local_to_global[words[:, 1]]
    return torch.stack([score, gidx, words[:, 2], words[:, 3]], dim=1)


def merge_hit_rows(stacked):
    """Reduce [W, Q, 4] rows over W with the tie-break: highest score, then smallest global
    index. Scores are bounded by the width proof (|s| < 2^30), so (score << 32) - index orders
    both keys in one int64."""
    import torch

    key = (stacked[..., 0] << 32) - stacked[..., 1]
    best = torch.argmax(key, dim=0)  # first maximum; keys are unique per (score, index)
    q = torch.arange(stacked.shape[1], device=stacked.device)
    return stacked[best, q]


def all_gather_best(rows, group=None):
    """Every rank's [Q, 4] rows all-gathered and merged; the same result on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if world == 1:
        return rows
    out = [torch.empty_like(rows) for _ in range(world)]
    dist.all_gather(out, rows, group=group)
    return merge_hit_rows(torch.stack(out))


def all_gather_scores(local_scores, local_to_global, n_total: int, group=None):
    """Per-target scores of every shard scattered into global order ([n_total] int32 on every
    rank). Shards may differ in size: each is padded to the largest before the all_gather."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = local_scores.device
    g = torch.as_tensor(np.asarray(local_to_global, dtype=np.int64), device=dev)
    n_local = torch.tensor([local_scores.numel()], dtype=torch.int64, device=dev)
    sizes = [torch.empty_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    m = int(max(int(s.item()) for s in sizes))
    pad_s = torch.zeros(m, dtype=torch.int32, device=dev)
    pad_s[: local_scores.numel()] = local_scores
    pad_g = torch.full((m,), -1, dtype=torch.int64, device=dev)
    pad_g[: g.numel()] = g
    all_s = [torch.empty_like(pad_s) for _ in range(world)]
    all_g = [torch.empty_like(pad_g) for _ in range(world)]
    dist.all_gather(all_s, pad_s, group=group)
    dist.all_gather(all_g, pad_g, group=group)
    out = torch.empty(n_total, dtype=torch.int32, device=dev)
    for s, gi, n in zip(all_s, all_g, sizes):
        k = int(n.item())
        out[gi[:k]] = s[:k]
    return out


class ShardedDatabase:
    """This rank's shard of a database spread over the process group, on the current CUDA device.

    ``configure`` receives a fresh DatabaseBuilder (sequences already set) and returns it with the
    scoring, mode, search type and limits applied; every rank must configure it identically.
    ``scan`` returns the same BestHit as a single Database over all sequences."""

    def __init__(self, sequences: Sequence, configure, group=None):
        import torch.distributed as dist

        from . import Database

        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.n_total = len(sequences)
        self.local_to_global = shard_indices([len(s) for s in sequences], self.world)[self.rank]
        local = [sequences[i] for i in self.local_to_global]
        self.db = configure(Database.builder().sequences(local)).build()

    def scan(self, scratch, query):
        from . import BestHit

        rows = hit_rows([self.db.scan(scratch, query)], self.local_to_global)
        m = self._gather(rows)[0].tolist()
        return BestHit(int(m[0]), int(m[1]), None if m[2] < 0 else int(m[2]), None if m[3] < 0 else int(m[3]))

    def scan_scores(self, scratch, query) -> np.ndarray:
        import torch

        local = torch.from_numpy(self.db.scan_scores_array(scratch, query)).to(self._device())
        return all_gather_scores(local, self.local_to_global, self.n_total, self.group).cpu().numpy()

    def _device(self):
        import torch
        import torch.distributed as dist

        if dist.is_initialized() and dist.get_backend(self.group) == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def _gather(self, rows):
        if self.world == 1:
            return rows
        return all_gather_best(rows.to(self._device()), self.group).cpu()
