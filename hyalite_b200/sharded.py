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


def take_sequences(residues, offsets, indices):
    """Sequences `indices` of a concatenated database, concatenated in that order: (residues,
    offsets)."""
    offsets = np.asarray(offsets, dtype=np.uint64)
    indices = np.asarray(indices, dtype=np.int64)
    starts = offsets[indices].astype(np.int64)
    lens = (offsets[indices + 1] - offsets[indices]).astype(np.int64)
    out_off = np.zeros(len(lens) + 1, np.uint64)
    out_off[1:] = np.cumsum(lens)
    idx = np.repeat(starts - out_off[:-1].astype(np.int64), lens) + np.arange(int(out_off[-1]), dtype=np.int64)
    return np.asarray(residues, dtype=np.uint8)[idx], out_off


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


def all_gather_scatter(local, local_to_global, n_total: int, group=None):
    """Per-target rows of every shard ([n_local, ...] on this rank) scattered into global order
    ([n_total, ...] on every rank). Shards may differ in size: each is padded to the largest
    before the all_gather."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = local.device
    g = torch.as_tensor(np.asarray(local_to_global, dtype=np.int64), device=dev)
    n_local = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.empty_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    m = int(max(int(s.item()) for s in sizes))
    pad_s = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=dev)
    pad_s[: local.shape[0]] = local
    pad_g = torch.full((m,), -1, dtype=torch.int64, device=dev)
    pad_g[: g.numel()] = g
    all_s = [torch.empty_like(pad_s) for _ in range(world)]
    all_g = [torch.empty_like(pad_g) for _ in range(world)]
    dist.all_gather(all_s, pad_s, group=group)
    dist.all_gather(all_g, pad_g, group=group)
    out = torch.empty((n_total,) + tuple(local.shape[1:]), dtype=local.dtype, device=dev)
    for s, gi, n in zip(all_s, all_g, sizes):
        k = int(n.item())
        out[gi[:k]] = s[:k]
    return out


def all_gather_scores(local_scores, local_to_global, n_total: int, group=None):
    """Per-target scores of every shard scattered into global order ([n_total] int32 on every
    rank)."""
    return all_gather_scatter(local_scores, local_to_global, n_total, group)


def all_gather_hits(local_rows, local_to_global, n_total: int, group=None):
    """scan_all across shards (src/database.rs:347-464): every shard's per-target rows (score,
    global index, query end, target end) scattered into global order ([n_total, 4] int64 on every
    rank). A target's row is its own, so no tie-break is involved."""
    return all_gather_scatter(local_rows, local_to_global, n_total, group)


def merge_aligned(candidates):
    """scan_aligned across shards (src/database.rs:527-536): from each rank's (score, global
    index, alignment) the winner under the scan's tie-break (highest score, then smallest global
    index)."""
    best = None
    for c in candidates:
        if best is None or c[0] > best[0] or (c[0] == best[0] and c[1] < best[1]):
            best = c
    return best


class ShardedDatabase:
    """This rank's shard of a database spread over the process group, on the current CUDA device.

    ``configure`` receives a fresh DatabaseBuilder (sequences already set) and returns it with the
    scoring, mode, search type and limits applied; every rank must configure it identically.
    ``scan`` returns the same BestHit as a single Database over all sequences."""

    def __init__(self, sequences: Sequence, configure, group=None):
        from . import Database

        self._init_group(group)
        self.n_total = len(sequences)
        self.local_to_global = shard_indices([len(s) for s in sequences], self.world)[self.rank]
        local = [sequences[i] for i in self.local_to_global]
        self.db = configure(Database.builder().sequences(local)).build()
        self._d_l2g = None

    def _init_group(self, group):
        import torch.distributed as dist

        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0

    @classmethod
    def from_concat(cls, residues, offsets, configure, group=None) -> "ShardedDatabase":
        """The same sharding over a database given as concatenated residues and offsets (every rank
        passes the whole database; each keeps only its shard on its device)."""
        from . import Database

        self = cls.__new__(cls)
        self._init_group(group)
        offsets = np.asarray(offsets, dtype=np.uint64)
        self.n_total = len(offsets) - 1
        self.local_to_global = shard_indices(np.diff(offsets.astype(np.int64)), self.world)[self.rank]
        loc_res, loc_off = take_sequences(residues, offsets, self.local_to_global)
        self.db = configure(Database.builder().sequences_concat(loc_res, loc_off)).build()
        self._d_l2g = None
        return self

    @classmethod
    def from_shard(cls, residues, offsets, local_to_global, n_total: int, configure,
                   group=None) -> "ShardedDatabase":
        """A rank that already holds its own shard (for example read from its own file): its
        sequences as concatenated residues and offsets, their global indices in ascending order,
        and the size of the whole database. Shards must partition 0..n_total."""
        from . import Database

        self = cls.__new__(cls)
        self._init_group(group)
        self.n_total = int(n_total)
        self.local_to_global = np.asarray(local_to_global, dtype=np.int64)
        if len(self.local_to_global) != len(offsets) - 1 or np.any(np.diff(self.local_to_global) <= 0):
            raise ValueError("local_to_global must give one ascending global index per sequence")
        self.db = configure(Database.builder().sequences_concat(residues, offsets)).build()
        self._d_l2g = None
        return self

    def merge_device_hits(self, hits_u8):
        """Per-query best hits of the whole database from this shard's device hit records ([Q, 32]
        uint8 hy_hit, as hy_scan_device writes them): rows (score, global index, query end,
        target end) on the device, after one all_gather over the group (NCCL)."""
        import torch

        if self._d_l2g is None or self._d_l2g.device != hits_u8.device:
            self._d_l2g = torch.as_tensor(self.local_to_global, dtype=torch.int64, device=hits_u8.device)
        rows = device_hit_rows(hits_u8, self._d_l2g)
        return rows if self.world == 1 else all_gather_best(rows, self.group)

    def scan(self, scratch, query):
        from . import BestHit

        rows = hit_rows([self.db.scan(scratch, query)], self.local_to_global)
        m = self._gather(rows)[0].tolist()
        return BestHit(int(m[0]), int(m[1]), None if m[2] < 0 else int(m[2]), None if m[3] < 0 else int(m[3]))

    def scan_scores(self, scratch, query) -> np.ndarray:
        import torch

        local = torch.from_numpy(self.db.scan_scores_array(scratch, query)).to(self._device())
        return all_gather_scores(local, self.local_to_global, self.n_total, self.group).cpu().numpy()

    def scan_all(self, scratch, query) -> list:
        """One BestHit per sequence of the whole database, in global order (db_index global)."""
        import torch

        from . import BestHit

        arr = self.db.scan_all_array(scratch, query)
        g = np.asarray(self.local_to_global, dtype=np.int64)
        rows = np.empty((len(g), HIT_COLUMNS), np.int64)
        for k in range(len(g)):
            rows[k] = (arr[k].score, g[k], arr[k].query_end, arr[k].target_end)
        local = torch.from_numpy(rows).to(self._device())
        if self.world == 1:
            full = local.cpu().numpy()
        else:
            full = all_gather_hits(local, self.local_to_global, self.n_total, self.group).cpu().numpy()
        return [BestHit(int(r[0]), int(r[1]), None if r[2] < 0 else int(r[2]), None if r[3] < 0 else int(r[3]))
                for r in full]

    def scan_aligned(self, scratch, query):
        """The winner's (global index, Alignment) over the whole database (SearchType.Alignment
        databases): every shard's own winner, the best of them by the scan's tie-break."""
        import torch.distributed as dist

        hit = self.db.scan_aligned(scratch, query)
        mine = (int(hit.alignment.score), int(self.local_to_global[hit.db_index]), hit.alignment)
        if self.world == 1:
            return mine[1], mine[2]
        cands = [None] * self.world
        dist.all_gather_object(cands, mine, group=self.group)
        best = merge_aligned(cands)
        return best[1], best[2]

    def scan_all_aligned(self, scratch, query) -> list:
        """Every sequence's Alignment over the whole database, in global order."""
        import torch.distributed as dist

        out = []
        self.db.scan_all_aligned(scratch, query, out)
        mine = list(zip((int(i) for i in self.local_to_global), out))
        if self.world == 1:
            parts = [mine]
        else:
            parts = [None] * self.world
            dist.all_gather_object(parts, mine, group=self.group)
        full = [None] * self.n_total
        for part in parts:
            for gi, a in part:
                full[gi] = a
        return full

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
