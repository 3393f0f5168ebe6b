"""The multi-GPU exchange of the sharded scan (hyalite_b200/sharded.py), run as two gloo ranks on
the CPU: each rank scans its shard with the oracle (standing in for its GPU), and the package's
all-gather and merge must reproduce the single-database results, ties across shards included
(src/database.rs:160-208: higher score, then smaller global index)."""
import os
import socket
from collections import namedtuple

import numpy as np
import pytest

import pyoracle as o
from conftest import DNA

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from hyalite_b200 import sharded  # noqa: E402

Hit = namedtuple("Hit", "score db_index query_end target_end")


def _workload(seed=7):
    rng = np.random.default_rng(seed)
    seqs = [list(rng.integers(0, 4, int(n))) for n in rng.integers(0, 120, 301)]
    q = list(rng.integers(0, 4, 60))
    # Planted ties: the same sequence at several global indices that land on different shards.
    for k in (5, 6, 150, 299):
        seqs[k] = q[10:50]
    queries = [q, list(rng.integers(0, 4, 30)), [], q[::-1]]
    return seqs, queries


def test_shard_indices_partition_and_balance():
    rng = np.random.default_rng(1)
    lengths = rng.integers(1, 1000, 10_001)
    for world in (1, 2, 3, 8):
        parts = sharded.shard_indices(lengths, world)
        allidx = np.concatenate(parts)
        assert sorted(allidx.tolist()) == list(range(len(lengths)))
        assert all(np.all(np.diff(p) > 0) for p in parts)  # ascending global order
        res = [int(lengths[p].sum()) for p in parts]
        assert max(res) - min(res) <= 2 * int(lengths.max())


def test_take_sequences_gathers_a_shard():
    rng = np.random.default_rng(2)
    seqs = [list(rng.integers(0, 20, int(n))) for n in rng.integers(0, 50, 200)]
    res, off = o.concat(seqs)
    for world in (1, 3):
        for mine in sharded.shard_indices([len(x) for x in seqs], world):
            r, f = sharded.take_sequences(res, off, mine)
            assert [list(r[int(f[i]):int(f[i + 1])]) for i in range(len(mine))] == [seqs[k] for k in mine]


def test_merge_aligned_tie_break():
    cands = [(30, 9, "a"), (31, 12, "b"), (31, 4, "c"), (29, 1, "d")]
    assert sharded.merge_aligned(cands) == (31, 4, "c")


def test_merge_hit_rows_tie_break():
    rows = torch.tensor([[[10, 7, 1, 2], [5, 3, -1, -1]],
                         [[10, 4, 3, 4], [6, 9, 0, 0]],
                         [[9, 0, 5, 5], [6, 8, 1, 1]]], dtype=torch.int64)
    m = sharded.merge_hit_rows(rows)
    assert m.tolist() == [[10, 4, 3, 4], [6, 8, 1, 1]]


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seqs, queries = _workload()
        mine = sharded.shard_indices([len(s) for s in seqs], world)[rank]
        local = [seqs[i] for i in mine]
        for mode, st in ((0, 1), (1, 1), (2, 0), (4, 1)):
            ref_local = o.OracleDb(local, DNA, 4, 2, 1, mode, st)
            ref_full = o.OracleDb(seqs, DNA, 4, 2, 1, mode, st)
            for q in queries:
                rows = sharded.hit_rows([Hit(*ref_local.scan(q))], mine)
                got = sharded.all_gather_best(rows)[0].tolist()
                want = ref_full.scan(q)
                want = [want[0], want[1], -1 if want[2] is None else want[2], -1 if want[3] is None else want[3]]
                assert got == want, (rank, mode, st, len(q), got, want)
                scores = sharded.all_gather_scores(torch.from_numpy(ref_local.scan_scores(q)), mine, len(seqs))
                assert np.array_equal(scores.numpy(), ref_full.scan_scores(q)), (rank, mode, len(q))
                # scan_all: every shard's per-target hits, scattered to global order.
                local_all = sharded.hit_rows([Hit(*h) for h in ref_local.scan_all(q)], mine)
                got_all = sharded.all_gather_hits(local_all, mine, len(seqs)).tolist()
                want_all = [[s, k, -1 if qe is None else qe, -1 if te is None else te]
                            for (s, _, qe, te), k in zip(ref_full.scan_all(q), range(len(seqs)))]
                assert got_all == want_all, (rank, mode, st, len(q))
            if mode in (0, 2):
                # scan_aligned / scan_all_aligned: the winner's alignment, and every alignment.
                for q in queries:
                    k, aln = ref_local.scan_aligned(q)
                    cands = [None] * world
                    dist.all_gather_object(cands, (aln[0], int(mine[k]), aln))
                    best = sharded.merge_aligned(cands)
                    assert (best[1], best[2]) == ref_full.scan_aligned(q), (rank, mode, len(q))
                    parts = [None] * world
                    dist.all_gather_object(parts, list(zip(mine.tolist(), ref_local.scan_all_aligned(q))))
                    full = [None] * len(seqs)
                    for part in parts:
                        for gi, a in part:
                            full[gi] = a
                    assert full == ref_full.scan_all_aligned(q), (rank, mode, len(q))
        open(os.path.join(out_dir, f"ok{rank}"), "w").close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reproduce_the_single_database_scan(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert os.path.exists(tmp_path / "ok0") and os.path.exists(tmp_path / "ok1")
