"""ShardedDatabase end to end on the device: two ranks (gloo for the exchange, both on cuda:0),
each scanning its shard with the CUDA kernels, must return the single-database answers of the
oracle for scan, scan_scores, scan_all, scan_aligned and scan_all_aligned, ties across shards
included (src/database.rs:83-565). The ranks' kernels never wait on one another: each rank scans
alone and the exchange runs on the host."""
import os
import socket

import numpy as np
import pytest

import pyoracle as o

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _workload():
    rng = np.random.default_rng(41)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = [rng.integers(0, 20, int(n)).astype(np.uint8) for n in rng.integers(0, 400, 1500)]
    seqs.append(rng.integers(0, 20, 3000).astype(np.uint8))  # an int32 sequence
    q = rng.integers(0, 20, 300).astype(np.uint8)
    for k in (10, 11, 700, 1499):  # the same best target on both shards: the smallest index wins
        seqs[k] = q[40:200].copy()
    queries = [q, rng.integers(0, 20, 1000).astype(np.uint8), np.zeros(0, np.uint8), q[::-1].copy()]
    return mat, seqs, queries


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        import hyalite_b200 as hy
        from hyalite_b200 import sharded

        mat, seqs, queries = _workload()
        res, off = o.concat(seqs)
        for st in (hy.SearchType.ScoreEnd, hy.SearchType.alignment(hy.USIZE_MAX)):
            conf = lambda b: b.scoring(hy.Scoring(20, mat, 11, 1)).mode(hy.Mode.Sw).search_type(st).max_query_len(1000)
            sdb = sharded.ShardedDatabase.from_concat(res, off, conf)
            assert sdb.db.sequence_count() < len(seqs)
            sc = hy.Scratch(sdb.db)
            ref = o.OracleDb((res, off), mat, 20, 11, 1, 0, 1)
            for q in queries:
                h = sdb.scan(sc, q)
                assert (h.score, h.db_index, h.query_end, h.target_end) == ref.scan(q), (rank, len(q))
                assert np.array_equal(sdb.scan_scores(sc, q), ref.scan_scores(q))
                got = [(h.score, h.db_index, h.query_end, h.target_end) for h in sdb.scan_all(sc, q)]
                assert got == ref.scan_all(q), (rank, len(q))
                if st != hy.SearchType.ScoreEnd:
                    k, aln = sdb.scan_aligned(sc, q)
                    assert (k, aln.as_tuple()) == ref.scan_aligned(q), (rank, len(q))
                    if len(q) <= 300:
                        alns = sdb.scan_all_aligned(sc, q)
                        assert [a.as_tuple() for a in alns] == ref.scan_all_aligned_mt(q), (rank, len(q))
            # The device merge of hy_scan_device records (the benchmark's timed path).
            if st == hy.SearchType.ScoreEnd:
                import ctypes as C

                d_hits = torch.zeros((len(queries), 32), dtype=torch.uint8, device="cuda")
                for i, q in enumerate(queries):
                    d_q = torch.tensor(q if len(q) else [0], dtype=torch.uint8, device="cuda")
                    torch.cuda.synchronize()
                    assert hy._abi.lib.hy_scan_device(sdb.db._h, sc._h, C.c_void_p(d_q.data_ptr()), len(q),
                                                      C.c_void_p(d_hits[i].data_ptr())) == 0
                    assert hy._abi.lib.hy_scratch_sync(sc._h) == 0
                rows = sdb.merge_device_hits(d_hits).cpu().tolist()
                for q, r in zip(queries, rows):
                    s, k, qe, te = ref.scan(q)
                    assert r == [s, k, -1 if qe is None else qe, -1 if te is None else te]
        open(os.path.join(out_dir, f"ok{rank}"), "w").close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_on_device_reproduce_the_single_database(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert os.path.exists(tmp_path / "ok0") and os.path.exists(tmp_path / "ok1")
