"""The batched form (hy_scan_batch): every query's hit must equal the plain scan's and the oracle's,
whatever the mix of modes, search types and query lengths, the launch configuration, the batch
size from call to call, and the autotuner's choices."""
import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, DNA
from gpu_helpers import build, hit_tuple, rand_seqs

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu


def _dbs(seqs, mat, al, go, ge, mql, sts=(1,)):
    """One database per (mode, search type) over the same sequences."""
    out = []
    for st in sts:
        for mode in ALL_MODES:
            out.append((mode, st, build(seqs, mat, al, go, ge, mode, st, mql)))
    return out


def _check_batch(batch, dbs, seqs, mat, al, go, ge, queries, dbq):
    hits = batch.scan(queries, dbq)
    sc = {}
    for i, (q, k) in enumerate(zip(queries, dbq)):
        mode, st, db = dbs[k]
        s = sc.setdefault(k, hy.Scratch(db))
        plain = hit_tuple(db.scan(s, q))
        got = hit_tuple(hits[i])
        want = o.OracleDb(seqs, mat, al, go, ge, mode, st).scan(q)
        assert got == plain == want, f"query {i} mode {mode} st {st} len {len(q)}: batch {got} plain {plain} oracle {want}"


def test_mixed_modes_lengths_and_search_types_dna():
    rng = np.random.default_rng(11)
    seqs = rand_seqs(rng, 300, 4, 0, 180)
    dbs = _dbs(seqs, DNA, 4, 2, 1, 700, sts=(0, 1))
    lengths = [0, 1, 5, 32, 63, 64, 65, 100, 192, 193, 256, 257, 400, 700]
    queries, dbq = [], []
    for i, L in enumerate(lengths * 2):
        queries.append(list(rng.integers(0, 4, L)))
        dbq.append(i % len(dbs))
    batch = hy.Batch([d for _, _, d in dbs], max_queries=64, autotune=False)
    _check_batch(batch, dbs, seqs, DNA, 4, 2, 1, queries, dbq)


def test_protein_long_targets_int32_and_long_pairs():
    # Targets wider than the long-pair split and sequences the device runs in int32 lanes.
    rng = np.random.default_rng(12)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = rand_seqs(rng, 120, 20, 1, 400) + rand_seqs(rng, 4, 20, 2100, 3000) + rand_seqs(rng, 3, 20, 4100, 5000)
    dbs = _dbs(seqs, mat, 20, 11, 1, 3000)
    queries, dbq = [], []
    for i, L in enumerate([100, 1000, 3000, 250, 600, 2999, 17, 64]):
        queries.append(list(rng.integers(0, 20, L)))
        dbq.append(i % len(dbs))
    batch = hy.Batch([d for _, _, d in dbs], max_queries=16, autotune=False)
    _check_batch(batch, dbs, seqs, mat, 20, 11, 1, queries, dbq)
    n16, n32 = dbs[0][2].partition()
    assert n32 > 0


@pytest.mark.parametrize("cfg", [(64, 192, 2048), (0, 0, 1024), (0, 256, 4096), (128, 512, 512), (1000, 1000, 64)])
def test_every_launch_configuration_gives_the_same_hits(cfg):
    rng = np.random.default_rng(13)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = rand_seqs(rng, 200, 20, 1, 300) + rand_seqs(rng, 3, 20, 1200, 2500)
    dbs = _dbs(seqs, mat, 20, 11, 1, 800)
    queries = [list(rng.integers(0, 20, L)) for L in (20, 70, 150, 300, 520, 800)]
    dbq = [i % 5 for i in range(len(queries))]
    batch = hy.Batch([d for _, _, d in dbs], max_queries=8, autotune=False)
    batch.set_config(*cfg)
    assert batch.config() == cfg
    _check_batch(batch, dbs, seqs, mat, 20, 11, 1, queries, dbq)


def test_graph_replay_with_changing_batches_and_autotune():
    rng = np.random.default_rng(14)
    seqs = rand_seqs(rng, 400, 4, 20, 200)
    dbs = _dbs(seqs, DNA, 4, 2, 1, 500)
    batch = hy.Batch([d for _, _, d in dbs], max_queries=40, autotune=True)
    for n in (40, 1, 7, 0, 23):
        queries = [list(rng.integers(0, 4, int(rng.integers(0, 501)))) for _ in range(n)]
        dbq = [int(rng.integers(0, 5)) for _ in range(n)]
        if n == 0:
            assert batch.scan([], []) == []
            continue
        _check_batch(batch, dbs, seqs, DNA, 4, 2, 1, queries, dbq)
    ms = batch.tune([list(rng.integers(0, 4, 300)) for _ in range(10)], [0] * 10, stride=2)
    assert ms > 0
    r8, r16, lw = batch.config()
    assert 1 <= lw <= 4096


def test_batch_validation_reports_the_first_failing_query():
    seqs = [[0, 1, 2, 3]] * 10
    dbs = _dbs(seqs, DNA, 4, 2, 1, 8)
    batch = hy.Batch([d for _, _, d in dbs], max_queries=4, autotune=False)
    with pytest.raises(hy.Error) as e:
        batch.scan([[0, 1], [0] * 9, [7]], [0, 1, 2])
    assert e.value.kind == "QueryTooLong" and e.value.failed_query == 1
    with pytest.raises(hy.Error) as e:
        batch.scan([[0, 1], [0, 4]], [0, 1])
    assert e.value.kind == "SymbolOutOfRange" and e.value.failed_query == 1
    assert e.value.fields == {"symbol": 4, "alphabet_len": 4}
    with pytest.raises(hy.Error) as e:
        batch.scan([[0]] * 5, [0] * 5)
    assert e.value.kind == "InvalidArgument"
    with pytest.raises(hy.Error) as e:
        batch.scan([[0]], [9])
    assert e.value.kind == "InvalidArgument"
    # The batch still works after the errors.
    assert hit_tuple(batch.scan([[0, 1, 2, 3]], [0])[0]) == o.OracleDb(seqs, DNA, 4, 2, 1, 0, 1).scan([0, 1, 2, 3])


def test_sharded_database_single_rank_equals_the_plain_scan():
    # ShardedDatabase over one gloo rank (the exchange runs, with one participant).
    import os
    import socket

    import torch.distributed as dist

    from hyalite_b200 import sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        rng = np.random.default_rng(15)
        seqs = rand_seqs(rng, 500, 20, 1, 300)
        mat = [int(v) for v in rng.integers(-4, 12, 400)]
        conf = lambda b: b.scoring(hy.Scoring(20, mat, 11, 1)).mode(hy.Mode.Sw).search_type(
            hy.SearchType.ScoreEnd).max_query_len(400)
        sdb = sharded.ShardedDatabase(seqs, conf)
        plain = build(seqs, mat, 20, 11, 1, 0, 1, 400)
        sc, sc2 = hy.Scratch(sdb.db), hy.Scratch(plain)
        for L in (0, 40, 400):
            q = list(rng.integers(0, 20, L))
            assert sdb.scan(sc, q) == plain.scan(sc2, q)
            assert np.array_equal(sdb.scan_scores(sc, q), plain.scan_scores_array(sc2, q))
    finally:
        dist.destroy_process_group()


def test_device_hit_rows_match_the_host_hits():
    import ctypes as C

    import torch

    from hyalite_b200 import sharded

    rng = np.random.default_rng(16)
    seqs = rand_seqs(rng, 300, 20, 1, 300)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    db = build(seqs, mat, 20, 11, 1, 0, 1, 300)
    sc = hy.Scratch(db)
    queries = [list(rng.integers(0, 20, L)) for L in (0, 30, 300)]
    d_hits = torch.zeros((len(queries), 32), dtype=torch.uint8, device="cuda")
    for i, q in enumerate(queries):
        d_q = torch.tensor(q if q else [0], dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        st = hy._abi.lib.hy_scan_device(db._h, sc._h, C.c_void_p(d_q.data_ptr()), len(q),
                                        C.c_void_p(d_hits[i].data_ptr()))
        assert st == 0
        lib_sync = hy._abi.lib.hy_scratch_sync(sc._h)
        assert lib_sync == 0
    g = torch.arange(len(seqs), dtype=torch.int64, device="cuda") + 1000
    rows = sharded.device_hit_rows(d_hits, g).cpu()
    want = sharded.hit_rows([db.scan(sc, q) for q in queries], np.arange(len(seqs)) + 1000)
    assert torch.equal(rows, want)
