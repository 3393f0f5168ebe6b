"""Layouts (src/inter.rs:317-351): forceable and reported back like the reference's
`layout_is_reported_and_overridable` (src/database.rs:1194-1240), and a forced Precomputed database
(pair-code columns, one pair table per pass) gives exactly the oracle's results."""
import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, DNA
from gpu_helpers import BLOSUM62, hit_tuple, rand_seqs

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu


def _build(seqs, mat, al, go, ge, mode, st, mql, layout=None):
    b = (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(al, mat, go, ge)).mode(hy.Mode(mode))
         .search_type(hy.SearchType(st)).max_query_len(mql))
    if layout is not None:
        b = b.layout(hy.LayoutChoice.Force(layout))
    return b.build()


def test_layout_is_reported_and_overridable():
    seqs = [[0, 1, 2, 3], [2, 2]]
    # Auto: a small alphabet's pair table is compact, so Precomputed; protein resolves to Gathered.
    assert _build(seqs, DNA, 4, 2, 1, 3, 1, 8).layout() == hy.Layout.Precomputed
    assert _build(seqs, BLOSUM62, 20, 11, 1, 3, 1, 8).layout() == hy.Layout.Gathered
    for layout in (hy.Layout.Gathered, hy.Layout.Precomputed):
        assert _build(seqs, DNA, 4, 2, 1, 3, 1, 8, layout).layout() == layout
        assert _build(seqs, BLOSUM62, 20, 11, 1, 3, 1, 8, layout).layout() == layout


def _check(seqs, mat, al, go, ge, mode, st, queries, mql, layout=hy.Layout.Precomputed):
    db = _build(seqs, mat, al, go, ge, mode, st, mql, layout)
    ref = o.OracleDb(seqs, mat, al, go, ge, mode, st)
    sc = hy.Scratch(db)
    for q in queries:
        assert hit_tuple(db.scan(sc, q)) == ref.scan(q), f"scan mode={mode} st={st} len={len(q)}"
        got = [(h.score, h.db_index, None if h.query_end < 0 else h.query_end,
                None if h.target_end < 0 else h.target_end) for h in db.scan_all_array(sc, q)]
        assert got == ref.scan_all(q), f"scan_all mode={mode} st={st} len={len(q)}"
        assert np.array_equal(db.scan_scores_array(sc, q), ref.scan_scores(q))
    return db


@pytest.mark.parametrize("mode", ALL_MODES)
def test_precomputed_dna_every_mode(mode):
    rng = np.random.default_rng(500 + mode)
    seqs = rand_seqs(rng, 90, 4, 0, 300) + rand_seqs(rng, 2, 4, 4100, 4600)
    queries = [list(rng.integers(0, 4, n)) for n in (0, 1, 40, 64, 65, 200, 257, 600)]
    for st in (0, 1):
        for layout in (hy.Layout.Precomputed, hy.Layout.Gathered):
            _check(seqs, DNA, 4, 2, 1, mode, st, queries, 600, layout)


def test_precomputed_protein_and_int32_partition():
    # A 441-letter pair table: the bulk kernel runs 8 rows per lane and the long pairs and band
    # read the table from global memory; large entries put the longest targets in int32.
    rng = np.random.default_rng(510)
    seqs = rand_seqs(rng, 60, 20, 1, 400) + rand_seqs(rng, 3, 20, 2100, 4600)
    queries = [list(rng.integers(0, 20, n)) for n in (30, 300, 1000)]
    for mode in (0, 2):
        _check(seqs, BLOSUM62, 20, 11, 1, mode, 1, queries, 1000)
    big = [int(v) for v in rng.integers(-20, 61, 16)]
    seqs = rand_seqs(rng, 40, 4, 1, 300) + rand_seqs(rng, 2, 4, 3000, 3200)
    db = _check(seqs, big, 4, 5, 1, 1, 1, [list(rng.integers(0, 4, n)) for n in (100, 700)], 700)
    assert db.partition()[1] > 0


def test_batch_server_and_noalloc_on_mixed_layouts():
    import ctypes as C

    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(520)
    seqs = rand_seqs(rng, 400, 4, 1, 250) + rand_seqs(rng, 2, 4, 4100, 4500)
    dbs = [_build(seqs, DNA, 4, 2, 1, m, 1, 700, lay)
           for m in (0, 1, 2) for lay in (hy.Layout.Precomputed, hy.Layout.Gathered)]
    pseqs = rand_seqs(rng, 200, 20, 1, 300)
    dbs.append(_build(pseqs, BLOSUM62, 20, 11, 1, 0, 1, 700))
    queries, dbq = [], []
    for i in range(21):
        k = i % len(dbs)
        al = 20 if k == len(dbs) - 1 else 4
        queries.append(list(rng.integers(0, al, int(rng.integers(0, 701)))))
        dbq.append(k)
    plain = [hit_tuple(dbs[k].scan(hy.Scratch(dbs[k]), q)) for q, k in zip(queries, dbq)]
    batch = hy.Batch(dbs, max_queries=32, autotune=False)
    assert [hit_tuple(h) for h in batch.scan(queries, dbq)] == plain
    srv = hy.Server(dbs, max_batch=8)
    hs = [srv.submit(q, db=k) for q, k in zip(queries, dbq)]
    assert [hit_tuple(srv.wait(h)) for h in hs] == plain
    srv.close()
    # The allocation-free scores on a Precomputed database equal the allocating scan's.
    db = dbs[0]
    q = rng.integers(0, 4, 500).astype(np.uint8)
    d_q = torch.from_numpy(q).cuda()
    out = torch.zeros(db.sequence_count(), dtype=torch.int32, device="cuda")
    st = hy._abi.lib.hy_scan_scores_noalloc(db._h, C.c_void_p(d_q.data_ptr()), len(q), C.c_void_p(out.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    assert np.array_equal(out.cpu().numpy(), db.scan_scores_array(hy.Scratch(db), q))
