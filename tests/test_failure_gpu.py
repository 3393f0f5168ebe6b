"""Failure paths of the device backend, driven from the host without faulting the GPU.

* Bounded device waits: hy_debug_set_wait_polls(0) makes every bounded wait give up at its first
  poll (a block waiting for its query-profile copy, a stripe waiting for the stripe above). The
  call must report Timeout (HY_ERR_TIMEOUT), and the same scratch must give the oracle's results
  once the limit is restored: the kernels let their in-flight copies land before they exit, and
  the error flag is cleared.
* Device allocation failure: hy_debug_fail_device_alloc(k) makes the k-th next device allocation
  fail as on a full device. Every allocation of hy_db_create, hy_scratch_create and
  hy_batch_create is failed in turn: each must return OutOfMemory and leave no allocation behind.
* hy_server_wait with a short timeout returns Timeout and the request stays waitable.

The reference's scan cannot fail (src/database.rs:79-89); these are the device backend's own
error paths (HY_ERR_TIMEOUT, HY_ERR_OUT_OF_MEMORY).
"""
import numpy as np
import pytest

import pyoracle as o
from gpu_helpers import BLOSUM62, hit_tuple

pytestmark = pytest.mark.gpu


def _hy():
    pytest.importorskip("torch")
    import hyalite_b200 as hy

    return hy


class _WaitPolls:
    """Sets the device wait limit for a block and always restores the default."""

    def __init__(self, hy, polls):
        self.lib, self.polls = hy._abi.lib, polls

    def __enter__(self):
        self.lib.hy_debug_set_wait_polls(self.polls)

    def __exit__(self, *exc):
        self.lib.hy_debug_set_wait_polls(-1)


def _protein_db(hy, rng, n=1500, st=None, mql=1000):
    seqs = [rng.integers(0, 20, int(k)).astype(np.uint8) for k in rng.integers(1, 500, n)]
    seqs.append(rng.integers(0, 20, 2500).astype(np.uint8))  # int32 partition
    st = hy.SearchType.ScoreEnd if st is None else st
    db = (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(20, BLOSUM62, 11, 1)).mode(hy.Mode.Sw)
          .search_type(st).max_query_len(mql).build())
    return seqs, db


def test_scan_wait_that_gives_up_is_a_timeout_and_the_scratch_recovers():
    hy = _hy()
    rng = np.random.default_rng(501)
    seqs, db = _protein_db(hy, rng)
    ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, 0, 1)
    sc = hy.Scratch(db)
    q = rng.integers(0, 20, 700).astype(np.uint8)  # several passes for every kernel
    want = ref.scan(q)
    assert hit_tuple(db.scan(sc, q)) == want  # also captures the call's graph
    with _WaitPolls(hy, 0):
        for call in (lambda: db.scan(sc, q), lambda: db.scan_scores_array(sc, q), lambda: db.scan_all_array(sc, q)):
            with pytest.raises(hy.Error) as e:
                call()
            assert e.value.kind == "Timeout"
    assert hit_tuple(db.scan(sc, q)) == want
    assert np.array_equal(db.scan_scores_array(sc, q), ref.scan_scores(q))
    got = [(h.score, h.db_index, None if h.query_end < 0 else h.query_end, None if h.target_end < 0 else h.target_end)
           for h in db.scan_all_array(sc, q)]
    assert got == ref.scan_all(q)


def test_band_cluster_wait_that_gives_up_is_a_timeout_and_the_scratch_recovers():
    # A 2000-residue query: 8 band passes of 256 rows, more than one block's shared memory holds
    # (4 pass slices of int16x2 pairs for this alphabet), so the winner's ends run on a cluster of
    # two blocks; every block gives up at its first profile wait and the whole cluster returns.
    hy = _hy()
    rng = np.random.default_rng(507)
    seqs, db = _protein_db(hy, rng, n=800, mql=2000)
    ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, 0, 1)
    sc = hy.Scratch(db)
    q = rng.integers(0, 20, 2000).astype(np.uint8)
    want = ref.scan(q)
    assert hit_tuple(db.scan(sc, q)) == want
    with _WaitPolls(hy, 0):
        with pytest.raises(hy.Error) as e:
            db.scan(sc, q)
        assert e.value.kind == "Timeout"
    assert hit_tuple(db.scan(sc, q)) == want


def test_int32_pipeline_wait_that_gives_up_is_a_timeout_and_the_scratch_recovers():
    # A 3000-residue query against targets longer than 2978 residues: those run in int32 lanes
    # (BLOSUM62's largest entry 11: 11 * 2979 + 11 > 32767), as pipelined passes.
    hy = _hy()
    rng = np.random.default_rng(506)
    seqs = [rng.integers(0, 20, int(k)).astype(np.uint8) for k in rng.integers(1, 400, 300)]
    seqs += [rng.integers(0, 20, int(k)).astype(np.uint8) for k in (3100, 3500, 4200)]
    db = (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(20, BLOSUM62, 11, 1)).mode(hy.Mode.Sw)
          .search_type(hy.SearchType.ScoreEnd).max_query_len(3000).build())
    assert db.partition()[1] > 0
    ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, 0, 1)
    sc = hy.Scratch(db)
    q = seqs[-2][:3000].copy()
    with _WaitPolls(hy, 0):
        with pytest.raises(hy.Error) as e:
            db.scan_scores_array(sc, q)
        assert e.value.kind == "Timeout"
    assert np.array_equal(db.scan_scores_array(sc, q), ref.scan_scores(q))
    assert hit_tuple(db.scan(sc, q)) == ref.scan(q)


def test_batch_wait_that_gives_up_is_a_timeout_and_the_batch_recovers():
    hy = _hy()
    rng = np.random.default_rng(502)
    seqs, db = _protein_db(hy, rng)
    ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, 0, 1)
    queries = [rng.integers(0, 20, int(n)).astype(np.uint8) for n in (50, 300, 900)]
    batch = hy.Batch([db], max_queries=8, autotune=False)
    assert [hit_tuple(h) for h in batch.scan(queries)] == [ref.scan(q) for q in queries]
    with _WaitPolls(hy, 0):
        with pytest.raises(hy.Error) as e:
            batch.scan(queries)
        assert e.value.kind == "Timeout"
    assert [hit_tuple(h) for h in batch.scan(queries)] == [ref.scan(q) for q in queries]


def test_stripe_wait_that_gives_up_is_a_timeout_and_the_next_call_is_exact():
    hy = _hy()
    rng = np.random.default_rng(503)
    q = rng.integers(0, 20, 2000).astype(np.uint8)  # 16 stripes of 128 rows
    t = q.copy()
    mut = rng.random(len(t)) < 0.2
    t[mut] = rng.integers(0, 20, int(mut.sum()))
    scoring = hy.Scoring(20, BLOSUM62, 11, 1)
    want_aln = o.align(q, t, BLOSUM62, 20, 11, 1, 0)[1]
    want_pair = o.align_pair(q, t, BLOSUM62, 20, 11, 1, 0)
    with _WaitPolls(hy, 0):
        with pytest.raises(hy.Error) as e:
            hy.align(q, t, scoring, hy.Mode.Sw, hy.USIZE_MAX)
        assert e.value.kind == "Timeout"
        with pytest.raises(hy.Error) as e:
            hy.align_pair(q, t, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
        assert e.value.kind == "Timeout"
    assert hy.align(q, t, scoring, hy.Mode.Sw, hy.USIZE_MAX).as_tuple() == want_aln
    h = hy.align_pair(q, t, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
    assert (h.score, h.query_end, h.target_end) == want_pair


def _alloc_failures(hy, create):
    """Fails each device allocation `create` makes, in turn; every failure must be OutOfMemory and
    leave the live allocation count where it was. Returns the number of allocations."""
    import gc

    lib = hy._abi.lib
    gc.collect()
    base = lib.hy_debug_live_device_allocations()
    obj = create()
    n = lib.hy_debug_live_device_allocations() - base
    del obj
    gc.collect()
    assert lib.hy_debug_live_device_allocations() == base
    assert n > 0
    try:
        for k in range(n):
            lib.hy_debug_fail_device_alloc(k)
            with pytest.raises(hy.Error) as e:
                create()
            assert e.value.kind == "OutOfMemory", k
            assert lib.hy_debug_live_device_allocations() == base, k
    finally:
        lib.hy_debug_fail_device_alloc(-1)
    obj = create()  # and it works again
    del obj
    gc.collect()
    assert lib.hy_debug_live_device_allocations() == base
    return n


def test_every_device_allocation_failure_is_out_of_memory_without_a_leak():
    hy = _hy()
    rng = np.random.default_rng(504)
    seqs = [rng.integers(0, 20, int(k)).astype(np.uint8) for k in rng.integers(1, 300, 400)]
    seqs.append(rng.integers(0, 20, 2500).astype(np.uint8))
    res, off = hy.concat(seqs)

    def build():
        return (hy.Database.builder().sequences_concat(res, off).scoring(hy.Scoring(20, BLOSUM62, 11, 1))
                .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(1000).build())

    assert _alloc_failures(hy, build) >= 4
    db = build()
    assert _alloc_failures(hy, lambda: hy.Scratch(db)) >= 10
    assert _alloc_failures(hy, lambda: hy.Batch([db], max_queries=4, autotune=False)) >= 4
    # The database still scans exactly after all of it.
    ref = o.OracleDb((res, off), BLOSUM62, 20, 11, 1, 0, 1)
    q = rng.integers(0, 20, 400).astype(np.uint8)
    assert hit_tuple(db.scan(hy.Scratch(db), q)) == ref.scan(q)


def test_server_wait_with_a_short_timeout():
    hy = _hy()
    rng = np.random.default_rng(505)
    seqs, db = _protein_db(hy, rng, n=40_000, mql=3000)
    srv = hy.Server([db], max_batch=4, in_flight=1)
    try:
        q = rng.integers(0, 20, 3000).astype(np.uint8)
        req = srv.submit(q)
        with pytest.raises(hy.Error) as e:
            srv.wait(req, timeout=1e-6)
        assert e.value.kind == "Timeout"
        got = srv.wait(req, timeout=600.0)
    finally:
        srv.close()
    assert hit_tuple(got) == hit_tuple(db.scan(hy.Scratch(db), q))
