"""The served form (hy_server): each request's result must be the same when it runs alone on an
idle server and when it is batched with others arriving at the same time, and equal to the
plain scan / scan_scores of its database. Admission by memory budget, rejection and statistics."""
import threading

import numpy as np
import pytest

import pyoracle as o
from gpu_helpers import build, hit_tuple, rand_seqs

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu


def _setup(seed=21):
    rng = np.random.default_rng(seed)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = rand_seqs(rng, 1500, 20, 1, 400) + rand_seqs(rng, 3, 20, 2200, 4300)
    dbs = [build(seqs, mat, 20, 11, 1, mode, 1, 1200) for mode in (0, 2, 4)]
    reqs = []
    for i in range(36):
        L = int(rng.choice([0, 10, 50, 100, 300, 700, 1200]))
        reqs.append((list(rng.integers(0, 20, L)), i % 3, bool(i % 4 == 1)))
    return rng, mat, seqs, dbs, reqs


def _result(hit, req):
    return hit_tuple(hit), (None if req.scores is None else req.scores.copy())


def test_same_result_alone_and_in_the_mix():
    rng, mat, seqs, dbs, reqs = _setup()
    srv = hy.Server(dbs, max_batch=16, in_flight=2)
    alone = []
    for q, k, sc in reqs:
        r = srv.submit(q, db=k, want_scores=sc)
        alone.append(_result(srv.wait(r), r))
    # The mix: every request submitted at once from four threads, then all waited for.
    handles = [None] * len(reqs)

    def submitter(part):
        for i in part:
            q, k, sc = reqs[i]
            handles[i] = srv.submit(q, db=k, want_scores=sc)

    ts = [threading.Thread(target=submitter, args=(range(t, len(reqs), 4),)) for t in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    mixed = [_result(srv.wait(h), h) for h in handles]
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["rejected"] == 0
    assert st["batches"] < 2 * len(reqs)  # the mix was batched
    for i, ((q, k, sc), a, m) in enumerate(zip(reqs, alone, mixed)):
        assert a[0] == m[0], f"request {i}: alone {a[0]} mixed {m[0]}"
        if sc:
            assert np.array_equal(a[1], m[1])
    # Both equal the plain calls of each database.
    scratch = [hy.Scratch(d) for d in dbs]
    for (q, k, sc), a in zip(reqs, alone):
        if sc:
            want = dbs[k].scan_scores_array(scratch[k], q)
            assert np.array_equal(a[1], want)
            assert a[0][0] == int(want.max()) and a[0][1] == int(np.argmax(want))
        else:
            assert a[0] == hit_tuple(dbs[k].scan(scratch[k], q))
    srv.close()


def test_results_match_the_oracle():
    rng, mat, seqs, dbs, reqs = _setup(22)
    srv = hy.Server(dbs, max_batch=8, in_flight=3)
    hs = [srv.submit(q, db=k) for q, k, _ in reqs[:12]]
    for h, (q, k, _) in zip(hs, reqs[:12]):
        mode = (0, 2, 4)[k]
        assert hit_tuple(srv.wait(h)) == o.OracleDb(seqs, mat, 20, 11, 1, mode, 1).scan(q)
        assert h.latency_ms is not None and h.latency_ms > 0.0  # submit to ready (hy_server_wait_timed)
    srv.close()


def test_admission_by_memory_budget_and_rejection():
    rng, mat, seqs, dbs, reqs = _setup(23)
    probe = hy.Server(dbs, max_batch=4)
    per, _ = probe.request_bytes(1200, db=0)
    probe.close()
    assert per > 0
    # A profile budget that holds two 1200-residue queries per batch.
    srv = hy.Server(dbs, max_batch=32, in_flight=1, profile_budget=2 * per + 64)
    qs = [list(rng.integers(0, 20, 1200)) for _ in range(6)]
    hs = [srv.submit(q, db=0) for q in qs]
    got = [srv.wait(h) for h in hs]
    st = srv.stats()
    assert st["completed"] == 6 and st["batches"] >= 3 and st["mean_batch"] <= 2.0
    scratch = hy.Scratch(dbs[0])
    for q, h in zip(qs, got):
        assert hit_tuple(h) == hit_tuple(dbs[0].scan(scratch, q))
    # A request larger than the profile budget alone can never be admitted.
    with pytest.raises(hy.Error) as e:
        hy.Server(dbs, max_batch=4, profile_budget=per // 2).submit(qs[0], db=0)
    assert e.value.kind == "Rejected"
    # A scores request larger than the score budget can never be admitted.
    small = hy.Server(dbs, max_batch=4, scores_budget=1024)
    with pytest.raises(hy.Error) as e:
        small.submit([1, 2, 3], db=0, want_scores=True)
    assert e.value.kind == "Rejected"
    assert small.stats()["rejected"] == 1
    small.close()
    srv.close()


def test_submit_validation_and_close_with_work_queued():
    rng, mat, seqs, dbs, reqs = _setup(24)
    srv = hy.Server(dbs, max_batch=4)
    with pytest.raises(hy.Error) as e:
        srv.submit([0] * 1201, db=0)
    assert e.value.kind == "QueryTooLong"
    with pytest.raises(hy.Error) as e:
        srv.submit([25], db=0)
    assert e.value.kind == "SymbolOutOfRange"
    with pytest.raises(hy.Error) as e:
        srv.submit([1], db=7)
    assert e.value.kind == "InvalidArgument"
    for q, k, sc in reqs:
        srv.submit(q, db=k, want_scores=sc)
    srv.close()  # completes the queued work before returning
