"""The benchmark workloads at (or near) their stated sizes, bit for bit against the oracle.

Each test uses bench.py's own seeded generators, so what is checked here is what the benchmark
measures:

* the small DNA scan (10,000 sequences of 50..300 bp, 50 planted 5%-substituted copies of the
  first 64-bp query): scan, scan_all and scan_scores of 20 queries;
* the batched multi-mode DNA scan (reads from the 5 Mb genome with substitutions and indels,
  queries of 32..2000 bp, SW/NW/HW/SHW/OV round-robin): a 50,000-read slice through hy_scan_batch
  and through Database.scan;
* the served protein scan (the log-normal protein generator at 100,000 sequences, log-normal query
  lengths, half scan and half scan_scores requests): every served result against the plain call,
  a sample against the oracle;
* align_pairs over (read, window) pairs (HW, gap_open 6): 1,000,000 pairs (16 chunks), a sample
  of 3,000 against the oracle.

The oracle's best hit of a scan is taken from its scan_all (per-target scores and ends, threaded):
the reference's scan returns the highest score with the smallest db_index on ties
(src/database.rs:117-130, 173-180), and its winner's ends are align_core's on that target, which
are the ends scan_all reports for it (src/database.rs:186-197, 395-402).
"""
import math

import numpy as np
import pytest

import bench
import pyoracle
from gpu_helpers import hit_tuple

pytestmark = pytest.mark.gpu

DNA = [2 if a == b else -1 for a in range(4) for b in range(4)]


def _hy():
    pytest.importorskip("torch")
    import hyalite_b200 as hy

    return hy


def best_of(all_hits, search_type):
    """The reference scan's BestHit from per-target (score, index, query_end, target_end)."""
    best = None
    for h in all_hits:
        if best is None or h[0] > best[0]:
            best = h
    if search_type == 0:  # Score: no ends
        return (best[0], best[1], None, None)
    return best


def test_small_dna_scan_at_benchmark_size():
    hy = _hy()
    from gpu_helpers import check

    seqs, queries, planted = bench.make_dna_small_workload(2024, 20)
    assert len(seqs) == 10_000 and len(planted) == 50
    db = check(seqs, DNA, 4, 2, 1, 0, 1, queries, mql=64)
    # The planted near-copies of the first query win its scan.
    assert db.scan(hy.Scratch(db), queries[0]).db_index in set(int(k) for k in planted)


def test_batched_multimode_reads_slice_against_the_oracle():
    hy = _hy()
    residues, offsets, queries = bench.make_reads_workload(2024, 50_000, 10)
    modes = [hy.Mode.Sw, hy.Mode.Nw, hy.Mode.Hw, hy.Mode.Shw, hy.Mode.Ov]
    dbs = [(hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(4, DNA, 2, 1))
            .mode(m).search_type(hy.SearchType.ScoreEnd).max_query_len(2000).build()) for m in modes]
    dbq = [i % len(modes) for i in range(len(queries))]
    batch = hy.Batch(dbs, max_queries=len(queries), autotune=False)
    got_b = [hit_tuple(h) for h in batch.scan(queries, dbq)]
    scratches = [hy.Scratch(d) for d in dbs]
    got_p = [hit_tuple(dbs[k].scan(scratches[k], q)) for q, k in zip(queries, dbq)]
    refs = [pyoracle.OracleDb((residues, offsets), DNA, 4, 2, 1, int(m), 1) for m in modes]
    for i, (q, k) in enumerate(zip(queries, dbq)):
        want = best_of(refs[k].scan_all(q, threads=32), 1)
        assert got_p[i] == want, (i, modes[k], len(q), got_p[i], want)
        assert got_b[i] == want, (i, modes[k], len(q), got_b[i], want)


def test_served_protein_scan_at_100k_sequences():
    hy = _hy()
    mat, residues, offsets, _ = bench.make_workload(2024, n_seqs=100_000)
    go, ge, al = bench.GO, bench.GE, bench.AL
    db = (hy.Database.builder().sequences_concat(residues, offsets).scoring(hy.Scoring(al, mat, go, ge))
          .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(3000).build())
    # Requests as the served workload draws them: log-normal lengths (median 350, 50..3000), the
    # generator's background, half ScoreEnd scans and half scan_scores.
    rng = np.random.default_rng(99)
    base = np.random.default_rng(12345)
    base.integers(-4, 4, size=(al, al))
    base.integers(4, 12, size=al)
    background = base.dirichlet(np.full(al, 4.0))
    reqs = []
    for i in range(16):
        n = int(np.clip(round(math.exp(math.log(350.0) + 0.8 * rng.standard_normal())), 50, 3000))
        reqs.append((rng.choice(al, size=n, p=background).astype(np.uint8), i % 2 == 1))
    srv = hy.Server([db], max_batch=8, in_flight=2)
    handles = [srv.submit(q, want_scores=s) for q, s in reqs]
    served = [(srv.wait(h), h.scores) for h in handles]
    srv.close()
    sc = hy.Scratch(db)
    for (q, s), (hit, scores) in zip(reqs, served):
        if s:
            assert np.array_equal(scores, db.scan_scores_array(sc, q))
        else:
            assert hit_tuple(hit) == hit_tuple(db.scan(sc, q))
    # The oracle on the shortest request of each kind.
    ref = pyoracle.OracleDb((residues, offsets), mat, al, go, ge, 0, 1)
    for want_scores in (False, True):
        i = min((i for i in range(len(reqs)) if reqs[i][1] == want_scores), key=lambda i: len(reqs[i][0]))
        q = reqs[i][0]
        if want_scores:
            assert np.array_equal(served[i][1], ref.scan_scores(q, threads=32))
        else:
            assert hit_tuple(served[i][0]) == best_of(ref.scan_all(q, threads=32), 1)


def test_align_pairs_reads_in_windows_sample_against_the_oracle():
    hy = _hy()
    q_res, q_off, t_res, t_off = bench.make_pairs_workload(2024, 1_000_000)
    scoring = hy.Scoring(4, DNA, 6, 1)
    hits, (err, _) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Hw, hy.SearchType.ScoreEnd)
    assert err is None
    rng = np.random.default_rng(1)
    sample = np.sort(np.concatenate([rng.choice(len(q_off) - 1, 3000, replace=False), [0, len(q_off) - 2]]))
    qs = [q_res[int(q_off[i]):int(q_off[i + 1])] for i in sample]
    ts = [t_res[int(t_off[i]):int(t_off[i + 1])] for i in sample]
    st, want, _ = pyoracle.align_pairs(qs, ts, DNA, 4, 6, 1, 2, 1, threads=32)
    assert st == 0
    got = [(hits[i].score, int(i), None if hits[i].query_end < 0 else hits[i].query_end,
            None if hits[i].target_end < 0 else hits[i].target_end) for i in sample]
    assert got == [(w[0], int(i), w[2], w[3]) for w, i in zip(want, sample)]
    # Reads placed in their windows: nearly every pair aligns the whole read.
    scores = np.array([hits[i].score for i in sample])
    assert np.median(scores) > 200
