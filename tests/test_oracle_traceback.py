"""Pins the oracle's traceback (hyo_traceback / hyo_align, restating src/align.rs) to the
reference before it checks the device traceback: every known answer of src/align/tests.rs,
tests/traceback.rs and tests/database_alignment.rs, the budget rule and its monotonicity
(src/align/tests.rs:345-365, 467-500), and the structural properties those files check over random
inputs (re-scoring, spans, symbol equality, optimality against the brute-force scorer)."""
import json
import os

import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, Lcg, identity_matrix

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "traceback_known_answers.json")) as f:
    G = json.load(f)

CODE = {c: i for i, c in enumerate(o.OPS)}


def scoring(name):
    s = G["scorings"][name]
    mat = identity_matrix(s["al"], *s["id"])
    for idx, v in s.get("set", []):
        mat[idx] = v
    return mat, s["al"], s["go"], s["ge"]


def gap(go, ge, n):
    return 0 if n == 0 else go + (n - 1) * ge


def rescore(a, q, t, mat, al, go, ge):
    """tests/traceback.rs:16-56: re-score from the ops, affine per maximal gap run."""
    score, qs, qe, ts, te, ops = a
    qi, tj, total, k = qs, ts, 0, 0
    while k < len(ops):
        op = ops[k]
        if op in (0, 1):
            total += mat[q[qi] * al + t[tj]]
            qi, tj, k = qi + 1, tj + 1, k + 1
        else:
            run = 0
            while k < len(ops) and ops[k] == op:
                run, k = run + 1, k + 1
                if op == 2:
                    qi += 1
                else:
                    tj += 1
            total -= gap(go, ge, run)
    return total


def assert_consistent(a, q, t, mat, al, go, ge, mode):
    """src/align/tests.rs:76-127."""
    score, qs, qe, ts, te, ops = a
    assert score == o.align_pair(q, t, mat, al, go, ge, mode, 0)[0]
    assert rescore(a, q, t, mat, al, go, ge) == score
    assert qs <= qe <= len(q) and ts <= te <= len(t)
    qi, tj, qc, tc = qs, ts, 0, 0
    for op in ops:
        if op in (0, 1):
            assert (q[qi] == t[tj]) == (op == 0)
            qi, tj, qc, tc = qi + 1, tj + 1, qc + 1, tc + 1
        elif op == 2:
            qi, qc = qi + 1, qc + 1
        else:
            tj, tc = tj + 1, tc + 1
    assert qc == qe - qs and tc == te - ts


@pytest.mark.parametrize("case", G["align"], ids=lambda c: c["cite"])
def test_known_alignments(case):
    mat, al, go, ge = scoring(case["scoring"])
    q, t = case["q"], case["t"]
    for mode in case["modes"]:
        st, a, _ = o.align(q, t, mat, al, go, ge, mode)
        assert st == 0
        score, qs, qe, ts, te, ops = a
        if "score" in case:
            assert score == case["score"], (case["cite"], mode)
        if "ops" in case:
            assert ops == bytes(CODE[c] for c in case["ops"]), (case["cite"], mode)
        if "cigar" in case:
            assert o.cigar(ops) == case["cigar"]
        if "cigar_extended" in case:
            assert o.cigar(ops, True) == case["cigar_extended"]
        if "query" in case:
            assert [qs, qe] == case["query"]
        if "target" in case:
            assert [ts, te] == case["target"]
        for letter, n in case.get("count", {}).items():
            assert o.cigar(ops).count(letter) == n
        if "first_op_if_any" in case and ops:
            assert ops[0] == CODE[case["first_op_if_any"]]
        if case.get("consistent"):
            assert_consistent(a, q, t, mat, al, go, ge, mode)


@pytest.mark.parametrize("case", G["cigar"], ids=lambda c: c["cite"])
def test_cigar_formatting(case):
    ops = [CODE[c] for c in case["ops"]]
    assert o.cigar(ops) == case["cigar"]
    assert o.cigar(ops, True) == case["cigar_extended"]


@pytest.mark.parametrize("case", G["budget"], ids=lambda c: c["cite"])
def test_budget_boundary_is_exact(case):
    mat, al, go, ge = scoring(case["scoring"])
    st, a, _ = o.align(case["q"], case["t"], mat, al, go, ge, case["mode"], case["ok_at"])
    assert st == 0
    st, a, (need, budget) = o.align(case["q"], case["t"], mat, al, go, ge, case["mode"], case["fails_at"])
    assert st == 11 and need == case["needed"] and budget == case["fails_at"]


@pytest.mark.parametrize("case", G["symbol"], ids=lambda c: c["cite"])
def test_out_of_range_symbol(case):
    mat, al, go, ge = scoring(case["scoring"])
    st, _, (sym, n) = o.align(case["q"], case["t"], mat, al, go, ge, case["mode"])
    assert st == 6 and sym == case["symbol"] and n == case["alphabet_len"]


@pytest.mark.parametrize("case", G["database"], ids=lambda c: c["cite"])
def test_database_alignment_cases(case):
    mat, al, go, ge = scoring(case["scoring"])
    seqs = case["seqs"]
    max_t = max(len(s) for s in seqs)
    need = o.traceback_min_bytes_for_database(case["max_query_len"], max_t)
    if "rejected_budget" in case:
        assert need > case["rejected_budget"]  # the build is rejected (src/database.rs:781-790)
    db = o.OracleDb(seqs, mat, al, go, ge, case["mode"], 1)
    k, a = db.scan_aligned(case["query"])
    assert k == case["winner"] and a[0] == case["score"] and o.cigar(a[5]) == case["cigar"]
    if "all_index" in case:
        out = db.scan_all_aligned(case["query"])
        assert len(out) == len(seqs) and out[case["all_index"]] == a


def test_database_budget_is_monotonic():
    """src/align/tests.rs:467-500."""
    for n in (0, 1, 2, 3, 5, 8, 21, 64, 100):
        prev = 0
        for m in range(401):
            v = o.traceback_min_bytes_for_database(m, n)
            assert v >= prev
            prev = v
    for m in (0, 1, 2, 3, 5, 8, 21, 64, 100):
        prev = 0
        for n in range(401):
            v = o.traceback_min_bytes_for_database(m, n)
            assert v >= prev
            prev = v


def test_checkpoint_rule_and_degenerate_edges():
    """src/align.rs:192-250: full matrix when it fits or a side is empty, else the sqrt(m)
    checkpoint peak; a side of 0 always traces."""
    assert o.traceback_needed(4, 3, 240) == 0 and o.traceback_needed(4, 3, 239) == 240
    assert o.traceback_needed(0, 10 ** 9, 1) == 0 and o.traceback_needed(10 ** 9, 0, 1) == 0
    m, n = 10000, 300
    k = int(np.sqrt(m))
    peak = (2 * (m // k + 1) + 3 * (k + 1)) * (n + 1) * 4
    assert o.traceback_needed(m, n, peak) == 0 and o.traceback_needed(m, n, peak - 1) == peak
    assert o.traceback_min_bytes_for_database(m, n) == min(peak, 3 * (m + 1) * (n + 1) * 4)


SCORINGS = [  # src/align/tests.rs:27-35
    (identity_matrix(4, 2, -1), 2, 1),
    (identity_matrix(4, 1, -3), 10, 5),
    (identity_matrix(4, 3, -2), 4, 0),
    (identity_matrix(4, 5, -1), 1, 1),
]


def test_traceback_is_consistent_everywhere():
    """src/align/tests.rs:380-411 over seeded random pairs of length 0..8, plus the end cell
    agreeing with align_core's ScoreEnd (the same Best rule)."""
    rng = Lcg(7)
    for _ in range(300):
        q = [(rng.next() % (4)) for _ in range((rng.next() % (9)))]
        t = [(rng.next() % (4)) for _ in range((rng.next() % (9)))]
        for mat, go, ge in SCORINGS:
            for mode in ALL_MODES:
                a = o.traceback(q, t, mat, 4, go, ge, mode)
                assert_consistent(a, q, t, mat, 4, go, ge, mode)
                s, qe, te = o.align_pair(q, t, mat, 4, go, ge, mode)
                assert a[2] == (0 if qe is None else qe + 1) and a[4] == (0 if te is None else te + 1)


def test_align_is_optimal_and_ops_rescore():
    """tests/traceback.rs:72-85: random scorings (al 2..4, entries -5..5, 0 <= ge <= go <= 8)."""
    rng = Lcg(11)
    for _ in range(400):
        al = 2 + (rng.next() % (3))
        mat = [(rng.next() % (11)) - 5 for _ in range(al * al)]
        go = (rng.next() % (9))
        ge = (rng.next() % (go + 1))
        q = [(rng.next() % (al)) for _ in range((rng.next() % (8)))]
        t = [(rng.next() % (al)) for _ in range((rng.next() % (8)))]
        for mode in ALL_MODES:
            st, a, _ = o.align(q, t, mat, al, go, ge, mode)
            assert st == 0
            assert a[0] == o.brute(mode, q, t, mat, al, go, ge)
            assert rescore(a, q, t, mat, al, go, ge) == a[0]


def test_database_alignment_matches_free_align():
    """tests/database_alignment.rs:28-81 at the oracle level: scan_all_aligned is the per-target
    align, scan_aligned's winner is the first best score."""
    rng = Lcg(13)
    for _ in range(150):
        al = 2 + (rng.next() % (3))
        mat = [(rng.next() % (11)) - 5 for _ in range(al * al)]
        go = (rng.next() % (9))
        ge = (rng.next() % (go + 1))
        seqs = [[(rng.next() % (al)) for _ in range((rng.next() % (8)))] for _ in range(1 + (rng.next() % (5)))]
        q = [(rng.next() % (al)) for _ in range((rng.next() % (8)))]
        for mode in ALL_MODES:
            want = [o.align(q, s, mat, al, go, ge, mode)[1] for s in seqs]
            db = o.OracleDb(seqs, mat, al, go, ge, mode, 1)
            assert db.scan_all_aligned(q) == want
            best = max(a[0] for a in want)
            k, a = db.scan_aligned(q)
            assert k == [a_[0] for a_ in want].index(best) and a == want[k]


def test_threaded_scan_all_aligned_equals_the_serial_one():
    rng = Lcg(3)
    seqs = [[(rng.next() % 4) for _ in range(rng.next() % 40)] for _ in range(60)]
    q = [(rng.next() % 4) for _ in range(30)]
    for mode in ALL_MODES:
        db = o.OracleDb(seqs, SCORINGS[0][0], 4, 2, 1, mode, 1)
        assert db.scan_all_aligned_mt(q, 4) == db.scan_all_aligned(q)
