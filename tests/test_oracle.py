"""Pins the CPU oracle (oracle/hyoracle.c) to the reference before it is trusted as the checker:
every known-answer vector of the reference's tests, the exhaustive brute-force differential of
tests/alignment.rs:185-214, the width-proof unit tests of src/width.rs:177-414, the database scan
semantics of tests/database.rs, and the AVX2 baseline restatement against the scalar oracle."""
import itertools

import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, DNA, Lcg, all_sequences, identity_matrix
from golden_cases import load, resolve

G = load()


def _scoring(name):
    s = G["scorings"][name]
    return s["matrix"], s["al"], s["go"], s["ge"]


@pytest.mark.parametrize("case", G["pairs"], ids=lambda c: c["cite"])
def test_pair_known_answers(case):
    mat, al, go, ge = _scoring(case["scoring"])
    q, t = resolve(case["q"]), resolve(case["t"])
    for mode in case["modes"]:
        s, qe, te = o.align_pair(q, t, mat, al, go, ge, mode)
        if "expect" in case:
            assert (s, qe, te) == tuple(case["expect"]), (case["cite"], mode)
        else:
            assert s == case["expect_score"], (case["cite"], mode)


def test_pair_known_answer_hw_is_not_symmetric():
    # tests/alignment.rs:419-424
    a = o.align_pair([1, 2], [0, 1, 2, 3], DNA, 4, 2, 1, 2)[0]
    b = o.align_pair([0, 1, 2, 3], [1, 2], DNA, 4, 2, 1, 2)[0]
    assert a != b


@pytest.mark.parametrize("case", G["scans"], ids=lambda c: c["cite"])
def test_scan_known_answers(case):
    mat, al, go, ge = _scoring(case["scoring"])
    db = [resolve(s) for s in case["db"]]
    q = resolve(case["q"])
    modes = ALL_MODES if case["mode"] == "all" else [case["mode"]]
    sts = (0, 1) if case["search_type"] == "all" else [case["search_type"]]
    for mode in modes:
        for st in sts:
            got = o.OracleDb(db, mat, al, go, ge, mode, st).scan(q)
            if "expect" in case:
                assert got == tuple(case["expect"])
            if "expect_score" in case:
                assert got[0] == case["expect_score"]
            if "expect_min_score" in case:
                assert got[0] >= case["expect_min_score"]
            if "expect_index" in case:
                assert got[1] == case["expect_index"]
            # Always: scan equals best-of-align_pair with the smallest index on ties
            # (tests/common/mod.rs:227-246).
            best = None
            for k, t in enumerate(db):
                s, qe, te = o.align_pair(q, t, mat, al, go, ge, mode, st)
                if best is None or s > best[0]:
                    best = (s, k, qe, te)
            assert got == best


def test_scan_scores_known_answer():
    case = G["scan_scores"][0]
    mat, al, go, ge = _scoring(case["scoring"])
    sc = o.OracleDb(case["db"], mat, al, go, ge, case["mode"], 0).scan_scores(case["q"])
    assert sc[1] == case["expect_index1"]
    order = case["expect_order"]
    assert sc[order[0]] > sc[order[1]] > sc[order[2]]


@pytest.mark.parametrize("scheme", [(2, 3, 2, -1, 2, 1), (2, 3, 1, -1, 3, 3), (2, 3, 3, -2, 4, 2), (3, 2, 2, -1, 2, 1)])
def test_oracle_matches_brute_force_over_all_short_pairs(scheme):
    # tests/alignment.rs:185-214
    al, max_len, m, x, go, ge = scheme
    mat = identity_matrix(al, m, x)
    seqs = all_sequences(al, max_len)
    for q in seqs:
        for t in seqs:
            for mode in ALL_MODES:
                assert o.align_pair(q, t, mat, al, go, ge, mode)[0] == o.brute(mode, q, t, mat, al, go, ge), (mode, q, t)


def test_small_penalty_affine_init_matches_brute():
    # tests/opal_regressions.rs:85-124
    seqs = all_sequences(2, 2)
    for go, ge in [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]:
        mat = identity_matrix(2, 2, -2)
        for q in seqs:
            for t in seqs:
                for mode in ALL_MODES:
                    assert o.align_pair(q, t, mat, 2, go, ge, mode)[0] == o.brute(mode, q, t, mat, 2, go, ge)
    deep = all_sequences(2, 4)
    for go, ge in [(1, 1), (2, 1), (0, 0)]:
        mat = identity_matrix(2, 3, -2)
        for q in deep[::3]:
            for t in deep[::3]:
                assert o.align_pair(q, t, mat, 2, go, ge, 1)[0] == o.brute(1, q, t, mat, 2, go, ge)


def test_random_schemes_match_brute_force():
    # tests/properties.rs:111-126 (seeded instead of proptest): al 2..3, entries -6..6, len <= 3.
    rng = np.random.default_rng(7)
    for _ in range(300):
        al = int(rng.integers(2, 4))
        mat = [int(v) for v in rng.integers(-6, 7, al * al)]
        go = int(rng.integers(0, 11))
        ge = int(rng.integers(0, go + 1))
        q = [int(v) for v in rng.integers(0, al, int(rng.integers(0, 4)))]
        t = [int(v) for v in rng.integers(0, al, int(rng.integers(0, 4)))]
        for mode in ALL_MODES:
            assert o.align_pair(q, t, mat, al, go, ge, mode)[0] == o.brute(mode, q, t, mat, al, go, ge)


def test_mode_score_ordering_and_score_end_consistency():
    # tests/alignment.rs:306-329, tests/properties.rs:131-160
    rng = np.random.default_rng(11)
    for _ in range(200):
        mat = [int(v) for v in rng.integers(-8, 9, 16)]
        go = int(rng.integers(0, 11))
        ge = int(rng.integers(0, go + 1))
        q = [int(v) for v in rng.integers(0, 4, int(rng.integers(0, 26)))]
        t = [int(v) for v in rng.integers(0, 4, int(rng.integers(0, 26)))]
        sc = {m: o.align_pair(q, t, mat, 4, go, ge, m)[0] for m in ALL_MODES}
        assert sc[0] >= 0 and sc[0] >= sc[3] >= sc[2] >= sc[1]
        for m in ALL_MODES:
            assert o.align_pair(q, t, mat, 4, go, ge, m, 0)[0] == sc[m]


def test_symmetric_modes_are_symmetric():
    seqs = all_sequences(4, 3)
    for q in seqs[::5]:
        for t in seqs[::5]:
            for mode in (0, 1, 3):
                assert o.align_pair(q, t, DNA, 4, 2, 1, mode)[0] == o.align_pair(t, q, DNA, 4, 2, 1, mode)[0]


# ---- width proof (src/width.rs:177-414) -------------------------------------------------------

def test_width_boundaries():
    W = {0: "i8", 1: "i16", 2: "i32", -1: None}
    # narrowest_for across boundaries (src/width.rs:196-213) via an SW gap_open magnitude
    for mag, want in [(0, 0), (127, 0), (128, 1), (32767, 1), (32768, 2), (536870911, 2), (536870912, -1),
                      (2147483647, -1)]:
        assert o.required_width(0, -1, 1, mag, 1, 4, 4)[0] == want, mag
    # i32 sentinel ceiling regressions (src/width.rs:216-270)
    w, b = o.required_width(1, 0, 0, 2_000_000_000, 1, 1, 1)
    assert (w, b) == (-1, 2_000_000_001)
    assert o.required_width(0, -1, 1, 1_100_000_000, 1_100_000_000, 9, 4)[0] == -1
    assert o.required_width(1, -2_000_000_000, 1, 1, 1, 2, 2)[0] == -1
    assert o.required_width(1, -1, 1, 2, 1, 30_000, 30_000)[0] == 2
    # small local fits i8; SW ignores mismatch negatives but not gap_open (275-309)
    assert o.required_width(0, -1, 2, 3, 1, 10, 10)[0] == 0
    assert o.required_width(0, -100, 1, 2, 1, 8, 8)[0] == 0
    for mode in (1, 2, 3):
        assert o.required_width(mode, -100, 1, 2, 1, 8, 8)[0] > 0
    assert o.required_width(0, -1, 1, 200, 1, 8, 8)[0] == 1
    # CR4 overlap stays i8, NW needs i16 (311-330)
    assert o.required_width(3, -2, 1, 2, 2, 91, 33)[0] == 0
    assert o.required_width(1, -2, 1, 2, 2, 91, 33)[0] == 1
    # escalation with length (332-368)
    for mode in ALL_MODES:
        prev = 0
        for n in [1, 2, 100, 300, 327, 328, 1000, 22_000, 50_000]:
            w = o.required_width(mode, 0, 100, 0, 0, n, n)[0]
            assert w >= prev
            prev = w
        assert o.required_width(mode, 0, 100, 0, 0, 1, 1)[0] == 0
        assert o.required_width(mode, 0, 100, 0, 0, 327, 327)[0] == 1
        assert o.required_width(mode, 0, 100, 0, 0, 328, 328)[0] == 2
        assert o.required_width(mode, 0, 100, 0, 0, 50_000, 50_000)[0] == 2
        assert o.required_width(mode, -5, 5, 4, 2, 0, 0)[0] == 0
    # positive reach uses min of the two lengths (370-381)
    assert o.required_width(0, 0, 100, 0, 0, 2, 1_000_000)[0] == 1
    assert o.required_width(0, 0, 100, 0, 0, 1, 1_000_000)[0] == 0
    # overflow is a typed error, pathological lengths do not overflow (393-410)
    w, b = o.required_width(1, -1, 1, 0, 1, 2_000_000_000, 2_000_000_000)
    assert w == -1 and b > 2**31 - 1
    assert o.required_width(3, -1, 1, 1, 1, 2**64 - 1, 2**64 - 1)[0] == -1
    # non-local overflow regressions (tests/opal_regressions.rs:126-140)
    assert o.required_width(1, -1, 1, 1, 1, 2_000_000_000, 2_000_000_000)[0] == -1
    assert o.required_width(1, -1, 1, 1, 1, 500, 500)[0] == 1
    # tests/real_data.rs:202-231
    assert o.required_width(1, -1, 1, 2, 1, 250, 250)[0] == 1
    assert o.required_width(1, -1, 1, 2, 1, 40_000, 40_000)[0] == 2
    # OV negative reach at the i8 edge (tests/sweeps.rs:288-318)
    assert o.required_width(3, -1, 1, 1, 1, 126, 126)[0] == 0
    assert o.required_width(3, -1, 1, 1, 1, 127, 127)[0] == 1
    # chosen width contains the bound and is minimal (383-391 of src/width.rs)
    for mode, mn, mx, go, ge, m, n in [(0, -1, 2, 3, 1, 50, 50), (1, -4, 5, 8, 2, 200, 200), (2, -2, 3, 6, 1, 500, 30),
                                       (3, -7, 7, 10, 3, 4000, 4000), (1, -1, 1, 0, 1, 40_000, 40_000)]:
        w, bound = o.required_width(mode, mn, mx, go, ge, m, n)
        caps = [127, 32767, 536870911]
        assert bound <= caps[w]
        assert all(bound > caps[k] for k in range(w))


def test_escalation_partition_widths():
    # src/database.rs:1366-1410: +20 match, SW, max_query_len 2000
    mat = identity_matrix(4, 20, -5)
    widths = [o.required_width(0, -5, 20, 8, 2, 2000, n)[0] for n in (4, 6, 10, 24, 2000)]
    assert widths == [0, 0, 1, 1, 2]


# ---- database scan semantics (tests/database.rs) -----------------------------------------------

def test_scan_matches_best_align_pair_over_all_short_databases():
    # tests/database.rs:68-98 (a strided subset of the 2-sequence databases, every query <= 3)
    seqs = all_sequences(4, 2)
    queries = all_sequences(4, 3)
    for a, b in list(itertools.product(seqs, seqs))[::7]:
        for mode in ALL_MODES:
            for st in (0, 1):
                db = o.OracleDb([a, b], DNA, 4, 2, 1, mode, st)
                for q in queries[::3]:
                    best = None
                    for k, t in enumerate([a, b]):
                        s, qe, te = o.align_pair(q, t, DNA, 4, 2, 1, mode, st)
                        if best is None or s > best[0]:
                            best = (s, k, qe, te)
                    assert db.scan(q) == best


def test_scan_all_and_scores_equal_per_target_align_pair():
    rng = Lcg(0x5EED)
    seqs = [rng.seq(rng.next() % 9, 4) for _ in range(40)]
    for mode in ALL_MODES:
        for st in (0, 1):
            db = o.OracleDb(seqs, DNA, 4, 2, 1, mode, st)
            for q in ([], [0], rng.seq(7, 4)):
                allh = db.scan_all(q)
                for k, t in enumerate(seqs):
                    s, qe, te = o.align_pair(q, t, DNA, 4, 2, 1, mode, st)
                    assert allh[k] == (s, k, qe, te)
                assert list(db.scan_scores(q)) == [h[0] for h in allh]


def test_align_pairs_validation_order():
    # src/kernel.rs:429-452: the first failing pair's error; hits before it are kept.
    st, hits, d = o.align_pairs([[0, 1], [0, 9], [1]], [[0], [0], [1]], DNA, 4, 2, 1, 0, 1)
    assert st == 6 and d == (9, 4)
    assert hits[0][0] == 2
    big = identity_matrix(2, 1, -1)
    st, hits, d = o.align_pairs([[0], [0] * 10], [[0], [0] * 10], big, 2, 2_000_000_000, 1, 1, 0)
    assert st == 5


# ---- the AVX2 baseline restatement equals the scalar oracle ---------------------------------------

@pytest.mark.parametrize("mode", ALL_MODES)
def test_avx2_port_matches_oracle(mode):
    rng = np.random.default_rng(100 + mode)
    for al, lo, hi, go, ge, maxlen in [(4, -1, 2, 2, 1, 40), (20, -4, 11, 11, 1, 60), (4, -80, 80, 5, 2, 30),
                                       (4, -5000, 5000, 7, 3, 12)]:
        mat = [int(v) for v in rng.integers(lo, hi + 1, al * al)]
        seqs = [list(rng.integers(0, al, int(rng.integers(0, maxlen)))) for _ in range(70)]
        res, off = o.concat(seqs)
        queries = [list(rng.integers(0, al, int(n))) for n in (0, 1, 9, maxlen)]
        mql = max(len(q) for q in queries)
        try:
            port = o.Avx2Db(res, off, mat, al, go, ge, mode, 1, mql, gathered_i8=(al <= 16))
        except ValueError:
            continue
        ref = o.OracleDb((res, off), mat, al, go, ge, mode, 1)
        got = port.scan_many(queries, 4)
        for q, g in zip(queries, got):
            assert g == ref.scan(q)
            assert list(port.scan_scores(q)) == list(ref.scan_scores(q))


@pytest.mark.parametrize("mode", ALL_MODES)
def test_avx2_sliced_stream_matches_oracle(mode):
    """The balanced CPU baseline (one database in slices, (query, slice) units over threads) gives
    the whole database's hits, ties across slice borders included."""
    rng = np.random.default_rng(300 + mode)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = [list(rng.integers(0, 20, int(rng.integers(0, 90)))) for _ in range(200)]
    for k in (3, 77, 78, 150):  # equal best candidates in several slices: the smallest index wins
        seqs[k] = list(range(20)) * 3
    res, off = o.concat(seqs)
    queries = [list(rng.integers(0, 20, int(n))) for n in (0, 1, 17, 60, 120)] + [list(range(20)) * 3]
    mql = max(len(q) for q in queries)
    port = o.Avx2SlicedDb(res, off, mat, 20, 11, 1, mode, 1, mql, n_slices=5)
    assert len(port.slices) == 5
    ref = o.OracleDb((res, off), mat, 20, 11, 1, mode, 1)
    for q, g in zip(queries, port.scan_stream(queries, 4)):
        assert g == ref.scan(q)
