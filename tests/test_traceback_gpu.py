"""Device traceback (the Alignment search type) against the oracle's restatement of
src/align.rs: align, Database::scan_aligned and Database::scan_all_aligned. Bit-exact: the same
score, spans and operation bytes for every pair, across the five modes, multi-pass queries,
every rows-per-lane choice, empty sequences, large alphabets and the reference's known answers."""
import json
import os

import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, DNA, Lcg, identity_matrix
from gpu_helpers import BLOSUM62

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "traceback_known_answers.json")) as f:
    G = json.load(f)


def _scoring(name):
    s = G["scorings"][name]
    mat = identity_matrix(s["al"], *s["id"])
    for idx, v in s.get("set", []):
        mat[idx] = v
    return mat, s["al"], s["go"], s["ge"]


def _mutate(rng, seq, al, rate=0.15):
    """A related sequence: substitutions, insertions and deletions at `rate`."""
    out = []
    for x in seq:
        r = rng.random()
        if r < rate / 3:
            continue
        if r < 2 * rate / 3:
            out.append(int(rng.integers(0, al)))
        elif r < rate:
            out.extend([x, int(rng.integers(0, al))])
        else:
            out.append(x)
    return out


def _align(q, t, mat, al, go, ge, mode):
    return hy.align(q, t, hy.Scoring(al, mat, go, ge), hy.Mode(mode), hy.USIZE_MAX).as_tuple()


@pytest.mark.parametrize("case", G["align"], ids=lambda c: c["cite"])
def test_known_alignments(case):
    mat, al, go, ge = _scoring(case["scoring"])
    for mode in case["modes"]:
        got = _align(case["q"], case["t"], mat, al, go, ge, mode)
        assert got == o.traceback(case["q"], case["t"], mat, al, go, ge, mode), (case["cite"], mode)
        if "score" in case:
            assert got[0] == case["score"]
        if "ops" in case:
            assert got[5] == bytes("MXID".index(c) for c in case["ops"])


def test_random_small_pairs_all_modes():
    """src/align/tests.rs:380-411 and tests/traceback.rs:72-85 shapes: al 2..4, lengths 0..12,
    random scorings with 0 <= ge <= go <= 8."""
    rng = Lcg(5)
    for _ in range(120):
        al = 2 + rng.next() % 3
        mat = [int(rng.next() % 11) - 5 for _ in range(al * al)]
        go = rng.next() % 9
        ge = rng.next() % (go + 1)
        q = [rng.next() % al for _ in range(rng.next() % 13)]
        t = [rng.next() % al for _ in range(rng.next() % 13)]
        for mode in ALL_MODES:
            assert _align(q, t, mat, al, go, ge, mode) == o.traceback(q, t, mat, al, go, ge, mode), \
                (mode, q, t, mat, go, ge)


@pytest.mark.parametrize("m", [1, 31, 127, 128, 129, 256, 257, 511, 512, 513, 1100])
def test_pass_boundaries_and_rows_per_lane(m):
    rng = np.random.default_rng(m)
    q = list(rng.integers(0, 20, m))
    for n in (1, 7, 40, 300, 1500):
        t = _mutate(rng, q[:n] if n <= m else q + list(rng.integers(0, 20, n - m)), 20)
        for mode in ALL_MODES:
            got = _align(q, t, BLOSUM62, 20, 11, 1, mode)
            assert got == o.traceback(q, t, BLOSUM62, 20, 11, 1, mode), (m, n, mode)


def test_long_pair_and_gap_regimes():
    rng = np.random.default_rng(3)
    q = list(rng.integers(0, 4, 2100))
    t = _mutate(rng, q, 4, 0.25)[:2900]
    for mat, go, ge in ((DNA, 2, 1), (identity_matrix(4, 1, -3), 10, 5), (identity_matrix(4, 3, -2), 4, 0),
                        (identity_matrix(4, 5, -1), 1, 1), (identity_matrix(4, 1, -1), 0, 0)):
        for mode in ALL_MODES:
            assert _align(q, t, mat, 4, go, ge, mode) == o.traceback(q, t, mat, 4, go, ge, mode), (mode, go, ge)


def test_large_alphabet():
    rng = np.random.default_rng(9)
    al = 200
    mat = [int(v) for v in rng.integers(-6, 9, al * al)]
    q = list(rng.integers(0, al, 700))
    t = _mutate(rng, q, al)
    for mode in ALL_MODES:
        assert _align(q, t, mat, al, 9, 2, mode) == o.traceback(q, t, mat, al, 9, 2, mode)


def _db(seqs, mat, al, go, ge, mode, mql, budget=hy.USIZE_MAX):
    return (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(al, mat, go, ge))
            .mode(hy.Mode(mode)).search_type(hy.SearchType.alignment(budget)).max_query_len(mql).build())


def test_scan_all_aligned_and_scan_aligned_match_the_oracle():
    rng = np.random.default_rng(17)
    base = list(rng.integers(0, 20, 500))
    seqs = [_mutate(rng, base[int(a): int(a) + int(L)], 20, 0.3)
            for a, L in zip(rng.integers(0, 300, 110), rng.integers(0, 400, 110))]
    seqs += [[], [3], list(rng.integers(0, 20, 1200))]
    for mode in ALL_MODES:
        db = _db(seqs, BLOSUM62, 20, 11, 1, mode, 800)
        ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, mode, 1)
        sc = hy.Scratch(db)
        for ql in (0, 1, 37, 260, 800):
            q = base[100: 100 + ql] if ql <= 400 else base + list(rng.integers(0, 20, ql - 500))
            out = []
            db.scan_all_aligned(sc, q, out)
            want = ref.scan_all_aligned(q)
            bad = [k for k in range(len(seqs)) if out[k].as_tuple() != want[k]]
            assert not bad, (mode, ql, bad[:5], [(out[k].as_tuple()[:5], want[k][:5]) for k in bad[:3]])
            hit = db.scan_aligned(sc, q)
            k, a = ref.scan_aligned(q)
            assert hit.db_index == k and hit.alignment.as_tuple() == a
            assert hit.db_index == db.scan(sc, q).db_index


def test_few_long_pairs_take_the_stripe_pipeline():
    """Up to 16 targets of a multi-stripe query fill with the stripe kernel (every 128-row stripe
    on its own warp, rows handed down column by column): several pairs in one launch, an empty
    target, targets shorter than one publish interval, and all five modes."""
    rng = np.random.default_rng(31)
    q = list(rng.integers(0, 20, 1500))
    seqs = [_mutate(rng, q[a: a + L], 20, 0.2) for a, L in ((0, 1500), (300, 900), (10, 5), (700, 40))]
    seqs += [[], [7], list(rng.integers(0, 20, 2600)), _mutate(rng, q, 20, 0.5)]
    for mode in ALL_MODES:
        db = _db(seqs, BLOSUM62, 20, 11, 1, mode, 1500)
        sc = hy.Scratch(db)
        out = []
        db.scan_all_aligned(sc, q, out)
        ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, mode, 1)
        assert [a.as_tuple() for a in out] == ref.scan_all_aligned(q), mode
        hit = db.scan_aligned(sc, q)
        assert (hit.db_index, hit.alignment.as_tuple()) == ref.scan_aligned(q)


@pytest.mark.parametrize("case", G["database"], ids=lambda c: c["cite"])
def test_database_known_answers(case):
    mat, al, go, ge = _scoring(case["scoring"])
    db = _db(case["seqs"], mat, al, go, ge, case["mode"], case["max_query_len"])
    sc = hy.Scratch(db)
    hit = db.scan_aligned(sc, case["query"])
    assert hit.db_index == case["winner"]
    assert hit.alignment.score == case["score"] and hit.alignment.cigar() == case["cigar"]
    if "all_index" in case:
        out = []
        db.scan_all_aligned(sc, case["query"], out)
        assert len(out) == len(case["seqs"]) and out[case["all_index"]] == hit.alignment


def test_score_only_database_rejects_the_aligned_scans():
    db = (hy.Database.builder().sequences([[0, 1, 2]]).scoring(hy.Scoring(4, DNA, 2, 1))
          .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(4).build())
    with pytest.raises(hy.Error) as e:
        db.scan_aligned(hy.Scratch(db), [0, 1])
    assert e.value.kind == "InvalidArgument"


def _rescore(a, q, t, mat, al, go, ge):
    qi, tj, total, k = a.query_start, a.target_start, 0, 0
    ops = a.ops_bytes
    while k < len(ops):
        op = ops[k]
        if op < 2:
            total += mat[q[qi] * al + t[tj]]
            qi, tj, k = qi + 1, tj + 1, k + 1
            continue
        run = 0
        while k < len(ops) and ops[k] == op:
            run, k = run + 1, k + 1
            if op == 2:
                qi += 1
            else:
                tj += 1
        total -= go + (run - 1) * ge
    assert (qi, tj) == (a.query_end, a.target_end)
    return total


@pytest.mark.parametrize("mode,n_seqs", [(0, 12000), (2, 3000)])
def test_database_scale_properties(mode, n_seqs):
    """A protein database against a 1000-residue query: every alignment's score is the scan score,
    its end cell is scan_all's end, its operations re-score to the score, and a sample matches the
    oracle exactly. 12,000 sequences hold about 2.4 GB of walk codes: more than one chunk, so the
    two-stream chunk pipeline and the whole-call compaction are exercised."""
    rng = np.random.default_rng(23)
    q = list(rng.integers(0, 20, 1000))
    seqs = []
    for _ in range(n_seqs):
        L = int(rng.integers(50, 700))
        a = int(rng.integers(0, 1000 - min(L, 999)))
        seqs.append(_mutate(rng, q[a: a + L], 20, 0.4) if rng.random() < 0.5 else list(rng.integers(0, 20, L)))
    db = _db(seqs, BLOSUM62, 20, 11, 1, mode, 1000)
    sc = hy.Scratch(db)
    out = []
    db.scan_all_aligned(sc, q, out)
    hits = db.scan_all_array(sc, q)
    for k, (a, h) in enumerate(zip(out, hits)):
        assert a.score == h.score
        assert a.query_end == (h.query_end + 1 if h.query_end >= 0 else 0)
        assert a.target_end == (h.target_end + 1 if h.target_end >= 0 else 0)
        assert _rescore(a, q, seqs[k], BLOSUM62, 20, 11, 1) == a.score
    for k in rng.integers(0, len(seqs), 6):
        assert out[k].as_tuple() == o.traceback(q, seqs[k], BLOSUM62, 20, 11, 1, mode)


@pytest.mark.parametrize("mode", ALL_MODES)
def test_wide_score_range_and_tiny_queries(mode):
    """Substitution scores of several hundred and gaps of tens (values far past 16 bits on the
    longer targets), targets from 1 to 400 residues, queries of 300, 130 and 7 residues."""
    rng = np.random.default_rng(41 + mode)
    al = 8
    mat = [int(v) for v in rng.integers(-120, 300, al * al)]
    q = list(rng.integers(0, al, 300))
    seqs = [_mutate(rng, q[a: a + L], al, 0.3) for a, L in
            ((0, 300), (10, 20), (40, 60), (0, 100), (100, 150), (5, 9), (0, 1))]
    seqs += [list(rng.integers(0, al, int(L))) for L in rng.integers(0, 400, 30)]
    db = _db(seqs, mat, al, 40, 7, mode, 300)
    sc = hy.Scratch(db)
    ref = o.OracleDb(seqs, mat, al, 40, 7, mode, 1)
    for ql in (300, 130, 7):
        out = []
        db.scan_all_aligned(sc, q[:ql], out)
        want = ref.scan_all_aligned(q[:ql])
        bad = [k for k in range(len(seqs)) if out[k].as_tuple() != want[k]]
        assert not bad, (ql, bad[:5])
