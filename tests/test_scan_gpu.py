"""Parity of the cuda backend's database scan with the CPU oracle, through the C ABI. Mirrors the
reference's sweeps (tests/sweeps.rs), cross-backend properties (tests/properties.rs), known answers
and real-data tests; every comparison is full-struct equality."""
import threading

import numpy as np
import pytest

from conftest import ALL_MODES, DNA, Lcg, identity_matrix
from golden_cases import load, resolve
from gpu_helpers import AMINO, BLOSUM62, build, check, hit_tuple, rand_seqs

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu
G = load()


def dna(m, x, go, ge):
    return identity_matrix(4, m, x), 4, go, ge


def test_backend_is_cuda():
    db = build([[0, 1, 2]], DNA, 4, 2, 1, 0, 1, 4)
    assert db.backend() == hy.Backend.Cuda
    assert hy.Backend.Cuda.is_available()


@pytest.mark.parametrize("case", G["scans"], ids=lambda c: c["cite"])
def test_known_answer_scans(case):
    s = G["scorings"][case["scoring"]]
    db_seqs = [resolve(x) for x in case["db"]]
    q = resolve(case["q"])
    modes = ALL_MODES if case["mode"] == "all" else [case["mode"]]
    sts = (0, 1) if case["search_type"] == "all" else [case["search_type"]]
    for mode in modes:
        for st in sts:
            db = check(db_seqs, s["matrix"], s["al"], s["go"], s["ge"], mode, st, [q], mql=case["mql"])
            got = hit_tuple(db.scan(hy.Scratch(db), q))
            if "expect" in case:
                assert got == tuple(case["expect"])
            if "expect_index" in case:
                assert got[1] == case["expect_index"]


@pytest.mark.parametrize("case", G["pairs"], ids=lambda c: c["cite"])
def test_known_answer_pairs_as_single_target_scans(case):
    s = G["scorings"][case["scoring"]]
    q, t = resolve(case["q"]), resolve(case["t"])
    for mode in case["modes"]:
        db = build([t], s["matrix"], s["al"], s["go"], s["ge"], mode, 1, max(len(q), 1))
        got = hit_tuple(db.scan(hy.Scratch(db), q))
        if "expect" in case:
            assert got == (case["expect"][0], 0, case["expect"][1], case["expect"][2])
        else:
            assert got[0] == case["expect_score"]


def test_scan_scores_known_answer():
    case = G["scan_scores"][0]
    db = build(case["db"], DNA, 4, 2, 1, 0, 0, 16)
    out = []
    db.scan_scores(hy.Scratch(db), case["q"], out)
    assert out[1] == 8 and out[1] > out[2] > out[0]


@pytest.mark.parametrize("n", [1, 2, 15, 16, 17, 31, 32, 33, 47, 48, 49, 63, 64, 65, 96, 129])
def test_database_sizes_around_every_lane_boundary(n):
    # tests/sweeps.rs:131-158
    rng = Lcg(0x5EED_1234 + n)
    seqs = [rng.seq(3 + rng.next() % 8, 4) for _ in range(n)]
    queries = [rng.seq(4 + rng.next() % 6, 4) for _ in range(6)]
    for mode in ALL_MODES:
        for st in (0, 1):
            check(seqs, DNA, 4, 2, 1, mode, st, queries)


def test_degenerate_sequences_and_queries():
    # tests/sweeps.rs:161-194
    cases = [
        [[]] * 20,
        [[] if i % 2 == 0 else [0, 1, 2] for i in range(33)],
        [[0] * 10] * 40,
        [[i % 4] for i in range(17)],
        [[0, 1, 2, 3]] * 32 + [[0] * 20],
    ]
    queries = [[], [0], [0, 1, 2, 3], [2, 2, 2, 2, 2]]
    for seqs in cases:
        for mode in ALL_MODES:
            for st in (0, 1):
                check(seqs, DNA, 4, 2, 1, mode, st, queries, mql=5)


def test_scoring_parameter_grid():
    # tests/sweeps.rs:197-236
    rng = Lcg(0xA11CE)
    seqs = [rng.seq(rng.next() % 9, 4) for _ in range(20)] + [[]]
    queries = [rng.seq(rng.next() % 9, 4) for _ in range(8)]
    for m, x in [(1, -1), (2, -1), (3, -2), (1, 0)]:
        for go, ge in [(1, 1), (2, 1), (3, 0), (5, 5), (4, 2), (0, 0), (100, 1), (127, 1)]:
            for mode in ALL_MODES:
                for st in (0, 1):
                    check(seqs, identity_matrix(4, m, x), 4, go, ge, mode, st, queries, mql=9)


@pytest.mark.parametrize("al", [16, 17])
def test_alphabet_at_and_past_the_shuffle_limit(al):
    # tests/sweeps.rs:239-262
    mat = identity_matrix(al, 1, -1)
    rng = Lcg(0xF00D + al)
    seqs = [rng.seq(4 + rng.next() % 5, al) for _ in range(40)]
    queries = [rng.seq(6, al) for _ in range(6)]
    for mode in ALL_MODES:
        check(seqs, mat, al, 2, 1, mode, 1, queries)


@pytest.mark.parametrize("length", [126, 127, 128, 129])
def test_score_width_boundaries(length):
    # tests/sweeps.rs:265-285
    check([[0] * length], [1, -1, -1, 1], 2, 2, 1, 0, 1, [[0] * length])


def test_overlap_negative_reach_at_the_i8_edge():
    # tests/sweeps.rs:288-318
    check([[1] * 126], [1, -1, -1, 1], 2, 1, 1, 3, 1, [[0] * 126])
    check([[1] * 6], [1, -1, -1, 1], 2, 1, 1, 3, 1, [[0] * 120 + [1] * 6])


def test_random_lane_crossing_databases():
    # tests/sweeps.rs:324-335 (seeded)
    rng = np.random.default_rng(1)
    for _ in range(25):
        seqs = rand_seqs(rng, int(rng.integers(1, 71)), 4, 0, 6)
        queries = rand_seqs(rng, int(rng.integers(1, 5)), 4, 0, 6)
        m = int(rng.integers(1, 3))
        go, ge = [(1, 1), (2, 1), (3, 0)][int(rng.integers(0, 3))]
        for mode in ALL_MODES:
            check(seqs, identity_matrix(4, m, -1), 4, go, ge, mode, 1, queries, mql=6)


@pytest.mark.parametrize("regime", ["i8", "i16", "i32", "mixed", "large_alphabet"])
def test_random_schemes_every_width(regime):
    # tests/properties.rs: scheme_db_query / _wide / _verywide / mixed_length / large_alphabet
    rng = np.random.default_rng({"i8": 3, "i16": 4, "i32": 5, "mixed": 6, "large_alphabet": 7}[regime])
    for _ in range(12):
        if regime == "large_alphabet":
            al = int(rng.integers(17, 26))
            lo, hi, gmax, maxlen, qlen = -6, 6, 6, 14, 14
        else:
            al = int(rng.integers(2, 5))
            lo, hi, gmax, maxlen, qlen = {"i8": (-8, 8, 10, 12, 12), "i16": (-80, 80, 10, 12, 12),
                                          "i32": (-5000, 5000, 10, 12, 12), "mixed": (-40, 70, 10, 40, 20)}[regime]
        mat = [int(v) for v in rng.integers(lo, hi + 1, al * al)]
        go = int(rng.integers(0, gmax + 1))
        ge = int(rng.integers(0, go + 1))
        seqs = rand_seqs(rng, int(rng.integers(1, 9)), al, 0 if regime != "mixed" else 1, maxlen)
        queries = rand_seqs(rng, 3, al, 0, qlen)
        for mode in ALL_MODES:
            for st in (0, 1):
                check(seqs, mat, al, go, ge, mode, st, queries, mql=qlen)


def test_escalated_widths_match_the_oracle():
    # src/database.rs:1359-1470: a database spanning i8/i16/i32 under SW with +20 matches
    mat = identity_matrix(4, 20, -5)
    seqs = [[i % 4 for i in range(n)] for n in (4, 6, 10, 24, 2000)]
    queries = [[(i * 3 + 1) % 4 for i in range(n)] for n in (3, 8, 30, 50)]
    for mode in ALL_MODES:
        for st in (0, 1):
            db = check(seqs, mat, 4, 8, 2, mode, st, queries, mql=2000)
            assert db.score_width() == hy.ScoreWidth.I32


def test_protein_blosum62_and_ubiquitin():
    # tests/real_data.rs:240-359
    ub = [AMINO.index(c) for c in "MQIFVKTLTGKTITLEVEPSDTIENVKAKIQDKEGIPPDQQRLIFAGKQLEDGRTLSDYNIQKESTLHLVLRLRGG"]
    diag = sum(BLOSUM62[a * 20 + a] for a in ub)

    def mutate(seq, subs):
        s = list(seq)
        for p, a in subs:
            s[p] = a
        return s

    db_seqs = [ub, mutate(ub, [(3, 9), (17, 4), (40, 0), (60, 19)]),
               mutate(ub, [(0, 5), (10, 5), (20, 5), (30, 5), (70, 5)]), ub[:50], ub[26:]]
    queries = [ub, mutate(ub, [(5, 0), (55, 11)]), ub[10:66]]
    for mode in ALL_MODES:
        for st in (0, 1):
            db = check(db_seqs, BLOSUM62, 20, 11, 1, mode, st, queries, mql=76)
            assert db.score_width() == hy.ScoreWidth.I16
        single = build([ub], BLOSUM62, 20, 11, 1, mode, 0, 76)
        assert single.scan(hy.Scratch(single), ub).score == diag


@pytest.mark.parametrize("mode", ALL_MODES)
def test_multi_pass_queries_and_long_targets(mode):
    # Queries longer than one pass of the device wavefront, targets of thousands of columns, and
    # both device partitions (int16 pairs and int32 singles) in one database.
    rng = np.random.default_rng(20 + mode)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = rand_seqs(rng, 30, 20, 0, 300) + rand_seqs(rng, 3, 20, 1500, 3000)
    queries = [list(rng.integers(0, 20, n)) for n in (127, 128, 129, 300, 777)]
    for st in (0, 1):
        check(seqs, mat, 20, 11, 1, mode, st, queries, mql=800)


def test_i32_partition_long_targets():
    # Sequences that only fit int32 on the device next to int16 ones (config-2 shape).
    rng = np.random.default_rng(99)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    seqs = rand_seqs(rng, 40, 20, 20, 400) + rand_seqs(rng, 4, 20, 3000, 4000)
    queries = [list(rng.integers(0, 20, n)) for n in (100, 1000, 5000)]
    for mode in (0, 2):
        db = check(seqs, mat, 20, 11, 1, mode, 1, queries, mql=5000)
        n16, n32 = db.partition()
        assert n16 > 0 and n32 > 0


def test_config1_shape_dna_sw_score_end():
    # Config-1 shape (DNA SW ScoreEnd, 64-bp query, lengths 50-300, planted near-copies), 2,000
    # sequences instead of 10,000 to keep the oracle fast.
    rng = np.random.default_rng(1)
    q = list(rng.integers(0, 4, 64))
    seqs = rand_seqs(rng, 2000, 4, 50, 300)
    for k in rng.choice(2000, 10, replace=False):
        s = list(q)
        for p in rng.choice(64, 3, replace=False):
            s[p] = int(rng.integers(0, 4))
        seqs[k] = s
    check(seqs, DNA, 4, 2, 1, 0, 1, [q, list(rng.integers(0, 4, 64))], mql=64)


def test_scratch_reuse_and_threads():
    # src/database.rs:1332-1357 and tests/database.rs:136-176
    seqs = [[0, 1], [0, 1, 2, 3, 3, 2, 1, 0], [2]]
    db = build(seqs, DNA, 4, 2, 1, 1, 1, 16)
    sc = hy.Scratch(db)
    first = None
    for q in ([0, 1, 2, 3], [2], [0, 1, 2, 3, 3, 2, 1, 0], [0, 1, 2, 3]):
        h = db.scan(sc, q)
        assert h == db.scan(hy.Scratch(db), q)
        if q == [0, 1, 2, 3]:
            first = first or h
            assert h == first
    db2 = build([[0, 1, 2, 3], [2, 2, 2, 2]], DNA, 4, 2, 1, 0, 1, 8)
    expected = db2.scan(hy.Scratch(db2), [0, 1, 2, 3])
    results = []

    def work():
        s = hy.Scratch(db2)
        for _ in range(50):
            r = db2.scan(s, [0, 1, 2, 3])
        results.append(r)

    ts = [threading.Thread(target=work) for _ in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert results == [expected] * 4


def test_query_validation():
    db = build([[0, 1, 2]], DNA, 4, 2, 1, 0, 1, 4)
    sc = hy.Scratch(db)
    with pytest.raises(hy.Error) as e:
        db.scan(sc, [0, 1, 2, 3, 0])
    assert e.value == hy.Error("QueryTooLong", len=5, max=4)
    with pytest.raises(hy.Error) as e:
        db.scan(sc, [0, 7])
    assert e.value == hy.Error("SymbolOutOfRange", symbol=7, alphabet_len=4)


@pytest.mark.parametrize("mode", [0, 2, 4])
def test_graph_replay_many_query_lengths(mode):
    """Small scans replay a CUDA graph per call kind and query length from the scratch (captured on
    first use, the least recently used of 32 evicted): 45 query lengths, each scanned, then scanned
    again in the reverse order with other residues (replays of evicted and kept graphs), every
    scan, scan_all and scan_scores equal to the oracle."""
    rng = np.random.default_rng(400 + mode)
    seqs = rand_seqs(rng, 3000, 4, 0, 120)
    first = [list(rng.integers(0, 4, n)) for n in range(1, 46)]
    second = [list(rng.integers(0, 4, n)) for n in range(45, 0, -1)]
    for st in (0, 1):
        check(seqs, DNA, 4, 2, 1, mode, st, first + second + first[:5], mql=45)
