"""Parity of the device align_pairs (src/kernel.rs:429-452) with the CPU oracle."""
import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES, DNA, identity_matrix
from gpu_helpers import BLOSUM62

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu


def _hits(out):
    return [(h.score, h.db_index, h.query_end, h.target_end) for h in out]


def run_both(qs, ts, mat, al, go, ge, mode, st):
    out = []
    hy.align_pairs(list(zip(qs, ts)), hy.Scoring(al, mat, go, ge), hy.Mode(mode), hy.SearchType(st), out)
    status, want, _ = o.align_pairs(qs, ts, mat, al, go, ge, mode, st)
    assert status == 0
    return _hits(out), want


@pytest.mark.parametrize("mode", ALL_MODES)
@pytest.mark.parametrize("st", [0, 1])
def test_random_pairs_match_oracle(mode, st):
    rng = np.random.default_rng(mode * 10 + st)
    qs = [list(rng.integers(0, 4, int(rng.integers(0, 40)))) for _ in range(300)]
    ts = [list(rng.integers(0, 4, int(rng.integers(0, 60)))) for _ in range(300)]
    got, want = run_both(qs, ts, DNA, 4, 2, 1, mode, st)
    assert got == want


@pytest.mark.parametrize("mode", ALL_MODES)
def test_pairs_equal_query_lengths_multi_pass_and_i32(mode):
    # Equal query lengths (packed two per int16x2 item), queries longer than one pass, and pairs
    # whose width proof needs int32.
    rng = np.random.default_rng(40 + mode)
    qs = [list(rng.integers(0, 20, 150)) for _ in range(64)] + [list(rng.integers(0, 20, 400)) for _ in range(9)]
    ts = [list(rng.integers(0, 20, int(rng.integers(100, 500)))) for _ in range(73)]
    got, want = run_both(qs, ts, BLOSUM62, 20, 11, 1, mode, 1)
    assert got == want
    big = [int(v) for v in rng.integers(-3000, 3000, 16)]
    qs = [list(rng.integers(0, 4, int(rng.integers(1, 30)))) for _ in range(40)]
    ts = [list(rng.integers(0, 4, int(rng.integers(1, 30)))) for _ in range(40)]
    got, want = run_both(qs, ts, big, 4, 9, 2, mode, 1)
    assert got == want


def test_config5_shape_hw_score_end():
    # Config-5 shape: 150-bp reads in 200-500-bp windows of a random genome, HW, go 6, ge 1.
    rng = np.random.default_rng(5)
    genome = rng.integers(0, 4, 200_000)
    qs, ts = [], []
    for _ in range(2000):
        start = int(rng.integers(300, len(genome) - 800))
        read = list(genome[start:start + 150])
        for p in rng.choice(150, 3, replace=False):
            read[p] = int(rng.integers(0, 4))
        wl = int(rng.integers(200, 501))
        off = int(rng.integers(0, wl - 150))
        qs.append(read)
        ts.append(list(genome[start - off:start - off + wl]))
    got, want = run_both(qs, ts, DNA, 4, 6, 1, 2, 1)
    assert got == want


def test_pairs_validation_returns_first_error_and_prefix():
    out = []
    with pytest.raises(hy.Error) as e:
        hy.align_pairs([([0, 1], [0]), ([0, 9], [0]), ([1], [1])], hy.Scoring(4, DNA, 2, 1), hy.Mode.Sw,
                       hy.SearchType.ScoreEnd, out)
    assert e.value == hy.Error("SymbolOutOfRange", symbol=9, alphabet_len=4)
    assert [h.score for h in out] == [2]
    with pytest.raises(hy.Error) as e:
        hy.align_pairs([([0], [0]), ([0] * 10, [0] * 10)], hy.Scoring(2, [1, -1, -1, 1], 2_000_000_000, 1),
                       hy.Mode.Nw, hy.SearchType.Score, out)
    assert e.value.kind == "ScoreRangeTooWide"
    assert len(out) == 0 or out[0].db_index == 0


@pytest.mark.parametrize("mode", ALL_MODES)
def test_every_rows_per_lane_choice_in_one_call(mode):
    # Query lengths around every pass height of the 8/12/16/20/24/32-row shapes, DNA and protein:
    # one call runs several launches (one per rows choice) over consecutive items.
    rng = np.random.default_rng(60 + mode)
    lengths = [1, 63, 64, 65, 96, 97, 128, 129, 150, 160, 161, 192, 193, 250, 256, 257, 400]
    for al, mat, go in ((4, DNA, 6), (20, BLOSUM62, 11)):
        qs, ts = [], []
        for L in lengths:
            for _ in range(3):  # three pairs per length: two share an int16x2 item
                qs.append(list(rng.integers(0, al, L)))
                ts.append(list(rng.integers(0, al, int(rng.integers(1, 520)))))
        got, want = run_both(qs, ts, mat, al, go, 1, mode, 1)
        assert got == want


def test_first_failure_found_in_a_later_host_chunk():
    # Enough pairs that validation runs in several host-thread chunks; the bad pair sits late.
    rng = np.random.default_rng(77)
    n = 200_000
    qs = [[int(x) for x in rng.integers(0, 4, 8)] for _ in range(n)]
    ts = [[int(x) for x in rng.integers(0, 4, 12)] for _ in range(n)]
    bad = 150_001
    ts[bad] = ts[bad][:5] + [7] + ts[bad][6:]
    out = []
    with pytest.raises(hy.Error) as e:
        hy.align_pairs(list(zip(qs, ts)), hy.Scoring(4, DNA, 2, 1), hy.Mode.Hw, hy.SearchType.ScoreEnd, out)
    assert e.value == hy.Error("SymbolOutOfRange", symbol=7, alphabet_len=4)
    assert len(out) == bad
    sample = list(range(0, bad, 9973)) + [bad - 1]
    status, want, _ = o.align_pairs([qs[i] for i in sample], [ts[i] for i in sample], DNA, 4, 2, 1, 2, 1)
    assert status == 0
    assert [(h.score, h.query_end, h.target_end) for h in (out[i] for i in sample)] == \
        [(w[0], w[2], w[3]) for w in want]


def _related(rng, seq, al, rate=0.2):
    out = []
    for x in seq:
        r = rng.random()
        if r < rate / 3:
            continue
        out.append(int(rng.integers(0, al)) if r < 2 * rate / 3 else int(x))
        if rate * 2 / 3 <= r < rate:
            out.append(int(rng.integers(0, al)))
    return out


@pytest.mark.parametrize("mode", ALL_MODES)
def test_long_pairs_take_the_stripe_kernel(mode):
    """src/kernel.rs:378-397 (the single long pair): pairs with a query of 256+ residues and 1 Mi+
    cells run on the score-only stripe kernel, mixed in one call with short pairs that keep the
    packed kernels; int16-range and int32-range scorings; Score and ScoreEnd."""
    rng = np.random.default_rng(70 + mode)
    base = list(rng.integers(0, 20, 3000))
    qs = [base[:2000], list(rng.integers(0, 20, 600)), base[500:1524], list(rng.integers(0, 20, 30))]
    ts = [_related(rng, base[:2000], 20), list(rng.integers(0, 20, 7000)), _related(rng, base, 20, 0.4),
          list(rng.integers(0, 20, 50))]
    qs += [list(rng.integers(0, 20, int(rng.integers(1, 200)))) for _ in range(50)]
    ts += [list(rng.integers(0, 20, int(rng.integers(1, 300)))) for _ in range(50)]
    for st in (0, 1):
        got, want = run_both(qs, ts, BLOSUM62, 20, 11, 1, mode, st)
        assert got == want, [(k, got[k], want[k]) for k in range(len(got)) if got[k] != want[k]][:4]
    big = [int(v) for v in rng.integers(-900, 900, 400)]
    got, want = run_both(qs[:3], ts[:3], big, 20, 50, 3, mode, 1)
    assert got == want


@pytest.mark.parametrize("mode", ALL_MODES)
def test_one_long_pair_among_short_pairs(mode):
    """Exactly one long pair in a call of many (src/kernel.rs:429-452): it runs on the band kernel
    inside the chunk pipeline while the short pairs keep the packed kernels; Score and ScoreEnd."""
    rng = np.random.default_rng(110 + mode)
    base = list(rng.integers(0, 20, 2500))
    qs = [list(rng.integers(0, 20, int(rng.integers(1, 200)))) for _ in range(40)]
    ts = [list(rng.integers(0, 20, int(rng.integers(1, 300)))) for _ in range(40)]
    qs.insert(17, base[:1500])
    ts.insert(17, _related(rng, base, 20, 0.3))
    for st in (0, 1):
        got, want = run_both(qs, ts, BLOSUM62, 20, 11, 1, mode, st)
        assert got == want, [(k, got[k], want[k]) for k in range(len(got)) if got[k] != want[k]][:4]


def test_single_long_pair_align_pair():
    """The 2000 x 2000 single pair of the single-pair path, every mode."""
    rng = np.random.default_rng(77)
    q = list(rng.integers(0, 20, 2000))
    t = _related(rng, q, 20, 0.3)
    for mode in ALL_MODES:
        h = hy.align_pair(q, t, hy.Scoring(20, BLOSUM62, 11, 1), hy.Mode(mode), hy.SearchType.ScoreEnd)
        assert (h.score, h.db_index, h.query_end, h.target_end) == \
            (lambda s: (s[0], 0, s[1], s[2]))(o.align_pair(q, t, BLOSUM62, 20, 11, 1, mode))


@pytest.mark.parametrize("mode", ALL_MODES)
def test_single_long_pair_band_shapes(mode):
    """One long pair runs on the band kernel in int32 lanes when its 256-row passes fit one round,
    on the warps of one block or of a cluster: 2000 rows (8 passes, one block), 5000 rows (20
    passes, a cluster of 3 blocks of 7 warps); 20000 rows against 60 columns (79 passes, more than
    one round) takes the stripe kernel; an int32-range scoring; Score and ScoreEnd
    (src/kernel.rs:331-397)."""
    rng = np.random.default_rng(90 + mode)
    base = list(rng.integers(0, 20, 5000))
    cases = [(base[:2000], _related(rng, base[:2000], 20, 0.3)),
             (base, _related(rng, base, 20, 0.15)),
             (list(rng.integers(0, 20, 20000)), list(rng.integers(0, 20, 60)))]
    sc = hy.Scoring(20, BLOSUM62, 11, 1)
    for q, t in cases:
        for st in (hy.SearchType.Score, hy.SearchType.ScoreEnd):
            h = hy.align_pair(q, t, sc, hy.Mode(mode), st)
            s, qe, te = o.align_pair(q, t, BLOSUM62, 20, 11, 1, mode)
            want = (s, 0, qe, te) if st == hy.SearchType.ScoreEnd else (s, 0, None, None)
            assert (h.score, h.db_index, h.query_end, h.target_end) == want, (len(q), len(t), st)
    big = [int(v) for v in rng.integers(-900, 900, 400)]
    q, t = cases[0]
    h = hy.align_pair(q, t, hy.Scoring(20, big, 50, 3), hy.Mode(mode), hy.SearchType.ScoreEnd)
    assert (h.score, h.query_end, h.target_end) == o.align_pair(q, t, big, 20, 50, 3, mode)


def _concat(seqs):
    off = np.zeros(len(seqs) + 1, np.uint64)
    off[1:] = np.cumsum([len(s) for s in seqs])
    return np.concatenate([np.asarray(s, np.uint8) for s in seqs]) if len(seqs) else np.zeros(0, np.uint8), off


def _arrays_call(qs, ts, mat, al, go, ge, mode, st):
    q_res, q_off = _concat(qs)
    t_res, t_off = _concat(ts)
    hits, (err, failed) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, hy.Scoring(al, mat, go, ge),
                                                hy.Mode(mode), hy.SearchType(st))
    return hits, err, failed


def _check_sample(hits, qs, ts, idx, mat, al, go, ge, mode, st):
    status, want, _ = o.align_pairs([qs[i] for i in idx], [ts[i] for i in idx], mat, al, go, ge, mode, st)
    assert status == 0
    got = [(hits[i].score, None if hits[i].query_end < 0 else hits[i].query_end,
            None if hits[i].target_end < 0 else hits[i].target_end, hits[i].db_index) for i in idx]
    assert got == [(w[0], w[2], w[3], i) for w, i in zip(want, idx)]


@pytest.mark.parametrize("case", ["query_symbol", "width_first", "same_pair", "long_pair_symbol"])
def test_first_failure_across_chunks(case):
    """The batch's first failure in input order (src/kernel.rs:429-452) when the length checks run
    on the host over all pairs and the symbol checks on the device per chunk: a bad query symbol
    in a later chunk with a width failure after it; a width failure before a symbol failure; a
    pair with both (symbols are checked first); a bad symbol inside a long pair of a many-chunk
    batch. The prefix before the failure is complete and exact."""
    rng = np.random.default_rng({"query_symbol": 1, "width_first": 2, "same_pair": 3, "long_pair_symbol": 4}[case])
    n = 300_000
    qs = [rng.integers(0, 4, int(rng.integers(5, 40))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(5, 60))) for _ in range(n)]
    go, ge = 2, 1
    # A wide matrix entry makes long pairs need int32 and very long ones exceed the width proof.
    mat = [2 if a == b else -1 for a in range(4) for b in range(4)]
    mat[5] = 3000
    width_bad = 250_000
    qs[width_bad] = rng.integers(0, 4, 200_000)
    ts[width_bad] = rng.integers(0, 4, 200_000)
    if case == "query_symbol":
        bad = 180_000
        qs[bad] = qs[bad].copy()
        qs[bad][3] = 9
        want_err, want_at = hy.Error("SymbolOutOfRange", symbol=9, alphabet_len=4), bad
    elif case == "width_first":
        bad = 260_000
        ts[bad] = ts[bad].copy()
        ts[bad][0] = 200
        want_at = width_bad
        want_err = None
    elif case == "same_pair":
        ts[width_bad] = ts[width_bad].copy()
        ts[width_bad][17] = 4
        want_err, want_at = hy.Error("SymbolOutOfRange", symbol=4, alphabet_len=4), width_bad
    else:
        # Long pairs (the stripe path) early in the batch; one carries a bad target symbol.
        base = rng.integers(0, 4, 3000)
        for j, k in enumerate((1_000, 70_000, 140_000)):
            qs[k] = base[:1200]
            ts[k] = rng.integers(0, 4, 1500)
        bad = 140_000
        ts[bad] = ts[bad].copy()
        ts[bad][1400] = 6
        want_err, want_at = hy.Error("SymbolOutOfRange", symbol=6, alphabet_len=4), bad
    hits, err, failed = _arrays_call(qs, ts, mat, 4, go, ge, hy.Mode.Sw, 1)
    assert failed == want_at
    if want_err is None:
        assert err.kind == "ScoreRangeTooWide"
    else:
        assert err == want_err
    sample = sorted(set(list(range(0, want_at, 7919)) + [want_at - 1, 1_000, 70_000]) & set(range(want_at)))
    _check_sample(hits, qs, ts, sample, mat, 4, go, ge, 0, 1)


@pytest.mark.parametrize("mode", ALL_MODES)
def test_many_chunks_mixed_widths_and_long_pairs(mode):
    """A batch of several chunks mixing int16x2 pairs, int32 pairs (a wide matrix entry on long
    pairs), empty sequences and a few long pairs on the stripe kernel: every result exact."""
    rng = np.random.default_rng(90 + mode)
    n = 200_000
    mat = [int(v) for v in rng.integers(-3, 4, 16)]
    mat[0] = 400
    qs = [rng.integers(0, 4, int(rng.integers(0, 30))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(0, 50))) for _ in range(n)]
    for k in rng.choice(n, 300, replace=False):
        qs[k] = rng.integers(0, 4, int(rng.integers(90, 200)))
        ts[k] = rng.integers(0, 4, int(rng.integers(100, 300)))
    for k in (5, 99_999, 150_001):
        qs[k] = rng.integers(0, 4, 1100)
        ts[k] = rng.integers(0, 4, 1300)
    hits, err, failed = _arrays_call(qs, ts, mat, 4, 9, 2, mode, 1)
    assert err is None and failed == n
    sample = sorted(set(list(range(0, n, 997)) + [5, 99_999, 150_001, n - 1]))
    _check_sample(hits, qs, ts, sample, mat, 4, 9, 2, mode, 1)


def test_pinned_buffers_give_the_same_results():
    """Residues (and, for position maxima, the column-maxima array) in page-locked memory are
    copied from and to where they are, with no staging: results identical to pageable buffers,
    across several chunks, with a failure in a later chunk."""
    rng = np.random.default_rng(31)
    n = 150_000
    qs = [rng.integers(0, 4, int(rng.integers(0, 40))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(0, 90))) for _ in range(n)]
    qs[120_001] = qs[120_001].copy()
    if len(qs[120_001]) == 0:
        qs[120_001] = np.array([0], np.uint8)
    qs[120_001][0] = 6
    q_res, q_off = _concat(qs)
    t_res, t_off = _concat(ts)

    def pinned(a):
        p = hy.pinned_empty(len(a), a.dtype)
        p[:] = a
        return p

    scoring = hy.Scoring(4, DNA, 2, 1)
    h1, (e1, f1) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
    pq, pt = pinned(q_res), pinned(t_res)
    h2, (e2, f2) = hy.align_pairs_arrays(pq, q_off, pt, t_off, scoring, hy.Mode.Sw, hy.SearchType.ScoreEnd)
    assert (e1, f1) == (e2, f2) and f1 == 120_001 and e1.kind == "SymbolOutOfRange"
    assert bytes(h1)[: 32 * f1] == bytes(h2)[: 32 * f2]
    cm1 = np.full(int(t_off[-1]), -3, np.int32)
    cm2 = pinned(cm1)
    r1 = hy.align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, scoring, 8, colmax_out=cm1)
    r2 = hy.align_pairs_position_max_arrays(pq, q_off, pt, t_off, scoring, 8, colmax_out=cm2)
    assert r1[3] == r2[3] and r1[3][1] == 120_001
    assert np.array_equal(cm1, cm2)
    assert bytes(r1[0])[: 32 * 120_001] == bytes(r2[0])[: 32 * 120_001]
    assert np.array_equal(r1[2][: 2 * 120_001], r2[2][: 2 * 120_001])
