"""Device align_pair_position_max / batched position maxima and score2 against the oracle
(src/kernel.rs:454-553, 741-792): every column maximum, the BestHit and score2, bit for bit."""
import json
import os

import numpy as np
import pytest

import pyoracle as o
from conftest import DNA
from gpu_helpers import BLOSUM62

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "position_max_known_answers.json")) as f:
    G = json.load(f)


@pytest.mark.parametrize("case", G["position_max"], ids=lambda c: c["cite"])
def test_known_answers(case):
    out = [9, 9, 9]  # cleared and refilled
    h = hy.align_pair_position_max(case["q"], case["t"], hy.Scoring(4, DNA, 2, 1), out)
    assert out == case["out"] and h.score == case["score"]
    assert h.query_end is None and h.target_end == case["target_end"]


def test_out_of_range_symbol():
    c = G["position_max_errors"][0]
    with pytest.raises(hy.Error) as e:
        hy.align_pair_position_max(c["q"], c["t"], hy.Scoring(4, DNA, 2, 1), [])
    assert e.value == hy.Error("SymbolOutOfRange", symbol=c["symbol"], alphabet_len=c["alphabet_len"])


def _batch(qs, ts, mat, al, go, ge, min_score):
    q_res, q_off = hy.concat(qs)
    t_res, t_off = hy.concat(ts)
    return hy.align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, hy.Scoring(al, mat, go, ge), min_score)


def _check(qs, ts, mat, al, go, ge, min_score=20):
    hits, cm, s2, (err, _) = _batch(qs, ts, mat, al, go, ge, min_score)
    assert err is None
    mmax = max(mat)
    at = 0
    for k, (q, t) in enumerate(zip(qs, ts)):
        want, score, te = o.position_max(q, t, mat, al, go, ge)
        got = [int(v) for v in cm[at: at + len(t)]]
        at += len(t)
        assert got == want, (k, len(q), len(t))
        h = hits[k]
        assert (h.score, h.db_index, h.query_end, h.target_end) == (score, k, -1, -1 if te is None else te)
        w2 = o.score2(want, score, 0 if te is None else te, mmax, min_score)
        assert (int(s2[2 * k]), int(s2[2 * k + 1])) == ((0, -1) if w2 is None else w2), k


def test_many_short_pairs_one_warp_each():
    """Mate-rescue shape: reads against windows, with empty and single-residue pairs mixed in."""
    rng = np.random.default_rng(3)
    genome = rng.integers(0, 4, 50_000)
    qs, ts = [], []
    for _ in range(400):
        a = int(rng.integers(0, 49_000))
        read = list(genome[a: a + int(rng.integers(50, 160))])
        w0 = max(0, a - int(rng.integers(0, 200)))
        qs.append(read)
        ts.append(list(genome[w0: w0 + int(rng.integers(100, 600))]))
    qs += [[], [1], [0, 1, 2], list(rng.integers(0, 4, 300))]
    ts += [[0, 1], [], [2], list(rng.integers(0, 4, 5))]
    _check(qs, ts, DNA, 4, 2, 1, min_score=10)
    _check(qs, ts, [int(v) for v in rng.integers(-3, 6, 16)], 4, 5, 2, min_score=3)


def test_long_pairs_take_the_stripe_kernel():
    rng = np.random.default_rng(8)
    q = list(rng.integers(0, 20, 1800))
    ts = [list(rng.integers(0, 20, 3000)), q[200:1500], list(rng.integers(0, 20, 700))]
    qs = [q, q, q[:300]]
    _check(qs, ts, BLOSUM62, 20, 11, 1, min_score=25)


def test_single_pair_entry_matches_batch_and_score2():
    rng = np.random.default_rng(9)
    q = list(rng.integers(0, 20, 400))
    t = list(rng.integers(0, 20, 200)) + q[50:350] + list(rng.integers(0, 20, 300)) + q[100:300]
    out = []
    h = hy.align_pair_position_max(q, t, hy.Scoring(20, BLOSUM62, 11, 1), out)
    want, score, te = o.position_max(q, t, BLOSUM62, 20, 11, 1)
    assert out == want and h.score == score and h.target_end == te
    assert hy.score2(out, h.score, h.target_end, max(BLOSUM62), 30) == o.score2(want, score, te, max(BLOSUM62), 30)
    assert hy.score2(out, h.score, h.target_end, max(BLOSUM62), 30) is not None  # the second copy


def _sample_check(qs, ts, idx, hits, cm, s2, t_off, mat, al, go, ge, min_score):
    mmax = max(mat)
    for k in idx:
        want, score, te = o.position_max(qs[k], ts[k], mat, al, go, ge)
        got = [int(v) for v in cm[int(t_off[k] - t_off[0]): int(t_off[k + 1] - t_off[0])]]
        assert got == want, k
        h = hits[k]
        assert (h.score, h.db_index, h.query_end, h.target_end) == (score, k, -1, -1 if te is None else te), k
        w2 = o.score2(want, score, 0 if te is None else te, mmax, min_score)
        assert (int(s2[2 * k]), int(s2[2 * k + 1])) == ((0, -1) if w2 is None else w2), k


def test_many_chunks_multi_pass_int32_and_long_pairs():
    """A batch of several chunks: mate-rescue pairs, queries longer than one pass (maxima of the
    passes combined), pairs whose width proof needs int32 (a large matrix entry on longer pairs),
    empty sequences and a few long pairs on the stripe kernel; the caller's column-maxima array
    refilled in place (every entry written)."""
    rng = np.random.default_rng(12)
    n = 150_000
    mat = [int(v) for v in rng.integers(-3, 5, 16)]
    mat[5] = 300
    qs = [rng.integers(0, 4, int(rng.integers(0, 40))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(0, 80))) for _ in range(n)]
    special = [int(k) for k in rng.choice(n, 400, replace=False)]
    for k in special[:200]:  # two or three passes of 256 rows
        qs[k] = rng.integers(0, 4, int(rng.integers(257, 700)))
        ts[k] = rng.integers(0, 4, int(rng.integers(50, 400)))
    for k in special[200:]:  # int32 by the width proof
        qs[k] = rng.integers(0, 4, int(rng.integers(120, 200)))
        ts[k] = rng.integers(0, 4, int(rng.integers(120, 300)))
    longs = [7, 80_001, 149_990]
    for k in longs:
        qs[k] = rng.integers(0, 4, 1100)
        ts[k] = np.concatenate([rng.integers(0, 4, 400), qs[k][100:900], rng.integers(0, 4, 300)])
    q_res, q_off = hy.concat(qs)
    t_res, t_off = hy.concat(ts)
    buf = np.full(int(t_off[-1]), -7, np.int32)
    hits, cm, s2, (err, failed) = hy.align_pairs_position_max_arrays(
        q_res, q_off, t_res, t_off, hy.Scoring(4, mat, 6, 1), 15, colmax_out=buf)
    assert err is None and failed == n and cm is buf
    assert int(buf.min()) >= 0  # every position written
    idx = sorted(set(list(range(0, n, 1009)) + special[::9] + longs + [n - 1]))
    _sample_check(qs, ts, idx, hits, cm, s2, t_off, mat, 4, 6, 1, 15)


def test_failure_in_a_later_chunk_leaves_a_correct_prefix():
    """The first bad symbol (a query's, in a later chunk) ends the batch there: its index and
    error, every earlier pair's maxima, hits and score2 exact, the positions from it on 0."""
    rng = np.random.default_rng(13)
    n = 140_000
    qs = [rng.integers(0, 4, int(rng.integers(1, 40))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(1, 80))) for _ in range(n)]
    bad = 100_003
    qs[bad] = qs[bad].copy()
    qs[bad][0] = 5
    ts[bad + 7] = ts[bad + 7].copy()
    ts[bad + 7][0] = 9
    q_res, q_off = hy.concat(qs)
    t_res, t_off = hy.concat(ts)
    buf = np.full(int(t_off[-1]), -7, np.int32)
    hits, cm, s2, (err, failed) = hy.align_pairs_position_max_arrays(
        q_res, q_off, t_res, t_off, hy.Scoring(4, DNA, 2, 1), 10, colmax_out=buf)
    assert err == hy.Error("SymbolOutOfRange", symbol=5, alphabet_len=4) and failed == bad
    assert int(buf[: int(t_off[bad])].min()) >= 0
    assert not buf[int(t_off[bad]):].any()
    idx = sorted(set(list(range(0, bad, 997)) + [bad - 1]))
    _sample_check(qs, ts, idx, hits, cm, s2, t_off, DNA, 4, 2, 1, 10)


def test_narrowed_chunks_every_column_maximum():
    """Chunks whose pairs all proved int16 send their column maxima back as int16 and the host
    widens them. A pageable column-maxima array over many such chunks (and, in the second call,
    one chunk made wide by int32 pairs among narrowed ones) must equal, entry for entry, the
    page-locked path, which copies the int32 maxima straight into the caller's array; a sample is
    checked against the oracle."""
    rng = np.random.default_rng(14)
    n = 400_000
    # Queries of at most 100 residues: int16 even under the large entry of the second call
    # (100 * 300 + 6 <= 32767).
    qs = [rng.integers(0, 4, int(rng.integers(1, 101))) for _ in range(n)]
    ts = [rng.integers(0, 4, int(rng.integers(1, 300))) for _ in range(n)]
    for mixed in (False, True):
        mat = list(DNA)
        if mixed:  # int32 by the width proof, only inside one range of the input (one chunk)
            mat = [int(v) for v in DNA]
            mat[5] = 300
            for k in range(200_000, 200_400):
                qs[k] = rng.integers(0, 4, 180)
                ts[k] = rng.integers(0, 4, 250)
        q_res, q_off = hy.concat(qs)
        t_res, t_off = hy.concat(ts)
        scoring = hy.Scoring(4, mat, 6, 1)
        page = np.full(int(t_off[-1]), -7, np.int32)
        hits, cm, s2, (err, _) = hy.align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, scoring, 20,
                                                                    colmax_out=page)
        assert err is None
        pq = hy.pinned_empty(len(q_res), np.uint8)
        pt = hy.pinned_empty(len(t_res), np.uint8)
        pcm = hy.pinned_empty(len(page), np.int32)
        pq[:] = q_res
        pt[:] = t_res
        pcm[:] = -7
        hits_p, cm_p, s2_p, (err_p, _) = hy.align_pairs_position_max_arrays(pq, q_off, pt, t_off, scoring, 20,
                                                                            colmax_out=pcm)
        assert err_p is None
        assert np.array_equal(page, pcm), int(np.flatnonzero(page != pcm)[0])
        assert bytes(hits) == bytes(hits_p) and np.array_equal(s2, s2_p)
        idx = sorted(set(list(range(0, n, 4999)) + list(range(200_000, 200_400, 37)) + [n - 1]))
        _sample_check(qs, ts, idx, hits, cm, s2, t_off, mat, 4, 6, 1, 20)
