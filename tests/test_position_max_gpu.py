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
