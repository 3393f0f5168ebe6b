"""align_pair_position_max and score2 (src/kernel.rs:454-553, 741-792) on the CPU side: the oracle
pinned to the reference's known answers and properties, and the product's host score2 (a scan of
a host array, as in the reference) against them."""
import json
import os

import numpy as np
import pytest

import pyoracle as o
from conftest import DNA, Lcg

import hyalite_b200 as hy

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "position_max_known_answers.json")) as f:
    G = json.load(f)


@pytest.mark.parametrize("case", G["position_max"], ids=lambda c: c["cite"])
def test_oracle_position_max_known_answers(case):
    out, score, te = o.position_max(case["q"], case["t"], DNA, 4, 2, 1)
    assert out == case["out"] and score == case["score"] and te == case["target_end"]


@pytest.mark.parametrize("case", G["score2"], ids=lambda c: c["cite"])
def test_score2_known_answers(case):
    want = None if case["want"] is None else tuple(case["want"])
    args = (case["colmax"], case["best"], case["te"], case["matrix_max"], case["min_score"])
    assert o.score2(*args) == want
    assert hy.score2(*args) == want


def score2_reference(colmax, best, te, matrix_max, min_score):
    """The reference test's explicit-peak-list transcription (src/kernel.rs:1207-1242)."""
    if matrix_max <= 0:
        return None
    peaks = []
    for i, v in enumerate(colmax):
        if v < min_score:
            continue
        if peaks and peaks[-1][1] + 1 == i:
            if peaks[-1][0] < v:
                peaks[-1] = (v, i)
        else:
            peaks.append((v, i))
    w = max((max(best, 0) + matrix_max - 1) // matrix_max, 0)
    low, high = te - w, te + w
    best2 = None
    for score, pos in peaks:
        if (pos < low or pos > high) and (best2 is None or score > best2[0]):
            best2 = (score, pos)
    return best2


def test_score2_matches_the_peak_list_form():
    """src/kernel.rs:1278-1293: random arrays, windows, thresholds and matrix maxima."""
    rng = Lcg(17)
    for _ in range(3000):
        colmax = [rng.next() % 21 for _ in range(rng.next() % 41)]
        args = (colmax, rng.next() % 41, rng.next() % 41, int(rng.next() % 11) - 2, 1 + rng.next() % 6)
        want = score2_reference(*args)
        assert o.score2(*args) == want and hy.score2(*args) == want, args


def test_oracle_position_max_matches_align_core():
    """src/kernel.rs:1081-1101: the array's maximum and first position equal the SW ScoreEnd
    score and target end; every entry >= 0; one entry per target position."""
    rng = Lcg(23)
    for _ in range(300):
        al = 2 + rng.next() % 3
        mat = [int(rng.next() % 11) - 5 for _ in range(al * al)]
        go = rng.next() % 9
        ge = rng.next() % (go + 1)
        q = [rng.next() % al for _ in range(rng.next() % 12)]
        t = [rng.next() % al for _ in range(rng.next() % 12)]
        out, score, te = o.position_max(q, t, mat, al, go, ge)
        s, qe, te2 = o.align_pair(q, t, mat, al, go, ge, 0)
        assert len(out) == len(t) and all(v >= 0 for v in out)
        assert score == s == max(out, default=0) and te == te2
        # Each entry is the column maximum of the full SW matrix (checked via single-column
        # targets: the best local score ending at target position j is the SW score of q against
        # t[:j + 1] restricted to alignments ending at j).
        for j in range(len(t)):
            pref, ps, pte = o.position_max(q, t[: j + 1], mat, al, go, ge)
            assert pref == out[: j + 1]
