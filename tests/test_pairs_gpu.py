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
