"""CPU-side checks of the traceback's host logic in the product library: the validation order of
align (src/align.rs:169-222) and of an Alignment database build (src/database.rs:776-790), and the
budget rule against the oracle. Every case here is refused before any device work, so it runs
without a GPU."""
import numpy as np
import pytest

import pyoracle as o
from conftest import DNA, identity_matrix

import hyalite_b200 as hy
from hyalite_b200 import _abi

DNA_SCORING = hy.Scoring(4, DNA, 2, 1)


def test_budget_rule_matches_the_oracle():
    for m in (0, 1, 2, 5, 17, 100, 1000, 65536):
        for n in (0, 1, 3, 64, 999, 100000):
            for budget in (0, 1, 240, 10 ** 4, 10 ** 6, 10 ** 9, hy.USIZE_MAX):
                assert _abi.lib.hy_traceback_needed(m, n, budget) == o.traceback_needed(m, n, budget)
            assert hy.traceback_min_bytes_for_database(m, n) == o.traceback_min_bytes_for_database(m, n)


def test_align_validation_order():
    # Scoring first (Scoring::new), then symbols (query before target), then the width proof,
    # then the budget (src/align.rs:176-186, 205-221).
    with pytest.raises(hy.Error) as e:
        hy.Scoring(4, DNA, 1, 2)
    assert e.value.kind == "GapOpenLessThanExtend"
    with pytest.raises(hy.Error) as e:
        hy.align([9], [0], DNA_SCORING, hy.Mode.Nw, hy.USIZE_MAX)
    assert e.value == hy.Error("SymbolOutOfRange", symbol=9, alphabet_len=4)
    with pytest.raises(hy.Error) as e:
        hy.align([0], [7], DNA_SCORING, hy.Mode.Nw, 0)
    assert e.value == hy.Error("SymbolOutOfRange", symbol=7, alphabet_len=4)
    wide = hy.Scoring(4, identity_matrix(4, 2, -1), 300_000_000, 100_000_000)
    with pytest.raises(hy.Error) as e:
        hy.align([0, 1], [0, 1], wide, hy.Mode.Nw, 0)
    assert e.value.kind == "ScoreRangeTooWide"
    # src/align/tests.rs:345-365: one byte short of 3 * 5 * 4 * 4 fails with both counts.
    with pytest.raises(hy.Error) as e:
        hy.align([0, 1, 2, 3], [0, 1, 2], DNA_SCORING, hy.Mode.Nw, 239)
    assert e.value == hy.Error("TracebackBudgetExceeded", needed_bytes=240, budget_bytes=239)


def test_alignment_database_budget_is_validated_at_build():
    # tests/database_alignment.rs:84-99: a one-byte budget cannot cover an 8 x 8 traceback.
    with pytest.raises(hy.Error) as e:
        (hy.Database.builder().sequences([[0, 1, 2, 3, 0, 1, 2, 3]]).scoring(DNA_SCORING)
         .mode(hy.Mode.Nw).search_type(hy.SearchType.alignment(1)).max_query_len(8).build())
    need = o.traceback_min_bytes_for_database(8, 8)
    assert e.value == hy.Error("TracebackBudgetExceeded", needed_bytes=need, budget_bytes=1)


def test_search_type_surface():
    # src/search.rs:62-88.
    assert not hy.SearchType.Score.tracks_end()
    assert hy.SearchType.ScoreEnd.tracks_end()
    a = hy.SearchType.alignment(4096)
    assert a.tracks_end() and a.max_bytes == 4096 and int(a) == 2
    assert str(a) == "Alignment { max_bytes: 4096 }"


def test_cigar_formatting():
    # src/align/tests.rs:317-339.
    ops = bytes([0, 0, 1, 2, 2, 3, 0])
    a = hy.Alignment(0, 0, 0, 0, 0, ops)
    assert a.cigar() == "3M2I1D1M" and a.cigar_extended() == "2=1X2I1D1="
    assert a.ops == [hy.AlignOp.Match, hy.AlignOp.Match, hy.AlignOp.Mismatch, hy.AlignOp.Ins,
                     hy.AlignOp.Ins, hy.AlignOp.Del, hy.AlignOp.Match]
    assert hy.Alignment(0, 0, 0, 0, 0, b"").cigar() == ""
