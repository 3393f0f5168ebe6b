"""The host worker pool behind the library's parallel loops, exercised on the CPU: align_pairs'
lengths pass (the width proof over every pair, chunked over the host threads) runs before any
device work, so a batch whose first pair fails the proof returns its error without a GPU. Repeated
calls reuse the pool; concurrent calls from several threads find it busy and run on threads of
their own. Every call must report the same error and index."""
import threading

import numpy as np

import hyalite_b200 as hy


def _batch(n, bad_at):
    rng = np.random.default_rng(5)
    ql = rng.integers(1, 40, n).astype(np.uint64)
    tl = rng.integers(1, 60, n).astype(np.uint64)
    ql[bad_at] = 40_000
    tl[bad_at] = 40_000
    q_off = np.zeros(n + 1, np.uint64)
    t_off = np.zeros(n + 1, np.uint64)
    q_off[1:] = np.cumsum(ql)
    t_off[1:] = np.cumsum(tl)
    q_res = rng.integers(0, 4, int(q_off[-1])).astype(np.uint8)
    t_res = rng.integers(0, 4, int(t_off[-1])).astype(np.uint8)
    return q_res, q_off, t_res, t_off


def _call(args, scoring):
    q_res, q_off, t_res, t_off = args
    _, (err, failed) = hy.align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, hy.Mode.Nw, hy.SearchType.Score)
    return err, failed


def test_width_failure_at_the_first_pair_repeated_and_concurrent():
    # NW with a wide matrix: 40,000 x 40,000 exceeds the int32 proof; every other pair fits.
    scoring = hy.Scoring(4, [10000 if a == b else -10000 for a in range(4) for b in range(4)], 10, 1)
    args = _batch(300_000, 0)
    want = _call(args, scoring)
    assert want[0] is not None and want[0].kind == "ScoreRangeTooWide" and want[1] == 0
    for _ in range(30):
        assert _call(args, scoring) == want
    results = [None] * 6

    def worker(i):
        results[i] = [_call(args, scoring) for _ in range(10)]

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert all(r == [want] * 10 for r in results)


def test_symbol_before_width_at_the_first_pair():
    # The first pair fails both ways: symbols are checked first (src/kernel.rs:354-415).
    scoring = hy.Scoring(4, [10000 if a == b else -10000 for a in range(4) for b in range(4)], 10, 1)
    q_res, q_off, t_res, t_off = _batch(100_000, 0)
    q_res = q_res.copy()
    q_res[3] = 7
    err, failed = _call((q_res, q_off, t_res, t_off), scoring)
    assert err == hy.Error("SymbolOutOfRange", symbol=7, alphabet_len=4) and failed == 0
