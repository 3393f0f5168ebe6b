"""Parity of the device scan at the launch-shape boundaries (rows per lane 8 / 16 / 32 chosen by
query length, query passes, the warp-per-pair path for targets wider than 4096 columns) and, on a
large protein database, full-size properties plus oracle parity on a sample of targets."""
import math

import numpy as np
import pytest

import pyoracle as o
from conftest import ALL_MODES
from gpu_helpers import build, check, hit_tuple, rand_seqs

import hyalite_b200 as hy

pytestmark = pytest.mark.gpu

# Query lengths around the rows-per-lane switches (64 and 192 residues) and around multiples of
# the pass heights (64, 128, 256 rows).
SHAPE_QLENS = (1, 8, 63, 64, 65, 127, 128, 129, 191, 192, 193, 255, 256, 257, 513)


@pytest.mark.parametrize("mode", ALL_MODES)
def test_rows_per_lane_and_pass_boundaries(mode):
    rng = np.random.default_rng(300 + mode)
    mat = [int(v) for v in rng.integers(-4, 12, 400)]
    # Mostly short targets (bulk int16x2 kernel), two wider than 4096 columns (one warp each).
    seqs = rand_seqs(rng, 70, 20, 1, 400) + rand_seqs(rng, 2, 20, 4097, 4600)
    queries = [list(rng.integers(0, 20, n)) for n in SHAPE_QLENS]
    for st in (0, 1):
        check(seqs, mat, 20, 11, 1, mode, st, queries, mql=max(SHAPE_QLENS))


@pytest.mark.parametrize("mode", ALL_MODES)
def test_winner_band_on_a_cluster_over_two_rounds(mode):
    # A 9000-residue ScoreEnd query: the winner's end recovery has 36 passes of 256 rows, more than
    # a cluster of 8 blocks holds slices for (4 int16x2 slices a block for this alphabet), so it
    # runs in two rounds on 8 blocks of 3 warps (src/database.rs:186-197).
    from gpu_helpers import BLOSUM62

    rng = np.random.default_rng(320 + mode)
    seqs = rand_seqs(rng, 120, 20, 20, 300)
    q = list(rng.integers(0, 20, 9000))
    seqs[37] = q[4000:4250]  # a clear winner inside the query
    db = build(seqs, BLOSUM62, 20, 11, 1, mode, 1, mql=9000)
    ref = o.OracleDb(seqs, BLOSUM62, 20, 11, 1, mode, 1)
    assert hit_tuple(db.scan(hy.Scratch(db), q)) == ref.scan(q)


def _protein(n_seqs, seed):
    rng = np.random.default_rng(seed)
    base = np.random.default_rng(12345)
    mat = base.integers(-4, 4, size=(20, 20))
    mat = np.triu(mat) + np.triu(mat, 1).T
    mat[np.diag_indices(20)] = base.integers(4, 12, size=20)
    bg = base.dirichlet(np.full(20, 4.0))
    lengths = np.clip(np.round(np.exp(math.log(300.0) + 0.8 * rng.standard_normal(n_seqs))), 20, 35_000)
    off = np.zeros(n_seqs + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lengths.astype(np.int64))
    res = rng.choice(20, size=int(off[-1]), p=bg).astype(np.uint8)
    return mat.reshape(-1).astype(np.int32), bg, res, off


def test_large_database_properties_and_sampled_parity():
    """200,000 log-normal protein sequences (the benchmark's generator at 2/5 size) with planted
    duplicates of one target. Properties at full size: scan's winner is the first argmax of
    scan_scores; scan_all's scores equal scan_scores; the winner's ends equal the oracle's. Parity:
    scan_all equals the oracle on a sample of 400 targets (the longest ones included)."""
    n = 200_000
    mat, bg, res, off = _protein(n, 4242)
    rng = np.random.default_rng(99)
    # Plant three identical copies of sequence 5000 further down the database (ties on score:
    # the smallest index must win).
    src = res[int(off[5000]):int(off[5001])].copy()
    seqs_res = [res]
    extra = [src, src, src]
    res2 = np.concatenate(seqs_res + extra)
    off2 = np.concatenate([off, off[-1] + np.cumsum([len(x) for x in extra]).astype(np.uint64)])
    n2 = n + 3
    lengths = np.diff(off2.astype(np.int64))
    qrng = np.random.default_rng(5)
    queries = [qrng.choice(20, size=L, p=bg).astype(np.uint8) for L in (150, 1000, 3000)]
    queries.append(src.copy())  # a query whose best hits are the planted copies and sequence 5000
    db = (hy.Database.builder().sequences_concat(res2, off2).scoring(hy.Scoring(20, [int(v) for v in mat], 11, 1))
          .mode(hy.Mode.Sw).search_type(hy.SearchType.ScoreEnd).max_query_len(3000).build())
    sc = hy.Scratch(db)
    order = np.argsort(-lengths, kind="stable")
    sample = np.unique(np.concatenate([order[:40], rng.choice(n2, 360, replace=False), [5000, n, n + 1, n + 2]]))
    for q in queries:
        scores = db.scan_scores_array(sc, q)
        hit = db.scan(sc, q)
        first = int(np.argmax(scores))
        assert hit.score == int(scores.max()) and hit.db_index == first
        allh = db.scan_all_array(sc, q)
        all_scores = np.array([h.score for h in allh], dtype=np.int32)
        assert np.array_equal(all_scores, scores)
        t = res2[int(off2[first]):int(off2[first + 1])]
        s, qe, te = o.align_pair(q, t, mat, 20, 11, 1, 0, 1)
        assert (hit.score, hit.query_end, hit.target_end) == (s, qe, te)
        for k in sample:
            k = int(k)
            t = res2[int(off2[k]):int(off2[k + 1])]
            want = o.align_pair(q, t, mat, 20, 11, 1, 0, 1)
            h = allh[k]
            got = (h.score, None if h.query_end < 0 else h.query_end, None if h.target_end < 0 else h.target_end)
            assert got == want, f"target {k} (len {len(t)}) qlen {len(q)}: {got} != {want}"
    # The self-query ties: sequence 5000 and its three copies score the same; 5000 wins.
    hit = db.scan(sc, src)
    assert hit.db_index == 5000


@pytest.mark.parametrize("al", [64, 200, 255])
def test_large_alphabets_read_the_profile_from_global_memory(al):
    # Alphabets whose query-profile slices do not fit in shared memory at every launch shape: the
    # bulk pairs drop to 8 rows per lane or read the profile from global memory, and so do the
    # int32 items and the winner's-ends recovery. Entries up to 60 put the long targets in int32.
    rng = np.random.default_rng(400 + al)
    mat = [int(v) for v in rng.integers(-20, 61, al * al)]
    seqs = rand_seqs(rng, 50, al, 1, 300) + rand_seqs(rng, 2, al, 2100, 4200)
    queries = [list(rng.integers(0, al, n)) for n in (1, 50, 300, 700)]
    for mode in (0, 1, 3):
        for st in (0, 1):
            db = check(seqs, mat, al, 5, 1, mode, st, queries, mql=700)
    n16, n32 = db.partition()
    assert n32 > 0


def test_large_alphabet_pairs_keep_group_profiles_in_global_memory():
    rng = np.random.default_rng(77)
    al = 200
    mat = [int(v) for v in rng.integers(-6, 9, al * al)]
    qs = [list(rng.integers(0, al, int(rng.integers(0, 200)))) for _ in range(120)]
    ts = [list(rng.integers(0, al, int(rng.integers(0, 300)))) for _ in range(120)]
    for mode in (0, 2, 4):
        out = []
        hy.align_pairs(list(zip(qs, ts)), hy.Scoring(al, mat, 5, 1), hy.Mode(mode), hy.SearchType.ScoreEnd, out)
        status, want, _ = o.align_pairs(qs, ts, mat, al, 5, 1, mode, 1)
        assert status == 0
        assert [(h.score, h.db_index, h.query_end, h.target_end) for h in out] == want


def test_noalloc_rejects_an_alphabet_beyond_shared_memory():
    import ctypes as C

    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    al = 120
    mat = [int(v) for v in rng.integers(-4, 5, al * al)]
    seqs = rand_seqs(rng, 20, al, 1, 100)
    db = build(seqs, mat, al, 5, 1, 0, 0, 600)
    qh = rng.integers(0, al, 600).astype(np.uint8)
    q = torch.from_numpy(qh).cuda()
    out = torch.zeros(20, dtype=torch.int32, device="cuda")
    st = hy._abi.lib.hy_scan_scores_noalloc(db._h, C.c_void_p(q.data_ptr()), 600, C.c_void_p(out.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert hy.Error.from_status(st).kind == "Unsupported"
    # The allocating scan handles it.
    want = o.OracleDb(seqs, mat, al, 5, 1, 0, 0).scan_scores(list(qh))
    assert np.array_equal(db.scan_scores_array(hy.Scratch(db), qh), want)
