"""The allocation-free scan (hy_scan_scores_noalloc) against the regular hy_scan_scores.

It serves callers that cannot call cudaMalloc while running: a process whose device memory is
already owned by another allocator, or a loop that cannot afford cudaMalloc's implicit device
synchronisation. Its scratch is a fixed array inside the library, shared by every call, so this
test makes two calls in a row (the second sees the first call's leftovers) and checks both against
the allocating entry point. Scores are integers: the tolerance is exact equality. Collected last
(file name) so a failure here never hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from gpu_helpers import BLOSUM62

pytestmark = pytest.mark.gpu


def _database(hy, rng, n_seqs):
    seqs = [rng.integers(0, 20, int(n)).astype(np.uint8) for n in rng.integers(0, 600, n_seqs)]
    seqs += [rng.integers(0, 20, 3500).astype(np.uint8)]  # a sequence in the int32 partition
    return (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(20, BLOSUM62, 11, 1))
            .mode(hy.Mode.Sw).search_type(hy.SearchType.Score).max_query_len(3000).build())


def _noalloc(hy, db, d_query, qlen, d_out, stream):
    return hy._abi.lib.hy_scan_scores_noalloc(db._h, C.c_void_p(d_query.data_ptr()), qlen,
                                              C.c_void_p(d_out.data_ptr()), C.c_void_p(stream))


def test_noalloc_scores_match_the_allocating_scan_twice_in_a_row():
    torch = pytest.importorskip("torch")
    import hyalite_b200 as hy

    rng = np.random.default_rng(2026)
    db = _database(hy, rng, 3000)
    sc = hy.Scratch(db)
    n = db.sequence_count()
    stream = torch.cuda.current_stream().cuda_stream
    # A single-pass query, then a multi-pass one that also needs boundary rows in the scratch.
    for qlen in (90, 1200):
        q = rng.integers(0, 20, qlen).astype(np.uint8)
        want = db.scan_scores_array(sc, q)
        d_q = torch.from_numpy(q).cuda()
        d_out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = _noalloc(hy, db, d_q, qlen, d_out, stream)
        assert st == 0, hy.Error.from_status(st)
        got = d_out.cpu().numpy()
        assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
        if qlen == 1200:
            # Not the first call of the process: nothing new may have been allocated on the device.
            assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_scratch_beyond_its_limit():
    torch = pytest.importorskip("torch")
    import hyalite_b200 as hy

    rng = np.random.default_rng(7)
    # 600,000 residues packed in pairs need 8 bytes of boundary row per pair column: ~2.4 MB per
    # 100k columns; a long query over a large database exceeds the fixed scratch.
    seqs = [rng.integers(0, 20, 1000).astype(np.uint8) for _ in range(5000)]
    db = (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(20, BLOSUM62, 11, 1))
          .mode(hy.Mode.Sw).search_type(hy.SearchType.Score).max_query_len(2000).build())
    q = torch.from_numpy(rng.integers(0, 20, 2000).astype(np.uint8)).cuda()
    out = torch.zeros(db.sequence_count(), dtype=torch.int32, device="cuda")
    st = _noalloc(hy, db, q, 2000, out, torch.cuda.current_stream().cuda_stream)
    err = hy.Error.from_status(st)
    assert err.kind == "Unsupported"
    needed, limit, _ = hy._abi.last_detail()
    assert needed > limit == 16 << 20
