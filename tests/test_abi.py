"""CPU-side checks of the product library: it loads, exports every symbol include/hyalite_cuda.h
declares, and its host logic (validation order, backend selection, width proof) mirrors the
reference. No kernel runs here."""
import ctypes as C
import os
import re
import subprocess
import sys

import pytest

from conftest import DNA, ROOT, identity_matrix

import hyalite_b200 as hy
from hyalite_b200 import _abi


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "hyalite_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hy_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = _declared_functions()
    assert len(names) >= 30
    lib = C.CDLL(_abi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_abi.SIGNATURES), set(names) ^ set(_abi.SIGNATURES)


def test_library_links_no_oracle_code():
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    assert "hyo_" not in out and "hyb_" not in out


def test_status_names_cover_error_variants():
    for code, name in _abi.STATUS_NAMES.items():
        assert _abi.lib.hy_status_name(code).decode() == name


def test_scoring_validation_order():
    # src/scoring.rs:65-100 and its tests
    with pytest.raises(hy.Error) as e:
        hy.Scoring(0, [], 1, 1)
    assert e.value.kind == "EmptyAlphabet"
    with pytest.raises(hy.Error) as e:
        hy.Scoring(3, [1, 2], 1, 1)
    assert e.value == hy.Error("MatrixShape", alphabet_len=3, expected=9, got=2)
    with pytest.raises(hy.Error) as e:
        hy.Scoring(2, [1, -1, -1, 1], -1, 0)
    assert e.value == hy.Error("NegativeGapPenalty", gap_open=-1, gap_ext=0)
    with pytest.raises(hy.Error) as e:
        hy.Scoring(2, identity_matrix(2, 1, -1), 1, 2)  # Opal #28 (tests/opal_regressions.rs:70-82)
    assert e.value == hy.Error("GapOpenLessThanExtend", gap_open=1, gap_ext=2)
    s = hy.Scoring(4, DNA, 2, 1)
    assert s.entry_bounds() == (-1, 2) and s.score(2, 2) == 2


def test_required_width_matches_reference_cases():
    assert hy.required_width(hy.Mode.Ov, -2, 1, 2, 2, 91, 33) == hy.ScoreWidth.I8
    assert hy.required_width(hy.Mode.Nw, -2, 1, 2, 2, 91, 33) == hy.ScoreWidth.I16
    assert hy.required_width(hy.Mode.Nw, -1, 1, 2, 1, 30_000, 30_000) == hy.ScoreWidth.I32
    with pytest.raises(hy.Error) as e:
        hy.required_width(hy.Mode.Nw, 0, 0, 2_000_000_000, 1, 1, 1)
    assert e.value == hy.Error("ScoreRangeTooWide", bound=2_000_000_001)


def test_backend_parse_mirrors_reference():
    # src/backend.rs:226-265
    assert hy.BackendChoice.parse("auto") == hy.BackendChoice.Auto()
    assert hy.BackendChoice.parse("AUTO") == hy.BackendChoice.Auto()
    assert hy.BackendChoice.parse("  SSE41 ") == hy.BackendChoice.Force(hy.Backend.Sse41)
    assert hy.BackendChoice.parse("sse4.1") == hy.BackendChoice.Force(hy.Backend.Sse41)
    assert hy.BackendChoice.parse("Avx2") == hy.BackendChoice.Force(hy.Backend.Avx2)
    assert hy.BackendChoice.parse("cuda") == hy.BackendChoice.Force(hy.Backend.Cuda)
    for b in hy.Backend:
        assert hy.BackendChoice.parse(b.name_str()) == hy.BackendChoice.Force(b)
    for bad in ["", "sse2", "ssse3", "avx512", "gpu", "x"]:
        with pytest.raises(hy.Error) as e:
            hy.BackendChoice.parse(bad)
        assert e.value == hy.Error("InvalidBackendName", name=bad)


def test_only_cuda_is_built():
    for b in (hy.Backend.Scalar, hy.Backend.Sse41, hy.Backend.Avx2, hy.Backend.Neon):
        assert not b.is_available()


def test_builder_reports_every_missing_required_field():
    # src/database.rs:1036-1066
    base = hy.Database.builder
    for builder, field in [
        (base(), "sequences"),
        (base().sequences([[0]]), "scoring"),
        (base().sequences([[0]]).scoring(hy.Scoring(4, DNA, 2, 1)), "mode"),
        (base().sequences([[0]]).scoring(hy.Scoring(4, DNA, 2, 1)).mode(hy.Mode.Sw), "max_query_len"),
    ]:
        with pytest.raises(hy.Error) as e:
            builder.build()
        assert e.value == hy.Error("IncompleteBuilder", field=field)


def _build(seqs, **kw):
    b = hy.Database.builder().sequences(seqs).scoring(kw.get("scoring", hy.Scoring(4, DNA, 2, 1)))
    return b.mode(kw.get("mode", hy.Mode.Sw)).max_query_len(kw.get("mql", 8)).backend(
        kw.get("backend", hy.BackendChoice.Auto())).build()


def test_build_validation_order_before_any_device_work():
    # src/database.rs:737-794: empty -> symbols -> width proof -> backend
    with pytest.raises(hy.Error) as e:
        _build([])
    assert e.value.kind == "EmptyDatabase"
    with pytest.raises(hy.Error) as e:
        _build([[0, 1], [2, 9]])
    assert e.value == hy.Error("SymbolOutOfRange", symbol=9, alphabet_len=4)
    with pytest.raises(hy.Error) as e:
        _build([[0]], scoring=hy.Scoring(2, [0, 0, 0, 0], 2_000_000_000, 1), mode=hy.Mode.Nw, mql=1)
    assert e.value.kind == "ScoreRangeTooWide"


@pytest.mark.skipif(hy.Backend.Cuda.is_available(), reason="only meaningful without a GPU")
def test_build_without_a_gpu_is_backend_unavailable():
    with pytest.raises(hy.Error) as e:
        _build([[0, 1, 2]])
    assert e.value == hy.Error("BackendUnavailable", backend=hy.Backend.Cuda)
    with pytest.raises(hy.Error) as e:
        _build([[0, 1, 2]], backend=hy.BackendChoice.Force(hy.Backend.Avx2))
    assert e.value == hy.Error("BackendUnavailable", backend=hy.Backend.Avx2)


def test_env_var_precedence_in_a_fresh_process():
    # tests/backend_env.rs:39-97: an invalid HYALITE_BACKEND is an error at build unless the builder
    # forces a backend explicitly.
    code = (
        "import hyalite_b200 as hy\n"
        "b = hy.Database.builder().sequences([[0]]).scoring(hy.Scoring(4, [2,-1,-1,-1,-1,2,-1,-1,-1,-1,2,-1,-1,-1,-1,2], 2, 1))"
        ".mode(hy.Mode.Sw).max_query_len(4)\n"
        "try:\n    b.build(); print('built')\nexcept hy.Error as e: print(e.kind)\n"
        "try:\n    b.backend(hy.BackendChoice.Force(hy.Backend.Avx2)).build(); print('built')\nexcept hy.Error as e: print(e.kind)\n"
    )
    env = dict(os.environ, HYALITE_BACKEND="definitely-not-a-backend", PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, cwd=ROOT)
    lines = out.stdout.split()
    assert lines[0] == "InvalidBackendName", out.stderr
    assert lines[1] == "BackendUnavailable"


def test_align_pairs_chunks_bound_their_residues_however_pairs_are_ordered():
    """hy_align_pairs cuts its pipeline chunks at equal residue shares: a batch whose long pairs
    cluster in one range still gives chunks of at most 512 MiB of residues plus one pair."""
    import numpy as np

    bound = 512 << 20
    rng = np.random.default_rng(9)
    for long_first in (True, False):
        n = 300_000
        t_len = np.full(n, 300, np.uint64)
        long_idx = np.arange(0, 1500) if long_first else np.arange(n - 1500, n)
        t_len[long_idx] = 1 << 20  # 1,500 windows of 1 MiB: 1.5 GiB in one range of the input
        q_len = rng.integers(50, 200, n).astype(np.uint64)
        q_off = np.zeros(n + 1, np.uint64)
        q_off[1:] = np.cumsum(q_len)
        t_off = np.zeros(n + 1, np.uint64)
        t_off[1:] = np.cumsum(t_len)
        out = np.zeros(64, np.uint64)
        k = _abi.lib.hy_debug_pair_chunks(q_off.ctypes.data_as(_abi._u64p), t_off.ctypes.data_as(_abi._u64p), n,
                                          out.ctypes.data_as(_abi._u64p), len(out))
        b = out[: k + 1].astype(np.int64)
        assert b[0] == 0 and b[-1] == n and np.all(np.diff(b) >= 1)
        res = (q_off[b[1:]] - q_off[b[:-1]]) + (t_off[b[1:]] - t_off[b[:-1]])
        assert int(res.max()) <= bound + (1 << 20) + 200, (long_first, k, res.max())
        assert int(res.sum()) == int(q_off[-1] + t_off[-1])


def test_band_kernel_launch_shape():
    """The end-recovery band kernel's launch shape: one pass slice per warp in shared memory (at
    most 200 KB of slices a block, 32 warps), a cluster of up to 8 blocks when the passes exceed one
    block, as few rounds as that allows and as few warps as those rounds need; slices larger than
    the budget read from global memory on one block."""
    import ctypes as C

    limit = 227 * 1024

    def shape(pass_bytes, n_passes):
        out = (C.c_int32 * 4)()
        _abi.lib.hy_debug_band_shape(pass_bytes, n_passes, limit, out)
        return tuple(out)

    i32_slice, i16_slice = 21 * 256 * 4, 21 * 256 * 8  # 20-letter alphabet, 256-row passes
    assert shape(i32_slice, 1) == (0, 1, 1, 1)
    assert shape(i32_slice, 8) == (0, 8, 1, 1)
    assert shape(i32_slice, 20) == (0, 7, 3, 1)  # a 5000-residue query: a cluster of 3 blocks
    assert shape(i32_slice, 79) == (0, 5, 8, 2)  # 20,000 rows: two rounds on 8 blocks
    assert shape(i16_slice, 36) == (0, 3, 8, 2)
    assert shape(300 * 1024, 5) == (1, 5, 1, 1)  # slices beyond the budget: global memory
    for pb in (1024, 10 * 1024, i32_slice, i16_slice, 100 * 1024, 200 * 1024):
        per_block = min(32, (200 * 1024) // pb)
        for n in range(1, 400, 7):
            g, w, b, r = shape(pb, n)
            assert g == 0 and 1 <= b <= 8 and 1 <= w <= per_block
            assert w * pb + 16 <= limit
            assert w * b * r >= n and (w - 1) * b * r < n  # every pass placed, no spare warp
            assert r == -(-n // (min(8, -(-n // per_block)) * per_block)) or n <= per_block
