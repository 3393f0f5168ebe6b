"""ctypes declarations of the C ABI in include/hyalite_cuda.h.

The shared library is built in-tree (hyalite_b200/libhyalite_cuda.so). There is no fallback:
importing the package without the library raises, so a missing build is never silently replaced by
CPU code. HYALITE_CUDA_BUILD=bounds loads the bounds-checked build instead
(hyalite_b200/libhyalite_cuda_bounds.so, `make -C hyalite_b200/csrc bounds`): every kernel checks the
indices each item's data can produce before using them and reports DeviceCheck instead of
reading outside an array.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILDS = {"release": "libhyalite_cuda.so", "bounds": "libhyalite_cuda_bounds.so"}
_BUILD = os.environ.get("HYALITE_CUDA_BUILD", "release")
if _BUILD not in _BUILDS:
    raise ImportError(f"HYALITE_CUDA_BUILD={_BUILD!r}: expected one of {sorted(_BUILDS)}")
LIB_PATH = os.path.join(_HERE, _BUILDS[_BUILD])

# Status codes (hy_status).
OK = 0
TIMEOUT = 24
STATUS_NAMES = {
    0: "Ok", 1: "EmptyAlphabet", 2: "MatrixShape", 3: "NegativeGapPenalty",
    4: "GapOpenLessThanExtend", 5: "ScoreRangeTooWide", 6: "SymbolOutOfRange",
    7: "IncompleteBuilder", 8: "EmptyDatabase", 9: "BackendUnavailable",
    10: "InvalidBackendName", 11: "TracebackBudgetExceeded", 20: "InvalidArgument",
    21: "QueryTooLong", 22: "Cuda", 23: "OutOfMemory", 24: "Timeout", 25: "Unsupported",
    26: "Rejected", 27: "DeviceCheck",
}
CHOICE_UNSET = -2
CHOICE_AUTO = -1
LAYOUT_AUTO = -1


class HyHit(C.Structure):
    _fields_ = [("score", C.c_int32), ("reserved", C.c_uint32), ("db_index", C.c_uint64),
                ("query_end", C.c_int64), ("target_end", C.c_int64)]


class HyServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("in_flight", C.c_uint32), ("max_pending", C.c_uint32),
                ("reserved", C.c_uint32), ("profile_budget", C.c_uint64), ("scores_budget", C.c_uint64),
                ("launch_config", C.c_int32 * 3)]


class HyServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("batches", C.c_uint64), ("pending", C.c_uint64), ("mean_batch", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("cells", C.c_double), ("seconds", C.c_double),
                ("gcups", C.c_double)]


class HyAlignment(C.Structure):
    _fields_ = [("score", C.c_int32), ("reserved", C.c_uint32), ("query_start", C.c_uint64),
                ("query_end", C.c_uint64), ("target_start", C.c_uint64), ("target_end", C.c_uint64),
                ("n_ops", C.c_uint64), ("ops_offset", C.c_uint64)]


_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p
_st = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "hy_last_error_detail": (None, [_i64p]),
    "hy_status_name": (C.c_char_p, [_st]),
    "hy_backend_parse": (_st, [C.c_char_p, C.POINTER(C.c_int)]),
    "hy_backend_is_available": (C.c_int, [C.c_int]),
    "hy_backend_resolve": (_st, [C.c_int, C.POINTER(C.c_int)]),
    "hy_backend_name": (C.c_char_p, [C.c_int]),
    "hy_scoring_validate": (_st, [C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32]),
    "hy_required_width": (_st, [C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                C.c_uint64, C.POINTER(C.c_int), _i64p]),
    "hy_db_create": (_st, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32,
                           C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.POINTER(_vp)]),
    "hy_db_traceback_max_bytes": (C.c_uint64, [_vp]),
    "hy_align": (_st, [_u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32,
                       C.c_int, C.c_uint64, C.POINTER(HyAlignment), _u8p]),
    "hy_scan_aligned": (_st, [_vp, _vp, _u8p, C.c_uint64, _u64p, C.POINTER(HyAlignment),
                              C.POINTER(_u8p)]),
    "hy_scan_all_aligned": (_st, [_vp, _vp, _u8p, C.c_uint64, C.POINTER(HyAlignment), C.POINTER(_u8p)]),
    "hy_traceback_min_bytes_for_database": (C.c_uint64, [C.c_uint64, C.c_uint64]),
    "hy_traceback_needed": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64]),
    "hy_traceback_timing": (_st, [_vp, C.POINTER(C.c_double)]),
    "hy_align_pairs_position_max": (_st, [_u8p, _u64p, _u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32,
                                          C.c_int32, _i32p, C.POINTER(HyHit), C.c_int32, _i32p, _u64p]),
    "hy_position_max_timing": (_st, [C.POINTER(C.c_double)]),
    "hy_score2": (C.c_int, [_i32p, C.c_uint64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, _i32p, _u64p]),
    "hy_db_destroy": (None, [_vp]),
    "hy_db_sequence_count": (C.c_uint64, [_vp]),
    "hy_db_mode": (C.c_int, [_vp]),
    "hy_db_search_type": (C.c_int, [_vp]),
    "hy_db_score_width": (C.c_int, [_vp]),
    "hy_db_backend": (C.c_int, [_vp]),
    "hy_db_layout": (C.c_int, [_vp]),
    "hy_db_max_query_len": (C.c_uint64, [_vp]),
    "hy_db_max_target_len": (C.c_uint64, [_vp]),
    "hy_db_device_bytes": (C.c_uint64, [_vp]),
    "hy_db_scratch_bytes": (C.c_uint64, [_vp]),
    "hy_db_partition": (None, [_vp, _u64p, _u64p]),
    "hy_scratch_create": (_st, [_vp, C.POINTER(_vp)]),
    "hy_scratch_destroy": (None, [_vp]),
    "hy_scratch_stream": (_vp, [_vp]),
    "hy_scan": (_st, [_vp, _vp, _u8p, C.c_uint64, C.POINTER(HyHit)]),
    "hy_scan_all": (_st, [_vp, _vp, _u8p, C.c_uint64, C.POINTER(HyHit)]),
    "hy_scan_scores": (_st, [_vp, _vp, _u8p, C.c_uint64, _i32p]),
    "hy_scan_device": (_st, [_vp, _vp, _vp, C.c_uint64, _vp]),
    "hy_scan_scores_device": (_st, [_vp, _vp, _vp, C.c_uint64, _vp]),
    "hy_query_validate": (_st, [_vp, _u8p, C.c_uint64]),
    "hy_scan_scores_noalloc": (_st, [_vp, _vp, C.c_uint64, _vp, _vp]),
    "hy_scratch_sync": (_st, [_vp]),
    "hy_scratch_profile": (_st, [_vp, C.c_int]),
    "hy_scratch_profile_read": (_st, [_vp, C.POINTER(C.c_double), _u64p, C.POINTER(C.c_double), _u64p]),
    "hy_measure_dpx_peak": (_st, [C.POINTER(C.c_double)]),
    "hy_measure_dpx_peak_i32": (_st, [C.POINTER(C.c_double)]),
    "hy_measure_dpx_peak_i8x4": (_st, [C.POINTER(C.c_double)]),
    "hy_debug_fail_device_alloc": (None, [C.c_int64]),
    "hy_debug_live_device_allocations": (C.c_int64, []),
    "hy_debug_set_wait_polls": (None, [C.c_int64]),
    "hy_debug_pair_chunks": (C.c_uint64, [_u64p, _u64p, C.c_uint64, _u64p, C.c_uint64]),
    "hy_debug_band_shape": (None, [C.c_uint32, C.c_int32, C.c_uint64, _i32p]),
    "hy_align_pairs": (_st, [_u8p, _u64p, _u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32,
                             C.c_int32, C.c_int, C.c_int, C.POINTER(HyHit), _u64p]),
    "hy_align_pairs_timing": (_st, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "hy_align_pairs_phases": (_st, [C.POINTER(C.c_double), C.c_uint32]),
    "hy_host_alloc": (_st, [C.c_uint64, C.POINTER(C.c_void_p)]),
    "hy_host_free": (_st, [C.c_void_p]),
    "hy_batch_create": (_st, [C.POINTER(_vp), C.c_uint32, C.c_uint32, C.c_int, C.POINTER(_vp)]),
    "hy_batch_destroy": (None, [_vp]),
    "hy_scan_batch": (_st, [_vp, C.c_uint32, _u32p, _u8p, _u64p, C.POINTER(HyHit), _u32p]),
    "hy_batch_tune": (_st, [_vp, C.c_uint32, _u32p, _u8p, _u64p, C.c_uint32, C.POINTER(C.c_double)]),
    "hy_batch_get_config": (_st, [_vp, _i32p]),
    "hy_batch_set_config": (_st, [_vp, _i32p]),
    "hy_batch_device_bytes": (C.c_uint64, [_vp]),
    "hy_batch_stream": (_vp, [_vp]),
    "hy_server_create": (_st, [C.POINTER(_vp), C.c_uint32, C.POINTER(HyServerConfig), C.POINTER(_vp)]),
    "hy_server_destroy": (None, [_vp]),
    "hy_server_submit": (_st, [_vp, C.c_uint32, _u8p, C.c_uint64, C.c_int, _i32p, _u64p]),
    "hy_server_request_bytes": (C.c_uint64, [_vp, C.c_uint32, C.c_uint64, C.c_int, _u64p]),
    "hy_server_poll": (_st, [_vp, C.c_uint64, C.POINTER(C.c_int)]),
    "hy_server_wait": (_st, [_vp, C.c_uint64, C.c_double, C.POINTER(HyHit)]),
    "hy_server_wait_timed": (_st, [_vp, C.c_uint64, C.c_double, C.POINTER(HyHit), C.POINTER(C.c_double)]),
    "hy_server_stats_read": (_st, [_vp, C.c_int, C.POINTER(HyServerStats)]),
}


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: the cuda backend has no CPU fallback. Build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (or `make -C hyalite_b200/csrc`).")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


def last_detail():
    d = (C.c_int64 * 3)()
    lib.hy_last_error_detail(d)
    return tuple(d)
