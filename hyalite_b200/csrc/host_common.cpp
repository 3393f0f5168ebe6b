// host_common.cpp -- status reporting, scoring validation, the width proof and backend selection.
// Pure host code: none of it touches the GPU except hy_backend_is_available.
#include "host_common.h"

#include <ctype.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>
#include <string>

#include <algorithm>
#include <atomic>

namespace hy {

static thread_local int64_t g_detail[3] = {0, 0, 0};

// Live device allocations, and the test hook's countdown to a failing one (-1: off).
static std::atomic<int64_t> g_live_allocs{0};
static std::atomic<int64_t> g_fail_countdown{-1};
static std::atomic<uint32_t> g_wait_polls{WAIT_POLLS_DEFAULT};
static std::atomic<uint64_t> g_wait_epoch{0};

cudaError_t dev_malloc_bytes(void **p, size_t bytes) {
    int64_t c = g_fail_countdown.load();
    while (c >= 0) {
        if (g_fail_countdown.compare_exchange_weak(c, c - 1)) {
            if (c == 0) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) g_live_allocs.fetch_add(1);
    return e;
}

cudaError_t dev_free(void *p) {
    if (!p) return cudaSuccess;
    g_live_allocs.fetch_sub(1);
    return cudaFree(p);
}

uint32_t wait_polls() { return g_wait_polls.load(); }
uint64_t wait_polls_epoch() { return g_wait_epoch.load(); }

hy_status fail(hy_status st, int64_t d0, int64_t d1, int64_t d2) {
    g_detail[0] = d0;
    g_detail[1] = d1;
    g_detail[2] = d2;
    return st;
}

int64_t magnitude_bound(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                        int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len) {
    __int128 m = (__int128)max_query_len, n = (__int128)max_target_len;
    __int128 min_ij = m < n ? m : n;
    __int128 max_pos = max_entry > 0 ? (__int128)max_entry : 0;
    __int128 max_neg = -(__int128)min_entry > 0 ? -(__int128)min_entry : 0;
    __int128 go = gap_open, ge = gap_ext;
    __int128 positive = min_ij * max_pos, negative;
    if (mode == HY_MODE_SW) {
        negative = go;
    } else if (mode == HY_MODE_OV) {
        negative = min_ij * max_neg + go;
    } else {
        __int128 run = m + n - 1;
        if (run < 0) run = 0;
        negative = (m + n) * max_neg + go + run * ge;
    }
    __int128 b = positive > negative ? positive : negative;
    if (b > (__int128)INT64_MAX) b = INT64_MAX;
    return (int64_t)b;
}

int narrowest_width(int64_t bound) {
    if (bound <= 127) return HY_WIDTH_I8;
    if (bound <= 32767) return HY_WIDTH_I16;
    if (bound <= 536870911) return HY_WIDTH_I32;
    return -1;
}

hy_status validate_scoring(uint64_t al, const int32_t *matrix, uint64_t matrix_len, int32_t go,
                           int32_t ge) {
    if (al == 0) return fail(HY_ERR_EMPTY_ALPHABET);
    unsigned __int128 sq = (unsigned __int128)al * al;
    if (sq != matrix_len) {
        int64_t expected = sq > (unsigned __int128)INT64_MAX ? INT64_MAX : (int64_t)sq;
        return fail(HY_ERR_MATRIX_SHAPE, (int64_t)al, expected, (int64_t)matrix_len);
    }
    if (matrix == nullptr && matrix_len > 0) return fail(HY_ERR_INVALID_ARGUMENT);
    if (go < 0 || ge < 0) return fail(HY_ERR_NEGATIVE_GAP_PENALTY, go, ge);
    if (go < ge) return fail(HY_ERR_GAP_OPEN_LESS_THAN_EXTEND, go, ge);
    return fail(HY_OK);
}

}  // namespace hy

using namespace hy;

extern "C" {

void hy_last_error_detail(int64_t detail[3]) {
    if (!detail) return;
    detail[0] = g_detail[0];
    detail[1] = g_detail[1];
    detail[2] = g_detail[2];
}

const char *hy_status_name(hy_status s) {
    switch (s) {
    case HY_OK: return "Ok";
    case HY_ERR_EMPTY_ALPHABET: return "EmptyAlphabet";
    case HY_ERR_MATRIX_SHAPE: return "MatrixShape";
    case HY_ERR_NEGATIVE_GAP_PENALTY: return "NegativeGapPenalty";
    case HY_ERR_GAP_OPEN_LESS_THAN_EXTEND: return "GapOpenLessThanExtend";
    case HY_ERR_SCORE_RANGE_TOO_WIDE: return "ScoreRangeTooWide";
    case HY_ERR_SYMBOL_OUT_OF_RANGE: return "SymbolOutOfRange";
    case HY_ERR_INCOMPLETE_BUILDER: return "IncompleteBuilder";
    case HY_ERR_EMPTY_DATABASE: return "EmptyDatabase";
    case HY_ERR_BACKEND_UNAVAILABLE: return "BackendUnavailable";
    case HY_ERR_INVALID_BACKEND_NAME: return "InvalidBackendName";
    case HY_ERR_TRACEBACK_BUDGET_EXCEEDED: return "TracebackBudgetExceeded";
    case HY_ERR_INVALID_ARGUMENT: return "InvalidArgument";
    case HY_ERR_QUERY_TOO_LONG: return "QueryTooLong";
    case HY_ERR_CUDA: return "Cuda";
    case HY_ERR_OUT_OF_MEMORY: return "OutOfMemory";
    case HY_ERR_TIMEOUT: return "Timeout";
    case HY_ERR_UNSUPPORTED: return "Unsupported";
    case HY_ERR_REJECTED: return "Rejected";
    case HY_ERR_DEVICE_CHECK: return "DeviceCheck";
    }
    return "Unknown";
}

const char *hy_backend_name(hy_backend b) {
    switch (b) {
    case HY_BACKEND_SCALAR: return "scalar";
    case HY_BACKEND_SSE41: return "sse4.1";
    case HY_BACKEND_AVX2: return "avx2";
    case HY_BACKEND_NEON: return "neon";
    case HY_BACKEND_CUDA: return "cuda";
    }
    return "unknown";
}

hy_status hy_backend_parse(const char *name, int *choice) {
    if (!name || !choice) return fail(HY_ERR_INVALID_ARGUMENT);
    std::string s(name);
    size_t a = 0, b = s.size();
    while (a < b && isspace((unsigned char)s[a])) ++a;
    while (b > a && isspace((unsigned char)s[b - 1])) --b;
    std::string t = s.substr(a, b - a);
    for (auto &c : t) c = (char)tolower((unsigned char)c);
    if (t == "auto") *choice = HY_CHOICE_AUTO;
    else if (t == "scalar") *choice = HY_BACKEND_SCALAR;
    else if (t == "sse4.1" || t == "sse41") *choice = HY_BACKEND_SSE41;
    else if (t == "avx2") *choice = HY_BACKEND_AVX2;
    else if (t == "neon") *choice = HY_BACKEND_NEON;
    else if (t == "cuda") *choice = HY_BACKEND_CUDA;
    else return fail(HY_ERR_INVALID_BACKEND_NAME);
    return fail(HY_OK);
}

int hy_backend_is_available(hy_backend b) {
    if (b != HY_BACKEND_CUDA) return 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0;
}

hy_status hy_backend_resolve(int choice, hy_backend *out) {
    if (!out) return fail(HY_ERR_INVALID_ARGUMENT);
    if (choice == HY_CHOICE_UNSET) {
        const char *env = getenv("HYALITE_BACKEND");
        choice = HY_CHOICE_AUTO;
        if (env) {
            std::string e(env);
            bool blank = true;
            for (char c : e) blank = blank && isspace((unsigned char)c);
            if (!blank) {
                hy_status st = hy_backend_parse(env, &choice);
                if (st != HY_OK) return st;
            }
        }
    }
    if (choice == HY_CHOICE_AUTO) {
        if (hy_backend_is_available(HY_BACKEND_CUDA)) {
            *out = HY_BACKEND_CUDA;
            return fail(HY_OK);
        }
        return fail(HY_ERR_BACKEND_UNAVAILABLE, HY_BACKEND_CUDA);
    }
    if (choice < HY_BACKEND_SCALAR || choice > HY_BACKEND_CUDA) return fail(HY_ERR_INVALID_ARGUMENT);
    if (!hy_backend_is_available((hy_backend)choice)) return fail(HY_ERR_BACKEND_UNAVAILABLE, choice);
    *out = (hy_backend)choice;
    return fail(HY_OK);
}

hy_status hy_scoring_validate(uint64_t alphabet_len, const int32_t *matrix, uint64_t matrix_len,
                              int32_t gap_open, int32_t gap_ext) {
    return validate_scoring(alphabet_len, matrix, matrix_len, gap_open, gap_ext);
}

hy_status hy_required_width(hy_mode mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                            int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len,
                            hy_score_width *width, int64_t *bound) {
    if ((int)mode < 0 || (int)mode > 4) return fail(HY_ERR_INVALID_ARGUMENT);
    int64_t b = magnitude_bound(mode, min_entry, max_entry, gap_open, gap_ext, max_query_len,
                                max_target_len);
    if (bound) *bound = b;
    int w = narrowest_width(b);
    if (w < 0) return fail(HY_ERR_SCORE_RANGE_TOO_WIDE, b);
    if (width) *width = (hy_score_width)w;
    return fail(HY_OK);
}

}  // extern "C"

extern "C" {

void hy_debug_fail_device_alloc(int64_t after) { hy::g_fail_countdown.store(after < 0 ? -1 : after); }

int64_t hy_debug_live_device_allocations(void) { return hy::g_live_allocs.load(); }

void hy_debug_set_wait_polls(int64_t polls) {
    hy::g_wait_polls.store(polls < 0 ? hy::WAIT_POLLS_DEFAULT : (uint32_t)std::min<int64_t>(polls, UINT32_MAX));
    hy::g_wait_epoch.fetch_add(1);
}

}  // extern "C"
