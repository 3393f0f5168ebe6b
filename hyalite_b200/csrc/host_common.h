// host_common.h -- host-side pieces shared by the runtime translation units: status reporting,
// the width proof and scoring validation (pure host code, callable without a GPU).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime.h>

#include "../../include/hyalite_cuda.h"

namespace hy {

// Every device allocation of the library goes through dev_malloc / dev_free: they count the live
// allocations and, when a test asks for it (hy_debug_fail_device_alloc), make a chosen request
// fail with cudaErrorMemoryAllocation as a full device would.
cudaError_t dev_malloc_bytes(void **p, size_t bytes);
template <class T>
inline cudaError_t dev_malloc(T **p, size_t bytes) {
    return dev_malloc_bytes(reinterpret_cast<void **>(p), bytes);
}
cudaError_t dev_free(void *p);

// Polls a bounded device wait makes before it gives up (the kernels take it as a launch
// parameter). The default bounds a wait to seconds; a test may lower it to make waits run out.
constexpr uint32_t WAIT_POLLS_DEFAULT = 1u << 24;
uint32_t wait_polls();
// Counts the changes of wait_polls(): work captured into a CUDA graph under an older value (the
// limit is a kernel parameter, frozen at capture) is captured again.
uint64_t wait_polls_epoch();

// The status of a device error word (ScanParams::err): 1 a bounded wait gave up, 2 the
// bounds-checked build found an item it could not index safely.
inline hy_status device_error(int word) { return word == 2 ? HY_ERR_DEVICE_CHECK : HY_ERR_TIMEOUT; }

// Records the detail fields of the status being returned on this thread (hy_last_error_detail).
hy_status fail(hy_status st, int64_t d0 = 0, int64_t d1 = 0, int64_t d2 = 0);

// width::magnitude_bound clamped to i64 (src/width.rs:107-137, 157).
int64_t magnitude_bound(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                        int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len);

// ScoreWidth::narrowest_for (src/width.rs:69-71): 0/1/2, or -1 when nothing fits.
int narrowest_width(int64_t bound);

// Scoring::new validation (src/scoring.rs:65-100), with error details recorded.
hy_status validate_scoring(uint64_t al, const int32_t *matrix, uint64_t matrix_len, int32_t go,
                           int32_t ge);

// The device's own per-sequence width rule: a sequence runs in packed int16 lanes when its
// magnitude bound plus gap_open fits int16 (every kernel intermediate is then exact), else in
// int32 lanes with the oracle's sentinel.
inline bool device_fits_i16(int64_t bound, int32_t gap_open) {
    return bound + (int64_t)gap_open <= 32767;
}

}  // namespace hy
