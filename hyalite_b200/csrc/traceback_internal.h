// traceback_internal.h -- the traceback pieces the runtime translation unit calls.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/hyalite_cuda.h"

namespace hy {

// Frees a traceback context (null is a no-op).
void tb_context_destroy(void *ctx);
// Kernels the context launched since the last call (then resets the count).
uint64_t tb_context_launches(void *ctx);
// Traces `query` (host, validated) back against database sequences idx[0 .. n_idx) on `stream`,
// creating the context in *ctx_slot on first use. out[x] is the alignment against idx[x]; the
// operations are concatenated in that order into `ops`.
hy_status tb_scan_targets(const hy_db *db, void **ctx_slot, cudaStream_t stream, const uint8_t *query,
                          uint64_t qlen, const uint32_t *idx, uint32_t n_idx, hy_alignment *out,
                          std::vector<uint8_t> &ops);

}  // namespace hy
