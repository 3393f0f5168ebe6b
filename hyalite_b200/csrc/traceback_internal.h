// traceback_internal.h -- the traceback pieces the runtime translation unit calls.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/hyalite_cuda.h"

namespace hy {

// Frees a traceback context (null is a no-op).
void tb_context_destroy(void *ctx);
// The last call's {fill ms, walk + compaction ms, device span ms, call ms, cells} (zeros for a
// null context).
void tb_context_timing(void *ctx, double out[5]);
// The traceback context of a scratch (null until its first traceback call).
void *scratch_tb(hy_scratch *scratch);
// Kernels the context launched since the last call (then resets the count).
uint64_t tb_context_launches(void *ctx);
// Traces `query` (host, validated) back against database sequences idx[0 .. n_idx) on `stream`,
// creating the context in *ctx_slot on first use. out[x] is the alignment against idx[x]; the
// operations are concatenated in that order into `ops`.
hy_status tb_scan_targets(const hy_db *db, void **ctx_slot, cudaStream_t stream, const uint8_t *query,
                          uint64_t qlen, const uint32_t *idx, uint32_t n_idx, hy_alignment *out,
                          std::vector<uint8_t> &ops);

// align_pairs' long pairs (src/kernel.rs:378-397, the single-pair path): whether a pair goes to
// the score-only stripe kernel, how many warps (stripes) it takes, and the run over the pairs idx
// (query residues already on the device at q_off): BestHit fields written at each pair's index
// into the device arrays, on `stream`; blocks until they are written. kernel_ms accumulates the
// stripe kernel's device time.
bool tb_long_pair(uint64_t qlen, uint64_t tlen);
uint64_t tb_long_pair_stripes(uint64_t qlen);
hy_status tb_long_pair_scores(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                              const uint64_t *t_off, const std::vector<uint32_t> &idx, const uint8_t *d_q,
                              const int32_t *d_matrix, uint64_t al, int32_t go, int32_t ge, int mode,
                              cudaStream_t stream, int32_t *d_scores, int32_t *d_qend, int32_t *d_tend,
                              double *kernel_ms);

}  // namespace hy
