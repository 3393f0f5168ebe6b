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
// stripe kernel's device time. With `cmx` (align_pair_position_max, mode SW): every column's
// maximum max-reduced into cmx->colmax + t_off[k] (zeroed by the caller), and the pair's BestHit
// and score2 from them (position_hits; d_qend unused).
bool tb_long_pair(uint64_t qlen, uint64_t tlen);
uint64_t tb_long_pair_stripes(uint64_t qlen);
struct TbColmaxOut {
    int32_t *colmax;     // device, indexed by absolute target offset
    int32_t *s2;         // device, {score, position} per pair, or null
    int32_t matrix_max;
    int32_t min_score;
};
hy_status tb_long_pair_scores(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                              const uint64_t *t_off, const std::vector<uint32_t> &idx, const uint8_t *d_q,
                              const int32_t *d_matrix, uint64_t al, int32_t go, int32_t ge, int mode,
                              cudaStream_t stream, int32_t *d_scores, int32_t *d_qend, int32_t *d_tend,
                              double *kernel_ms, const TbColmaxOut *cmx = nullptr);

// align_pair_position_max's BestHit from one pair's column maxima cm[0 .. n) (src/kernel.rs:541-553:
// score = the maximum, target end = its first position, -1 when the score is 0) and, with s2, bwa's
// score2 (src/kernel.rs:741-792) with that best and target end (position 0 when -1): runs of
// adjacent columns >= min_score collapsed to their maximum, the highest such peak outside
// [te - w, te + w] with w = ceil(best / matrix_max), ties to the smallest position; s2 = {0, -1}
// when none qualifies.
__device__ inline void position_hits(const int32_t *cm, uint32_t n, int32_t matrix_max, int32_t min_score,
                                     int32_t *score, int32_t *tend, int32_t *s2) {
    int32_t best = 0;
    int64_t te = -1;
    for (uint32_t x = 0; x < n; ++x)
        if (cm[x] > best) {
            best = cm[x];
            te = x;
        }
    *score = best;
    *tend = (int32_t)te;
    if (!s2) return;
    int32_t s2_score = -1;
    int64_t s2_pos = -1;
    if (matrix_max > 0) {
        const int64_t w = ((int64_t)best + matrix_max - 1) / matrix_max;
        const int64_t c = te < 0 ? 0 : te;
        const int64_t low = c - w, high = c + w;
        auto consider = [&](int32_t sc, int64_t pos) {
            if ((pos < low || pos > high) && (s2_pos < 0 || sc > s2_score)) {
                s2_score = sc;
                s2_pos = pos;
            }
        };
        int32_t cs = 0;
        int64_t cp = -1;  // the open peak (score, position), none while cp < 0
        for (uint32_t x = 0; x < n; ++x) {
            const int32_t v = cm[x];
            if (v < min_score) continue;
            if (cp >= 0 && cp + 1 == (int64_t)x) {
                if (cs < v) {
                    cs = v;
                    cp = x;
                }
            } else {
                if (cp >= 0) consider(cs, cp);
                cs = v;
                cp = x;
            }
        }
        if (cp >= 0) consider(cs, cp);
    }
    s2[0] = s2_pos < 0 ? 0 : s2_score;
    s2[1] = (int32_t)s2_pos;
}

}  // namespace hy
