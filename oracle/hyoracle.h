/*
 * hyoracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of hyalite's scalar oracle and of the result semantics of its database
 * scan. It exists so the tests can check the CUDA backend, and so bench.py can time a CPU
 * baseline. Nothing in the shipped library links, loads or calls this code: the product path
 * (hyalite_b200/csrc, libhyalite_cuda.so) has no CPU fallback.
 *
 * Each function cites the reference file:line it follows (paths inside Psy-Fer/hyalite).
 * Parity status: pinned. tests/test_oracle.py checks this oracle against every known-answer
 * vector the reference's own tests hold for this path, against an exhaustive brute-force
 * enumeration (restated from tests/common/mod.rs:65-171), and against the reference's width-proof
 * unit tests (src/width.rs:177-414).
 *
 * Conventions shared with the C-ABI (include/hyalite_cuda.h):
 *   mode:        0 SW, 1 NW, 2 HW, 3 OV, 4 SHW          (src/mode.rs:11-27)
 *   search type: 0 Score, 1 ScoreEnd, 2 Alignment      (src/search.rs:13-27)
 *   width:       0 i8, 1 i16, 2 i32                    (src/width.rs:26-34)
 *   ends:        -1 means None                         (src/hit.rs:16-25)
 *   status:      the HY_* codes of include/hyalite_cuda.h
 */
#ifndef HYORACLE_H
#define HYORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t score;
    uint64_t db_index;
    int64_t query_end;
    int64_t target_end;
} hyo_hit;

/* Scoring::new validation order (src/scoring.rs:65-100). Returns a status code; *d1,*d2,*d3
 * receive the error's fields (see include/hyalite_cuda.h). */
int hyo_scoring_validate(uint64_t alphabet_len, const int32_t *matrix, uint64_t matrix_len,
                         int32_t gap_open, int32_t gap_ext, int64_t *d1, int64_t *d2, int64_t *d3);

/* width::magnitude_bound clamped to i64 (src/width.rs:107-137, 157). */
int64_t hyo_magnitude_bound(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                            int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len);

/* width::required_width (src/width.rs:145-169): returns 0/1/2 for i8/i16/i32, or -1 when even
 * i32 is too narrow (ScoreRangeTooWide); *bound_out receives the clamped bound either way. */
int hyo_required_width(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                       int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len,
                       int64_t *bound_out);

/* kernel::align_core = fill_dp + reduce_answer (src/kernel.rs:168-277). */
void hyo_align_core(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                    const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                    int mode, int32_t *score, int64_t *query_end, int64_t *target_end);

/* Database scan semantics over a concatenated database: sequence k is
 * residues[offsets[k] .. offsets[k+1]]. Database::scan (src/database.rs:83-144, 160-208),
 * scan_all (347-464), scan_scores (481-515). The caller has validated the database. */
void hyo_scan(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
              const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
              int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out);
void hyo_scan_all(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                  const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
                  int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out);
void hyo_scan_scores(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                     const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                     int mode, const uint8_t *query, uint64_t qlen, int32_t *out);

/* The same three entry points spread over `threads` OpenMP threads (targets split statically);
 * identical results. */
void hyo_scan_scores_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                        const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                        int mode, const uint8_t *query, uint64_t qlen, int32_t *out, int threads);
void hyo_scan_all_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                     const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                     int mode, int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out,
                     int threads);

/* align_pairs (src/kernel.rs:429-452 via align_pair_with 354-415): validation first, pair by
 * pair (symbols, then width); returns a status and fills `out` on success. */
int hyo_align_pairs(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                    const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix, uint64_t al,
                    int32_t gap_open, int32_t gap_ext, int mode, int search_type, hyo_hit *out,
                    int threads, int64_t *d1, int64_t *d2);

/* Exhaustive brute-force scorer (restated from tests/common/mod.rs:65-171): an independent
 * second oracle for tiny inputs. */
int32_t hyo_brute(int mode, const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                  const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext);

/* Alignment (src/align.rs:57-83): half-open spans; ops[0 .. n_ops) hold AlignOp codes 0 Match,
 * 1 Mismatch, 2 Ins, 3 Del (src/align.rs:47-56). */
typedef struct {
    int32_t score;
    uint64_t query_start, query_end, target_start, target_end;
    uint64_t n_ops;
} hyo_alignment;

/* traceback_full + walk (src/align.rs:345-545) on validated input (no budget): ops needs room
 * for m + n codes. */
void hyo_traceback(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                   const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
                   hyo_alignment *out, uint8_t *ops);
/* align (src/align.rs:169-222): symbols, width proof, then the traceback budget (status 11 with
 * *d1 = needed bytes, *d2 = budget), then hyo_traceback. */
int hyo_align(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n, const int32_t *matrix,
              uint64_t al, int32_t gap_open, int32_t gap_ext, int mode, uint64_t max_bytes,
              hyo_alignment *out, uint8_t *ops, int64_t *d1, int64_t *d2);
/* Database::scan_all_aligned over `threads` threads (src/database.rs:538-549): alignment k's
 * codes go to ops + k * qlen + (offsets[k] - offsets[0]). */
void hyo_scan_all_aligned_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                             const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                             int mode, const uint8_t *query, uint64_t qlen, hyo_alignment *out,
                             uint8_t *ops, int threads);
/* align_pair_position_max's scalar path (src/kernel.rs:526-553): out[0 .. n) column maxima;
 * returns the best score, *target_end its first position (-1 when 0). */
int32_t hyo_position_max(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n, const int32_t *matrix,
                         uint64_t al, int32_t gap_open, int32_t gap_ext, int32_t *out, int64_t *target_end);
/* hyo_position_max over many pairs on `threads` threads: pair k's maxima at out + t_off[k] - t_off[0]. */
void hyo_position_max_mt(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                         const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix, uint64_t al,
                         int32_t gap_open, int32_t gap_ext, int32_t *out, int32_t *scores, int threads);
/* score2 (src/kernel.rs:741-792). */
int hyo_score2(const int32_t *colmax, uint64_t n, int32_t best_score, uint64_t best_target_end,
               int32_t matrix_max, int32_t min_score, int32_t *score, uint64_t *pos);
/* traceback's budget rule (src/align.rs:192-222): 0 if traceable in max_bytes, else needed. */
uint64_t hyo_traceback_needed(uint64_t m, uint64_t n, uint64_t max_bytes);
/* traceback_min_bytes_for_database (src/align.rs:228-250). */
uint64_t hyo_traceback_min_bytes_for_database(uint64_t max_m, uint64_t max_n);

#ifdef __cplusplus
}
#endif
#endif
