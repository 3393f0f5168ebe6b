/*
 * hyoracle.c -- TEST INFRASTRUCTURE ONLY (see hyoracle.h).
 *
 * Plain-C restatement of hyalite's scalar reference kernel and of its database/pairwise result
 * semantics. Arithmetic is carried in int64 so no intermediate can overflow; for every input the
 * reference's width proof accepts, the reference's i32 arithmetic never wraps either, so the two
 * compute identical values.
 */
#include "hyoracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* Status codes: must equal the HY_* values of include/hyalite_cuda.h. */
enum {
    ST_OK = 0,
    ST_EMPTY_ALPHABET = 1,
    ST_MATRIX_SHAPE = 2,
    ST_NEGATIVE_GAP_PENALTY = 3,
    ST_GAP_OPEN_LESS_THAN_EXTEND = 4,
    ST_SCORE_RANGE_TOO_WIDE = 5,
    ST_SYMBOL_OUT_OF_RANGE = 6,
    ST_TRACEBACK_BUDGET_EXCEEDED = 11,
};

/* kernel::NEG = i32::MIN / 4 (src/kernel.rs:39). */
#define ORC_NEG ((int64_t)(INT32_MIN / 4))

/* Flags::for_mode (src/kernel.rs:43-98). */
typedef struct {
    int top_row_free, left_col_free, answer_last_row, answer_last_col, local;
} flags_t;

static flags_t flags_for_mode(int mode) {
    flags_t f = {0, 0, 0, 0, 0};
    switch (mode) {
    case 0: /* SW */ f.top_row_free = 1; f.left_col_free = 1; f.local = 1; break;
    case 1: /* NW */ break;
    case 2: /* HW */ f.top_row_free = 1; f.answer_last_row = 1; break;
    case 3: /* OV */
        f.top_row_free = 1; f.left_col_free = 1; f.answer_last_row = 1; f.answer_last_col = 1;
        break;
    default: /* SHW */ f.left_col_free = 1; f.answer_last_col = 1; break;
    }
    return f;
}

/* gap_penalty (src/kernel.rs:103-109): computed in i64, cast to i32 like the reference. */
static int64_t gap_penalty(int32_t go, int32_t ge, uint64_t len) {
    if (len == 0) return 0;
    int64_t v = (int64_t)go + ((int64_t)len - 1) * (int64_t)ge;
    return (int64_t)(int32_t)v;
}

/* Best::consider (src/kernel.rs:113-129): maximise score, then minimise (grid_col, grid_row). */
typedef struct {
    int64_t score;
    uint64_t row, col;
} best_t;

static inline void consider(best_t *b, int64_t s, uint64_t row, uint64_t col) {
    if (s > b->score || (s == b->score && (col < b->col || (col == b->col && row < b->row)))) {
        b->score = s;
        b->row = row;
        b->col = col;
    }
}

int hyo_scoring_validate(uint64_t alphabet_len, const int32_t *matrix, uint64_t matrix_len,
                         int32_t gap_open, int32_t gap_ext, int64_t *d1, int64_t *d2, int64_t *d3) {
    (void)matrix;
    if (alphabet_len == 0) return ST_EMPTY_ALPHABET;
    unsigned __int128 sq = (unsigned __int128)alphabet_len * alphabet_len;
    if (sq != matrix_len) {
        if (d1) *d1 = (int64_t)alphabet_len;
        if (d2) *d2 = sq > (unsigned __int128)INT64_MAX ? INT64_MAX : (int64_t)sq;
        if (d3) *d3 = (int64_t)matrix_len;
        return ST_MATRIX_SHAPE;
    }
    if (gap_open < 0 || gap_ext < 0) {
        if (d1) *d1 = gap_open;
        if (d2) *d2 = gap_ext;
        return ST_NEGATIVE_GAP_PENALTY;
    }
    if (gap_open < gap_ext) {
        if (d1) *d1 = gap_open;
        if (d2) *d2 = gap_ext;
        return ST_GAP_OPEN_LESS_THAN_EXTEND;
    }
    return ST_OK;
}

/* magnitude_bound (src/width.rs:107-137), in 128-bit so products cannot wrap, then the i64 clamp
 * of required_width (src/width.rs:157). */
int64_t hyo_magnitude_bound(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                            int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len) {
    __int128 m = (__int128)max_query_len;
    __int128 n = (__int128)max_target_len;
    __int128 min_ij = m < n ? m : n;
    __int128 max_pos = max_entry > 0 ? (__int128)max_entry : 0;
    __int128 max_neg = -(__int128)min_entry > 0 ? -(__int128)min_entry : 0;
    __int128 go = gap_open, ge = gap_ext;
    __int128 positive = min_ij * max_pos;
    __int128 negative;
    if (mode == 0) {
        negative = go;
    } else if (mode == 3) {
        negative = min_ij * max_neg + go;
    } else {
        __int128 run = m + n - 1;
        if (run < 0) run = 0;
        negative = (m + n) * max_neg + go + run * ge;
    }
    __int128 bound = positive > negative ? positive : negative;
    if (bound > (__int128)INT64_MAX) bound = INT64_MAX;
    return (int64_t)bound;
}

/* required_width + ScoreWidth::narrowest_for/max_abs (src/width.rs:49-71, 145-169). */
int hyo_required_width(int mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                       int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len,
                       int64_t *bound_out) {
    int64_t b = hyo_magnitude_bound(mode, min_entry, max_entry, gap_open, gap_ext, max_query_len,
                                    max_target_len);
    if (bound_out) *bound_out = b;
    if (b <= 127) return 0;
    if (b <= 32767) return 1;
    if (b <= 536870911) return 2;
    return -1;
}

/* fill_dp + reduce_answer (src/kernel.rs:168-260), restated with rolling rows: the same cells are
 * computed in the same order with the same arithmetic, and the answer region and tie-break of
 * reduce_answer are applied to them (the tie-break is an explicit comparison, so visiting order
 * does not matter). */
void hyo_align_core(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                    const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                    int mode, int32_t *score, int64_t *query_end, int64_t *target_end) {
    flags_t fl = flags_for_mode(mode);
    const int64_t go = gap_open, ge = gap_ext;
    uint64_t cols = n + 1;
    int64_t *prev = (int64_t *)malloc(sizeof(int64_t) * cols);
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * cols);
    int64_t *f = (int64_t *)malloc(sizeof(int64_t) * cols);
    int64_t *lastcol = (int64_t *)malloc(sizeof(int64_t) * (m + 1));
    best_t best = {ORC_NEG, 0, 0};

    for (uint64_t j = 0; j <= n; ++j) {
        prev[j] = (j == 0 || fl.top_row_free) ? 0 : -gap_penalty(gap_open, gap_ext, j);
        f[j] = ORC_NEG;
    }
    if (fl.local)
        for (uint64_t j = 0; j <= n; ++j) consider(&best, prev[j], 0, j);
    lastcol[0] = prev[n];

    for (uint64_t i = 1; i <= m; ++i) {
        cur[0] = fl.left_col_free ? 0 : -gap_penalty(gap_open, gap_ext, i);
        int64_t e = ORC_NEG;
        const int32_t *qrow = matrix + (uint64_t)q[i - 1] * al;
        for (uint64_t j = 1; j <= n; ++j) {
            int64_t a = cur[j - 1] - go, b = e - ge;
            e = a > b ? a : b;
            int64_t c = prev[j] - go, d = f[j] - ge;
            f[j] = c > d ? c : d;
            int64_t diag = prev[j - 1] + (int64_t)qrow[t[j - 1]];
            int64_t cell = diag > e ? diag : e;
            if (f[j] > cell) cell = f[j];
            if (fl.local && cell < 0) cell = 0;
            cur[j] = cell;
        }
        if (fl.local)
            for (uint64_t j = 0; j <= n; ++j) consider(&best, cur[j], i, j);
        lastcol[i] = cur[n];
        int64_t *tmp = prev;
        prev = cur;
        cur = tmp;
    }
    /* prev holds row m. */
    if (!fl.local) {
        consider(&best, prev[n], m, n);
        if (fl.answer_last_row)
            for (uint64_t j = 0; j <= n; ++j) consider(&best, prev[j], m, j);
        if (fl.answer_last_col)
            for (uint64_t i = 0; i <= m; ++i) consider(&best, lastcol[i], i, n);
    }
    *score = (int32_t)best.score;
    *query_end = best.row == 0 ? -1 : (int64_t)best.row - 1;
    *target_end = best.col == 0 ? -1 : (int64_t)best.col - 1;
    free(prev);
    free(cur);
    free(f);
    free(lastcol);
}

/* Database::scan: highest score, smallest db_index on a tie (src/database.rs:117-130, 173-180);
 * ScoreEnd ends come from one scalar re-alignment of the winner (186-197), Score drops them. */
void hyo_scan(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
              const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
              int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out) {
    int64_t best_score = INT32_MIN;
    uint64_t best_index = 0;
    int64_t bq = -1, bt = -1;
    for (uint64_t k = 0; k < n_seqs; ++k) {
        int32_t s;
        int64_t qe, te;
        hyo_align_core(query, qlen, residues + offsets[k], offsets[k + 1] - offsets[k], matrix,
                       al, gap_open, gap_ext, mode, &s, &qe, &te);
        if (s > best_score) {
            best_score = s;
            best_index = k;
            bq = qe;
            bt = te;
        }
    }
    out->score = (int32_t)best_score;
    out->db_index = best_index;
    out->query_end = search_type == 1 ? bq : -1;
    out->target_end = search_type == 1 ? bt : -1;
}

static void scan_all_range(const uint8_t *residues, const uint64_t *offsets, uint64_t lo,
                           uint64_t hi, const int32_t *matrix, uint64_t al, int32_t go,
                           int32_t ge, int mode, int search_type, const uint8_t *query,
                           uint64_t qlen, hyo_hit *out) {
    for (uint64_t k = lo; k < hi; ++k) {
        int32_t s;
        int64_t qe, te;
        hyo_align_core(query, qlen, residues + offsets[k], offsets[k + 1] - offsets[k], matrix,
                       al, go, ge, mode, &s, &qe, &te);
        out[k].score = s;
        out[k].db_index = k;
        out[k].query_end = search_type == 1 ? qe : -1;
        out[k].target_end = search_type == 1 ? te : -1;
    }
}

/* Database::scan_all (src/database.rs:347-464): one hit per sequence in db order; ScoreEnd ends
 * equal the scalar oracle's (end = grid - 1, None at grid 0: 395-402). */
void hyo_scan_all(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                  const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
                  int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out) {
    scan_all_range(residues, offsets, 0, n_seqs, matrix, al, gap_open, gap_ext, mode, search_type,
                   query, qlen, out);
}

/* Database::scan_scores (src/database.rs:481-515): every sequence's best score in db order. */
void hyo_scan_scores(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                     const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                     int mode, const uint8_t *query, uint64_t qlen, int32_t *out) {
    for (uint64_t k = 0; k < n_seqs; ++k) {
        int64_t qe, te;
        hyo_align_core(query, qlen, residues + offsets[k], offsets[k + 1] - offsets[k], matrix,
                       al, gap_open, gap_ext, mode, &out[k], &qe, &te);
    }
}

void hyo_scan_scores_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                        const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                        int mode, const uint8_t *query, uint64_t qlen, int32_t *out, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int64_t k = 0; k < (int64_t)n_seqs; ++k) {
        int64_t qe, te;
        hyo_align_core(query, qlen, residues + offsets[k], offsets[k + 1] - offsets[k], matrix,
                       al, gap_open, gap_ext, mode, &out[k], &qe, &te);
    }
}

void hyo_scan_all_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                     const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                     int mode, int search_type, const uint8_t *query, uint64_t qlen, hyo_hit *out,
                     int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int64_t k = 0; k < (int64_t)n_seqs; ++k)
        scan_all_range(residues, offsets, (uint64_t)k, (uint64_t)k + 1, matrix, al, gap_open,
                       gap_ext, mode, search_type, query, qlen, out);
}

/* align_pairs (src/kernel.rs:429-452) -> align_pair_with (354-415): per pair, symbols are checked
 * query-then-target (362-370), then the width proof on the pair's exact lengths (373); the first
 * failing pair's error is returned and the hits of the pairs before it stay written. The striped
 * Score fast path (378-397) is bit-identical to align_core, so align_core stands for both. */
int hyo_align_pairs(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                    const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix, uint64_t al,
                    int32_t gap_open, int32_t gap_ext, int mode, int search_type, hyo_hit *out,
                    int threads, int64_t *d1, int64_t *d2) {
    int32_t min_e = INT32_MAX, max_e = INT32_MIN;
    for (uint64_t i = 0; i < al * al; ++i) {
        if (matrix[i] < min_e) min_e = matrix[i];
        if (matrix[i] > max_e) max_e = matrix[i];
    }
    uint64_t n_ok = n_pairs;
    int status = ST_OK;
    for (uint64_t p = 0; p < n_pairs && status == ST_OK; ++p) {
        const uint8_t *seqs[2] = {q_res + q_off[p], t_res + t_off[p]};
        uint64_t lens[2] = {q_off[p + 1] - q_off[p], t_off[p + 1] - t_off[p]};
        for (int s = 0; s < 2 && status == ST_OK; ++s)
            for (uint64_t i = 0; i < lens[s]; ++i)
                if (seqs[s][i] >= al) {
                    status = ST_SYMBOL_OUT_OF_RANGE;
                    if (d1) *d1 = seqs[s][i];
                    if (d2) *d2 = (int64_t)al;
                    break;
                }
        if (status == ST_OK) {
            int64_t bound;
            if (hyo_required_width(mode, min_e, max_e, gap_open, gap_ext, lens[0], lens[1],
                                   &bound) < 0) {
                status = ST_SCORE_RANGE_TOO_WIDE;
                if (d1) *d1 = bound;
            }
        }
        if (status != ST_OK) n_ok = p;
    }
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t p = 0; p < (int64_t)n_ok; ++p) {
        int32_t s;
        int64_t qe, te;
        hyo_align_core(q_res + q_off[p], q_off[p + 1] - q_off[p], t_res + t_off[p],
                       t_off[p + 1] - t_off[p], matrix, al, gap_open, gap_ext, mode, &s, &qe, &te);
        out[p].score = s;
        out[p].db_index = (uint64_t)p;
        out[p].query_end = search_type == 1 ? qe : -1;
        out[p].target_end = search_type == 1 ? te : -1;
    }
    return status;
}

/* ---- brute force (tests/common/mod.rs:65-171) ------------------------------------------- */

typedef struct {
    const uint8_t *q, *t;
    uint64_t m, n;
    const int32_t *mat;
    uint64_t al;
    int32_t go, ge;
} prob_t;

static int32_t sat_add(int32_t a, int32_t b) {
    int64_t s = (int64_t)a + b;
    if (s > INT32_MAX) return INT32_MAX;
    if (s < INT32_MIN) return INT32_MIN;
    return (int32_t)s;
}

/* brute_nw's recursion: every path, affine gaps charged from maximal same-direction runs.
 * last: 0 start/diagonal, 1 right (gap in query), 2 down (gap in target). */
static int32_t brute_rec(const prob_t *p, uint64_t i, uint64_t j, int last) {
    if (i == p->m && j == p->n) return 0;
    int32_t best = INT32_MIN;
    if (i < p->m && j < p->n) {
        int32_t s = p->mat[(uint64_t)p->q[i] * p->al + p->t[j]];
        int32_t v = sat_add(s, brute_rec(p, i + 1, j + 1, 0));
        if (v > best) best = v;
    }
    if (j < p->n) {
        int32_t cost = last == 1 ? p->ge : p->go;
        int32_t v = sat_add(-cost, brute_rec(p, i, j + 1, 1));
        if (v > best) best = v;
    }
    if (i < p->m) {
        int32_t cost = last == 2 ? p->ge : p->go;
        int32_t v = sat_add(-cost, brute_rec(p, i + 1, j, 2));
        if (v > best) best = v;
    }
    return best;
}

static int32_t brute_nw(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                        const int32_t *mat, uint64_t al, int32_t go, int32_t ge) {
    prob_t p = {q, t, m, n, mat, al, go, ge};
    return brute_rec(&p, 0, 0, 0);
}

int32_t hyo_brute(int mode, const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                  const int32_t *mat, uint64_t al, int32_t go, int32_t ge) {
    int32_t best;
    switch (mode) {
    case 1: /* NW */
        return brute_nw(q, m, t, n, mat, al, go, ge);
    case 0: /* SW: best over every substring pair, floored at 0 */
        best = 0;
        for (uint64_t a = 0; a <= m; ++a)
            for (uint64_t b = a; b <= m; ++b)
                for (uint64_t c = 0; c <= n; ++c)
                    for (uint64_t d = c; d <= n; ++d) {
                        int32_t v = brute_nw(q + a, b - a, t + c, d - c, mat, al, go, ge);
                        if (v > best) best = v;
                    }
        return best;
    case 2: /* HW: whole query against the best target window */
        best = INT32_MIN;
        for (uint64_t c = 0; c <= n; ++c)
            for (uint64_t d = c; d <= n; ++d) {
                int32_t v = brute_nw(q, m, t + c, d - c, mat, al, go, ge);
                if (v > best) best = v;
            }
        return best;
    case 3: /* OV: substring pairs touching a border at both ends, floored at 0 */
        best = 0;
        for (uint64_t a = 0; a <= m; ++a)
            for (uint64_t b = a; b <= m; ++b)
                for (uint64_t c = 0; c <= n; ++c)
                    for (uint64_t d = c; d <= n; ++d)
                        if ((a == 0 || c == 0) && (b == m || d == n)) {
                            int32_t v = brute_nw(q + a, b - a, t + c, d - c, mat, al, go, ge);
                            if (v > best) best = v;
                        }
        return best;
    default: /* SHW: whole target against the best query window */
        best = INT32_MIN;
        for (uint64_t a = 0; a <= m; ++a)
            for (uint64_t b = a; b <= m; ++b) {
                int32_t v = brute_nw(q + a, b - a, t, n, mat, al, go, ge);
                if (v > best) best = v;
            }
        return best;
    }
}

/* ---- traceback (src/align.rs) --------------------------------------------------------------- */

/* full_matrix_bytes (src/align.rs:252-258): three i32 matrices of (m+1)(n+1) cells, saturating. */
static uint64_t sat_mul(uint64_t a, uint64_t b) {
    unsigned __int128 p = (unsigned __int128)a * b;
    return p > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (uint64_t)p;
}
static uint64_t full_matrix_bytes(uint64_t m, uint64_t n) {
    return sat_mul(sat_mul(sat_mul(m + 1, n + 1), 3), 4);
}
/* checkpoint_bytes (src/align.rs:261-268). */
static uint64_t checkpoint_bytes(uint64_t m, uint64_t n, uint64_t k) {
    uint64_t num_ckpt = m / k + 1, strip_rows = k + 1;
    return sat_mul(sat_mul(2 * num_ckpt + 3 * strip_rows, n + 1), 4);
}
/* u64::isqrt, then .max(1) (src/align.rs:210, 236). */
static uint64_t strip_height(uint64_t m) {
    uint64_t r = 0;
    for (uint64_t bit = (uint64_t)1 << 62; bit; bit >>= 2) {
        if (m >= r + bit) {
            m -= r + bit;
            r = (r >> 1) + bit;
        } else {
            r >>= 1;
        }
    }
    return r ? r : 1;
}

/* traceback's budget rule (src/align.rs:192-222): 0 when the problem is traceable in max_bytes,
 * else the bytes it needs (the checkpoint peak). */
uint64_t hyo_traceback_needed(uint64_t m, uint64_t n, uint64_t max_bytes) {
    if (full_matrix_bytes(m, n) <= max_bytes || m == 0 || n == 0) return 0;
    uint64_t peak = checkpoint_bytes(m, n, strip_height(m));
    return peak > max_bytes ? peak : 0;
}

/* traceback_min_bytes (src/align.rs:228-236) and traceback_min_bytes_for_database (245-250). */
static uint64_t traceback_min_bytes(uint64_t m, uint64_t n) {
    uint64_t full = full_matrix_bytes(m, n);
    if (m == 0 || n == 0) return full;
    uint64_t cp = checkpoint_bytes(m, n, strip_height(m));
    return full < cp ? full : cp;
}
uint64_t hyo_traceback_min_bytes_for_database(uint64_t max_m, uint64_t max_n) {
    uint64_t v = traceback_min_bytes(max_m, max_n);
    uint64_t a = full_matrix_bytes(max_m, 0), b = full_matrix_bytes(0, max_n);
    if (a > v) v = a;
    if (b > v) v = b;
    return v;
}

/* traceback_full (src/align.rs:487-545) with fill_row (446-483), consider_row (309-327) and the
 * shared walk (345-420): full H/E/F matrices (int64 here; every value the reference's i32
 * arithmetic produces for an input its width proof accepts is the same), the end cell by
 * Best::consider, then the backward walk with the reference's tie-break and stop rules, reading
 * the three matrices' values (not a direction encoding). ops receives codes 0 Match, 1 Mismatch,
 * 2 Ins, 3 Del (AlignOp, src/align.rs:47-56) in forward order; room for m + n codes. */
void hyo_traceback(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n,
                   const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext, int mode,
                   hyo_alignment *out, uint8_t *ops) {
    flags_t fl = flags_for_mode(mode);
    const int64_t go = gap_open, ge = gap_ext;
    const uint64_t cols = n + 1, cells = (m + 1) * cols;
    int64_t *h = (int64_t *)malloc(sizeof(int64_t) * cells);
    int64_t *e = (int64_t *)malloc(sizeof(int64_t) * cells);
    int64_t *f = (int64_t *)malloc(sizeof(int64_t) * cells);
    for (uint64_t c = 0; c < cells; ++c) {
        h[c] = 0;
        e[c] = ORC_NEG;
        f[c] = ORC_NEG;
    }
    for (uint64_t j = 1; j <= n; ++j) {
        h[j] = fl.top_row_free ? 0 : -gap_penalty(gap_open, gap_ext, j);
        e[j] = fl.top_row_free ? ORC_NEG : h[j];
    }
    for (uint64_t i = 1; i <= m; ++i) {
        const uint64_t b = i * cols, pb = (i - 1) * cols;
        h[b] = fl.left_col_free ? 0 : -gap_penalty(gap_open, gap_ext, i);
        e[b] = ORC_NEG;
        f[b] = fl.left_col_free ? ORC_NEG : h[b];
        for (uint64_t j = 1; j <= n; ++j) {
            int64_t x = h[b + j - 1] - go, y = e[b + j - 1] - ge;
            e[b + j] = x > y ? x : y;
            x = h[pb + j] - go;
            y = f[pb + j] - ge;
            f[b + j] = x > y ? x : y;
            int64_t cell = h[pb + j - 1] + matrix[(uint64_t)q[i - 1] * al + t[j - 1]];
            if (e[b + j] > cell) cell = e[b + j];
            if (f[b + j] > cell) cell = f[b + j];
            if (fl.local && cell < 0) cell = 0;
            h[b + j] = cell;
        }
    }
    best_t best = {ORC_NEG, 0, 0};
    for (uint64_t i = 0; i <= m; ++i) {
        const int64_t *row = h + i * cols;
        if (fl.local) {
            for (uint64_t j = 0; j <= n; ++j) consider(&best, row[j], i, j);
        } else {
            if (fl.answer_last_col) consider(&best, row[n], i, n);
            if (i == m) {
                consider(&best, row[n], m, n);
                if (fl.answer_last_row)
                    for (uint64_t j = 0; j <= n; ++j) consider(&best, row[j], m, j);
            }
        }
    }
    /* walk: state 0 H, 1 E, 2 F. */
    uint64_t i = best.row, j = best.col, k = 0;
    int state = 0;
    uint8_t *rev = (uint8_t *)malloc(m + n + 1);
    for (;;) {
        if (state == 0) {
            const int64_t hij = h[i * cols + j];
            if (fl.local && hij == 0) break;
            if (i == 0 && j == 0) break;
            if (i == 0) {
                if (fl.top_row_free) break;
                state = 1;
                continue;
            }
            if (j == 0) {
                if (fl.left_col_free) break;
                state = 2;
                continue;
            }
            const int64_t sub = matrix[(uint64_t)q[i - 1] * al + t[j - 1]];
            if (hij == h[(i - 1) * cols + j - 1] + sub) {
                rev[k++] = q[i - 1] == t[j - 1] ? 0 : 1;
                --i;
                --j;
            } else if (hij == e[i * cols + j]) {
                state = 1;
            } else {
                state = 2;
            }
        } else if (state == 1) {
            rev[k++] = 3;
            const int64_t ev = e[i * cols + j];
            --j;
            if (ev == h[i * cols + j] - go) state = 0;
        } else {
            rev[k++] = 2;
            const int64_t fv = f[i * cols + j];
            --i;
            if (fv == h[i * cols + j] - go) state = 0;
        }
    }
    for (uint64_t x = 0; x < k; ++x) ops[x] = rev[k - 1 - x];
    out->score = (int32_t)best.score;
    out->query_start = i;
    out->query_end = best.row;
    out->target_start = j;
    out->target_end = best.col;
    out->n_ops = k;
    free(rev);
    free(h);
    free(e);
    free(f);
}

/* align (src/align.rs:169-186) then traceback's budget rule (192-222). */
int hyo_align(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n, const int32_t *matrix,
              uint64_t al, int32_t gap_open, int32_t gap_ext, int mode, uint64_t max_bytes,
              hyo_alignment *out, uint8_t *ops, int64_t *d1, int64_t *d2) {
    for (uint64_t x = 0; x < m + n; ++x) {
        const uint8_t s = x < m ? q[x] : t[x - m];
        if (s >= al) {
            if (d1) *d1 = s;
            if (d2) *d2 = (int64_t)al;
            return ST_SYMBOL_OUT_OF_RANGE;
        }
    }
    int32_t mn = matrix[0], mx = matrix[0];
    for (uint64_t x = 1; x < al * al; ++x) {
        if (matrix[x] < mn) mn = matrix[x];
        if (matrix[x] > mx) mx = matrix[x];
    }
    int64_t bound;
    if (hyo_required_width(mode, mn, mx, gap_open, gap_ext, m, n, &bound) < 0) {
        if (d1) *d1 = bound;
        return ST_SCORE_RANGE_TOO_WIDE;
    }
    uint64_t need = hyo_traceback_needed(m, n, max_bytes);
    if (need) {
        if (d1) *d1 = (int64_t)need;
        if (d2) *d2 = (int64_t)max_bytes;
        return ST_TRACEBACK_BUDGET_EXCEEDED;
    }
    hyo_traceback(q, m, t, n, matrix, al, gap_open, gap_ext, mode, out, ops);
    return ST_OK;
}

/* Database::scan_all_aligned (src/database.rs:538-549): hyo_traceback of the query against every
 * sequence, spread over `threads` OpenMP threads. Alignment k's operations go to the slot at
 * ops + k * qlen + (offsets[k] - offsets[0]) (room for qlen + |t_k| codes). */
void hyo_scan_all_aligned_mt(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                             const int32_t *matrix, uint64_t al, int32_t gap_open, int32_t gap_ext,
                             int mode, const uint8_t *query, uint64_t qlen, hyo_alignment *out,
                             uint8_t *ops, int threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
#endif
    for (int64_t k = 0; k < (int64_t)n_seqs; ++k) {
        const uint64_t a = offsets[k], b = offsets[k + 1];
        hyo_traceback(query, qlen, residues + a, b - a, matrix, al, gap_open, gap_ext, mode, &out[k],
                      ops + (uint64_t)k * qlen + (a - offsets[0]));
    }
    (void)threads;
}

/* align_pair_position_max's scalar path (src/kernel.rs:526-553): the full SW matrix's column
 * maxima (floor 0), then score = their maximum, target_end = its first position (-1 when 0). */
int32_t hyo_position_max(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t n, const int32_t *matrix,
                         uint64_t al, int32_t gap_open, int32_t gap_ext, int32_t *out, int64_t *target_end) {
    const int64_t go = gap_open, ge = gap_ext;
    int64_t *prev = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    int64_t *f = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    for (uint64_t j = 0; j <= n; ++j) {
        prev[j] = 0;
        f[j] = ORC_NEG;
    }
    for (uint64_t j = 0; j < n; ++j) out[j] = 0;
    for (uint64_t i = 1; i <= m; ++i) {
        cur[0] = 0;
        int64_t e = ORC_NEG;
        for (uint64_t j = 1; j <= n; ++j) {
            int64_t a = cur[j - 1] - go, b = e - ge;
            e = a > b ? a : b;
            a = prev[j] - go;
            b = f[j] - ge;
            f[j] = a > b ? a : b;
            int64_t c = prev[j - 1] + matrix[(uint64_t)q[i - 1] * al + t[j - 1]];
            if (e > c) c = e;
            if (f[j] > c) c = f[j];
            if (c < 0) c = 0;
            cur[j] = c;
            if (c > out[j - 1]) out[j - 1] = (int32_t)c;
        }
        int64_t *tmp = prev;
        prev = cur;
        cur = tmp;
    }
    int32_t best = 0;
    int64_t te = -1;
    for (uint64_t j = 0; j < n; ++j)
        if (out[j] > best) {
            best = out[j];
            te = (int64_t)j;
        }
    *target_end = te;
    free(prev);
    free(cur);
    free(f);
    return best;
}

/* score2 (src/kernel.rs:741-792): 1 and the peak when one qualifies, else 0. */
int hyo_score2(const int32_t *colmax, uint64_t n, int32_t best_score, uint64_t best_target_end,
               int32_t matrix_max, int32_t min_score, int32_t *score, uint64_t *pos) {
    if (matrix_max <= 0) return 0;
    int64_t w = ((int64_t)(best_score > 0 ? best_score : 0) + matrix_max - 1) / matrix_max;
    if (w < 0) w = 0;
    const int64_t low = (int64_t)best_target_end - w, high = (int64_t)best_target_end + w;
    int have = 0, open = 0;
    int32_t bs = 0, cs = 0;
    uint64_t bp = 0, cp = 0;
    for (uint64_t i = 0; i <= n; ++i) {
        const int finish = i == n;
        if (!finish) {
            const int32_t v = colmax[i];
            if (v < min_score) continue;
            if (open && cp + 1 == i) {
                if (cs < v) {
                    cs = v;
                    cp = i;
                }
                continue;
            }
        }
        if (open) {
            const int64_t p = (int64_t)cp;
            if ((p < low || p > high) && (!have || cs > bs)) {
                have = 1;
                bs = cs;
                bp = cp;
            }
        }
        if (!finish) {
            open = 1;
            cs = colmax[i];
            cp = i;
        }
    }
    if (have) {
        *score = bs;
        *pos = bp;
    }
    return have;
}

/* hyo_position_max over many pairs on `threads` OpenMP threads (the CPU baseline of the
 * mate-rescue workload): pair k's column maxima go to out + (t_off[k] - t_off[0]). */
void hyo_position_max_mt(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                         const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix, uint64_t al,
                         int32_t gap_open, int32_t gap_ext, int32_t *out, int32_t *scores, int threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
#endif
    for (int64_t k = 0; k < (int64_t)n_pairs; ++k) {
        int64_t te;
        scores[k] = hyo_position_max(q_res + q_off[k], q_off[k + 1] - q_off[k], t_res + t_off[k],
                                     t_off[k + 1] - t_off[k], matrix, al, gap_open, gap_ext,
                                     out + (t_off[k] - t_off[0]), &te);
    }
    (void)threads;
}
