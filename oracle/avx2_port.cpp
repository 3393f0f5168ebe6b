// avx2_port.cpp -- TEST/BENCH INFRASTRUCTURE ONLY.
//
// A C++ restatement of hyalite's AVX2 inter-sequence backend, the CPU baseline bench.py times
// beside the CUDA backend (the reference is Rust and cannot be built here). It follows:
//   - packing: PackedDb::build, db-order chunks of LANES, per-batch width w (src/inter.rs:431-509)
//   - kernel:  scan_batch (src/inter.rs:683-831), score only
//   - lanes:   Avx2 i8x32 / Avx2I16 i16x16 / Avx2I32 i32x8 (src/inter.rs:1986-2627): saturating
//              adds/subs at i8/i16, wrapping add/sub at i32 with NEG = i32::MIN/4
//   - per-sequence width groups: build_width_groups (src/database.rs:884-948) and the grouped
//              single-best reduction + scalar re-alignment of the winner (160-208)
// Layout Precomputed is forced for every width (the reference's Auto layout rejects these
// databases and would fall back to scalar, src/inter.rs:299-315); Gathered is offered for
// i8 with alphabet <= 16. Nothing in the shipped library uses this file.
#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
#include "hyoracle.h"
}

namespace {

struct Flags {
    bool top_row_free, left_col_free, answer_last_row, answer_last_col, local;
};

Flags flags_for_mode(int mode) {
    switch (mode) {
    case 0: return {true, true, false, false, true};
    case 1: return {false, false, false, false, false};
    case 2: return {true, false, true, false, false};
    case 3: return {true, true, true, true, false};
    default: return {false, true, false, true, false};
    }
}

int32_t gap_penalty(int32_t go, int32_t ge, size_t len) {
    if (len == 0) return 0;
    return (int32_t)((int64_t)go + ((int64_t)len - 1) * (int64_t)ge);
}

// ---- lane backends ---------------------------------------------------------------------------

struct L8 {
    typedef int8_t E;
    static const int LANES = 32;
    static const E NEG = INT8_MIN;
    static E sat(int32_t v) { return (E)std::min(127, std::max(-128, v)); }
    static __m256i splat(E v) { return _mm256_set1_epi8(v); }
    static __m256i add(__m256i a, __m256i b) { return _mm256_adds_epi8(a, b); }
    static __m256i sub(__m256i a, __m256i b) { return _mm256_subs_epi8(a, b); }
    static __m256i max(__m256i a, __m256i b) { return _mm256_max_epi8(a, b); }
};
struct L16 {
    typedef int16_t E;
    static const int LANES = 16;
    static const E NEG = INT16_MIN;
    static E sat(int32_t v) { return (E)std::min(32767, std::max(-32768, v)); }
    static __m256i splat(E v) { return _mm256_set1_epi16(v); }
    static __m256i add(__m256i a, __m256i b) { return _mm256_adds_epi16(a, b); }
    static __m256i sub(__m256i a, __m256i b) { return _mm256_subs_epi16(a, b); }
    static __m256i max(__m256i a, __m256i b) { return _mm256_max_epi16(a, b); }
};
struct L32 {
    typedef int32_t E;
    static const int LANES = 8;
    static const E NEG = INT32_MIN / 4;
    static E sat(int32_t v) { return v; }
    static __m256i splat(E v) { return _mm256_set1_epi32(v); }
    static __m256i add(__m256i a, __m256i b) { return _mm256_add_epi32(a, b); }
    static __m256i sub(__m256i a, __m256i b) { return _mm256_sub_epi32(a, b); }
    static __m256i max(__m256i a, __m256i b) { return _mm256_max_epi32(a, b); }
};

static inline __m256i sel(__m256i mask, __m256i a, __m256i b) { return _mm256_blendv_epi8(b, a, mask); }
static inline __m256i ld(const void *p) { return _mm256_loadu_si256((const __m256i *)p); }
static inline void st(void *p, __m256i v) { _mm256_storeu_si256((__m256i *)p, v); }

// ---- packing ------------------------------------------------------------------------------

template <class L>
struct Batch {
    size_t real = 0, w = 0;
    std::vector<typename L::E> mask_le, mask_eq, table;  // Precomputed table
    std::vector<uint8_t> residues;                        // Gathered
};

template <class L>
struct PackedDb {
    bool gathered = false;
    size_t al = 0;
    std::vector<typename L::E> letter_profile;  // Gathered only, al*al
    std::vector<Batch<L>> batches;
    std::vector<uint64_t> indices;              // global db index of each packed sequence

    void build(const std::vector<const uint8_t *> &seqs, const std::vector<size_t> &lens,
               const int32_t *matrix, size_t al_, bool gathered_) {
        typedef typename L::E E;
        const int lanes = L::LANES;
        al = al_;
        gathered = gathered_;
        for (size_t start = 0; start < seqs.size(); start += lanes) {
            Batch<L> b;
            b.real = std::min((size_t)lanes, seqs.size() - start);
            for (size_t k = 0; k < b.real; ++k) b.w = std::max(b.w, lens[start + k]);
            std::vector<size_t> len(lanes, 0);
            std::vector<uint8_t> res(b.w * lanes, 0);
            for (size_t k = 0; k < b.real; ++k) {
                len[k] = lens[start + k];
                for (size_t j0 = 0; j0 < len[k]; ++j0) res[j0 * lanes + k] = seqs[start + k][j0];
            }
            b.mask_le.assign((b.w + 1) * lanes, 0);
            b.mask_eq.assign((b.w + 1) * lanes, 0);
            for (size_t j = 0; j <= b.w; ++j)
                for (int k = 0; k < lanes; ++k) {
                    b.mask_le[j * lanes + k] = j <= len[k] ? (E)-1 : (E)0;
                    b.mask_eq[j * lanes + k] = j == len[k] ? (E)-1 : (E)0;
                }
            if (gathered) {
                b.residues = res;
            } else {
                b.table.assign(al * b.w * lanes, 0);
                for (size_t q = 0; q < al; ++q)
                    for (size_t j0 = 0; j0 < b.w; ++j0)
                        for (int k = 0; k < lanes; ++k)
                            b.table[(q * b.w + j0) * lanes + k] =
                                L::sat(matrix[q * al + res[j0 * lanes + k]]);
            }
            batches.push_back(std::move(b));
        }
        if (gathered) {
            letter_profile.assign(al * al, 0);
            for (size_t q = 0; q < al; ++q)
                for (size_t s = 0; s < al; ++s) letter_profile[q * al + s] = L::sat(matrix[q * al + s]);
        }
    }
};

// ---- kernel: scan_batch (src/inter.rs:683-831) ---------------------------------------------

template <class L>
void scan_batch(const uint8_t *query, size_t qlen, const PackedDb<L> &db, const Batch<L> &batch,
                int32_t go, int32_t ge, const Flags &fl, typename L::E *hbuf, typename L::E *f,
                typename L::E *out) {
    typedef typename L::E E;
    const int lanes = L::LANES;
    const size_t w = batch.w;
    const size_t cols = (w + 1) * lanes;
    const __m256i go_v = L::splat(L::sat(go)), ge_v = L::splat(L::sat(ge));
    const __m256i zero = _mm256_setzero_si256(), neg = L::splat(L::NEG);
    E *prev = hbuf, *cur = hbuf + cols;

    for (size_t j = 0; j <= w; ++j) {
        __m256i border = fl.top_row_free ? zero : L::splat(L::sat(-gap_penalty(go, ge, j)));
        st(prev + j * lanes, border);
        st(f + j * lanes, neg);
    }
    __m256i sw_ans = zero, ov_lastcol = zero;
    if (fl.answer_last_col) {
        ov_lastcol = neg;
        for (size_t j = 0; j <= w; ++j)
            ov_lastcol = sel(ld(&batch.mask_eq[j * lanes]), L::max(ov_lastcol, ld(prev + j * lanes)),
                             ov_lastcol);
    }
    __m256i lp_tab = zero;
    for (size_t i = 1; i <= qlen; ++i) {
        __m256i border = fl.left_col_free ? zero : L::splat(L::sat(-gap_penalty(go, ge, i)));
        st(cur, border);
        const size_t qi = query[i - 1];
        if (db.gathered) {
            int8_t padded[16] = {0};
            for (size_t s = 0; s < db.al; ++s) padded[s] = (int8_t)db.letter_profile[qi * db.al + s];
            lp_tab = _mm256_broadcastsi128_si256(_mm_loadu_si128((const __m128i *)padded));
        }
        __m256i e = neg;
        for (size_t j = 1; j <= w; ++j) {
            const size_t col = j * lanes, prevcol = (j - 1) * lanes;
            e = L::max(L::sub(ld(cur + prevcol), go_v), L::sub(e, ge_v));
            __m256i fj = L::max(L::sub(ld(prev + col), go_v), L::sub(ld(f + col), ge_v));
            st(f + col, fj);
            __m256i sub;
            if (db.gathered)
                sub = _mm256_shuffle_epi8(lp_tab, ld(&batch.residues[prevcol]));
            else
                sub = ld(&batch.table[(qi * w + (j - 1)) * lanes]);
            __m256i diag = L::add(ld(prev + prevcol), sub);
            __m256i cell = L::max(diag, L::max(e, fj));
            if (fl.local) {
                cell = L::max(cell, zero);
                sw_ans = sel(ld(&batch.mask_le[col]), L::max(sw_ans, cell), sw_ans);
            }
            if (fl.answer_last_col)
                ov_lastcol = sel(ld(&batch.mask_eq[col]), L::max(ov_lastcol, cell), ov_lastcol);
            st(cur + col, cell);
        }
        std::swap(prev, cur);
    }
    __m256i ans;
    if (fl.local) {
        ans = sw_ans;
    } else if (fl.answer_last_row) {
        __m256i lastrow = ld(prev);
        for (size_t j = 1; j <= w; ++j)
            lastrow = sel(ld(&batch.mask_le[j * lanes]), L::max(lastrow, ld(prev + j * lanes)), lastrow);
        ans = fl.answer_last_col ? L::max(lastrow, ov_lastcol) : lastrow;
    } else if (fl.answer_last_col) {
        ans = ov_lastcol;
    } else {
        __m256i nw = ld(prev);
        for (size_t j = 1; j <= w; ++j) nw = sel(ld(&batch.mask_eq[j * lanes]), ld(prev + j * lanes), nw);
        ans = nw;
    }
    E tmp[32];
    st(tmp, ans);
    memcpy(out, tmp, batch.real * sizeof(E));
}

// ---- a whole database: width groups + scratch ----------------------------------------------

struct Database {
    int mode = 0, search_type = 0;
    int32_t go = 0, ge = 0;
    size_t al = 0, n = 0, max_t = 0;
    std::vector<int32_t> matrix;
    std::vector<uint8_t> residues;
    std::vector<uint64_t> offsets;
    PackedDb<L8> g8;
    PackedDb<L16> g16;
    PackedDb<L32> g32;
};

struct Scratch {
    std::vector<int8_t> h8, f8, s8;
    std::vector<int16_t> h16, f16, s16;
    std::vector<int32_t> h32, f32, s32;
};

template <class L>
void fill_scores(const Database &db, const PackedDb<L> &p, const uint8_t *q, size_t qlen,
                 std::vector<typename L::E> &h, std::vector<typename L::E> &f,
                 std::vector<typename L::E> &scores) {
    const Flags fl = flags_for_mode(db.mode);
    const size_t lanes = L::LANES;
    if (scores.size() < p.indices.size() + lanes) scores.resize(p.indices.size() + lanes);
    for (size_t b = 0; b < p.batches.size(); ++b) {
        const Batch<L> &batch = p.batches[b];
        size_t need = 2 * (batch.w + 1) * lanes;
        if (h.size() < need) h.resize(need);
        if (f.size() < (batch.w + 1) * lanes) f.resize((batch.w + 1) * lanes);
        scan_batch<L>(q, qlen, p, batch, db.go, db.ge, fl, h.data(), f.data(), &scores[b * lanes]);
    }
}

}  // namespace

extern "C" {

// Build a baseline database with per-sequence width groups (all Precomputed unless
// `gathered_i8` and al <= 16, which packs the i8 group Gathered). Returns nullptr on a width-proof
// failure. The caller validated symbols and scoring.
void *hyb_db_create(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                    const int32_t *matrix, uint64_t al, int32_t go, int32_t ge, int mode,
                    int search_type, uint64_t max_query_len, int gathered_i8) {
    Database *db = new Database;
    db->mode = mode;
    db->search_type = search_type;
    db->go = go;
    db->ge = ge;
    db->al = al;
    db->n = n_seqs;
    db->matrix.assign(matrix, matrix + al * al);
    db->residues.assign(residues, residues + offsets[n_seqs]);
    db->offsets.assign(offsets, offsets + n_seqs + 1);
    int32_t mn = *std::min_element(db->matrix.begin(), db->matrix.end());
    int32_t mx = *std::max_element(db->matrix.begin(), db->matrix.end());
    for (uint64_t k = 0; k < n_seqs; ++k) db->max_t = std::max<size_t>(db->max_t, offsets[k + 1] - offsets[k]);
    std::vector<const uint8_t *> seqs[3];
    std::vector<size_t> lens[3];
    std::vector<uint64_t> idx[3];
    for (uint64_t k = 0; k < n_seqs; ++k) {
        size_t len = offsets[k + 1] - offsets[k];
        int w = hyo_required_width(mode, mn, mx, go, ge, max_query_len, len, nullptr);
        if (w < 0) {
            delete db;
            return nullptr;
        }
        seqs[w].push_back(db->residues.data() + offsets[k]);
        lens[w].push_back(len);
        idx[w].push_back(k);
    }
    db->g8.build(seqs[0], lens[0], matrix, al, gathered_i8 && al <= 16);
    db->g8.indices = idx[0];
    db->g16.build(seqs[1], lens[1], matrix, al, false);
    db->g16.indices = idx[1];
    db->g32.build(seqs[2], lens[2], matrix, al, false);
    db->g32.indices = idx[2];
    return db;
}

void hyb_db_destroy(void *p) { delete (Database *)p; }

void *hyb_scratch_create(void) { return new Scratch; }
void hyb_scratch_destroy(void *p) { delete (Scratch *)p; }

// Per-target scores in db order (scan_scores semantics).
void hyb_scan_scores(const void *dbp, void *scp, const uint8_t *q, uint64_t qlen, int32_t *out) {
    const Database &db = *(const Database *)dbp;
    Scratch &sc = *(Scratch *)scp;
    fill_scores(db, db.g8, q, qlen, sc.h8, sc.f8, sc.s8);
    for (size_t i = 0; i < db.g8.indices.size(); ++i) out[db.g8.indices[i]] = sc.s8[i];
    fill_scores(db, db.g16, q, qlen, sc.h16, sc.f16, sc.s16);
    for (size_t i = 0; i < db.g16.indices.size(); ++i) out[db.g16.indices[i]] = sc.s16[i];
    fill_scores(db, db.g32, q, qlen, sc.h32, sc.f32, sc.s32);
    for (size_t i = 0; i < db.g32.indices.size(); ++i) out[db.g32.indices[i]] = sc.s32[i];
}

// Single best hit (grouped scan semantics, src/database.rs:160-208).
void hyb_scan(const void *dbp, void *scp, const uint8_t *q, uint64_t qlen, hyo_hit *out) {
    const Database &db = *(const Database *)dbp;
    Scratch &sc = *(Scratch *)scp;
    int64_t best = INT32_MIN;
    uint64_t best_idx = 0;
    auto reduce = [&](const std::vector<uint64_t> &ix, auto &scores) {
        for (size_t i = 0; i < ix.size(); ++i) {
            int64_t s = scores[i];
            if (s > best || (s == best && ix[i] < best_idx)) {
                best = s;
                best_idx = ix[i];
            }
        }
    };
    fill_scores(db, db.g8, q, qlen, sc.h8, sc.f8, sc.s8);
    reduce(db.g8.indices, sc.s8);
    fill_scores(db, db.g16, q, qlen, sc.h16, sc.f16, sc.s16);
    reduce(db.g16.indices, sc.s16);
    fill_scores(db, db.g32, q, qlen, sc.h32, sc.f32, sc.s32);
    reduce(db.g32.indices, sc.s32);
    out->score = (int32_t)best;
    out->db_index = best_idx;
    out->query_end = out->target_end = -1;
    if (db.search_type == 1) {
        int32_t s;
        hyo_align_core(q, qlen, db.residues.data() + db.offsets[best_idx],
                       db.offsets[best_idx + 1] - db.offsets[best_idx], db.matrix.data(), db.al,
                       db.go, db.ge, db.mode, &s, &out->query_end, &out->target_end);
    }
}

// The best score of a query over one database and its smallest db index among ties (the grouped
// scan's reduction, src/database.rs:160-208), without the winner's ends.
static void best_score(const Database &db, Scratch &sc, const uint8_t *q, uint64_t qlen, int64_t *best_out,
                       uint64_t *idx_out) {
    int64_t best = INT32_MIN;
    uint64_t best_idx = 0;
    auto reduce = [&](const std::vector<uint64_t> &ix, auto &scores) {
        for (size_t i = 0; i < ix.size(); ++i) {
            int64_t s = scores[i];
            if (s > best || (s == best && ix[i] < best_idx)) {
                best = s;
                best_idx = ix[i];
            }
        }
    };
    fill_scores(db, db.g8, q, qlen, sc.h8, sc.f8, sc.s8);
    reduce(db.g8.indices, sc.s8);
    fill_scores(db, db.g16, q, qlen, sc.h16, sc.f16, sc.s16);
    reduce(db.g16.indices, sc.s16);
    fill_scores(db, db.g32, q, qlen, sc.h32, sc.f32, sc.s32);
    reduce(db.g32.indices, sc.s32);
    *best_out = best;
    *idx_out = best_idx;
}

// A query stream against one database held as `n_slices` consecutive slices (slice s holds global
// indices slice_base[s] ..), balanced over `threads` threads so that no thread idles while a long
// query runs: the (query, slice) units go longest query first to threads that take them one at a
// time, each thread with its own Scratch. Per query the slices' best hits reduce to the grouped
// scan's answer (highest score, then smallest global index), and ScoreEnd takes the winner's ends
// from align_core, as hyb_scan does for a whole database.
void hyb_scan_stream(const void *const *dbs, const uint64_t *slice_base, uint64_t n_slices,
                     const uint8_t *queries, const uint64_t *qoff, uint64_t nq, hyo_hit *out,
                     int threads) {
    if (threads < 1) threads = 1;
    std::vector<uint64_t> order(nq);
    for (uint64_t k = 0; k < nq; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) {
        return qoff[a + 1] - qoff[a] > qoff[b + 1] - qoff[b];
    });
    std::vector<int64_t> bs(nq * n_slices);
    std::vector<uint64_t> bi(nq * n_slices);
    const int64_t units = (int64_t)(nq * n_slices);
#pragma omp parallel num_threads(threads)
    {
        Scratch sc;
#pragma omp for schedule(dynamic, 1)
        for (int64_t u = 0; u < units; ++u) {
            const uint64_t k = order[(uint64_t)u / n_slices], s = (uint64_t)u % n_slices;
            best_score(*(const Database *)dbs[s], sc, queries + qoff[k], qoff[k + 1] - qoff[k],
                       &bs[k * n_slices + s], &bi[k * n_slices + s]);
        }
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)nq; ++i) {
            const uint64_t k = order[(uint64_t)i];
            uint64_t ws = 0;
            for (uint64_t s = 1; s < n_slices; ++s)
                if (bs[k * n_slices + s] > bs[k * n_slices + ws]) ws = s;
            const Database &db = *(const Database *)dbs[ws];
            const uint64_t local = bi[k * n_slices + ws];
            out[k].score = (int32_t)bs[k * n_slices + ws];
            out[k].db_index = slice_base[ws] + local;
            out[k].query_end = out[k].target_end = -1;
            if (db.search_type == 1) {
                int32_t sc2;
                hyo_align_core(queries + qoff[k], qoff[k + 1] - qoff[k], db.residues.data() + db.offsets[local],
                               db.offsets[local + 1] - db.offsets[local], db.matrix.data(), db.al, db.go,
                               db.ge, db.mode, &sc2, &out[k].query_end, &out[k].target_end);
            }
        }
    }
}

// A query stream over `threads` threads, one Scratch per thread (tests/database.rs:136-176):
// query k is queries[qoff[k] .. qoff[k+1]].
void hyb_scan_many(const void *dbp, const uint8_t *queries, const uint64_t *qoff, uint64_t nq,
                   hyo_hit *out, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel num_threads(threads)
    {
        Scratch sc;
#pragma omp for schedule(dynamic, 1)
        for (int64_t k = 0; k < (int64_t)nq; ++k)
            hyb_scan(dbp, &sc, queries + qoff[k], qoff[k + 1] - qoff[k], &out[k]);
    }
}

}  // extern "C"
