// db_internal.h -- the device-resident database as the runtime translation units see it.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <vector>

#include "host_common.h"
#include "scan_kernel.cuh"

namespace hy {

// Launch shapes. Main scan: int16x2 pairs in groups of MAIN_G lanes with MAIN_R16 query rows per
// lane; int32 items (the long sequences) one full warp each. Winner end recovery: the band kernel,
// one warp per band of WIN_G * WIN_R query rows.
constexpr int MAIN_G = 8;
constexpr int MAIN_R16 = 16;
constexpr int MAIN_G32 = 32;
constexpr int MAIN_R32 = 16;
constexpr int WIN_G = 32;
constexpr int WIN_R = 8;
// The batched form's pairs longer than LONG_W columns run one full warp each (LONG_G lanes of
// LONG_R rows) in a class of their own, whose boundary regions the bulk classes then need not
// size for. Plain scans keep every pair in the bulk kernel (measured: the same time as a separate
// long-pair kernel on the protein benchmark, with one kernel and stream fewer).
constexpr int LONG_G = 32;
constexpr int LONG_R = 8;
constexpr uint32_t LONG_W = 4096;
constexpr uint32_t NO_LONG_SPLIT = 0xffffffffu;
constexpr int BLOCK = 256;
// Rows per lane of the bulk int16x2 kernel for a query of length qlen (passes of MAIN_G * rows).
// SW scores run the two-column sweep at 8 or 16 rows per lane: 16 unless 8 pads the query to so
// many fewer rows that it wins at 8 rows' rate per padded row (measured 0.853 of 16 rows' rate,
// 4813 against 5641 GCUPS for 1000-residue queries on the protein benchmark: 150 residues take 192
// rows at 8 against 256 at 16). The other kinds run one column of up to 32 rows.
inline int bulk_rows(uint64_t qlen, bool two_col) {
    if (qlen <= 64) return 8;
    if (two_col) {
        const uint64_t rows8 = (qlen + 63) / 64 * 64, rows16 = (qlen + 127) / 128 * 128;
        return 7 * rows8 < 6 * rows16 ? 8 : 16;
    }
    return qlen <= 192 ? 16 : 32;
}
constexpr int BULK_MAX_RPP = 8 * 32;
constexpr size_t BAND_SMEM_BUDGET = 200 * 1024;
// Blocks of one band-kernel cluster at most (the portable cluster size).
constexpr int BAND_CLUSTER_MAX = 8;

// One long pair's BestHit cell on the band kernel (int32 lanes): the query already on the device
// (d_q, m residues), the target on the host (t, tl residues, copied here). Writes the score and the
// 0-based query and target ends (-1 for row or column 0) at index `slot` of d_scores / d_qend /
// d_tend on stream `st` and waits for them; adds the band kernel's time to *kernel_ms.
// Whether a long pair with an m-residue query runs its band passes in one round of one block or
// cluster (band_long_pair's shape); longer queries take the stripe kernel.
bool band_long_pair_fits(uint64_t m, uint64_t al);
hy_status band_long_pair(const uint8_t *d_q, uint64_t m, const uint8_t *t, uint64_t tl, const int32_t *d_matrix,
                         uint64_t al, int32_t go, int32_t ge, int mode, cudaStream_t st, uint32_t slot,
                         int32_t *d_scores, int32_t *d_qend, int32_t *d_tend, double *kernel_ms);
// The same for a lone pair whose query, target and matrix are on the host (align_pair's direct
// path): one copy in, the profile and band kernels, one copy out. out = {score, query end, target
// end}.
hy_status band_single_pair(const uint8_t *q, uint64_t m, const uint8_t *t, uint64_t tl, const int32_t *matrix,
                           uint64_t al, int32_t go, int32_t ge, int mode, int32_t out[3], double *kernel_ms);

struct Partition {
    uint32_t n_items = 0;
    uint64_t n_seqs = 0;
    uint64_t total_cols = 0;
    std::vector<uint64_t> res_prefix;  // host: residues of items [0, i) (both halves of a pair)
    ItemMeta *d_meta = nullptr;
    void *d_res = nullptr;
};

template <class A>
struct ElemSize {
    static constexpr size_t pe = sizeof(typename A::PE);
};

struct QueryPlan {
    int32_t n_passes = 0;
    int32_t vrow0 = 1;
    uint32_t pass_bytes = 0;
};

inline QueryPlan plan(uint64_t qlen, int rpp, uint64_t al, size_t pe) {
    QueryPlan q;
    q.n_passes = (int32_t)((qlen + rpp - 1) / rpp);
    q.vrow0 = (int32_t)qlen - q.n_passes * rpp + 1;
    q.pass_bytes = (uint32_t)((al + 1) * (uint64_t)rpp * pe);
    return q;
}

// The plan of lane arithmetic A (its profile has A::letters(al) letters per table).
template <class A>
inline QueryPlan plan_for(uint64_t qlen, int rpp, uint64_t al) {
    QueryPlan q = plan(qlen, rpp, al, profile_row_bytes<A>());
    q.pass_bytes = (uint32_t)(profile_slice_row_bytes<A>((int64_t)al) * (uint64_t)rpp);
    return q;
}

}  // namespace hy

struct hy_db {
    int device = 0;
    // Largest dynamic shared memory one block may use on the device (opt-in): launch shapes whose
    // query-profile slices exceed it read the profile from global memory instead.
    size_t smem_limit = 48 * 1024;
    uint64_t n_seqs = 0, mql = 0, max_t = 0, al = 0;
    int32_t go = 0, ge = 0, min_e = 0, max_e = 0;
    int mode = 0, search_type = 0, layout = HY_LAYOUT_GATHERED;
    hy_score_width width = HY_WIDTH_I8;
    hy_backend backend = HY_BACKEND_CUDA;
    int32_t *d_matrix = nullptr;
    // Every sequence in int16x2 pairs over the global length order (longest first); the longest
    // ones (those the whole-database proof cannot place in int16) also as int32 singles.
    hy::Partition p16, p32;
    std::vector<uint32_t> pair_w;  // host: longer length of each pair, non-increasing
    uint32_t *d_rank = nullptr;    // device: rank of each global index in the length order
    uint64_t device_bytes = 0;
    // Alignment search type: its budget, and every sequence's residues in db order (sequence k is
    // d_tb_res[tb_off[k] .. tb_off[k+1]]), the targets of the traceback.
    uint64_t tb_max_bytes = 0;
    uint8_t *d_tb_res = nullptr;
    std::vector<uint64_t> tb_off;
};

namespace hy {

// The extents a bounds-checked build (HY_BOUNDS) verifies each item of `part` against: the
// partition's residue columns, `bnd_cols` columns of boundary region, the database's indices and
// the profile letters of lane arithmetic A.
template <class A>
inline void set_extents(ScanParams &p, const hy_db *db, const Partition &part, uint64_t bnd_cols) {
    p.res_cols = part.total_cols;
    p.bnd_cols = bnd_cols;
    p.n_seqs = (uint32_t)db->n_seqs;
    p.letters = (uint32_t)A::letters((int64_t)db->al);
}

// Which items one query runs in which lanes. The width proof is redone with the actual query
// length: pairs [k0, n) fit int16 for this query and run packed; the 2*k0 longest sequences run
// in int32 (always inside the int32 layout, which holds the static int32 set plus one).
struct QuerySplit {
    uint32_t k0 = 0;      // first int16x2 pair item
    uint32_t kl = 0;      // pairs [k0, kl) are long (one warp each), [kl, n) the bulk
    uint32_t n_i32 = 0;   // int32 items [0, n_i32)
};

inline QuerySplit split_for_query(const hy_db *db, uint64_t qlen, uint32_t long_w = NO_LONG_SPLIT) {
    QuerySplit q;
    // Longest target length t whose bound for this query keeps the int16 kernel exact.
    auto fits = [&](uint64_t n) {
        return device_fits_i16(magnitude_bound(db->mode, db->min_e, db->max_e, db->go, db->ge, qlen, n), db->go);
    };
    uint64_t t;
    if (fits(db->max_t)) {
        t = db->max_t;
    } else {
        uint64_t lo = 0, hi = db->max_t;  // fits(lo) may be false only if even length 0 fails
        if (!fits(0)) {
            t = 0;
            lo = hi = 0;
        }
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo + 1) / 2;
            if (fits(mid)) lo = mid; else hi = mid - 1;
        }
        t = lo;
    }
    // First pair whose longer sequence is <= t (pair_w is non-increasing).
    uint32_t a = 0, b = (uint32_t)db->pair_w.size();
    while (a < b) {
        uint32_t mid = a + (b - a) / 2;
        if (db->pair_w[mid] <= t) b = mid; else a = mid + 1;
    }
    q.k0 = a;
    q.n_i32 = (uint32_t)std::min<uint64_t>(2ull * a, db->n_seqs);
    b = (uint32_t)db->pair_w.size();
    while (a < b) {
        uint32_t mid = a + (b - a) / 2;
        if (db->pair_w[mid] <= long_w) b = mid; else a = mid + 1;
    }
    q.kl = a;
    return q;
}

}  // namespace hy

