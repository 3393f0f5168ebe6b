// batch_internal.h -- the batch runner shared by the batched scan (hy_scan_batch) and the server.
#pragma once

#include <stdint.h>

#include <map>
#include <vector>

#include "db_internal.h"

namespace hy {

// Launch classes (one persistent kernel each; the T classes run databases of the Precomputed
// layout; the SW classes the bulk pairs of SW databases, in a kernel of that mode alone with the
// plain scan's register budget) and profile kinds (one query profile each).
enum {
    BC_BULK8 = 0, BC_BULK16 = 1, BC_BULK32 = 2, BC_LONG = 3, BC_I32 = 4,
    BC_TBULK8 = 5, BC_TBULK16 = 6, BC_TBULK32 = 7, BC_TLONG = 8,
    BC_SW8 = 9, BC_SW16 = 10, BC_TSW8 = 11, BC_TSW16 = 12, BC_N = 13
};
enum { PK_BULK = 0, PK_W16 = 1, PK_I32 = 2, PK_W32 = 3, PK_N = 4 };

// One query slot of a batch, as the device kernels read it.
struct BatchQuery {
    // Per profile kind: everything its launches need except the block's boundary region.
    ScanParams sp[PK_N];
    const int32_t *matrix;
    const uint8_t *q;
    const uint32_t *rank;
    int32_t qlen, mode, ends, bulk_rows, top_free, al, lim16;
    int32_t tab;  // the database's pair columns are Precomputed codes (PairTab16)
    uint32_t k0, kl, n_i32, n16;
};

struct BatchCtl {
    uint32_t count[BC_N];     // query slots in each class's order list
    uint32_t n_chunks[BC_N];  // item chunks each class's queue walks
    uint32_t head[BC_N];      // work counters (zeroed by the graph)
    uint32_t n_queries;
    uint32_t chunk_stride;    // 1, or k to run only every k-th chunk (autotuner samples)
};

struct BatchConfig {
    int32_t rows8_max = 64;    // queries up to this length: 8 rows per lane
    int32_t rows16_max = 192;  // up to this length: 16 rows per lane; longer: 32
    uint32_t long_w = LONG_W;  // pairs wider than this run one warp each
};

// What one query of a batch asks for.
struct BatchItem {
    uint32_t db;             // index into the batch's databases
    const uint8_t *q;        // host residues
    uint64_t qlen;
    int32_t *d_scores;       // device per-target scores (n_seqs of the database), or null
    bool ends;               // recover the winner's ends (ScoreEnd databases only)
};

}  // namespace hy

struct hy_batch {
    int device = 0;
    std::vector<const hy_db *> dbs;
    uint32_t max_queries = 0;
    uint64_t max_q_res = 0;
    int32_t al_max = 0;
    uint64_t mql_max = 0, max_t = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    hy::BatchQuery *d_queries = nullptr, *h_queries = nullptr;
    hy::BatchCtl *d_ctl = nullptr, *h_ctl = nullptr;
    uint32_t *d_order = nullptr, *h_order = nullptr;  // BC_N lists of max_queries slots
    uint8_t *d_qres = nullptr, *h_qres = nullptr;
    uint8_t *d_prof = nullptr;
    uint64_t prof_cap = 0;  // bytes of query profiles one batch may hold
    uint8_t *d_bnd_bulk = nullptr, *d_bnd_side = nullptr, *d_bnd_band = nullptr;
    size_t stride_bulk = 0, stride_side = 0, stride_band = 0;
    unsigned long long *d_keys = nullptr;
    int32_t *d_ends = nullptr;
    hy_hit *d_hits = nullptr, *h_hits = nullptr;
    int *d_err = nullptr, *h_err = nullptr;
    int grid[hy::BC_N] = {};
    size_t smem[hy::BC_N] = {};
    int band_threads = 32;
    size_t band_smem = 0;
    cudaGraphExec_t exec = nullptr;
    hy::BatchConfig cfg;
    bool autotune = true;
    std::map<uint64_t, hy::BatchConfig> tuned;  // batch shape signature -> configuration
    uint64_t device_bytes = 0;
    uint64_t runs = 0;
    uint64_t kernels_per_run = 0;
};

namespace hy {

// A batch runner over `dbs` for up to max_queries queries holding at most prof_cap bytes of query
// profiles per batch (0: enough for max_queries queries of the largest max_query_len).
hy_status batch_create(const hy_db *const *dbs, uint32_t n_dbs, uint32_t max_queries,
                       uint64_t prof_cap, bool autotune, hy_batch **out);
void batch_free(hy_batch *b);
// Device bytes of query profiles a query of length qlen against `db` takes in a batch.
uint64_t batch_profile_bytes(const hy_batch *b, const hy_db *db, uint64_t qlen, bool ends);
// Validates the items (length, then symbols; *failed = the first bad item) and writes the
// batch's descriptors into the pinned staging buffers.
hy_status batch_stage(hy_batch *b, const BatchItem *items, uint32_t n, const BatchConfig &cfg,
                      uint32_t chunk_stride, uint32_t *failed);
// Copies the staged batch to the device, replays the graph and queues the hits' read-back, all
// asynchronously on b->stream.
hy_status batch_launch(hy_batch *b, uint32_t n);
// After b->stream has completed: the hits of the last launch (HY_ERR_TIMEOUT if a device wait
// ran out).
hy_status batch_collect(hy_batch *b, uint32_t n, hy_hit *out);

}  // namespace hy
