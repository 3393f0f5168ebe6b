/*
 * hyalite_cuda.h -- C ABI of the B200 `cuda` backend for hyalite's inter-sequence database scan.
 *
 * Plain pointers and sizes only; no CUDA or torch types cross this boundary (the one stream
 * accessor hands out an opaque pointer). Each declaration names the reference interface it
 * replaces (paths inside Psy-Fer/hyalite), for the Rust-side `extern "C"` binding a maintainer
 * adds over it.
 *
 * Threading (src/database.rs:1-7, tests/database.rs:136-176): an hy_db is immutable after
 * creation and may be shared by any number of host threads; an hy_scratch belongs to one thread
 * at a time. Every call returns a status; error details are per thread (hy_last_error_detail).
 * Residues are pre-encoded alphabet indices (0..alphabet_len), never ASCII (DETERMINISM.md).
 */
#ifndef HYALITE_CUDA_H
#define HYALITE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. 1..11 mirror hyalite's Error variants one to one (src/error.rs:16-96); the rest
 * are conditions the reference expresses as panics or that only a device backend has. */
typedef enum {
    HY_OK = 0,
    HY_ERR_EMPTY_ALPHABET = 1,           /* Error::EmptyAlphabet */
    HY_ERR_MATRIX_SHAPE = 2,             /* Error::MatrixShape {alphabet_len, expected, got} */
    HY_ERR_NEGATIVE_GAP_PENALTY = 3,     /* Error::NegativeGapPenalty {gap_open, gap_ext} */
    HY_ERR_GAP_OPEN_LESS_THAN_EXTEND = 4,/* Error::GapOpenLessThanExtend {gap_open, gap_ext} */
    HY_ERR_SCORE_RANGE_TOO_WIDE = 5,     /* Error::ScoreRangeTooWide {bound} */
    HY_ERR_SYMBOL_OUT_OF_RANGE = 6,      /* Error::SymbolOutOfRange {symbol, alphabet_len} */
    HY_ERR_INCOMPLETE_BUILDER = 7,       /* Error::IncompleteBuilder (raised by host bindings) */
    HY_ERR_EMPTY_DATABASE = 8,           /* Error::EmptyDatabase */
    HY_ERR_BACKEND_UNAVAILABLE = 9,      /* Error::BackendUnavailable {backend} */
    HY_ERR_INVALID_BACKEND_NAME = 10,    /* Error::InvalidBackendName {name} */
    HY_ERR_TRACEBACK_BUDGET_EXCEEDED = 11,/* Error::TracebackBudgetExceeded (traceback not built) */
    HY_ERR_INVALID_ARGUMENT = 20,        /* null pointer, bad enum value */
    HY_ERR_QUERY_TOO_LONG = 21,          /* query longer than max_query_len (reference: debug_assert) */
    HY_ERR_CUDA = 22,                    /* a CUDA runtime call failed; detail[0] = cudaError_t */
    HY_ERR_OUT_OF_MEMORY = 23,           /* device or pinned allocation failed */
    HY_ERR_TIMEOUT = 24,                 /* a bounded device wait ran out; the context stays usable */
    HY_ERR_UNSUPPORTED = 25,             /* a search type or option this backend does not build */
    HY_ERR_REJECTED = 26,                /* serving: admission refused (queue or memory full) */
    HY_ERR_DEVICE_CHECK = 27             /* bounds-checked build: a kernel skipped an item whose
                                          * indices fell outside their arrays */
} hy_status;

typedef enum { HY_MODE_SW = 0, HY_MODE_NW = 1, HY_MODE_HW = 2, HY_MODE_OV = 3, HY_MODE_SHW = 4 } hy_mode;
/* SearchType (src/search.rs:13-27). HY_SEARCH_ALIGNMENT carries its max_bytes budget in the
 * traceback_max_bytes argument of hy_db_create; it tracks ends like HY_SEARCH_SCORE_END. */
typedef enum { HY_SEARCH_SCORE = 0, HY_SEARCH_SCORE_END = 1, HY_SEARCH_ALIGNMENT = 2 } hy_search_type;

/* AlignOp (src/align.rs:47-56): one byte per operation. */
typedef enum { HY_OP_MATCH = 0, HY_OP_MISMATCH = 1, HY_OP_INS = 2, HY_OP_DEL = 3 } hy_align_op;
typedef enum { HY_WIDTH_I8 = 0, HY_WIDTH_I16 = 1, HY_WIDTH_I32 = 2 } hy_score_width;
/* Backend names of src/backend.rs:25-36 plus the new `Cuda` (the enum is #[non_exhaustive]). */
typedef enum {
    HY_BACKEND_SCALAR = 0, HY_BACKEND_SSE41 = 1, HY_BACKEND_AVX2 = 2, HY_BACKEND_NEON = 3,
    HY_BACKEND_CUDA = 4
} hy_backend;
/* BackendChoice (src/backend.rs:123-133) as an int: HY_CHOICE_UNSET consults HYALITE_BACKEND,
 * HY_CHOICE_AUTO detects, a hy_backend value forces that backend. */
#define HY_CHOICE_UNSET (-2)
#define HY_CHOICE_AUTO (-1)
/* Layout / LayoutChoice (src/inter.rs:317-351): on the device, Gathered interleaves two per-letter
 * query profiles per cell pair; Precomputed loads a pre-packed pair profile. Results identical. */
#define HY_LAYOUT_AUTO (-1)
#define HY_LAYOUT_GATHERED 0
#define HY_LAYOUT_PRECOMPUTED 1

/* BestHit (src/hit.rs:16-25). query_end / target_end are 0-based; -1 encodes None. */
typedef struct {
    int32_t score;
    uint32_t reserved;
    uint64_t db_index;
    int64_t query_end;
    int64_t target_end;
} hy_hit;

/* Alignment (src/align.rs:57-83): half-open spans [start, end); its operations are the n_ops bytes
 * (hy_align_op) at ops_offset of the operation buffer the call returned or was given. */
typedef struct {
    int32_t score;
    uint32_t reserved;
    uint64_t query_start, query_end;
    uint64_t target_start, target_end;
    uint64_t n_ops;
    uint64_t ops_offset;
} hy_alignment;

typedef struct hy_db hy_db;
typedef struct hy_scratch hy_scratch;

/* ---- errors -------------------------------------------------------------------------------- */

/* The fields of the last error raised on this thread: MatrixShape {alphabet_len, expected, got};
 * NegativeGapPenalty / GapOpenLessThanExtend {gap_open, gap_ext}; ScoreRangeTooWide {bound};
 * SymbolOutOfRange {symbol, alphabet_len}; BackendUnavailable {backend}; QueryTooLong {len, max};
 * Cuda {cudaError_t}. Unused fields are 0. */
void hy_last_error_detail(int64_t detail[3]);
/* A static, human-readable name for a status ("ScoreRangeTooWide", ...). */
const char *hy_status_name(hy_status status);

/* ---- backend selection (src/backend.rs) ------------------------------------------------------ */

/* BackendChoice::parse (src/backend.rs:143-155), plus "cuda": case-insensitive, trimmed. Writes
 * HY_CHOICE_AUTO or a hy_backend to *choice. */
hy_status hy_backend_parse(const char *name, int *choice);
/* Backend::is_available (src/backend.rs:77-84): only HY_BACKEND_CUDA is built here, and it is
 * available iff a CUDA device can be used. */
int hy_backend_is_available(hy_backend backend);
/* resolve (src/backend.rs:176-187) + choice_from_env (195-204): HY_CHOICE_UNSET reads
 * HYALITE_BACKEND, then falls back to auto. */
hy_status hy_backend_resolve(int choice, hy_backend *out);
/* Backend::name (src/backend.rs:40-48). */
const char *hy_backend_name(hy_backend backend);

/* ---- scoring and width proof ----------------------------------------------------------------- */

/* Scoring::new validation (src/scoring.rs:65-100). */
hy_status hy_scoring_validate(uint64_t alphabet_len, const int32_t *matrix, uint64_t matrix_len,
                              int32_t gap_open, int32_t gap_ext);
/* width::required_width (src/width.rs:145-169). *bound receives the clamped magnitude bound. */
hy_status hy_required_width(hy_mode mode, int32_t min_entry, int32_t max_entry, int32_t gap_open,
                            int32_t gap_ext, uint64_t max_query_len, uint64_t max_target_len,
                            hy_score_width *width, int64_t *bound);

/* ---- database (src/database.rs) -------------------------------------------------------------- */

/* DatabaseBuilder::build (src/database.rs:737-877): sequence k is residues[offsets[k] ..
 * offsets[k+1]] (offsets has n_seqs + 1 entries). Validates in the reference's order (scoring,
 * empty database, symbols in db order, whole-database width proof, for HY_SEARCH_ALIGNMENT the
 * traceback budget traceback_max_bytes against hy_traceback_min_bytes_for_database(max_query_len,
 * longest sequence) (src/database.rs:776-790), backend), then packs the database into device
 * memory on the current CUDA device, where it stays until hy_db_destroy. traceback_max_bytes is
 * ignored for the other search types. backend_choice: HY_CHOICE_UNSET / HY_CHOICE_AUTO / a
 * hy_backend. layout: HY_LAYOUT_*. */
hy_status hy_db_create(const uint8_t *residues, const uint64_t *offsets, uint64_t n_seqs,
                       const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open,
                       int32_t gap_ext, hy_mode mode, hy_search_type search_type,
                       uint64_t traceback_max_bytes, uint64_t max_query_len, int backend_choice,
                       int layout, hy_db **out);
void hy_db_destroy(hy_db *db);

/* Accessors (src/database.rs:570-638). score_width is the reference's whole-database proof (the
 * widest width); the device partitions sequences by its own per-sequence rule (bound + gap_open
 * must fit int16 for the packed int16x2 kernel, else int32), which never changes results. */
uint64_t hy_db_sequence_count(const hy_db *db);
hy_mode hy_db_mode(const hy_db *db);
hy_search_type hy_db_search_type(const hy_db *db);
hy_score_width hy_db_score_width(const hy_db *db);
hy_backend hy_db_backend(const hy_db *db);
int hy_db_layout(const hy_db *db);
uint64_t hy_db_max_query_len(const hy_db *db);
uint64_t hy_db_max_target_len(const hy_db *db);
/* Device bytes held by the database, and device bytes one hy_scratch needs. */
uint64_t hy_db_device_bytes(const hy_db *db);
uint64_t hy_db_scratch_bytes(const hy_db *db);
/* Number of sequences the device runs in packed int16x2 pairs and in int32 lanes. */
void hy_db_partition(const hy_db *db, uint64_t *n_i16, uint64_t *n_i32);

/* Scratch::new (src/database.rs:965-998): one CUDA stream plus device work and output buffers,
 * sized for the database. Exclusive to one host thread at a time. */
hy_status hy_scratch_create(const hy_db *db, hy_scratch **out);
void hy_scratch_destroy(hy_scratch *scratch);
/* The scratch's cudaStream_t, as an opaque pointer (for event timing and graph capture). */
void *hy_scratch_stream(hy_scratch *scratch);

/* Database::scan (src/database.rs:83-144): the single best hit; ties go to the smallest db_index.
 * Host query in, host hit out; blocks until the result is in *out. */
hy_status hy_scan(const hy_db *db, hy_scratch *scratch, const uint8_t *query, uint64_t qlen,
                  hy_hit *out);
/* Database::scan_all (src/database.rs:347-464): one hit per sequence in db order (out has
 * hy_db_sequence_count entries). */
hy_status hy_scan_all(const hy_db *db, hy_scratch *scratch, const uint8_t *query, uint64_t qlen,
                      hy_hit *out);
/* Database::scan_scores (src/database.rs:481-515): every sequence's best score in db order. */
hy_status hy_scan_scores(const hy_db *db, hy_scratch *scratch, const uint8_t *query,
                         uint64_t qlen, int32_t *out);

/* Device-resident forms of scan / scan_scores: the query is already in device memory and the
 * result is written to device memory, asynchronously on the scratch's stream (no host sync).
 * The query's symbols must already be validated (hy_query_validate). */
hy_status hy_scan_device(const hy_db *db, hy_scratch *scratch, const uint8_t *d_query,
                         uint64_t qlen, hy_hit *d_out);
hy_status hy_scan_scores_device(const hy_db *db, hy_scratch *scratch, const uint8_t *d_query,
                                uint64_t qlen, int32_t *d_out);
/* No counterpart in the reference: an allocation-free form of hy_scan_scores for callers that cannot
 * call cudaMalloc once running (device memory already owned by another allocator, or a loop that
 * cannot take cudaMalloc's implicit synchronisation). Query and scores are the caller's device
 * buffers; the kernels' scratch is a fixed 16 MiB __device__ array inside this library, which
 * every GPU that loads the library holds until exit. A call needing more scratch than that (the
 * boundary rows of a multi-pass query grow with the database) returns HY_ERR_UNSUPPORTED with
 * detail {needed_bytes, limit}; so does an alphabet whose query-profile slices do not fit in the
 * device's shared memory (about 54 letters and up; hy_scan_scores handles those). Runs on
 * `stream` (a cudaStream_t, or NULL for the legacy default stream) and returns once the scores
 * are written. Calls share the array: calls whose kernels
 * overlap on the GPU race and must be serialised by the caller. The query's symbols must already
 * be validated (hy_query_validate); the current device must be the database's. The first call on
 * each device does a one-time set-up (the array's device address, and loading every kernel this
 * entry point launches, which CUDA's lazy module loading would otherwise do, allocating, at each
 * kernel's first launch): make it before device memory is fully reserved and before any stream
 * capture. Later calls allocate nothing. */
hy_status hy_scan_scores_noalloc(const hy_db *db, const uint8_t *d_query, uint64_t qlen,
                                 int32_t *d_scores, void *stream);
/* The checks hy_scan performs on a host query (length, then symbols). */
hy_status hy_query_validate(const hy_db *db, const uint8_t *query, uint64_t qlen);
/* Waits for the scratch's stream; returns HY_ERR_TIMEOUT if a kernel's bounded wait ran out. */
hy_status hy_scratch_sync(hy_scratch *scratch);

/* ---- measurement (no reference counterpart: the reference benches with criterion) ------------ */

/* While enabled, every main scan-kernel launch on this scratch is bracketed by CUDA events on the
 * stream it runs on. _read synchronises and returns, since the last read (or enable), the summed
 * kernel time, launch count and real DP cells of the bulk int16x2 pair kernel ([0]) and the int32
 * kernel ([1]) ([2] is kept for a separate long-pair kernel, which plain scans no longer launch:
 * zero), plus the number of kernels of every kind this scratch launched; then resets them. */
hy_status hy_scratch_profile(hy_scratch *scratch, int enable);
hy_status hy_scratch_profile_read(hy_scratch *scratch, double kernel_ms[3], uint64_t launches[3],
                                  double cells[3], uint64_t *all_launches);
/* The packed-int16 DPX roofline of the current device: the scan's per-cell instruction mix run
 * register resident on every SM, in DP cells per second. */
hy_status hy_measure_dpx_peak(double *cells_per_second);
/* The same recurrence in int32 DPX lanes (one cell per op): the roofline of the int32 kernels
 * (the traceback fill and the int32 scan items), in DP cells per second. */
hy_status hy_measure_dpx_peak_i32(double *cells_per_second);
/* The same recurrence in packed int8x4 lanes (four cells per op, saturating SIMD-video
 * intrinsics, as the reference's i8 lanes saturate), in DP cells per second: the measurement
 * behind keeping i8-proven sequences in int16x2 lanes. */
hy_status hy_measure_dpx_peak_i8x4(double *cells_per_second);

/* ---- failure injection for tests (no reference counterpart: the reference's scan cannot fail) -- */

/* Makes the `after`-th next device allocation of this library fail as a full device would (0: the
 * very next one), so that tests can drive every allocation's error path; -1 turns it off. The
 * failing call returns HY_ERR_OUT_OF_MEMORY and frees what it had allocated. */
void hy_debug_fail_device_alloc(int64_t after);
/* Device allocations this library holds right now (a test's leak check). */
int64_t hy_debug_live_device_allocations(void);
/* Polls every bounded device wait makes before it gives up (a wait for a query-profile copy into
 * shared memory, a stripe waiting on the stripe above); -1 restores the default, which bounds a
 * wait to seconds. 0 makes every such wait give up at once, which a test uses to see
 * HY_ERR_TIMEOUT reported and the scratch still usable afterwards. */
void hy_debug_set_wait_polls(int64_t polls);
/* The chunks hy_align_pairs would run pairs [0, n_pairs) in, for these offsets: writes up to `cap`
 * chunk boundaries (the first pair of each chunk, then n_pairs) and returns the number of chunks.
 * Chunks are cut at equal shares of the residues, so that no chunk's staging much exceeds its
 * bound (512 MiB) however long and short pairs are ordered. */
uint64_t hy_debug_pair_chunks(const uint64_t *q_off, const uint64_t *t_off, uint64_t n_pairs,
                              uint64_t *bounds, uint64_t cap);
/* The launch shape of the end-recovery band kernel (a scan's winner, a long pair) for a query of
 * n_passes pass slices of pass_bytes each, with smem_limit bytes of shared memory a block: out =
 * {slices read from global memory (1) or shared memory (0), warps a block, blocks of the cluster,
 * rounds}. One slice per warp; more passes than one block holds take a cluster of up to 8 blocks. */
void hy_debug_band_shape(uint32_t pass_bytes, int32_t n_passes, uint64_t smem_limit, int32_t out[4]);

/* ---- batched scan (no reference counterpart: the reference scans one query per call) ---------- */

/* A batch runner over a fixed set of databases on one device. hy_scan_batch computes, for many
 * queries at once, exactly what hy_scan returns for each (same score, db_index and ends), with
 * every query against its own database (any mode and search type). The device work is persistent
 * kernels over a work queue (chunks of length-sorted targets x queries, largest first), one
 * recovery of the winner's ends per ScoreEnd query, all captured once into a CUDA graph that
 * every call replays. max_queries bounds the queries of one call (at most 16000); query
 * residues of one call are bounded by max_queries x the largest max_query_len. With autotune
 * set, the first call of each batch shape (the mix of modes and query lengths) first times
 * candidate launch configurations on a sampled part of the batch and keeps the fastest.
 * Returns HY_ERR_UNSUPPORTED when the largest alphabet's query profiles do not fit in shared
 * memory. The databases must outlive the batch. One host thread at a time per batch. */
typedef struct hy_batch hy_batch;
hy_status hy_batch_create(const hy_db *const *dbs, uint32_t n_dbs, uint32_t max_queries,
                          int autotune, hy_batch **out);
void hy_batch_destroy(hy_batch *batch);
/* Query i is q_res[q_off[i] - q_off[0] .. q_off[i+1] - q_off[0]) against dbs[db_of_query[i]];
 * out[i] receives its BestHit. Queries are validated in order like hy_scan's (length, then
 * symbols); on the first failing query the call returns its error, writes its index to
 * *failed_query (if not NULL) and runs nothing. Blocks until the hits are in `out`. */
hy_status hy_scan_batch(hy_batch *batch, uint32_t n_queries, const uint32_t *db_of_query,
                        const uint8_t *q_res, const uint64_t *q_off, hy_hit *out,
                        uint32_t *failed_query);
/* Runs the autotuner on this batch now (every `stride`-th item chunk; 0 picks a stride leaving
 * about 256 chunks) and keeps the fastest configuration; *best_ms is its sampled time. */
hy_status hy_batch_tune(hy_batch *batch, uint32_t n_queries, const uint32_t *db_of_query,
                        const uint8_t *q_res, const uint64_t *q_off, uint32_t stride,
                        double *best_ms);
/* The launch configuration in use: {largest query length run with 8 rows per lane, largest with
 * 16 rows (longer: 32), the pair width above which a pair runs one warp each}. Setting one turns
 * autotuning off; the width must be 1..4096. */
hy_status hy_batch_get_config(const hy_batch *batch, int32_t cfg[3]);
hy_status hy_batch_set_config(hy_batch *batch, const int32_t cfg[3]);
uint64_t hy_batch_device_bytes(const hy_batch *batch);
/* The batch's cudaStream_t, as an opaque pointer. */
void *hy_batch_stream(hy_batch *batch);

/* ---- served scan (no reference counterpart) ------------------------------------------------- */

/* A request loop on its own host thread over a fixed set of databases. Requests ask for the best
 * hit of a query (like hy_scan, with ends for ScoreEnd databases) or for every target's score
 * (like hy_scan_scores; the hit then carries the best score and index without ends). Queued
 * requests are admitted in arrival order into device batches while a batch's query-profile and
 * score-output budgets hold; up to `in_flight` batches run on the GPU at once, so requests that
 * arrive while others run are batched and overlap them on the device. Results equal the plain
 * calls' for the same query. Zero fields take the defaults named below. */
typedef struct {
    uint32_t max_batch;        /* queries per device batch (64) */
    uint32_t in_flight;        /* device batches that may run at once (2) */
    uint32_t max_pending;      /* queued requests beyond which hy_server_submit rejects (4096) */
    uint32_t reserved;
    uint64_t profile_budget;   /* device bytes of query profiles per batch (max_batch queries of
                                  the largest max_query_len) */
    uint64_t scores_budget;    /* device (and pinned host) bytes of score outputs per batch
                                  (max_batch x 4 x the largest database's sequence count) */
    int32_t launch_config[3];  /* as hy_batch_set_config; {0, 0, 0}: the defaults */
} hy_server_config;

typedef struct {
    uint64_t submitted, completed, rejected, batches, pending;
    double mean_batch;                      /* requests per device batch */
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> result ready, completed requests */
    double cells;                           /* DP cells of the completed requests */
    double seconds;                         /* first submit -> last completion */
    double gcups;                           /* cells / seconds / 1e9 */
} hy_server_stats;

typedef struct hy_server hy_server;
hy_status hy_server_create(const hy_db *const *dbs, uint32_t n_dbs, const hy_server_config *config,
                           hy_server **out);
/* Stops accepting requests, completes every queued and running one, and frees the server.
 * Results not yet waited for are discarded. */
void hy_server_destroy(hy_server *server);
/* Queues a query against dbs[db]. With want_scores, `scores_out` (the database's sequence count
 * of int32, owned by the caller) receives every target's score when the request completes, so it
 * must stay valid until the request is waited for or the server is destroyed. Validates like
 * hy_scan; HY_ERR_REJECTED when the queue is full or the request alone exceeds a batch budget.
 * Thread-safe. */
hy_status hy_server_submit(hy_server *server, uint32_t db, const uint8_t *query, uint64_t qlen,
                           int want_scores, int32_t *scores_out, uint64_t *request_id);
/* The query-profile bytes a request of length qlen against dbs[db] takes from its batch's
 * profile budget (the admission rule); *score_bytes (if not NULL) receives its score-output
 * bytes. 0 for a bad server or database index. */
uint64_t hy_server_request_bytes(const hy_server *server, uint32_t db, uint64_t qlen,
                                 int want_scores, uint64_t *score_bytes);
/* *done = 1 once the request's result is ready. */
hy_status hy_server_poll(hy_server *server, uint64_t request_id, int *done);
/* Waits up to timeout_s for the request; on completion writes its hit, releases the request and
 * returns its status. HY_ERR_TIMEOUT leaves the request queued. */
hy_status hy_server_wait(hy_server *server, uint64_t request_id, double timeout_s, hy_hit *out);
/* hy_server_wait that also returns the request's latency, submit to result ready, in ms. */
hy_status hy_server_wait_timed(hy_server *server, uint64_t request_id, double timeout_s, hy_hit *out,
                               double *latency_ms);
/* Counters and latency percentiles since the last reset (reset != 0 clears them). */
hy_status hy_server_stats_read(hy_server *server, int reset, hy_server_stats *out);

/* Page-locked host memory (no reference counterpart): buffers from hy_host_alloc given to
 * hy_align_pairs / hy_align_pairs_position_max as residues or column maxima are copied from and to
 * where they are, without the calls' staging copies. Freed with hy_host_free. */
hy_status hy_host_alloc(uint64_t bytes, void **out);
hy_status hy_host_free(void *p);

/* ---- pairwise batch (src/kernel.rs:429-452) -------------------------------------------------- */

/* align_pairs: pair p is (q_res[q_off[p]..q_off[p+1]], t_res[t_off[p]..t_off[p+1]]). Each pair is
 * validated in order (symbols query-then-target, then the width proof on its exact lengths); on
 * the first failing pair the call returns its error, *failed_pair receives its index and out[0 ..
 * index) holds the hits of the pairs before it. db_index of each hit is its pair index. The calling
 * thread keeps grow-only device buffers, a ring of pinned host staging slots and host work arrays
 * between calls (freed at thread exit). Internally the width proof runs on the host over every
 * pair and the symbol check on the device while it packs each chunk; the reported error, index and
 * prefix are those of the in-order validation. */
hy_status hy_align_pairs(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                         const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix,
                         uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext, hy_mode mode,
                         hy_search_type search_type, hy_hit *out, uint64_t *failed_pair);
/* Timing of this thread's last hy_align_pairs call (no reference counterpart): the device time of
 * its kernels (CUDA events around each chunk's packing and pair kernels, plus the long pairs'
 * stripe kernel, or a lone long pair's band kernel) and the wall time of the whole call. */
hy_status hy_align_pairs_timing(double *kernel_ms, double *call_ms);
/* Phases of this thread's last hy_align_pairs call, in ms (no reference counterpart): up to n of
 * {the host lengths pass and routing, host sort and item packing (summed over chunks), waits for the
 * staging copies (which run on their own threads beside the next chunk's sort and packing), the
 * chunk pipeline (wall time to the device's end, overlapping the two before),
 * results back, host waits for a staging slot, host copies of the column maxima into the caller's
 * array (hy_align_pairs_position_max)}. The last call of either entry point. */
hy_status hy_align_pairs_phases(double *ms, uint32_t n);

/* ---- traceback: the Alignment search type (src/align.rs, src/database.rs:517-565) -------------- */

/* align (src/align.rs:169-222): validates the scoring (src/scoring.rs:65-100), the symbols of the
 * query then the target, the width proof on (qlen, tlen), then the traceback budget (the
 * reference's full-matrix / sqrt-checkpoint footprint rule: HY_ERR_TRACEBACK_BUDGET_EXCEEDED with
 * detail {needed_bytes, budget_bytes}); then traces the pair back on the current CUDA device.
 * max_bytes = UINT64_MAX is usize::MAX. ops receives out->n_ops operations (room for qlen + tlen;
 * out->ops_offset is 0). The device path keeps 4 bits a cell whatever the budget, and its result is
 * the reference's for every budget that passes. The calling thread keeps grow-only buffers. */
hy_status hy_align(const uint8_t *query, uint64_t qlen, const uint8_t *target, uint64_t tlen,
                   const int32_t *matrix, uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext,
                   hy_mode mode, uint64_t max_bytes, hy_alignment *out, uint8_t *ops);
/* Database::scan_aligned (src/database.rs:527-536): the winner of hy_scan (same tie-break) and its
 * alignment. *ops points to the operations, owned by the scratch and valid until its next
 * traceback call or its destruction. The database must be built with HY_SEARCH_ALIGNMENT
 * (otherwise HY_ERR_INVALID_ARGUMENT, where the reference panics). */
hy_status hy_scan_aligned(const hy_db *db, hy_scratch *scratch, const uint8_t *query, uint64_t qlen,
                          uint64_t *db_index, hy_alignment *out, const uint8_t **ops);
/* Database::scan_all_aligned (src/database.rs:538-549): out[k] (hy_db_sequence_count entries) is
 * the alignment against sequence k; the operations of all of them are concatenated in db order at
 * *ops (owned by the scratch as above), out[k].ops_offset indexing into it. */
hy_status hy_scan_all_aligned(const hy_db *db, hy_scratch *scratch, const uint8_t *query,
                              uint64_t qlen, hy_alignment *out, const uint8_t **ops);
/* The budget a database built with HY_SEARCH_ALIGNMENT needs (traceback_min_bytes_for_database,
 * src/align.rs:228-250), and traceback's rule for one problem (src/align.rs:192-222): 0 when an
 * m x n problem traces within max_bytes, else the bytes it needs. */
uint64_t hy_traceback_min_bytes_for_database(uint64_t max_m, uint64_t max_n);
uint64_t hy_traceback_needed(uint64_t m, uint64_t n, uint64_t max_bytes);
/* Timing of the last traceback call of a scratch (scratch NULL: of this thread's hy_align), no
 * reference counterpart: out = {fill kernels' device ms, walk and compaction kernels' device ms,
 * device span from the first fill to the end of compaction in ms (walks overlap the next chunk's
 * fill), whole call ms, DP cells traced}. Device times are CUDA events. */
hy_status hy_traceback_timing(hy_scratch *scratch, double out[5]);
/* ---- per-position maxima and score2 (src/kernel.rs:454-553, 741-792) -------------------------- */

/* align_pair_position_max over n_pairs independent (query, target) pairs (SW; the reference's
 * entry is one pair, align_pair_position_max_with in a loop): pair k is q_res[q_off[k] ..
 * q_off[k+1]] against t_res[t_off[k] .. t_off[k+1]]. Validation as align_pairs (symbols of the query
 * then the target, then the SW width proof, pair by pair; the first failure is returned with its
 * index in *failed_pair and the pairs before it are computed). out[k]: score = max of the pair's
 * column maxima, query_end -1 (not tracked), target_end = first position of that maximum or -1 when
 * the score is 0, db_index k. colmax (NULL: not copied) receives every pair's per-target-position
 * maxima at t_off[k] - t_off[0] (|t_k| entries, each >= 0; on an error, the positions of the
 * pairs from the failing one on are 0). score2 (NULL: not computed) receives {score, position} per
 * pair: bwa's score2 (hy_score2) of the pair's maxima with its best score, its target end
 * (position 0 when -1), the matrix's largest entry and min_score; {0, -1} when no peak qualifies.
 * The pairs run through align_pairs' chunked pipeline and pair kernels (their column-maxima
 * form); a few long pairs on the stripe kernel. */
hy_status hy_align_pairs_position_max(const uint8_t *q_res, const uint64_t *q_off, const uint8_t *t_res,
                                      const uint64_t *t_off, uint64_t n_pairs, const int32_t *matrix,
                                      uint64_t alphabet_len, int32_t gap_open, int32_t gap_ext,
                                      int32_t *colmax, hy_hit *out, int32_t min_score, int32_t *score2,
                                      uint64_t *failed_pair);
/* Timing of this thread's last hy_align_pairs_position_max call (no reference counterpart):
 * out = {device ms of its kernels (CUDA events), whole call ms, DP cells}. */
hy_status hy_position_max_timing(double out[3]);
/* score2 (src/kernel.rs:741-792) over a host array of column maxima: returns 1 and the peak's
 * {score, position} when a secondary peak qualifies, 0 (None) otherwise. Host code, as in the
 * reference: a scan of one array. */
int hy_score2(const int32_t *colmax, uint64_t n, int32_t best_score, uint64_t best_target_end,
              int32_t matrix_max, int32_t min_score, int32_t *score, uint64_t *pos);

/* The budget the database was built with (0 unless HY_SEARCH_ALIGNMENT). */
uint64_t hy_db_traceback_max_bytes(const hy_db *db);

#ifdef __cplusplus
}
#endif
#endif
