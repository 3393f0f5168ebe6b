// server.cu -- the served form of the scan: a request loop on its own host thread.
//
// Requests (a query against one of the server's databases, asking for the best hit or for every
// target's score) are queued by hy_server_submit from any thread. The loop admits queued requests
// into a device batch in arrival order while the batch's query-profile and score-output memory
// budgets hold, launches the batch (the persistent kernels of the batch runner under its CUDA
// graph) asynchronously on the batch's own stream, and keeps up to `in_flight` batches on the
// device at once: requests that arrive while a batch runs go into the next batch, whose kernels
// start on SMs as the running batch's queue drains. A finished batch is detected by its event;
// its hits and scores are handed to the waiting callers. Each request's result equals what
// hy_scan / hy_scan_scores returns for it alone: every query of a batch runs the same kernels
// with its own descriptors, profiles, key and outputs.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_internal.h"

using namespace hy;
using Clock = std::chrono::steady_clock;

namespace {

struct ServerRequest {
    uint64_t id = 0;
    uint32_t db = 0;
    std::vector<uint8_t> q;
    bool want_scores = false;
    int32_t *scores_out = nullptr;  // caller's host array, n_seqs of the database
    uint64_t prof_bytes = 0, score_bytes = 0;
    double cells = 0.0;
    Clock::time_point t_submit, t_done;
    hy_hit hit{};
    hy_status status = HY_OK;
    bool done = false;
};

struct ServerSlot {
    hy_batch *b = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<ServerRequest *> reqs;
    std::vector<uint64_t> score_off;  // int32 offset of each request's scores in the arena
    int32_t *d_scores = nullptr, *h_scores = nullptr;
    std::vector<hy_hit> hits;
};

}  // namespace

struct hy_server {
    int device = 0;
    std::vector<const hy_db *> dbs;
    std::vector<double> db_residues;
    hy_server_config cfg{};
    std::vector<ServerSlot> slots;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServerRequest *> pending;
    std::unordered_map<uint64_t, ServerRequest *> reqs;
    uint64_t next_id = 1;
    bool stopping = false;
    hy_status fatal = HY_OK;
    // Statistics since the last reset.
    std::vector<double> lat_ms;
    uint64_t submitted = 0, completed = 0, rejected = 0, batches = 0, batched = 0;
    double cells = 0.0;
    bool have_t0 = false;
    Clock::time_point t0, t_last;
};

namespace {

void free_slots(hy_server *s) {
    for (ServerSlot &sl : s->slots) {
        if (sl.b) batch_free(sl.b);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.d_scores) hy::dev_free(sl.d_scores);
        if (sl.h_scores) cudaFreeHost(sl.h_scores);
    }
    s->slots.clear();
    cudaGetLastError();
}

// Completes the requests of a finished slot (called with the lock held).
void finish_slot(hy_server *s, ServerSlot &sl) {
    const uint32_t n = (uint32_t)sl.reqs.size();
    sl.hits.resize(std::max<uint32_t>(n, 1));
    const hy_status st = batch_collect(sl.b, n, sl.hits.data());
    const Clock::time_point now = Clock::now();
    for (uint32_t i = 0; i < n; ++i) {
        ServerRequest *r = sl.reqs[i];
        r->status = st;
        if (st == HY_OK) {
            r->hit = sl.hits[i];
            if (r->want_scores)
                memcpy(r->scores_out, sl.h_scores + sl.score_off[i], r->score_bytes);
            ++s->completed;
            s->cells += r->cells;
            s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
        }
        r->t_done = now;
        r->done = true;
    }
    s->t_last = now;
    sl.reqs.clear();
    sl.busy = false;
    s->cv_done.notify_all();
}

// Stages and launches the selected requests on a free slot (called without the lock).
hy_status launch_slot(hy_server *s, ServerSlot &sl) {
    const uint32_t n = (uint32_t)sl.reqs.size();
    std::vector<BatchItem> items(n);
    sl.score_off.assign(n, 0);
    uint64_t off = 0;
    for (uint32_t i = 0; i < n; ++i) {
        ServerRequest *r = sl.reqs[i];
        items[i].db = r->db;
        items[i].q = r->q.data();
        items[i].qlen = r->q.size();
        items[i].ends = !r->want_scores;
        items[i].d_scores = nullptr;
        if (r->want_scores) {
            sl.score_off[i] = off;
            items[i].d_scores = sl.d_scores + off;
            off += r->score_bytes / sizeof(int32_t);
        }
    }
    hy_status st = batch_stage(sl.b, items.data(), n, sl.b->cfg, 1, nullptr);
    if (st != HY_OK) return st;
    st = batch_launch(sl.b, n);
    if (st != HY_OK) return st;
    for (uint32_t i = 0; i < n; ++i) {
        if (!sl.reqs[i]->want_scores) continue;
        if (cudaMemcpyAsync(sl.h_scores + sl.score_off[i], sl.d_scores + sl.score_off[i],
                            sl.reqs[i]->score_bytes, cudaMemcpyDeviceToHost, sl.b->stream) != cudaSuccess) {
            cudaGetLastError();
            return fail(HY_ERR_CUDA);
        }
    }
    if (cudaEventRecord(sl.done, sl.b->stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(HY_ERR_CUDA);
    }
    return HY_OK;
}

void worker_main(hy_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        bool any_busy = false;
        for (ServerSlot &sl : s->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaSuccess) {
                finish_slot(s, sl);
                progressed = true;
            } else if (q != cudaErrorNotReady) {
                cudaGetLastError();
                for (ServerRequest *r : sl.reqs) {
                    r->status = HY_ERR_CUDA;
                    r->done = true;
                }
                sl.reqs.clear();
                sl.busy = false;
                s->cv_done.notify_all();
                progressed = true;
            } else {
                any_busy = true;
            }
        }
        for (ServerSlot &sl : s->slots) {
            if (sl.busy || s->pending.empty()) continue;
            // Admission in arrival order while the batch's slots and memory budgets hold.
            uint64_t prof = 0, sco = 0;
            while (!s->pending.empty() && sl.reqs.size() < s->cfg.max_batch) {
                ServerRequest *r = s->pending.front();
                if (prof + r->prof_bytes > s->cfg.profile_budget || sco + r->score_bytes > s->cfg.scores_budget)
                    break;
                prof += r->prof_bytes;
                sco += r->score_bytes;
                sl.reqs.push_back(r);
                s->pending.pop_front();
            }
            if (sl.reqs.empty()) continue;
            sl.busy = true;
            ++s->batches;
            s->batched += sl.reqs.size();
            lk.unlock();
            const hy_status st = launch_slot(s, sl);
            lk.lock();
            if (st != HY_OK) {
                for (ServerRequest *r : sl.reqs) {
                    r->status = st;
                    r->done = true;
                }
                sl.reqs.clear();
                sl.busy = false;
                s->cv_done.notify_all();
            } else {
                any_busy = true;
            }
            progressed = true;
        }
        if (s->stopping && s->pending.empty() && !any_busy) break;
        if (!progressed) {
            if (any_busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lk.lock();
            } else {
                s->cv_work.wait(lk, [&] { return s->stopping || !s->pending.empty(); });
            }
        }
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t lo = (size_t)pos;
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

extern "C" {

hy_status hy_server_create(const hy_db *const *dbs, uint32_t n_dbs, const hy_server_config *config,
                           hy_server **out) {
    if (!dbs || n_dbs == 0 || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    for (uint32_t i = 0; i < n_dbs; ++i)
        if (!dbs[i] || dbs[i]->device != dbs[0]->device) return fail(HY_ERR_INVALID_ARGUMENT, i);
    hy_server *s = new hy_server();
    s->device = dbs[0]->device;
    s->dbs.assign(dbs, dbs + n_dbs);
    uint64_t n_max = 0;
    for (const hy_db *db : s->dbs) {
        s->db_residues.push_back((double)db->p16.res_prefix.back());
        n_max = std::max(n_max, db->n_seqs);
    }
    hy_server_config c{};
    if (config) c = *config;
    if (c.max_batch == 0) c.max_batch = 64;
    if (c.in_flight == 0) c.in_flight = 2;
    if (c.max_pending == 0) c.max_pending = 4096;
    if (c.scores_budget == 0) c.scores_budget = (uint64_t)c.max_batch * n_max * sizeof(int32_t);
    s->cfg = c;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    hy_status st = HY_OK;
    s->slots.resize(c.in_flight);
    for (ServerSlot &sl : s->slots) {
        st = batch_create(dbs, n_dbs, c.max_batch, c.profile_budget, false, &sl.b);
        if (st != HY_OK) break;
        if (c.launch_config[2] != 0) {
            sl.b->cfg.rows8_max = c.launch_config[0];
            sl.b->cfg.rows16_max = c.launch_config[1];
            sl.b->cfg.long_w = (uint32_t)std::min<int32_t>(std::max<int32_t>(c.launch_config[2], 1), 4096);
        }
        if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            hy::dev_malloc(&sl.d_scores, std::max<uint64_t>(c.scores_budget, 16)) != cudaSuccess ||
            cudaMallocHost(&sl.h_scores, std::max<uint64_t>(c.scores_budget, 16)) != cudaSuccess) {
            cudaGetLastError();
            st = fail(HY_ERR_OUT_OF_MEMORY);
            break;
        }
    }
    if (st == HY_OK) s->cfg.profile_budget = s->slots[0].b->prof_cap;
    if (st != HY_OK) {
        int64_t d[3];
        hy_last_error_detail(d);
        free_slots(s);
        if (prev >= 0) cudaSetDevice(prev);
        delete s;
        return fail(st, d[0], d[1], d[2]);
    }
    if (prev >= 0) cudaSetDevice(prev);
    s->worker = std::thread(worker_main, s);
    *out = s;
    return fail(HY_OK);
}

void hy_server_destroy(hy_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    free_slots(s);
    if (prev >= 0) cudaSetDevice(prev);
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
}

hy_status hy_server_submit(hy_server *s, uint32_t db, const uint8_t *query, uint64_t qlen,
                           int want_scores, int32_t *scores_out, uint64_t *id) {
    if (!s || !id || db >= s->dbs.size() || (qlen && !query) || (want_scores && !scores_out))
        return fail(HY_ERR_INVALID_ARGUMENT);
    const hy_db *d = s->dbs[db];
    if (qlen > d->mql) return fail(HY_ERR_QUERY_TOO_LONG, (int64_t)qlen, (int64_t)d->mql);
    for (uint64_t k = 0; k < qlen; ++k)
        if (query[k] >= d->al) return fail(HY_ERR_SYMBOL_OUT_OF_RANGE, query[k], (int64_t)d->al);
    ServerRequest *r = new ServerRequest();
    r->db = db;
    r->q.assign(query, query + qlen);
    r->want_scores = want_scores != 0;
    r->scores_out = scores_out;
    r->prof_bytes = batch_profile_bytes(s->slots[0].b, d, qlen, !r->want_scores);
    r->score_bytes = r->want_scores ? d->n_seqs * sizeof(int32_t) : 0;
    r->cells = (double)qlen * s->db_residues[db];
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stopping || s->pending.size() >= s->cfg.max_pending ||
        r->prof_bytes > s->cfg.profile_budget || r->score_bytes > s->cfg.scores_budget) {
        ++s->rejected;
        delete r;
        return fail(HY_ERR_REJECTED);
    }
    r->id = s->next_id++;
    r->t_submit = Clock::now();
    if (!s->have_t0) {
        s->t0 = r->t_submit;
        s->have_t0 = true;
    }
    ++s->submitted;
    s->reqs[r->id] = r;
    s->pending.push_back(r);
    *id = r->id;
    lk.unlock();
    s->cv_work.notify_one();
    return fail(HY_OK);
}

uint64_t hy_server_request_bytes(const hy_server *s, uint32_t db, uint64_t qlen, int want_scores,
                                 uint64_t *score_bytes) {
    if (!s || db >= s->dbs.size()) return 0;
    const hy_db *d = s->dbs[db];
    const uint64_t sb = want_scores ? d->n_seqs * sizeof(int32_t) : 0;
    if (score_bytes) *score_bytes = sb;
    return batch_profile_bytes(s->slots[0].b, d, qlen, want_scores == 0);
}

hy_status hy_server_poll(hy_server *s, uint64_t id, int *done) {
    if (!s || !done) return fail(HY_ERR_INVALID_ARGUMENT);
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(HY_ERR_INVALID_ARGUMENT);
    *done = it->second->done ? 1 : 0;
    return fail(HY_OK);
}

hy_status hy_server_wait(hy_server *s, uint64_t id, double timeout_s, hy_hit *out) {
    return hy_server_wait_timed(s, id, timeout_s, out, nullptr);
}

hy_status hy_server_wait_timed(hy_server *s, uint64_t id, double timeout_s, hy_hit *out, double *latency_ms) {
    if (!s) return fail(HY_ERR_INVALID_ARGUMENT);
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(HY_ERR_INVALID_ARGUMENT);
    ServerRequest *r = it->second;
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(std::max(0.0, timeout_s)));
    if (!s->cv_done.wait_until(lk, deadline, [&] { return r->done; })) return fail(HY_ERR_TIMEOUT);
    const hy_status st = r->status;
    if (out) *out = r->hit;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    s->reqs.erase(it);
    delete r;
    return fail(st);
}

hy_status hy_server_stats_read(hy_server *s, int reset, hy_server_stats *out) {
    if (!s || !out) return fail(HY_ERR_INVALID_ARGUMENT);
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->batches = s->batches;
    out->mean_batch = s->batches ? (double)s->batched / (double)s->batches : 0.0;
    out->p50_ms = percentile(s->lat_ms, 0.50);
    out->p99_ms = percentile(s->lat_ms, 0.99);
    out->max_ms = s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end());
    double sum = 0.0;
    for (double v : s->lat_ms) sum += v;
    out->mean_ms = s->lat_ms.empty() ? 0.0 : sum / (double)s->lat_ms.size();
    out->cells = s->cells;
    out->seconds = (s->have_t0 && s->completed) ? std::chrono::duration<double>(s->t_last - s->t0).count() : 0.0;
    out->gcups = out->seconds > 0 ? s->cells / out->seconds / 1e9 : 0.0;
    out->pending = s->pending.size();
    if (reset) {
        s->lat_ms.clear();
        s->submitted = s->completed = s->rejected = s->batches = s->batched = 0;
        s->cells = 0.0;
        s->have_t0 = false;
    }
    return fail(HY_OK);
}

}  // extern "C"
