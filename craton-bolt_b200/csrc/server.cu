// server.cu — continuous-batching request loop for filter + GROUP BY queries.
//
// No counterpart in the reference: its Engine runs one query at a time on
// one synchronous stream (src/exec/launch.rs:308-368). Here:
//   * `n_lanes` worker threads, each owning a bolt_ctx (scratch arena) and a
//     CUDA stream, so batches on different lanes overlap on the device;
//   * a queue of submitted queries; an idle lane admits a large query at
//     the head alone, else small queries in arrival order while their summed
//     HBM footprint (bolt_groupby_footprint) fits its share of the budget,
//     their summed rows stay below a work cap and the batch is below
//     `max_batch`;
//   * the lane runs its batch as one bolt_batch_groupby call (one persistent
//     aggregation launch + one batched finalize) and completes the tickets;
//   * queries that arrive while lanes are busy wait only until some lane
//     frees, then join the next batch (continuous batching).
// Results are identical alone or in any mix: every accumulator is order-
// independent (integer states, fixed-point float sums).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ctx.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    bolt_query* q = nullptr;
    uint64_t ticket = 0;
    uint64_t footprint = 0;
    Clock::time_point t_submit, t_done;
    bool done = false;
    bolt_status st = BOLT_OK;
};

}  // namespace

struct bolt_server {
    bolt_server_config cfg{};
    std::vector<bolt_ctx*> ctx;
    std::vector<cudaStream_t> streams;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> queue;
    std::unordered_map<uint64_t, Req*> reqs;
    uint64_t next_ticket = 1;
    uint64_t lane_budget = 0;
    uint64_t n_big = 0;  // queued queries of at least BIG_QUERY_ROWS rows
    bool stop = false;
};

namespace {

uint64_t query_rows(const bolt_query* q) { return q->row_end > q->row_begin ? q->row_end - q->row_begin : 0; }

// Queries with at least this many rows are admitted alone, and a batch of
// smaller ones holds at most BATCH_ROWS_MAX rows (a few milliseconds of
// device work), which bounds how long a query waits for its batch.
constexpr uint64_t BIG_QUERY_ROWS = 4ull << 20;
constexpr uint64_t BATCH_ROWS_MAX = 32ull << 20;

void lane_loop(bolt_server* srv, int lane) {
    cudaSetDevice(srv->cfg.device);
    bolt_ctx* ctx = srv->ctx[lane];
    cudaStream_t s = srv->streams[lane];
    std::vector<Req*> batch;
    std::vector<bolt_query> qs;
    for (;;) {
        batch.clear();
        {
            // The first half of the lanes serve the large queries (at most
            // that many run at once, so they do not all stretch each other's
            // tail latency) and small ones when none is queued; the other
            // lanes serve only small queries. With one lane it goes by arrival.
            const bool big_lane = lane < std::max(1, srv->cfg.n_lanes / 2);
            const bool solo = srv->cfg.n_lanes == 1;
            std::unique_lock<std::mutex> lk(srv->mu);
            srv->cv_work.wait(lk, [&] {
                return srv->stop || (big_lane ? !srv->queue.empty() : srv->queue.size() > srv->n_big);
            });
            if (big_lane ? srv->queue.empty() : srv->queue.size() <= srv->n_big) return;  // stopping
            Req* big = nullptr;
            if (big_lane && srv->n_big > 0 &&
                (!solo || query_rows(srv->queue.front()->q) >= BIG_QUERY_ROWS)) {
                for (auto it = srv->queue.begin(); it != srv->queue.end(); ++it)
                    if (query_rows((*it)->q) >= BIG_QUERY_ROWS) {
                        big = *it;
                        srv->queue.erase(it);
                        --srv->n_big;
                        break;
                    }
            }
            if (big) {
                batch.push_back(big);
            } else {
                // Small queries in arrival order (passing over large ones),
                // while the summed footprint fits the lane's share and the
                // summed rows the work cap.
                uint64_t used = 0, rows = 0;
                std::deque<Req*> rest;
                while (!srv->queue.empty()) {
                    Req* r = srv->queue.front();
                    srv->queue.pop_front();
                    const uint64_t qr = query_rows(r->q);
                    const bool take = qr < BIG_QUERY_ROWS && (int)batch.size() < srv->cfg.max_batch &&
                                      (batch.empty() || (used + r->footprint <= srv->lane_budget &&
                                                         rows + qr <= BATCH_ROWS_MAX));
                    if (take) {
                        used += r->footprint;
                        rows += qr;
                        batch.push_back(r);
                    } else {
                        rest.push_back(r);
                    }
                }
                srv->queue.swap(rest);
            }
        }
        if (!srv->queue.empty()) srv->cv_work.notify_all();
        qs.resize(batch.size());
        for (size_t i = 0; i < batch.size(); ++i) qs[i] = *batch[i]->q;
        const bolt_status st = bolt_batch_groupby(ctx, qs.data(), (int32_t)qs.size(), 0, (bolt_stream)s);
        const auto now = Clock::now();
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            for (size_t i = 0; i < batch.size(); ++i) {
                Req* r = batch[i];
                r->q->out.n_groups = qs[i].out.n_groups;
                r->q->status = qs[i].status;
                r->st = (st == BOLT_OK || qs[i].status != BOLT_OK) ? qs[i].status : st;
                r->t_done = now;
                r->done = true;
            }
        }
        srv->cv_done.notify_all();
    }
}

}  // namespace

using namespace bolt;

extern "C" bolt_status bolt_server_create(const bolt_server_config* cfg, bolt_server** out) {
    if (!cfg || !out) return BOLT_ERR_INVALID;
    *out = nullptr;
    bolt_server* srv = new bolt_server();
    srv->cfg = *cfg;
    if (srv->cfg.n_lanes < 1) srv->cfg.n_lanes = 2;
    if (srv->cfg.max_batch < 1) srv->cfg.max_batch = 256;
    if (cudaSetDevice(cfg->device) != cudaSuccess) {
        delete srv;
        return BOLT_ERR_CUDA;
    }
    uint64_t total = cfg->scratch_bytes;
    if (total == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        total = (uint64_t)fr / 2;
    }
    const uint64_t per_lane = total / (uint64_t)srv->cfg.n_lanes;
    srv->lane_budget = per_lane - per_lane / 8;  // headroom for finalize scratch
    for (int i = 0; i < srv->cfg.n_lanes; ++i) {
        bolt_ctx* c = nullptr;
        bolt_status st = bolt_ctx_create(cfg->device, per_lane, &c);
        cudaStream_t s = nullptr;
        // The large-query lanes get the highest stream priority: their
        // blocks are scheduled first as SMs free up, so a large query runs
        // at close to its solo speed while the small batches fill in.
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        const int prio = (i < std::max(1, srv->cfg.n_lanes / 2) && srv->cfg.n_lanes > 1) ? hi : lo;
        if (st != BOLT_OK || cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio) != cudaSuccess) {
            if (c) bolt_ctx_destroy(c);
            bolt_server_destroy(srv);
            return st != BOLT_OK ? st : BOLT_ERR_CUDA;
        }
        srv->ctx.push_back(c);
        srv->streams.push_back(s);
    }
    for (int i = 0; i < srv->cfg.n_lanes; ++i) srv->workers.emplace_back(lane_loop, srv, i);
    *out = srv;
    return BOLT_OK;
}

extern "C" bolt_status bolt_server_submit(bolt_server* srv, bolt_query* q, uint64_t* ticket) {
    if (!srv || !q || !ticket) return BOLT_ERR_INVALID;
    Req* r = new Req();
    r->q = q;
    r->footprint = bolt_groupby_footprint(&q->desc, query_rows(q));
    if (r->footprint > srv->lane_budget) {
        delete r;
        return BOLT_ERR_CAPACITY;
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        r->ticket = srv->next_ticket++;
        srv->reqs[r->ticket] = r;
        srv->queue.push_back(r);
        if (query_rows(q) >= BIG_QUERY_ROWS) ++srv->n_big;
    }
    *ticket = r->ticket;
    srv->cv_work.notify_all();
    return BOLT_OK;
}

// A burst of queries enqueued under one lock and announced once, so the
// lanes see it whole and form full batches (one call per query lets the
// lanes drain the queue as the queries trickle in, a few at a time).
extern "C" bolt_status bolt_server_submit_batch(bolt_server* srv, bolt_query* qs, int32_t n, uint64_t* tickets) {
    if (!srv || n < 0 || (n > 0 && (!qs || !tickets))) return BOLT_ERR_INVALID;
    std::vector<Req*> rs((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        Req* r = new Req();
        r->q = &qs[i];
        r->footprint = bolt_groupby_footprint(&qs[i].desc, query_rows(&qs[i]));
        if (r->footprint > srv->lane_budget) {
            delete r;
            for (int32_t j = 0; j < i; ++j) delete rs[(size_t)j];
            return BOLT_ERR_CAPACITY;
        }
        rs[(size_t)i] = r;
    }
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        for (int32_t i = 0; i < n; ++i) {
            Req* r = rs[(size_t)i];
            r->t_submit = now;
            r->ticket = srv->next_ticket++;
            srv->reqs[r->ticket] = r;
            srv->queue.push_back(r);
            if (query_rows(r->q) >= BIG_QUERY_ROWS) ++srv->n_big;
            tickets[i] = r->ticket;
        }
    }
    srv->cv_work.notify_all();
    return BOLT_OK;
}

extern "C" bolt_status bolt_server_wait(bolt_server* srv, uint64_t ticket, double* latency_us) {
    if (!srv) return BOLT_ERR_INVALID;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return BOLT_ERR_INVALID;
    Req* r = it->second;
    srv->cv_done.wait(lk, [&] { return r->done; });
    if (latency_us) latency_us[0] = std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count();
    const bolt_status st = r->st;
    srv->reqs.erase(it);
    delete r;
    return st;
}

extern "C" void bolt_server_destroy(bolt_server* srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    for (auto& t : srv->workers)
        if (t.joinable()) t.join();
    for (auto s : srv->streams) cudaStreamDestroy(s);
    for (auto c : srv->ctx) bolt_ctx_destroy(c);
    for (auto& kv : srv->reqs) delete kv.second;
    delete srv;
}
