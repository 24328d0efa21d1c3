// xm_serve.cu -- resident catalog, continuous batching of query catalogs.
//
// The reference runs one catalog pair per process (_main,
// BoostXmatch.cpp:247-330: load, sort, match, exit).  Here a server keeps
// the catalog segment resident and answers a stream of query catalogs:
//
//   submit    copies the query records into a host queue entry (ticket)
//   builder   host thread with its own context (stream, memory pool): admits
//             queued queries in order while their estimated device bytes fit
//             the budget, zone-builds each on the device
//   matcher   host thread on the caller's context: takes every built query
//             (up to max_batch) as one batch of jobs (query = A, catalog = B),
//             one persistent pair-kernel launch, groups the matches by query,
//             copies them to the host, releases the memory reservation
//
// A query that arrives while a batch is on the GPU is admitted and built on
// the builder's stream while that batch runs, and joins the next batch.  The
// pair set of a query does not depend on its batch: each job is matched by the
// same kernel over the same two segments as xm_match.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "xm_internal.h"

namespace {

enum QState { Q_QUEUED, Q_ADMITTED, Q_BUILT, Q_DONE, Q_FAILED };

struct Query {
    uint64_t ticket = 0;
    std::vector<xm_obj> objs;
    double sr_deg = 0;
    uint64_t bytes = 0;            // reserved device bytes while in flight
    xm_segment *seg = nullptr;
    QState state = Q_QUEUED;
    xm_status err = XM_OK;
    std::string msg;
    std::vector<int64_t> pairs;    // 2 per match
    std::vector<double> dist;
    xm_serve_info info{};
};

using QPtr = std::shared_ptr<Query>;

}  // namespace

struct xm_server {
    xm_ctx *mctx = nullptr;        // caller's context: matching
    xm_ctx *bctx = nullptr;        // own context: query builds
    const xm_segment *cat = nullptr;
    xm_serve_cfg cfg{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<QPtr> queue;        // submitted, not admitted
    std::deque<QPtr> ready;        // built, waiting for a batch
    std::vector<xm_segment *> garbage;   // matched query segments, freed by the builder
    std::unordered_map<uint64_t, QPtr> tickets;
    uint64_t next_ticket = 1;
    uint64_t in_flight = 0;        // reserved bytes of admitted queries
    uint32_t n_batches = 0;
    std::string last_error;        // message of the last failed query polled (guarded by mu)
    bool stop = false, builder_done = false;
    std::thread builder, matcher;
    std::vector<int64_t> hp;       // host staging of a batch's pairs
    std::vector<double> hd;

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// Device bytes a query holds while in flight: its segment (40 B per object:
// id, ra/dec, FP32 unit vector; and the zone offsets) and room for 2 n matches
// (16 B pairs, 8 B distance, 4 B job index), the default output size of
// Worker.cu:296-297.
uint64_t query_bytes(uint64_t n, int32_t n_zones)
{
    return 40 * n + 4 * ((uint64_t)n_zones + 8) + 28 * std::max<uint64_t>(2 * n, 1024);
}

void builder_loop(xm_server *S)
{
    for (;;) {
        QPtr q;
        std::vector<xm_segment *> trash;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [&] {
                if (!S->garbage.empty()) return true;
                if (S->queue.empty()) return S->stop;
                return S->in_flight == 0 || S->in_flight + S->queue.front()->bytes <= S->cfg.mem_budget;
            });
            trash.swap(S->garbage);
            if (!S->queue.empty() &&
                (S->in_flight == 0 || S->in_flight + S->queue.front()->bytes <= S->cfg.mem_budget)) {
                q = S->queue.front();
                S->queue.pop_front();
                S->in_flight += q->bytes;
                q->state = Q_ADMITTED;
                q->info.t_admit_ms = S->now_ms();
            } else if (S->queue.empty() && S->stop && trash.empty()) {
                S->builder_done = true;
                S->cv.notify_all();
                return;
            }
        }
        for (xm_segment *g : trash) xm_segment_free(g);
        if (!q) continue;
        xm_segment *seg = nullptr;
        xm_status rc = xm_segment_build(S->bctx, (uint32_t)q->ticket, q->objs.data(), q->objs.size(), S->cat->zh_deg,
                                        &seg, nullptr);
        std::lock_guard<std::mutex> lk(S->mu);
        q->objs.clear();
        q->objs.shrink_to_fit();
        if (rc != XM_OK) {
            q->state = Q_FAILED;
            q->err = rc;
            q->msg = xm_last_error(S->bctx);
            q->info.t_done_ms = S->now_ms();
            S->in_flight -= q->bytes;
        } else {
            q->seg = seg;
            q->state = Q_BUILT;
            q->info.t_built_ms = S->now_ms();
            S->ready.push_back(q);
        }
        S->cv.notify_all();
    }
}

void matcher_loop(xm_server *S)
{
    for (;;) {
        std::vector<QPtr> batch;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv.wait(lk, [&] { return !S->ready.empty() || S->builder_done; });
            if (S->ready.empty() && S->builder_done) return;
            const double t = S->now_ms();
            while (!S->ready.empty() && batch.size() < S->cfg.max_batch) {
                batch.push_back(S->ready.front());
                S->ready.pop_front();
                batch.back()->info.t_batch_ms = t;
            }
        }
        const uint32_t nb = (uint32_t)batch.size();
        std::vector<xm_job> jobs(nb);
        for (uint32_t j = 0; j < nb; ++j) jobs[j] = {batch[j]->seg, S->cat, batch[j]->sr_deg};
        xm_ctx *ctx = S->mctx;
        const bool dist = (S->cfg.flags & XM_NO_DIST) == 0;
        xm_status rc = xm_run_jobs(ctx, jobs.data(), nb, S->cfg.flags, nullptr, nb > 1, nullptr, nullptr);
        uint32_t launches = 0;
        if (rc == XM_OK) {
            if (nb > 1) {
                rc = xm_group_by_job(ctx, nb, &launches);
            } else {
                ctx->res.job_off = {0ull, (uint64_t)ctx->res.count};
                ctx->res.grouped = false;
            }
        }
        const double t_matched = S->now_ms();
        uint64_t total = 0;
        if (rc == XM_OK) {
            total = ctx->res.count;
            const int64_t *P = ctx->res.grouped ? ctx->res.pairs_g : ctx->res.pairs;
            const double *D = ctx->res.grouped ? ctx->res.dist_g : ctx->res.dist;
            if (S->hp.size() < 2 * total) S->hp.resize(2 * total);
            if (dist && S->hd.size() < total) S->hd.resize(total);
            cudaError_t e = cudaSuccess;
            if (total) e = cudaMemcpyAsync(S->hp.data(), P, total * 16, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess && total && dist)
                e = cudaMemcpyAsync(S->hd.data(), D, total * 8, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) {
                ctx->last_error = cudaGetErrorString(e);
                rc = XM_ERR_CUDA;
            }
        }
        std::lock_guard<std::mutex> lk(S->mu);
        const uint32_t b = S->n_batches++;
        const double t = S->now_ms();
        for (uint32_t j = 0; j < nb; ++j) {
            Query &q = *batch[j];
            if (rc == XM_OK) {
                const uint64_t o = ctx->res.job_off[j], c = ctx->res.job_off[j + 1] - o;
                q.pairs.assign(S->hp.begin() + 2 * o, S->hp.begin() + 2 * (o + c));
                if (dist) q.dist.assign(S->hd.begin() + o, S->hd.begin() + o + c);
                q.info.count = c;
                q.state = Q_DONE;
            } else {
                q.state = Q_FAILED;
                q.err = rc;
                q.msg = ctx->last_error;
            }
            q.info.batch = b;
            q.info.batch_size = nb;
            q.info.t_matched_ms = t_matched;
            q.info.t_done_ms = t;
            S->in_flight -= q.bytes;
            S->garbage.push_back(q.seg);
            q.seg = nullptr;
        }
        S->cv.notify_all();
    }
}

}  // namespace

extern "C" xm_status xm_serve_open(xm_ctx *ctx, const xm_segment *catalog, const xm_serve_cfg *cfg, xm_server **out)
{
    if (!ctx || !catalog || !out || catalog->ctx->device != ctx->device) return XM_ERR_INVALID;
    *out = nullptr;
    if (!catalog->store) {
        ctx->last_error = "the catalog segment is offloaded (xm_segment_page_in it first)";
        return XM_ERR_INVALID;
    }
    cudaSetDevice(ctx->device);
    auto *S = new xm_server();
    S->mctx = ctx;
    S->cat = catalog;
    if (cfg) S->cfg = *cfg;
    if (!S->cfg.max_batch) S->cfg.max_batch = 1024;
    if (!S->cfg.mem_budget) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete S;
            return XM_ERR_CUDA;
        }
        S->cfg.mem_budget = fr / 2;
    }
    xm_status rc = xm_ctx_create(ctx->device, &S->bctx);
    if (rc != XM_OK) {
        delete S;
        return rc;
    }
    S->t0 = std::chrono::steady_clock::now();
    S->builder = std::thread([S] {
        cudaSetDevice(S->bctx->device);
        builder_loop(S);
    });
    S->matcher = std::thread([S] {
        cudaSetDevice(S->mctx->device);
        matcher_loop(S);
    });
    *out = S;
    return XM_OK;
}

extern "C" xm_status xm_serve_submit(xm_server *S, const xm_obj *objs, uint64_t n, double sr_deg, uint64_t *ticket)
{
    if (!S || !ticket || (n && !objs) || !(sr_deg > 0)) return XM_ERR_INVALID;
    auto q = std::make_shared<Query>();
    q->objs.assign(objs, objs + n);
    q->sr_deg = sr_deg;
    q->bytes = query_bytes(n, S->cat->n_zones);
    std::lock_guard<std::mutex> lk(S->mu);
    if (q->bytes > S->cfg.mem_budget) return XM_ERR_TOO_LARGE;
    if (S->stop) return XM_ERR_INVALID;
    q->ticket = S->next_ticket++;
    q->info.t_submit_ms = S->now_ms();
    S->tickets[q->ticket] = q;
    S->queue.push_back(q);
    *ticket = q->ticket;
    S->cv.notify_all();
    return XM_OK;
}

extern "C" xm_status xm_serve_poll(xm_server *S, uint64_t ticket, int wait, xm_pairs *out, xm_serve_info *info)
{
    if (!S) return XM_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->tickets.find(ticket);
    if (it == S->tickets.end()) return XM_ERR_INVALID;
    QPtr q = it->second;
    auto finished = [&] { return q->state == Q_DONE || q->state == Q_FAILED; };
    if (!finished()) {
        if (!wait) return XM_ERR_BUSY;
        S->cv.wait(lk, finished);
    }
    if (info) *info = q->info;
    if (q->state == Q_FAILED) {
        S->last_error = q->msg;   // the matcher thread owns mctx; the text is kept per server
        S->tickets.erase(it);
        return q->err;
    }
    const uint64_t c = q->info.count;
    if (!out || (!out->pairs && !out->dist)) {   // count only; the result is kept
        if (out) out->count = c;
        return XM_OK;
    }
    out->count = c;
    if (out->capacity < c) return XM_ERR_CAPACITY;
    if (out->dist && c && q->dist.size() < c) return XM_ERR_INVALID;   // served with XM_NO_DIST
    if (out->pairs && c) std::memcpy(out->pairs, q->pairs.data(), c * 16);
    if (out->dist && c) std::memcpy(out->dist, q->dist.data(), c * 8);
    S->tickets.erase(it);
    return XM_OK;
}

extern "C" xm_status xm_serve_last_error(xm_server *S, char *buf, uint64_t cap)
{
    if (!S || !buf || cap == 0) return XM_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    const size_t n = std::min<size_t>(S->last_error.size(), (size_t)cap - 1);
    std::memcpy(buf, S->last_error.data(), n);
    buf[n] = 0;
    return XM_OK;
}

extern "C" xm_status xm_serve_close(xm_server *S)
{
    if (!S) return XM_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    S->builder.join();
    S->matcher.join();
    for (xm_segment *g : S->garbage) xm_segment_free(g);
    for (auto &kv : S->tickets)
        if (kv.second->seg) xm_segment_free(kv.second->seg);
    xm_ctx_destroy(S->bctx);
    delete S;
    return XM_OK;
}
