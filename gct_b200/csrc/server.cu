// Serving loop with continuous batching (include/gct_fdk.h, gct_fdk_server_*).
//
// One worker thread per server drives four streams: uploads, filter stages, backprojection
// rounds and downloads. Admission is first-come first-served against a device memory budget
// reserved once (Arena) and a cap on admitted requests. Each backprojection round is one launch
// of the work-queue kernel (per storage type and depth class) over the tiles of every active
// request, each
// request contributing its next chunk of views; chunk 0 overwrites the volume and later chunks
// add to it in view order, so a result does not depend on which other requests share the rounds.
// Two rounds are in flight at most (double-buffered work lists in pinned host memory).
//
// No counterpart in the reference (one synchronous reconstruction per call,
// src/cuda/recon/recon_wrappers.cuh:15-43).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "arena.hpp"
#include "plan.hpp"
#include "queue.hpp"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
    void reserve(size_t n)
    {
        if (n <= bytes) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        cuda_check(cudaMallocHost(&p, n), "pinned work list");
        bytes = n;
    }
};

struct Request {
    uint64_t ticket = 0;
    gct_fdk_plan *plan = nullptr;
    const float *proj_host = nullptr;
    float *vol_host = nullptr;
    size_t proj_bytes = 0, vol_bytes = 0, block_bytes = 0;
    size_t block = SIZE_MAX;  // arena offset
    float *proj_dev = nullptr, *vol_dev = nullptr;
    StackRef st;
    gct::TileConfig cfg;
    int chunk = 0, next_view = 0;  // views per round and the next view (base views for quarter-turn stacks)
    uint32_t rounds = 0;
    gct_req_state state = GCT_REQ_QUEUED;
    gct_status status = GCT_OK;
    Clock::time_point t_submit, t_admit, t_done;
    cudaEvent_t e_in = nullptr, e_prep = nullptr, e_out = nullptr;

    ~Request()
    {
        for (cudaEvent_t e : {e_in, e_prep, e_out})
            if (e) cudaEventDestroy(e);
    }
};

}  // namespace

struct gct_fdk_server {
    int device = 0, num_sms = 148;
    uint32_t max_active = 64;
    bool autotune = false;
    double round_updates = 2e9;
    DevBuf<unsigned char> budget;
    gct::Arena arena;
    cudaStream_t s_in = nullptr, s_prep = nullptr, s_bp = nullptr, s_out = nullptr;
    int grid[2 * gct::kQueueClasses] = {};

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stopping = false;
    bool failed = false;
    std::string fail_msg;
    uint64_t next_ticket = 1;
    std::deque<Request *> queued;                         // guarded by mu
    std::map<uint64_t, std::unique_ptr<Request>> table;   // guarded by mu (requests stay until destroy)
    std::vector<double> latencies;                        // guarded by mu
    uint64_t n_submitted = 0, n_completed = 0, n_failed = 0, n_cancelled = 0, n_rejected = 0, n_rounds = 0;
    uint32_t peak_active = 0;
    Clock::time_point t_first_submit, t_last_done;
    bool any_submit = false;

    // worker-only state (admit() reads the sizes under mu)
    std::vector<Request *> preparing, active, draining;
    struct Slot {
        DevBuf<gct::BpItem> items;
        DevBuf<gct::BpWork> work;
        DevBuf<int> counters;
        PinnedBuf h_items, h_work;
        cudaEvent_t done = nullptr;
        bool used = false;
    } slot[2];
    uint64_t round = 0;
    std::thread worker;

    ~gct_fdk_server()
    {
        for (auto &s : slot)
            if (s.done) cudaEventDestroy(s.done);
        for (cudaStream_t s : {s_in, s_prep, s_bp, s_out})
            if (s) cudaStreamDestroy(s);
    }
};

namespace {

size_t footprint(const gct_fdk_plan *p, size_t *proj_bytes, size_t *vol_bytes)
{
    *proj_bytes = sizeof(float) * static_cast<size_t>(p->nv) * p->nr * p->nc;
    *vol_bytes = sizeof(float) * static_cast<size_t>(p->vol.nx) * p->vol.ny * p->vol.nz;
    return gct::Arena::round_up(*proj_bytes) + gct::Arena::round_up(p->workspace_bytes()) +
           gct::Arena::round_up(*vol_bytes);
}

// Views per round of a request: about round_updates voxel-view updates, at least 16 views.
// Views per round (at least 16) for about round_updates voxel-view updates; for a quarter-turn
// stack the views of a round are base views, each worth four.
int chunk_views(const gct_fdk_plan *p, const StackRef &st, double round_updates)
{
    const double vox = static_cast<double>(p->vol.nx) * p->vol.ny * p->vol.nz * (st.quarter ? 4 : 1);
    const double v = std::floor(round_updates / std::max(vox, 1.0));
    const int views = gct::item_views(p, st);
    return static_cast<int>(std::max(st.quarter ? 4.0 : 16.0, std::min(static_cast<double>(views), v)));
}

void finish(gct_fdk_server *s, Request *r, gct_req_state state, gct_status status)
{
    // caller holds s->mu
    r->state = state;
    r->status = status;
    r->t_done = Clock::now();
    if (r->block != SIZE_MAX) {
        s->arena.release(r->block);
        r->block = SIZE_MAX;
    }
    if (state == GCT_REQ_DONE) {
        ++s->n_completed;
        s->latencies.push_back(ms_between(r->t_submit, r->t_done));
        s->t_last_done = r->t_done;
    } else if (state == GCT_REQ_FAILED) {
        ++s->n_failed;
    } else if (state == GCT_REQ_CANCELLED) {
        ++s->n_cancelled;
    }
    s->cv_done.notify_all();
}

// Admission: first-come first-served while the head request fits in the budget.
std::vector<Request *> admit(gct_fdk_server *s)
{
    std::vector<Request *> out;
    std::lock_guard<std::mutex> lock(s->mu);
    const size_t inflight = s->preparing.size() + s->active.size() + s->draining.size();
    while (!s->queued.empty() && inflight + out.size() < s->max_active) {
        Request *r = s->queued.front();
        const size_t off = s->arena.alloc(r->block_bytes);
        if (off == SIZE_MAX) break;
        s->queued.pop_front();
        r->block = off;
        r->state = GCT_REQ_RUNNING;
        r->t_admit = Clock::now();
        out.push_back(r);
    }
    s->peak_active = std::max<uint32_t>(s->peak_active, static_cast<uint32_t>(inflight + out.size()));
    return out;
}

void start(gct_fdk_server *s, Request *r)
{
    unsigned char *base = s->budget.p + r->block;
    r->proj_dev = reinterpret_cast<float *>(base);
    unsigned char *ws = base + gct::Arena::round_up(r->proj_bytes);
    r->vol_dev = reinterpret_cast<float *>(ws + gct::Arena::round_up(r->plan->workspace_bytes()));
    // quarter-turn plans keep their interleaved partner stacks (the quarter-turn queue class)
    r->st = stack_of(r->plan, ws, false);
    for (cudaEvent_t *e : {&r->e_in, &r->e_prep, &r->e_out})
        cuda_check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "request event");
    cuda_check(cudaMemcpyAsync(r->proj_dev, r->proj_host, r->proj_bytes, cudaMemcpyHostToDevice, s->s_in),
               "projection upload");
    cuda_check(cudaEventRecord(r->e_in, s->s_in), "event record");
    cuda_check(cudaStreamWaitEvent(s->s_prep, r->e_in, 0), "stream wait");
    if (r->st.quarter) prepare_partners(r->plan, r->proj_dev, r->st, 0, r->st.quarter, s->s_prep);
    else prepare(r->plan, r->proj_dev, r->st, 0, r->plan->nv, s->s_prep);
    cuda_check(cudaEventRecord(r->e_prep, s->s_prep), "event record");
    r->chunk = chunk_views(r->plan, r->st, s->round_updates);
}

void activate(gct_fdk_server *s, Request *r)
{
    cuda_check(cudaStreamWaitEvent(s->s_bp, r->e_prep, 0), "stream wait");
    r->cfg = s->autotune ? gct::autotune(r->plan, r->st, r->vol_dev, s->num_sms, s->s_bp).cfg
                         : gct::default_config(r->plan, r->st.quarter > 0);
    s->active.push_back(r);
}

// One backprojection round over the next view chunk of every active request.
void run_round(gct_fdk_server *s)
{
    auto &sl = s->slot[s->round % 2];
    if (sl.used) cuda_check(cudaEventSynchronize(sl.done), "round slot");
    constexpr int NQ = 2 * gct::kQueueClasses;  // index storage * kQueueClasses + depth class
    std::vector<gct::BpItem> items[NQ];
    std::vector<gct::BpWork> work[NQ];
    std::vector<std::pair<Request *, int>> advanced;
    for (Request *r : s->active) {
        const int q = (r->plan->opts.storage == GCT_STORAGE_F16 ? 1 : 0) * gct::kQueueClasses +
                      gct::item_class(r->st, r->cfg);
        const int vb = r->next_view, vc = std::min(r->chunk, gct::item_views(r->plan, r->st) - vb);
        const gct::BpItem it = gct::make_item(r->plan, r->st, r->vol_dev, r->cfg);
        const int idx = static_cast<int>(items[q].size());
        items[q].push_back(it);
        const auto w = gct::tile_entries(idx, gct::item_tiles(it), vb, vc, vb == 0 ? gct::kBpStore : gct::kBpAccumulate);
        work[q].insert(work[q].end(), w.begin(), w.end());
        advanced.emplace_back(r, vc);
    }
    size_t ni = 0, nw = 0;
    for (int q = 0; q < NQ; ++q) {
        ni += items[q].size();
        nw += work[q].size();
    }
    if (sl.items.n < ni) sl.items.alloc(ni, "round items");
    if (sl.work.n < nw) sl.work.alloc(nw, "round work");
    if (!sl.counters.p) sl.counters.alloc(NQ, "round counters");
    sl.h_items.reserve(ni * sizeof(gct::BpItem));
    sl.h_work.reserve(nw * sizeof(gct::BpWork));
    auto *hi = static_cast<gct::BpItem *>(sl.h_items.p);
    auto *hw = static_cast<gct::BpWork *>(sl.h_work.p);
    for (int q = 0, io = 0, wo = 0; q < NQ; ++q) {
        std::copy(items[q].begin(), items[q].end(), hi + io);
        std::copy(work[q].begin(), work[q].end(), hw + wo);
        io += static_cast<int>(items[q].size());
        wo += static_cast<int>(work[q].size());
    }
    cuda_check(cudaMemcpyAsync(sl.items.p, hi, ni * sizeof(gct::BpItem), cudaMemcpyHostToDevice, s->s_bp),
               "round items upload");
    cuda_check(cudaMemcpyAsync(sl.work.p, hw, nw * sizeof(gct::BpWork), cudaMemcpyHostToDevice, s->s_bp),
               "round work upload");
    cuda_check(cudaMemsetAsync(sl.counters.p, 0, NQ * sizeof(int), s->s_bp), "round counters");
    size_t item_off = 0, work_off = 0;
    for (int q = 0; q < NQ; ++q) {
        if (!work[q].empty()) {
            gct::launch_backproject_queue(sl.items.p + item_off, sl.work.p + work_off, static_cast<int>(work[q].size()),
                                          sl.counters.p + q, q / gct::kQueueClasses, q % gct::kQueueClasses,
                                          s->grid[q], s->s_bp);
            cuda_check(cudaGetLastError(), "round launch");
        }
        item_off += items[q].size();
        work_off += work[q].size();
    }
    cuda_check(cudaEventRecord(sl.done, s->s_bp), "event record");
    sl.used = true;
    ++s->round;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        ++s->n_rounds;
    }
    std::vector<Request *> still;
    for (auto &a : advanced) {
        Request *r = a.first;
        r->next_view += a.second;
        ++r->rounds;
        if (r->next_view < gct::item_views(r->plan, r->st)) {
            still.push_back(r);
            continue;
        }
        cuda_check(cudaStreamWaitEvent(s->s_out, sl.done, 0), "stream wait");
        cuda_check(cudaMemcpyAsync(r->vol_host, r->vol_dev, r->vol_bytes, cudaMemcpyDeviceToHost, s->s_out),
                   "volume download");
        cuda_check(cudaEventRecord(r->e_out, s->s_out), "event record");
        s->draining.push_back(r);
    }
    s->active.swap(still);
}

void retire(gct_fdk_server *s)
{
    std::vector<Request *> still;
    for (Request *r : s->draining) {
        const cudaError_t e = cudaEventQuery(r->e_out);
        if (e == cudaErrorNotReady) {
            still.push_back(r);
            continue;
        }
        cuda_check(e, "volume download");
        std::lock_guard<std::mutex> lock(s->mu);
        finish(s, r, GCT_REQ_DONE, GCT_OK);
    }
    s->draining.swap(still);
}

void fail_all(gct_fdk_server *s, const std::string &msg)
{
    std::lock_guard<std::mutex> lock(s->mu);
    s->failed = true;
    s->fail_msg = msg;
    for (auto *list : {&s->preparing, &s->active, &s->draining})
        for (Request *r : *list) finish(s, r, GCT_REQ_FAILED, GCT_ERR_CUDA);
    s->preparing.clear();
    s->active.clear();
    s->draining.clear();
    for (Request *r : s->queued) finish(s, r, GCT_REQ_FAILED, GCT_ERR_CUDA);
    s->queued.clear();
}

void worker_main(gct_fdk_server *s)
{
    cudaSetDevice(s->device);
    try {
        for (;;) {
            for (Request *r : admit(s)) {
                start(s, r);
                s->preparing.push_back(r);
            }
            // filtered requests join the rounds
            std::vector<Request *> still;
            for (Request *r : s->preparing) {
                const cudaError_t e = cudaEventQuery(r->e_prep);
                if (e == cudaErrorNotReady) {
                    still.push_back(r);
                    continue;
                }
                cuda_check(e, "filter stage");
                activate(s, r);
            }
            s->preparing.swap(still);
            if (s->active.empty() && !s->preparing.empty()) {
                cuda_check(cudaEventSynchronize(s->preparing.front()->e_prep), "filter stage");
                continue;
            }
            if (!s->active.empty()) run_round(s);
            retire(s);
            if (s->active.empty() && s->preparing.empty()) {
                if (!s->draining.empty()) {
                    cuda_check(cudaEventSynchronize(s->draining.front()->e_out), "volume download");
                    continue;
                }
                std::unique_lock<std::mutex> lock(s->mu);
                if (s->stopping && s->queued.empty()) break;
                // wait for a submission, or for budget that a retired request returned
                s->cv_work.wait_for(lock, std::chrono::milliseconds(50));
            }
        }
    } catch (const gct::GctError &e) {
        fail_all(s, e.msg);
    } catch (const std::exception &e) {
        fail_all(s, e.what());
    }
}

void create_server(gct_fdk_server *s, const gct_server_opts *o)
{
    if (!o || o->memory_budget_bytes == 0) gct::fail(GCT_ERR_INVALID_ARG, "a memory budget is required");
    s->max_active = o->max_active ? o->max_active : 64;
    s->autotune = o->autotune != 0;
    s->round_updates = o->round_updates > 0 ? o->round_updates : 2e9;
    cuda_check(cudaGetDevice(&s->device), "cudaGetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, s->device), "cudaGetDeviceProperties");
    s->num_sms = prop.multiProcessorCount;
    for (int q = 0; q < 2 * gct::kQueueClasses; ++q)
        s->grid[q] = std::max(1, gct::queue_blocks_per_sm(q / gct::kQueueClasses, q % gct::kQueueClasses)) * s->num_sms;
    s->budget.alloc(o->memory_budget_bytes, "server memory budget");
    s->arena.reset(o->memory_budget_bytes);
    for (cudaStream_t *st : {&s->s_in, &s->s_prep, &s->s_bp, &s->s_out})
        cuda_check(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "server stream");
    for (auto &sl : s->slot) cuda_check(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "event");
    s->worker = std::thread(worker_main, s);
}

struct ServerHolder {
    gct_fdk_server *s = nullptr;
    ~ServerHolder() { delete s; }
};

Request *find(gct_fdk_server *s, uint64_t ticket)
{
    auto it = s->table.find(ticket);
    if (it == s->table.end()) gct::fail(GCT_ERR_INVALID_ARG, "unknown ticket");
    return it->second.get();
}

}  // namespace

extern "C" {

gct_status gct_fdk_server_create(const gct_server_opts *opts, gct_fdk_server **out)
{
    return guarded([&] {
        if (!out) gct::fail(GCT_ERR_INVALID_ARG, "NULL server output");
        *out = nullptr;
        ServerHolder h;
        h.s = new gct_fdk_server();
        create_server(h.s, opts);
        *out = h.s;
        h.s = nullptr;
    });
}

gct_status gct_fdk_server_submit(gct_fdk_server *server, gct_fdk_plan *plan, const float *proj_host,
                                 float *vol_host, uint64_t *ticket)
{
    return guarded([&] {
        if (!server || !plan || !proj_host || !vol_host || !ticket) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (plan->device != server->device) gct::fail(GCT_ERR_INVALID_ARG, "plan was built on another device");
        auto r = std::make_unique<Request>();
        r->plan = plan;
        r->proj_host = proj_host;
        r->vol_host = vol_host;
        r->block_bytes = footprint(plan, &r->proj_bytes, &r->vol_bytes);
        std::lock_guard<std::mutex> lock(server->mu);
        if (server->failed) gct::fail(GCT_ERR_CUDA, "server stopped after a device error: " + server->fail_msg);
        if (server->stopping) gct::fail(GCT_ERR_CANCELLED, "server is shutting down");
        if (r->block_bytes > server->arena.size()) {
            ++server->n_rejected;
            gct::fail(GCT_ERR_BUDGET, "request needs " + std::to_string(r->block_bytes) + " device bytes; the budget is " +
                                          std::to_string(server->arena.size()));
        }
        r->ticket = server->next_ticket++;
        r->t_submit = Clock::now();
        if (!server->any_submit) {
            server->any_submit = true;
            server->t_first_submit = r->t_submit;
        }
        ++server->n_submitted;
        *ticket = r->ticket;
        server->queued.push_back(r.get());
        server->table.emplace(r->ticket, std::move(r));
        server->cv_work.notify_all();
    });
}

gct_status gct_fdk_server_info(gct_fdk_server *server, uint64_t ticket, gct_request_info *info)
{
    return guarded([&] {
        if (!server || !info) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        std::lock_guard<std::mutex> lock(server->mu);
        const Request *r = find(server, ticket);
        info->state = r->state;
        info->status = r->status;
        const bool admitted = r->state != GCT_REQ_QUEUED && r->state != GCT_REQ_CANCELLED;
        info->queued_ms = admitted ? ms_between(r->t_submit, r->t_admit) : ms_between(r->t_submit, Clock::now());
        info->latency_ms = r->state == GCT_REQ_DONE ? ms_between(r->t_submit, r->t_done) : 0.0;
        info->rounds = r->rounds;
        info->views_per_round = static_cast<uint32_t>(r->chunk);
    });
}

gct_status gct_fdk_server_wait(gct_fdk_server *server, uint64_t ticket, double timeout_ms)
{
    gct_status result = GCT_OK;
    const gct_status st = guarded([&] {
        if (!server) gct::fail(GCT_ERR_INVALID_ARG, "NULL server");
        std::unique_lock<std::mutex> lock(server->mu);
        Request *r = find(server, ticket);
        auto finished = [&] {
            return r->state == GCT_REQ_DONE || r->state == GCT_REQ_FAILED || r->state == GCT_REQ_CANCELLED;
        };
        if (timeout_ms < 0) {
            server->cv_done.wait(lock, finished);
        } else if (!server->cv_done.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms), finished)) {
            result = set_error(GCT_ERR_NOT_READY, "request still running");
            return;
        }
        if (r->state == GCT_REQ_FAILED)
            result = set_error(r->status, "request failed: " + server->fail_msg);
        else if (r->state == GCT_REQ_CANCELLED)
            result = set_error(GCT_ERR_CANCELLED, "request cancelled");
    });
    return st != GCT_OK ? st : result;
}

gct_status gct_fdk_server_cancel(gct_fdk_server *server, uint64_t ticket)
{
    return guarded([&] {
        if (!server) gct::fail(GCT_ERR_INVALID_ARG, "NULL server");
        std::lock_guard<std::mutex> lock(server->mu);
        Request *r = find(server, ticket);
        if (r->state != GCT_REQ_QUEUED) gct::fail(GCT_ERR_NOT_READY, "request already admitted");
        server->queued.erase(std::find(server->queued.begin(), server->queued.end(), r));
        finish(server, r, GCT_REQ_CANCELLED, GCT_ERR_CANCELLED);
    });
}

gct_status gct_fdk_server_stats(gct_fdk_server *server, gct_server_stats *out)
{
    return guarded([&] {
        if (!server || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        std::lock_guard<std::mutex> lock(server->mu);
        *out = gct_server_stats{};
        out->submitted = server->n_submitted;
        out->completed = server->n_completed;
        out->failed = server->n_failed;
        out->cancelled = server->n_cancelled;
        out->rejected = server->n_rejected;
        out->rounds = server->n_rounds;
        out->peak_bytes = server->arena.peak();
        out->peak_active = server->peak_active;
        std::vector<double> l = server->latencies;
        if (!l.empty()) {
            std::sort(l.begin(), l.end());
            auto pct = [&](double q) {
                const double pos = q * (l.size() - 1);
                const size_t lo = static_cast<size_t>(std::floor(pos)), hi = std::min(lo + 1, l.size() - 1);
                return l[lo] + (l[hi] - l[lo]) * (pos - lo);
            };
            out->p50_ms = pct(0.50);
            out->p99_ms = pct(0.99);
            double sum = 0.0;
            for (double x : l) sum += x;
            out->mean_ms = sum / l.size();
            const double span = ms_between(server->t_first_submit, server->t_last_done);
            out->recons_per_s = span > 0.0 ? 1000.0 * l.size() / span : 0.0;
        }
    });
}

gct_status gct_fdk_server_destroy(gct_fdk_server *server)
{
    return guarded([&] {
        if (!server) return;
        {
            std::lock_guard<std::mutex> lock(server->mu);
            server->stopping = true;
            server->cv_work.notify_all();
        }
        if (server->worker.joinable()) server->worker.join();
        DeviceGuard dg(server->device);
        cudaStreamSynchronize(server->s_out);
        delete server;
    });
}

}  // extern "C"
