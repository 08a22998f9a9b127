// Batched FDK: many reconstructions of uneven sizes and geometries in one persistent
// backprojection launch over a work queue of (volume tile, view chunk) entries, with the filter
// stages of all items and the queue launch captured in one CUDA graph. Tile shape, z-voxels per
// thread and views per coefficient stage come from an on-device autotuner whose results are
// cached per device and item shape.
//
// No counterpart in the reference, which reconstructs one stack per call
// (src/cuda/recon/recon_wrappers.cuh:15-43) with one backprojection launch per view
// (src/cuda/recon/fdk_axial.cuh:189-193).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "plan.hpp"
#include "queue.hpp"

namespace gct {

bool vol3d(const gct_fdk_plan *p) { return p->kz > 1 || is_2d_detector(p->kind); }

BpItem make_item(const gct_fdk_plan *p, const StackRef &st, float *vol, const TileConfig &c)
{
    if (c.bx * c.by != kQueueThreads || c.bx < 1 || !queue_zpt_ok(c.zpt) || c.vps < 1 || c.vps > kQueueMaxVps)
        fail(GCT_ERR_INVALID_ARG, "queue tile shape must cover 256 threads with z per thread 1, 4, 8 or 16");
    if (p->spiral) fail(GCT_ERR_NOT_SUPPORTED, "spiral plans run through gct_fdk_execute*, not batches or the server");
    BpItem it;
    it.a = bp_args(p, st, vol, 0, p->nv);
    it.family = static_cast<int>(p->family);
    it.z_affine = p->z_affine ? 1 : 0;
    it.zpt = c.zpt;
    it.bx = c.bx;
    it.by = c.by;
    it.vps = c.vps;
    if (st.quarter) {  // quarter-turn item: tiles of first-quadrant columns
        if (!sym_queue_zpt_ok(c.zpt))
            fail(GCT_ERR_INVALID_ARG, "quarter-turn queue tiles hold 8 voxels per thread (1 for 2D images)");
        it.a.sym = p->sym;
        it.a.v_count = st.quarter;
        it.tiles_x = (p->kx / 2 + c.bx - 1) / c.bx;
        it.tiles_y = (p->ky / 2 + c.by - 1) / c.by;
    } else {
        it.tiles_x = (p->kx + c.bx - 1) / c.bx;
        it.tiles_y = (p->ky + c.by - 1) / c.by;
    }
    it.tiles_z = (p->kz + c.zpt - 1) / c.zpt;
    return it;
}

int item_views(const gct_fdk_plan *p, const StackRef &st) { return st.quarter ? st.quarter : p->nv; }
int item_class(const StackRef &st, const TileConfig &c) { return st.quarter ? kQueueSymClass : queue_class(c.zpt); }

long long item_tiles(const BpItem &it) { return static_cast<long long>(it.tiles_x) * it.tiles_y * it.tiles_z; }

std::vector<BpWork> tile_entries(int item, long long tiles, int vb, int vc, int mode)
{
    std::vector<BpWork> w(static_cast<size_t>(tiles));
    for (long long t = 0; t < tiles; ++t) w[t] = BpWork{item, static_cast<int>(t), vb, vc, mode};
    return w;
}

TileConfig default_config(const gct_fdk_plan *p, bool quarter_turn)
{
    TileConfig c;
    if (quarter_turn) {
        c.zpt = vol3d(p) ? 8 : 1;
        c.bx = vol3d(p) ? 8 : 16;
        c.by = vol3d(p) ? 32 : 16;
    } else if (p->ky == 1 && vol3d(p)) {  // one row of columns (the transposed 1D parallel kind)
        c.bx = 256;
        c.by = 1;
        c.zpt = 16;
    } else if (!vol3d(p)) {
        c.zpt = 1;
        c.bx = 32;
        c.by = 8;
    }
    return c;
}

namespace {

// Candidate (zpt, block) shapes; views per stage is tuned afterwards for the best shape.
std::vector<TileConfig> shape_candidates(bool three_d, bool one_row, bool quarter_turn)
{
    std::vector<TileConfig> c;
    if (quarter_turn) {
        for (auto b : {std::make_pair(8, 32), std::make_pair(4, 64), std::make_pair(16, 16), std::make_pair(32, 8)})
            c.push_back({three_d ? 8 : 1, b.first, b.second, 32});
    } else if (one_row) {
        for (int zpt : {8, 16}) c.push_back({zpt, 256, 1, 32});
    } else if (three_d) {
        for (int zpt : {8, 16})
            for (auto b : {std::make_pair(8, 32), std::make_pair(16, 16), std::make_pair(32, 8)})
                c.push_back({zpt, b.first, b.second, 32});
    } else {
        for (auto b : {std::make_pair(32, 8), std::make_pair(16, 16), std::make_pair(8, 32), std::make_pair(64, 4)})
            c.push_back({1, b.first, b.second, 32});
    }
    return c;
}

// Device scratch of one timing run: the item, its work entries and the queue counter.
struct QueueScratch {
    DevBuf<BpItem> item;
    DevBuf<BpWork> work;
    DevBuf<int> counter;
};

// Updates per second of one configuration: all tiles of the item over its first views, on the
// grid of the configuration's queue kernel.
double time_config(const gct_fdk_plan *p, const StackRef &st, float *vol, const TileConfig &c, int num_sms,
                   QueueScratch &sc, cudaStream_t s)
{
    const int zc = item_class(st, c);
    const int grid = std::max(1, queue_blocks_per_sm(p->opts.storage, zc)) * num_sms;
    const BpItem it = make_item(p, st, vol, c);
    const int nvt = std::min(item_views(p, st), st.quarter ? 16 : 64);
    const std::vector<BpWork> w = tile_entries(0, item_tiles(it), 0, nvt, kBpStore);
    sc.item.upload(&it, 1, "autotune item");
    sc.work.upload(w.data(), w.size(), "autotune work");
    if (!sc.counter.p) sc.counter.alloc(1, "autotune counter");
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {  // the first run warms up
        cuda_check(cudaMemsetAsync(sc.counter.p, 0, sizeof(int), s), "counter reset");
        cuda_check(cudaEventRecord(e0, s), "event record");
        launch_backproject_queue(sc.item.p, sc.work.p, static_cast<int>(w.size()), sc.counter.p, p->opts.storage, zc,
                                 grid, s);
        cuda_check(cudaGetLastError(), "autotune launch");
        cuda_check(cudaEventRecord(e1, s), "event record");
        cuda_check(cudaEventSynchronize(e1), "autotune timing");
        float ms = 0.f;
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double upd = static_cast<double>(p->vol.nx) * p->vol.ny * p->vol.nz * nvt * (st.quarter ? 4 : 1);
    return upd / (static_cast<double>(best) * 1e-3);
}

std::mutex g_tune_mu;
std::map<std::string, Tuned> g_tune_cache;

std::string tune_key(const gct_fdk_plan *p, int num_sms)
{
    return std::to_string(p->device) + "/" + std::to_string(static_cast<int>(p->kind)) + "/" +
           std::to_string(p->opts.storage) + "/" + std::to_string(p->z_affine) + "/" + std::to_string(p->kx) +
           "x" + std::to_string(p->ky) + "x" + std::to_string(p->kz) + "/" + std::to_string(p->nr) + "x" +
           std::to_string(p->nc) + "/" + std::to_string(num_sms) + "/q" + std::to_string(p->sym);
}

}  // namespace

Tuned autotune(const gct_fdk_plan *p, const StackRef &st, float *vol, int num_sms, cudaStream_t s)
{
    const std::string key = tune_key(p, num_sms);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return it->second;
    }
    QueueScratch sc;
    Tuned best;
    for (const TileConfig &c : shape_candidates(vol3d(p), p->ky == 1 && vol3d(p), st.quarter > 0)) {
        const double ups = time_config(p, st, vol, c, num_sms, sc, s);
        if (ups > best.ups) best = {c, ups};
    }
    for (int vps : {16, 64}) {
        TileConfig c = best.cfg;
        c.vps = vps;
        const double ups = time_config(p, st, vol, c, num_sms, sc, s);
        if (ups > best.ups) best = {c, ups};
    }
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = best;
    return best;
}

}  // namespace gct

struct gct_fdk_batch {
    struct Item {
        gct_fdk_plan *plan = nullptr;
        const float *proj = nullptr;
        float *vol = nullptr;
        DevBuf<unsigned char> ws;
        StackRef st;
        gct::TileConfig cfg;
        double tuned_ups = 0.0;
        int view_split = 1;
        int stream = 0;  // side stream of its filter stage
    };
    int device = 0;
    int num_sms = 148;
    bool use_graph = true;
    std::vector<std::unique_ptr<Item>> items;
    // one queue per storage type and depth class present: index storage * kQueueClasses + class
    struct Queue {
        DevBuf<gct::BpItem> d_items;
        DevBuf<gct::BpWork> d_work;
        int n_work = 0;
        int grid = 0;
        std::vector<int> atomic_items;  // items whose volumes start at zero (view-split)
    } queue[2 * gct::kQueueClasses];
    DevBuf<int> counters;  // one per queue
    unsigned long long updates = 0;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> events;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~gct_fdk_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (cudaStream_t s : side) cudaStreamDestroy(s);
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace gct {
namespace {

// Issues the whole batch on `s`: filter stages forked onto the side streams, then, once all are
// done, one queue launch per storage type.
void issue(gct_fdk_batch *b, cudaStream_t s)
{
    size_t ev = 0;
    auto next_event = [&]() {
        if (ev == b->events.size()) {
            cudaEvent_t e;
            cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            b->events.push_back(e);
        }
        return b->events[ev++];
    };
    cudaEvent_t fork = next_event();
    cuda_check(cudaEventRecord(fork, s), "event record");
    std::vector<bool> used(b->side.size(), false);
    for (auto &ip : b->items) {
        gct_fdk_batch::Item &it = *ip;
        cudaStream_t ss = b->side[it.stream];
        if (!used[it.stream]) cuda_check(cudaStreamWaitEvent(ss, fork, 0), "stream wait");
        used[it.stream] = true;
        if (it.st.quarter) prepare_partners(it.plan, it.proj, it.st, 0, it.st.quarter, ss);
        else prepare(it.plan, it.proj, it.st, 0, it.plan->nv, ss);
    }
    for (size_t k = 0; k < b->side.size(); ++k) {
        if (!used[k]) continue;
        cudaEvent_t join = next_event();
        cuda_check(cudaEventRecord(join, b->side[k]), "event record");
        cuda_check(cudaStreamWaitEvent(s, join, 0), "stream wait");
    }
    for (int q = 0; q < 2 * kQueueClasses; ++q) {
        const auto &Q = b->queue[q];
        if (Q.n_work == 0) continue;
        for (int i : Q.atomic_items) {
            const gct_fdk_plan *p = b->items[i]->plan;
            cuda_check(cudaMemsetAsync(b->items[i]->vol, 0, sizeof(float) * p->vol.nx * p->vol.ny * p->vol.nz, s),
                       "volume reset");
        }
        cuda_check(cudaMemsetAsync(b->counters.p + q, 0, sizeof(int), s), "queue counter reset");
        launch_backproject_queue(Q.d_items.p, Q.d_work.p, Q.n_work, b->counters.p + q, q / kQueueClasses,
                                 q % kQueueClasses, Q.grid, s);
        cuda_check(cudaGetLastError(), "queue backprojection launch");
    }
}

void build_batch(gct_fdk_batch *b, const gct_batch_item *items, uint32_t n, const gct_batch_opts *opts)
{
    if (!items || n == 0) fail(GCT_ERR_INVALID_ARG, "empty batch");
    const bool tune = opts ? opts->autotune != 0 : true;
    b->use_graph = opts ? opts->use_graph != 0 : true;
    const int bps_opt = opts ? opts->blocks_per_sm : 0;
    cuda_check(cudaGetDevice(&b->device), "cudaGetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, b->device), "cudaGetDeviceProperties");
    b->num_sms = prop.multiProcessorCount;
    for (uint32_t i = 0; i < n; ++i) {
        const gct_batch_item &src = items[i];
        if (!src.plan || !src.proj_dev || !src.vol_dev)
            fail(GCT_ERR_INVALID_ARG, "batch item " + std::to_string(i) + " has a NULL plan or buffer");
        if (src.plan->device != b->device)
            fail(GCT_ERR_INVALID_ARG, "batch item " + std::to_string(i) + " was planned on another device");
        auto it = std::make_unique<gct_fdk_batch::Item>();
        it->plan = src.plan;
        it->proj = src.proj_dev;
        it->vol = src.vol_dev;
        it->ws.alloc(src.plan->workspace_bytes(), "batch item workspace");
        // quarter-turn plans keep their interleaved partner stacks and run in the quarter-turn queue
        it->st = stack_of(src.plan, it->ws.p, false);
        b->items.push_back(std::move(it));
    }
    // filter stages: items of one plan share its filter scratch, so they run on one side stream
    std::map<const gct_fdk_plan *, int> plan_stream;
    const int max_side = 4;
    for (auto &ip : b->items) {
        auto f = plan_stream.find(ip->plan);
        if (f == plan_stream.end())
            f = plan_stream.emplace(ip->plan, static_cast<int>(plan_stream.size()) % max_side).first;
        ip->stream = f->second;
    }
    const int nside = std::min(max_side, static_cast<int>(plan_stream.size()));
    for (int k = 0; k < nside; ++k) {
        cudaStream_t s;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "side stream");
        b->side.push_back(s);
    }
    cuda_check(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "capture stream");

    // tile configurations
    for (int q = 0; q < 2 * kQueueClasses; ++q) {
        int bps = bps_opt > 0 ? bps_opt : queue_blocks_per_sm(q / kQueueClasses, q % kQueueClasses);
        if (bps <= 0) bps = 1;
        b->queue[q].grid = bps * b->num_sms;
    }
    for (auto &ip : b->items) {
        if (tune) {
            const Tuned t = autotune(ip->plan, ip->st, ip->vol, b->num_sms, b->cap);
            ip->cfg = t.cfg;
            ip->tuned_ups = t.ups;
        } else {
            ip->cfg = default_config(ip->plan, ip->st.quarter > 0);
        }
    }

    // work queues: items by decreasing cost; an item whose single tile costs more than an even
    // share of the queue over 8 entries per block is split into view chunks (atomic adds)
    auto queue_of = [&](const gct_fdk_batch::Item &it) {
        return (it.plan->opts.storage == GCT_STORAGE_F16 ? 1 : 0) * kQueueClasses + item_class(it.st, it.cfg);
    };
    for (int q = 0; q < 2 * kQueueClasses; ++q) {
        auto &Q = b->queue[q];
        std::vector<int> idx;
        for (int i = 0; i < static_cast<int>(b->items.size()); ++i)
            if (queue_of(*b->items[i]) == q) idx.push_back(i);
        if (idx.empty()) continue;
        std::vector<BpItem> qitems;
        std::vector<double> cost;
        double total = 0.0;
        for (int i : idx) {
            const gct_fdk_plan *p = b->items[i]->plan;
            const double c = static_cast<double>(p->vol.nx) * p->vol.ny * p->vol.nz * p->nv;
            cost.push_back(c);
            total += c;
        }
        std::vector<int> order(idx.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
        const double target = total / (static_cast<double>(Q.grid) * 8.0);
        std::vector<BpWork> work;
        for (int o : order) {
            const int i = idx[o];
            auto &it = *b->items[i];
            const gct_fdk_plan *p = it.plan;
            const BpItem bi = make_item(p, it.st, it.vol, it.cfg);
            const long long tiles = item_tiles(bi);
            const int views = item_views(p, it.st);
            const double tile_cost = cost[o] / static_cast<double>(tiles);
            int split = static_cast<int>(std::ceil(tile_cost / std::max(target, 1.0)));
            split = std::max(1, std::min(split, views / 16));
            it.view_split = split;
            const int qi = static_cast<int>(qitems.size());
            qitems.push_back(bi);
            if (split > 1) Q.atomic_items.push_back(i);
            for (int c = 0; c < split; ++c) {
                const int vb = static_cast<int>(static_cast<long long>(views) * c / split);
                const int ve = static_cast<int>(static_cast<long long>(views) * (c + 1) / split);
                const auto w = tile_entries(qi, tiles, vb, ve - vb, split > 1 ? kBpAtomic : kBpStore);
                work.insert(work.end(), w.begin(), w.end());
            }
            b->updates += static_cast<unsigned long long>(p->vol.nx) * p->vol.ny * p->vol.nz * p->nv;
        }
        if (work.size() > static_cast<size_t>(INT32_MAX)) fail(GCT_ERR_NOT_SUPPORTED, "work queue too long");
        Q.d_items.upload(qitems.data(), qitems.size(), "queue items");
        Q.d_work.upload(work.data(), work.size(), "queue work");
        Q.n_work = static_cast<int>(work.size());
    }
    b->counters.alloc(2 * kQueueClasses, "queue counters");

    if (b->use_graph) {
        cuda_check(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "graph capture begin");
        try {
            issue(b, b->cap);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->cap, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cuda_check(cudaStreamEndCapture(b->cap, &b->graph), "graph capture end");
        cuda_check(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
    }
}

struct BatchHolder {
    gct_fdk_batch *b = nullptr;
    ~BatchHolder() { delete b; }
};

}  // namespace
}  // namespace gct

extern "C" {

gct_status gct_fdk_batch_create(const gct_batch_item *items, uint32_t count, const gct_batch_opts *opts,
                                gct_fdk_batch **out)
{
    return guarded([&] {
        if (!out) gct::fail(GCT_ERR_INVALID_ARG, "NULL batch output");
        *out = nullptr;
        gct::BatchHolder h;
        h.b = new gct_fdk_batch();
        gct::build_batch(h.b, items, count, opts);
        *out = h.b;
        h.b = nullptr;
    });
}

gct_status gct_fdk_batch_launch(gct_fdk_batch *batch, void *stream)
{
    return guarded([&] {
        if (!batch) gct::fail(GCT_ERR_INVALID_ARG, "NULL batch");
        DeviceGuard dg(batch->device);
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (batch->use_graph)
            cuda_check(cudaGraphLaunch(batch->exec, s), "graph launch");
        else
            gct::issue(batch, s);
    });
}

gct_status gct_fdk_batch_item_config(const gct_fdk_batch *batch, uint32_t item, gct_batch_item_config *out)
{
    return guarded([&] {
        if (!batch || !out) gct::fail(GCT_ERR_INVALID_ARG, "NULL argument");
        if (item >= batch->items.size()) gct::fail(GCT_ERR_INVALID_ARG, "item index out of range");
        const auto &it = *batch->items[item];
        out->z_per_thread = it.cfg.zpt;
        out->block_x = it.cfg.bx;
        out->block_y = it.cfg.by;
        out->views_per_stage = it.cfg.vps;
        out->view_split = it.view_split;
        out->tuned_gups = it.tuned_ups * 1e-9;
    });
}

gct_status gct_fdk_batch_work(const gct_fdk_batch *batch, uint64_t *work_entries, uint64_t *updates)
{
    return guarded([&] {
        if (!batch) gct::fail(GCT_ERR_INVALID_ARG, "NULL batch");
        if (work_entries)
            *work_entries = 0;
        for (const auto &q : batch->queue)
            if (work_entries) *work_entries += static_cast<uint64_t>(q.n_work);
        if (updates) *updates = batch->updates;
    });
}

gct_status gct_fdk_batch_destroy(gct_fdk_batch *batch)
{
    return guarded([&] {
        if (!batch) return;
        DeviceGuard dg(batch->device);
        delete batch;
    });
}

}  // extern "C"
