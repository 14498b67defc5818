// skg_serve.cpp -- continuous batching of many simulations on one device behind two calls,
// skg_submit and skg_poll.
//
// The caller is FitSKIRT's variant loop (FitSKIRTcore/OligoFitScheme.cpp:123-149 evaluates each
// parameter set through AdjustableSkirtSimulation::performWith, AdjustableSkirtSimulation.cpp:
// 145-194): many short simulations of one ski file with a few values substituted, each waiting for
// its frames.  A server owns three host threads and works through the public C ABI (and the
// device's memory pool, below):
//
//   loop thread     admits submitted requests in arrival order while a batch slot is free and the
//                   request's device-memory bound fits the budget (admission by HBM footprint);
//                   runs ticks -- one skg_batch_run carrying the next packet slice of every
//                   admitted request whose context is ready, oldest requests first up to a packet
//                   budget per tick -- so that requests arriving meanwhile join a later tick and
//                   their work overlaps on the device; retires a request once all its packets
//                   have run: reads its tallies into the caller's buffers and hands its context
//                   to the clean-up thread;
//   set-up thread   builds the contexts of admitted requests (skg_ctx_create: uploads, density
//                   sampling) while the ticks run;
//   clean-up thread frees retired contexts, then releases their reservations: the next tick does
//                   not wait for it.
//
// The device's default memory pool, from which contexts allocate (stream-ordered), keeps up to the
// server's HBM budget of freed memory instead of returning it to the driver at each
// synchronisation: a retired context's memory goes to the next one without being unmapped and
// mapped again.  (Returned and mapped again, context set-up took 20-50 ms and release up to 0.75 s
// on the fit-variant stream, and releases under the loop's lock left the device idle for 2.3 of
// 17.6 s.)
//
// A request's packets draw from streams keyed by its seed and the packet index, so its result is
// the same in whichever ticks it runs, alone or mixed with others, up to the summation order of
// the FP64 tally atomics.
#include "../../include/skirt_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

// A deep copy of a scene: every array the struct points to is owned here, so the caller's scene
// may go away as soon as skg_submit returns.
struct SceneCopy {
    skg_scene sc;
    std::vector<std::vector<char>> blocks;
    std::vector<skg_dust_comp> dust;
    std::vector<skg_stellar_comp> stellar;
    std::vector<skg_instrument> instr;
    int64_t ncells = 0;

    template<typename T> const T* keep(const T* p, size_t n) {
        if (!p || n == 0) return nullptr;
        blocks.emplace_back(n * sizeof(T));
        std::memcpy(blocks.back().data(), p, n * sizeof(T));
        return reinterpret_cast<const T*>(blocks.back().data());
    }
    void keep_geometry(skg_geometry& g) {
        if (g.clump_count > 0) g.clump_pos = keep(g.clump_pos, 3 * (size_t)g.clump_count);
    }

    explicit SceneCopy(const skg_scene& s) : sc(s) {
        skg_grid& g = sc.grid;
        if (g.type == SKG_GRID_CARTESIAN) {
            g.xv = keep(g.xv, (size_t)g.nx + 1); g.yv = keep(g.yv, (size_t)g.ny + 1); g.zv = keep(g.zv, (size_t)g.nz + 1);
            ncells = (int64_t)g.nx * g.ny * g.nz;
        } else if (g.type == SKG_GRID_OCTREE || g.type == SKG_GRID_BINTREE) {
            const size_t n = (size_t)g.nnodes;
            for (size_t l = 0; l < n; l++) if (g.node_cell[l] >= 0) ncells++;
            const int64_t nn = g.nbr_offsets ? g.nbr_offsets[6 * n] : 0;
            g.node_box = keep(g.node_box, 6 * n); g.node_child = keep(g.node_child, n);
            g.node_father = keep(g.node_father, n); g.node_cell = keep(g.node_cell, n); g.node_dir = keep(g.node_dir, n);
            g.nbr_ids = g.nbr_offsets ? keep(g.nbr_ids, (size_t)nn) : nullptr;
            g.nbr_offsets = keep(g.nbr_offsets, g.nbr_offsets ? 6 * n + 1 : 0);
        } else {
            const size_t n = (size_t)g.nsites, nb3 = (size_t)g.nb * g.nb * g.nb;
            ncells = g.nsites;
            g.vnbr_ids = keep(g.vnbr_ids, (size_t)g.vnbr_offsets[n]);
            g.block_ids = keep(g.block_ids, (size_t)g.block_offsets[nb3]);
            g.sites = keep(g.sites, 3 * n); g.vnbr_offsets = keep(g.vnbr_offsets, n + 1);
            g.block_offsets = keep(g.block_offsets, nb3 + 1);
            g.cell_volume = keep(g.cell_volume, g.cell_volume ? n : 0);
            g.cell_bbox = keep(g.cell_bbox, g.cell_bbox ? 6 * n : 0);
        }
        const size_t nl = (size_t)sc.nlambda;
        sc.lambda = keep(sc.lambda, nl); sc.dlambda = keep(sc.dlambda, nl);
        dust.assign(s.dust, s.dust + std::max(s.ncomp, 0));
        for (auto& d : dust) {
            keep_geometry(d.geometry);
            d.kappaext = keep(d.kappaext, nl); d.albedo = keep(d.albedo, nl); d.asymmpar = keep(d.asymmpar, nl);
        }
        sc.dust = dust.data();
        sc.rho = keep(sc.rho, sc.rho ? (size_t)std::max(s.ncomp, 0) * ncells : 0);
        stellar.assign(s.stellar, s.stellar + std::max(s.nstellar, 0));
        for (auto& c : stellar) { keep_geometry(c.geometry); c.luminosity = keep(c.luminosity, nl); }
        sc.stellar = stellar.data();
        instr.assign(s.instr, s.instr + std::max(s.ninstr, 0));
        sc.instr = instr.data();
    }
    size_t host_bytes() const {
        size_t b = 0;
        for (auto& v : blocks) b += v.size();
        return b;
    }
};

enum ReqState { QUEUED, BUILDING, READY, DONE };

struct Req {
    int64_t id = 0;
    std::unique_ptr<SceneCopy> scene;
    std::vector<int32_t> ells;
    uint64_t npp = 0, seed = 0;
    int instr = 0;
    double* cube = nullptr;
    double* sed = nullptr;
    int64_t footprint = 0;
    int64_t held = 0;         // the reservation it holds (its footprint once admitted)
    ReqState state = QUEUED;
    skg_ctx* ctx = nullptr;
    uint64_t next = 0;        // first packet of the next slice
    uint64_t ran = 0;         // packets whose ticks have completed
    int status = SKG_OK;
    std::string error;
    Clock::time_point submitted, done;
};

// Device-memory bound of a request's context, before it exists: the densities (FP64 and FP32) and
// the grid records per cell, the grid arrays as given, the tallies, and a fixed allowance for
// the remaining tables.
int64_t footprint(const SceneCopy& s) {
    int64_t b = s.ncells * (int64_t)(12 * std::max(s.sc.ncomp, 1) + 96) + (int64_t)s.host_bytes() + (16 << 20);
    for (const auto& in : s.instr) {
        int64_t nc = 1;
        if (in.type == SKG_INSTR_FRAME && in.stellar_comps) nc = 1 + std::max(s.sc.nstellar, 0);
        if (in.type == SKG_INSTR_FULL) nc = SKG_FULL_NBASE + in.nscatt_levels;
        b += nc * s.sc.nlambda * 8 * (1 + (in.type == SKG_INSTR_SED ? 0 : (int64_t)in.nxp * in.nyp));
    }
    if (s.sc.store_absorption || s.sc.dust_emission) b += s.ncells * (int64_t)s.sc.nlambda * 16;
    if (s.sc.dust_emission) b += s.ncells * (int64_t)s.sc.nlambda * 24;
    return b;
}

}  // namespace

struct skg_server {
    int device = 0;
    skg_server_opts opts{};
    skg_batch* batch = nullptr;
    std::mutex mu;
    std::condition_variable cv;          // the loop's wake-up (submissions, built contexts, stop)
    std::condition_variable done_cv;     // completions (skg_poll)
    std::condition_variable setup_cv;
    std::map<int64_t, std::unique_ptr<Req>> reqs;
    std::deque<Req*> pending;            // submitted, not admitted (arrival order)
    std::deque<Req*> to_build;           // admitted, context not built yet
    std::vector<Req*> admitted;          // admitted, in arrival order
    std::condition_variable free_cv;
    std::deque<std::pair<skg_ctx*, int64_t>> to_free;   // retired contexts and their reservations
    int64_t next_id = 1, reserved = 0;
    bool stop = false, stop_free = false;
    std::thread loop_thread, setup_thread, free_thread;
    // statistics
    int64_t ticks = 0, completed = 0, packets = 0;
    double tick_ms = 0;

    void setup_main();
    void loop_main();
    void free_main();
    void finish(Req* r, int status, const std::string& msg);
};

void skg_server::finish(Req* r, int status, const std::string& msg) {
    // caller holds mu; the context and the reservation go to the clean-up thread
    r->status = status; r->error = msg; r->state = DONE; r->done = Clock::now();
    to_free.emplace_back(r->ctx, r->held);
    r->ctx = nullptr; r->held = 0;
    r->scene.reset();
    completed++;
    done_cv.notify_all();
    free_cv.notify_one();
}

void skg_server::free_main() {
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        free_cv.wait(lk, [&] { return stop_free || !to_free.empty(); });
        if (to_free.empty()) return;             // stop_free and nothing left
        auto [ctx, bytes] = to_free.front();
        to_free.pop_front();
        lk.unlock();
        if (ctx) skg_ctx_destroy(ctx);
        lk.lock();
        reserved -= bytes;
        cv.notify_all();                         // admission may proceed
    }
}

void skg_server::setup_main() {
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        setup_cv.wait(lk, [&] { return stop || !to_build.empty(); });
        if (stop) return;                      // the loop cancels what is left
        Req* r = to_build.front();
        to_build.pop_front();
        r->state = BUILDING;
        const skg_scene* sc = &r->scene->sc;
        lk.unlock();
        skg_ctx* ctx = nullptr;
        const int rc = skg_ctx_create(sc, device, &ctx);
        std::string msg = rc ? skg_last_error(nullptr) : "";
        lk.lock();
        if (rc) {
            admitted.erase(std::find(admitted.begin(), admitted.end(), r));
            finish(r, rc, msg);
        } else {
            r->ctx = ctx;
            r->state = READY;
        }
        cv.notify_all();
    }
}

void skg_server::loop_main() {
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        if (stop) {
            // destroyed: a context being built is waited for, then every request that has not
            // finished ends with an error (its buffers are not written)
            bool building = false;
            for (Req* r : admitted) building |= r->state == BUILDING;
            if (building) { cv.wait_for(lk, std::chrono::milliseconds(20)); continue; }
            for (Req* r : pending) finish(r, SKG_ERR_INVALID, "server destroyed before the request ran");
            for (Req* r : admitted) finish(r, SKG_ERR_INVALID, "server destroyed before the request finished");
            pending.clear(); admitted.clear(); to_build.clear();
            return;
        }
        // admission: arrival order, a free slot, the footprint within the budget (a request that
        // alone exceeds the budget is admitted when nothing else holds memory)
        while (!pending.empty() && (int)admitted.size() < opts.max_slots) {
            Req* r = pending.front();
            if (!admitted.empty() && reserved + r->footprint > opts.hbm_budget) break;
            pending.pop_front();
            reserved += r->footprint;
            r->held = r->footprint;
            admitted.push_back(r);
            to_build.push_back(r);
            setup_cv.notify_one();
        }
        // one tick: the next slices of the ready requests, oldest first, up to the tick budget
        std::vector<skg_work> work;
        std::vector<std::pair<Req*, uint64_t>> given;
        int64_t budget = opts.tick_budget;
        for (Req* r : admitted) {
            if (r->state != READY || r->next >= r->npp) continue;
            if (budget <= 0) break;
            const int64_t nell = (int64_t)r->ells.size();
            uint64_t cnt = std::min<uint64_t>((uint64_t)opts.tick_packets, r->npp - r->next);
            cnt = std::max<uint64_t>(1, std::min<uint64_t>(cnt, (uint64_t)std::max<int64_t>(budget / nell, 1)));
            budget -= (int64_t)cnt * nell;
            skg_work w;
            w.ctx = r->ctx; w.ells = r->ells.data(); w.nell = (int32_t)nell;
            w.npp = r->npp; w.first = r->next; w.count = cnt; w.seed = r->seed;
            work.push_back(w);
            given.emplace_back(r, cnt);
            r->next += cnt;
        }
        // budget left after every ready request had its slice: the oldest requests take more of
        // their packets in this tick (no per-request cap), so that a lightly loaded server runs a
        // large request in fewer ticks (the 256-request stream at 10/s: p99 0.74 -> 0.64 s)
        for (size_t k = 0; k < given.size() && budget > 0; k++) {
            Req* r = given[k].first;
            const int64_t nell = (int64_t)r->ells.size();
            const uint64_t extra = std::min<uint64_t>(r->npp - r->next, (uint64_t)(budget / nell));
            if (extra == 0) continue;
            work[k].count += extra;
            given[k].second += extra;
            r->next += extra;
            budget -= (int64_t)extra * nell;
        }
        if (!work.empty()) {
            lk.unlock();
            skg_run_opts ro;
            std::memset(&ro, 0, sizeof(ro));
            ro.precision = opts.precision; ro.dedupe_peeloff = 1;
            int rc = skg_batch_run(batch, SKG_PHASE_STELLAR, work.data(), (int)work.size(), &ro, 0, nullptr);
            if (rc == SKG_OK) rc = skg_batch_sync(batch, -1);
            float ms = 0;
            if (rc == SKG_OK) skg_batch_last_ms(batch, &ms);
            const std::string msg = rc ? skg_last_error(nullptr) : "";
            // retire the requests whose last packets ran (their tallies into the caller's buffers)
            std::vector<std::pair<Req*, int>> out;
            for (auto& [r, cnt] : given) {
                r->ran += cnt;
                if (rc != SKG_OK) { out.emplace_back(r, rc); continue; }
                if (r->ran < r->npp) continue;
                int rrc = skg_read_instrument(r->ctx, r->instr, r->cube, r->sed);
                out.emplace_back(r, rrc);
            }
            lk.lock();
            ticks++; tick_ms += ms;
            for (auto& [r, cnt] : given) packets += (int64_t)cnt * (int64_t)r->ells.size();
            for (auto& [r, st] : out) {
                admitted.erase(std::find(admitted.begin(), admitted.end(), r));
                finish(r, st, st ? (rc ? msg : std::string(skg_last_error(nullptr))) : "");
            }
            continue;
        }
        cv.wait_for(lk, std::chrono::milliseconds(20));
    }
}

extern "C" {

int skg_scene_tally_sizes(const skg_scene* sc, int instr, int64_t* cube_len, int64_t* sed_len) {
    if (!sc || instr < 0 || instr >= sc->ninstr) return SKG_ERR_INVALID;
    const skg_instrument& in = sc->instr[instr];
    int64_t nc = 1;
    if (in.type == SKG_INSTR_FRAME && in.stellar_comps) nc = 1 + std::max(sc->nstellar, 0);
    if (in.type == SKG_INSTR_FULL) nc = SKG_FULL_NBASE + in.nscatt_levels;
    if (cube_len) *cube_len = in.type == SKG_INSTR_SED ? 0 : nc * sc->nlambda * (int64_t)in.nxp * in.nyp;
    if (sed_len) *sed_len = nc * sc->nlambda;
    return SKG_OK;
}

int skg_server_create(int device, const skg_server_opts* opts, skg_server** out) {
    if (!out) return SKG_ERR_INVALID;
    *out = nullptr;
    skg_server* s = new skg_server();
    s->device = device;
    if (opts) s->opts = *opts;
    if (s->opts.hbm_budget <= 0) s->opts.hbm_budget = (int64_t)40 << 30;
    if (s->opts.max_slots <= 0) s->opts.max_slots = 64;
    // tick sizes measured on the 256-request fit-variant stream (p99 at 10/s and 20/s arrivals):
    // 2^22 per request and 48 * 2^20 per tick 0.64 / 4.32 s, 2^23 and 24 * 2^20 0.74 / 3.89 s,
    // 2^23 and 16 * 2^20 0.61 / 3.94 s
    if (s->opts.tick_packets <= 0) s->opts.tick_packets = (int64_t)1 << 23;
    if (s->opts.tick_budget <= 0) s->opts.tick_budget = (int64_t)16 << 20;
    if (s->opts.max_slots > 64 ||
        (s->opts.precision != SKG_PREC_FP32 && s->opts.precision != SKG_PREC_FP64)) { delete s; return SKG_ERR_INVALID; }
    const int rc = skg_batch_create(device, s->opts.max_slots, s->opts.max_slots, 64 * s->opts.max_slots, &s->batch);
    if (rc) { delete s; return rc; }
    // freed context memory stays in the device's default pool up to the budget (see above)
    cudaMemPool_t pool;
    if (cudaSetDevice(device) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        keep = std::max<uint64_t>(keep, (uint64_t)s->opts.hbm_budget);
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    s->loop_thread = std::thread([s] { s->loop_main(); });
    s->setup_thread = std::thread([s] { s->setup_main(); });
    s->free_thread = std::thread([s] { s->free_main(); });
    *out = s;
    return SKG_OK;
}

int skg_submit(skg_server* s, const skg_request* q, int64_t* id) {
    if (!s || !q || !q->scene || !q->ells || q->nell <= 0 || q->nell > 64 || q->packages == 0 || !id)
        return SKG_ERR_INVALID;
    if (q->instr < 0 || q->instr >= q->scene->ninstr) return SKG_ERR_INVALID;
    for (int e = 0; e < q->nell; e++) if (q->ells[e] < 0 || q->ells[e] >= q->scene->nlambda) return SKG_ERR_INVALID;
    auto r = std::make_unique<Req>();
    r->scene = std::make_unique<SceneCopy>(*q->scene);
    r->ells.assign(q->ells, q->ells + q->nell);
    r->npp = q->packages; r->seed = q->seed; r->instr = q->instr; r->cube = q->cube; r->sed = q->sed;
    r->footprint = footprint(*r->scene);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return SKG_ERR_INVALID;
    r->id = s->next_id++;
    *id = r->id;
    s->pending.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->cv.notify_all();
    return SKG_OK;
}

int skg_poll(skg_server* s, int64_t id, int timeout_ms, double* latency_s) {
    if (!s) return SKG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SKG_ERR_INVALID;
    Req* r = it->second.get();
    auto ready = [&] { return r->state == DONE; };
    if (timeout_ms < 0) s->done_cv.wait(lk, ready);
    else if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return SKG_ERR_TIMEOUT;
    if (latency_s) *latency_s = std::chrono::duration<double>(r->done - r->submitted).count();
    const int st = r->status;
    s->reqs.erase(it);                       // reported once
    return st;
}

int skg_server_stats(skg_server* s, int64_t* ticks, int64_t* completed, int64_t* packets, double* tick_ms) {
    if (!s) return SKG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (ticks) *ticks = s->ticks;
    if (completed) *completed = s->completed;
    if (packets) *packets = s->packets;
    if (tick_ms) *tick_ms = s->tick_ms;
    return SKG_OK;
}

int skg_server_destroy(skg_server* s) {
    if (!s) return SKG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
        s->setup_cv.notify_all();
    }
    s->setup_thread.join();
    s->loop_thread.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_free = true;
        s->free_cv.notify_all();
    }
    s->free_thread.join();                   // the retired contexts are freed
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& kv : s->reqs) if (kv.second->ctx) { skg_ctx_destroy(kv.second->ctx); kv.second->ctx = nullptr; }
    }
    skg_batch_destroy(s->batch);
    delete s;
    return SKG_OK;
}

}  // extern "C"
