// Batching and serving behind axc_serve_configure / axc_submit / axc_poll / axc_partition_batch:
// continuous batching over a pool of lanes. Each lane is a worker thread with its own stream; a
// job runs on one lane in a device arena of its estimated size. Jobs start in submission order
// as lanes and device memory free up, with smaller jobs allowed past one that does not fit yet,
// so independent jobs overlap on the device; a job of 1M pins or more runs alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "axc_host.h"

struct axc_ctx;

namespace axc {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    HostGraph g;
    axc_hgraph view{};
    axc_params p{};
    std::vector<uint32_t> part;
    axc_stats st{};
    size_t est = 0;  // device bytes granted
    uint64_t pins = 0;
    bool exclusive = false;  // running alone on the device
    int retries = 0;
    int rc = 0;
    bool done = false;
    std::string err;
    Clock::time_point t_submit, t_start, t_end;
};

// Device bytes a job's arena needs: the level hierarchy, one refinement round's scratch (the
// inbound transitions, at most two per destination pin, dominate it) and the sorts' buffers.
// A job that runs out is retried once with twice as much.
static size_t estimate_bytes(const axc_hgraph *g) {
    const uint64_t P = g->e ? g->hedge_off[g->e] : 0;
    const double b = 192.0 * (double)P + 160.0 * (double)g->n + 96.0 * (double)g->e + (64u << 20);
    return (size_t)b;
}

// Tile and table sizes for the jobs of one size class: jobs of at least min_pins pins (the largest
// such class applies; a job below every class uses the context's own values).
struct TuneClass {
    bool set = false;
    uint64_t min_pins = 0;
    uint32_t rate_try = 2048, rate_mid = 8192, cascade_movers = 0;
};
constexpr int TUNE_CLASSES = 8;

// The executor's settings, given before the first submit (axc_serve_configure, axc_tune_set).
struct ServeConfig {
    uint32_t lanes = 1;
    size_t budget = 0;
    bool excl_set = false;
    uint64_t excl_pins = 1000000;
    TuneClass cls[TUNE_CLASSES];
};

struct Executor {
    int device = 0;
    uint32_t defaults[3] = {2048, 8192, 0};
    TuneClass cls[TUNE_CLASSES];
    uint32_t nlanes = 1;
    size_t budget = 0;
    std::vector<Lane *> lanes;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    size_t in_use = 0;
    uint32_t running = 0;
    bool stop = false;
    uint64_t next_id = 1;
    // Jobs of at least excl_pins pins (0: none) run alone: one such job keeps the GPU busy by
    // itself, and overlapping it only adds contention; smaller, launch-bound jobs overlap. The
    // environment variable AXC_SERVE_EXCLUSIVE_PINS overrides the default of 1M pins.
    uint64_t excl_pins = 1000000;
    bool excl_running = false;

    // The first queued job that fits next to the running ones; with nothing running, the head.
    // A large job waits until the device drains, and no later job passes it meanwhile.
    Job *pick() {
        if (excl_running) return nullptr;
        for (auto it = queue.begin(); it != queue.end(); ++it) {
            Job *j = *it;
            if (excl_pins && j->pins >= excl_pins) {
                if (running) return nullptr;
                queue.erase(it);
                j->exclusive = true;
                excl_running = true;
                return j;
            }
            if (running == 0 || j->est <= budget - std::min(budget, in_use)) {
                queue.erase(it);
                return j;
            }
        }
        return nullptr;
    }

    void run(uint32_t li) {
        Lane *lane = lanes[li];
        for (;;) {
            Job *j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || (!queue.empty() && (j = pick()) != nullptr); });
                if (!j) return;  // stopping
                in_use += j->est;
                ++running;
            }
            j->t_start = Clock::now();
            {  // the job's size class picks the lane's tile and table sizes
                const TuneClass *best = nullptr;
                for (const TuneClass &t : cls)
                    if (t.set && j->pins >= t.min_pins && (!best || t.min_pins > best->min_pins)) best = &t;
                if (best) lane_tune(lane, best->rate_try, best->rate_mid, best->cascade_movers);
                else lane_tune(lane, defaults[0], defaults[1], defaults[2]);
            }
            std::string err;
            const int rc = lane_partition(lane, j->est, &j->view, &j->p, j->part.data(), &j->st, &err);
            j->t_end = Clock::now();
            bool requeued = false;
            {
                std::lock_guard<std::mutex> lk(mu);
                in_use -= j->est;
                --running;
                if (j->exclusive) {
                    j->exclusive = false;
                    excl_running = false;
                }
                if (rc == AXC_ENOMEM && j->retries == 0) {
                    j->retries = 1;
                    j->est *= 2;
                    queue.push_front(j);
                    requeued = true;
                } else {
                    j->rc = rc;
                    j->err = err;
                    j->st.ms_queued = std::chrono::duration<double, std::milli>(j->t_start - j->t_submit).count();
                    j->st.ms_run = std::chrono::duration<double, std::milli>(j->t_end - j->t_start).count();
                    j->done = true;
                }
            }
            cv_work.notify_all();
            if (!requeued) cv_done.notify_all();
        }
    }

    int start(int dev) {
        device = dev;
        for (uint32_t i = 0; i < nlanes; ++i) {
            int rc = AXC_OK;
            Lane *l = lane_create(device, &rc);
            if (!l) return rc;
            lanes.push_back(l);
        }
        for (uint32_t i = 0; i < nlanes; ++i) threads.emplace_back([this, i] { run(i); });
        return AXC_OK;
    }

    // Stops the lanes after their running jobs, answers every job still queued with
    // AXC_ECANCELED and wakes its pollers. Idempotent.
    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        for (auto &t : threads)
            if (t.joinable()) t.join();
        {
            std::lock_guard<std::mutex> lk(mu);
            for (Job *j : queue) {
                j->rc = AXC_ECANCELED;
                j->err = "the context shut down before the job ran";
                j->done = true;
            }
            queue.clear();
        }
        cv_done.notify_all();
        for (Lane *l : lanes) lane_destroy(l);
        lanes.clear();
    }

    ~Executor() { shutdown(); }
};

// per-context executor, created at the first submit with the configured lanes and budget; held
// by shared_ptr so that a poller waiting on it keeps it alive while the context shuts down
static std::mutex g_mu;
static std::map<axc_ctx *, std::shared_ptr<Executor>> g_exec;
static std::map<axc_ctx *, ServeConfig> g_config;

static std::shared_ptr<Executor> executor_for(axc_ctx *ctx, int *rc) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_exec.find(ctx);
    if (it != g_exec.end()) {
        *rc = AXC_OK;
        return it->second;
    }
    auto x = std::make_shared<Executor>();
    ServeConfig cfg;
    if (auto it2 = g_config.find(ctx); it2 != g_config.end()) cfg = it2->second;
    x->nlanes = cfg.lanes;
    size_t budget = cfg.budget;
    if (budget == 0) budget = device_free_bytes(ctx_device(ctx)) / 2;
    x->budget = budget;
    x->excl_pins = cfg.excl_pins;
    if (const char *e = std::getenv("AXC_SERVE_EXCLUSIVE_PINS"); e && !cfg.excl_set)
        x->excl_pins = std::strtoull(e, nullptr, 10);
    for (int i = 0; i < TUNE_CLASSES; ++i) x->cls[i] = cfg.cls[i];
    ctx_tune_get(ctx, x->defaults);
    *rc = x->start(ctx_device(ctx));
    if (*rc) return nullptr;
    g_exec[ctx] = x;
    return x;
}

}  // namespace axc

using namespace axc;

extern "C" void axc_batch_free(axc_ctx *ctx) {
    std::shared_ptr<Executor> e;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_config.erase(ctx);
        auto it = g_exec.find(ctx);
        if (it == g_exec.end()) return;
        e = std::move(it->second);
        g_exec.erase(it);
    }
    e->shutdown();  // joins the lane threads, cancels queued jobs, wakes their pollers
}

extern "C" int axc_serve_configure(axc_ctx *ctx, uint32_t lanes, size_t device_budget) {
    if (!ctx || lanes == 0 || lanes > 256) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_exec.count(ctx)) return AXC_EBUSY;  // already serving
    ServeConfig &cfg = g_config[ctx];
    cfg.lanes = lanes;
    cfg.budget = device_budget;
    return AXC_OK;
}

extern "C" int axc_tune_set(axc_ctx *ctx, const char *key, uint64_t value) {
    if (!ctx || !key) return AXC_EINVAL;
    const std::string k(key);
    if (k.rfind("serve.", 0) != 0 && k.rfind("class.", 0) != 0) return ctx_tune_set(ctx, k, value);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_exec.count(ctx)) return AXC_EBUSY;  // the executor has started
    ServeConfig &cfg = g_config[ctx];
    if (k == "serve.exclusive_pins") {
        cfg.excl_pins = value;
        cfg.excl_set = true;
        return AXC_OK;
    }
    // class.<i>.<field>
    const size_t dot = k.find('.', 6);
    if (dot == std::string::npos || dot != 7) return AXC_ENOTFOUND;
    const char ci = k[6];
    if (ci < '0' || ci >= '0' + TUNE_CLASSES) return AXC_ENOTFOUND;
    TuneClass &t = cfg.cls[ci - '0'];
    const std::string field = k.substr(dot + 1);
    if (field == "min_pins") {
        t.min_pins = value;
    } else if (field == "rate.try_slots") {
        if (!tune_pow2_in(value, 64, 16384)) return AXC_EINVAL;
        t.rate_try = (uint32_t)value;
    } else if (field == "rate.mid_slots") {
        if (!tune_pow2_in(value, 64, 16384)) return AXC_EINVAL;
        t.rate_mid = (uint32_t)value;
    } else if (field == "cascade.block_movers") {
        if (value != 0 && !tune_pow2_in(value, 128, 2048)) return AXC_EINVAL;
        t.cascade_movers = (uint32_t)value;
    } else {
        return AXC_ENOTFOUND;
    }
    t.set = true;
    return AXC_OK;
}

extern "C" int axc_submit(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, uint64_t *job_id) {
    if (!ctx || !g || !p || !job_id) return AXC_EINVAL;
    if (g->e && (!g->hedge_off || !g->src_count)) return AXC_EINVAL;
    const uint64_t P = g->e ? g->hedge_off[g->e] : 0;
    if (P && !g->pins) return AXC_EINVAL;
    auto j = std::make_unique<Job>();
    j->t_submit = Clock::now();
    j->g.n = g->n;
    if (g->e) j->g.off.assign(g->hedge_off, g->hedge_off + g->e + 1);
    else j->g.off.assign(1, 0);
    j->g.pins.assign(g->pins, g->pins + P);
    j->g.nsrc.assign(g->src_count, g->src_count + g->e);
    if (g->hedge_w) j->g.w.assign(g->hedge_w, g->hedge_w + g->e);
    else j->g.w.assign(g->e, 1.0f);
    j->view.n = j->g.n;
    j->view.e = g->e;
    j->view.hedge_off = j->g.off.data();
    j->view.pins = j->g.pins.data();
    j->view.src_count = j->g.nsrc.data();
    j->view.hedge_w = j->g.w.data();
    j->p = *p;
    j->part.assign(g->n ? g->n : 1, 0);
    j->est = estimate_bytes(g);
    j->pins = P;
    int rc = AXC_OK;
    std::shared_ptr<Executor> x = executor_for(ctx, &rc);
    if (!x) return rc;
    {
        std::lock_guard<std::mutex> lk(x->mu);
        if (x->stop) return AXC_ECANCELED;
        j->id = x->next_id++;
        *job_id = j->id;
        x->queue.push_back(j.get());
        x->jobs[j->id] = std::move(j);
    }
    x->cv_work.notify_all();
    return AXC_OK;
}

extern "C" int axc_poll(axc_ctx *ctx, uint64_t job_id, uint32_t *out_part, axc_stats *stats, int timeout_ms) {
    if (!ctx) return AXC_EINVAL;
    int rc = AXC_OK;
    std::shared_ptr<Executor> x = executor_for(ctx, &rc);  // kept alive while this call waits
    if (!x) return rc;
    std::unique_lock<std::mutex> lk(x->mu);
    auto it = x->jobs.find(job_id);
    if (it == x->jobs.end()) return AXC_ENOTFOUND;
    Job *j = it->second.get();
    auto ready = [&] { return j->done; };
    if (timeout_ms < 0) x->cv_done.wait(lk, ready);
    else if (!x->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return AXC_ETIMEDOUT;
    rc = j->rc;
    if (out_part && j->g.n) std::memcpy(out_part, j->part.data(), (size_t)j->g.n * 4);
    if (stats) *stats = j->st;
    x->jobs.erase(it);
    return rc;
}

extern "C" int axc_partition_batch(axc_ctx *ctx, uint32_t count, const axc_hgraph *g, const axc_params *p,
                                   uint32_t *const *out_parts, axc_stats *stats) {
    if (!ctx || (count && (!g || !p || !out_parts))) return AXC_EINVAL;
    std::vector<uint64_t> ids(count, 0);
    int first = AXC_OK;
    for (uint32_t i = 0; i < count; ++i) {
        const int rc = axc_submit(ctx, &g[i], &p[i], &ids[i]);
        if (rc) {
            ids[i] = 0;
            if (!first) first = rc;
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (!ids[i]) continue;
        const int rc = axc_poll(ctx, ids[i], out_parts[i], stats ? &stats[i] : nullptr, -1);
        if (rc && !first) first = rc;
    }
    return first;
}
