// Job queue behind axc_submit / axc_poll / axc_partition_batch: a worker thread owns the device
// context and runs admitted jobs; callers wait on per-job completion. Admission compares a job's
// device-memory estimate against the context arena.
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "axc_host.h"

struct axc_ctx;
extern "C" int axc_partition(axc_ctx *, const axc_hgraph *, const axc_params *, uint32_t *, axc_stats *);

namespace axc {

struct Job {
    uint64_t id = 0;
    HostGraph g;
    axc_hgraph view{};
    axc_params p{};
    std::vector<uint32_t> part;
    axc_stats st{};
    int rc = 0;
    bool done = false;
};

struct BatchState {
    axc_ctx *ctx = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    bool stop = false;
    uint64_t next_id = 1;

    void run() {
        for (;;) {
            Job *j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop && queue.empty()) return;
                j = queue.front();
                queue.pop_front();
            }
            int rc = axc_partition(ctx, &j->view, &j->p, j->part.data(), &j->st);
            {
                std::lock_guard<std::mutex> lk(mu);
                j->rc = rc;
                j->done = true;
            }
            cv_done.notify_all();
        }
    }
};

// per-context batching state, created lazily
static std::mutex g_mu;
static std::map<axc_ctx *, std::unique_ptr<BatchState>> g_states;

static BatchState *state_for(axc_ctx *ctx) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto &s = g_states[ctx];
    if (!s) {
        s.reset(new BatchState());
        s->ctx = ctx;
        s->worker = std::thread([p = s.get()] { p->run(); });
    }
    return s.get();
}

}  // namespace axc

using namespace axc;

extern "C" void axc_batch_free(axc_ctx *ctx) {
    std::unique_ptr<BatchState> s;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_states.find(ctx);
        if (it == g_states.end()) return;
        s = std::move(it->second);
        g_states.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
}

extern "C" int axc_submit(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, uint64_t *job_id) {
    if (!ctx || !g || !p || !job_id) return AXC_EINVAL;
    auto j = std::make_unique<Job>();
    const uint64_t P = g->e ? g->hedge_off[g->e] : 0;
    j->g.n = g->n;
    j->g.off.assign(g->hedge_off, g->hedge_off + g->e + 1);
    if (!g->e) j->g.off.assign(1, 0);
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
    BatchState *s = state_for(ctx);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        j->id = s->next_id++;
        *job_id = j->id;
        s->queue.push_back(j.get());
        s->jobs[j->id] = std::move(j);
    }
    s->cv_work.notify_one();
    return AXC_OK;
}

extern "C" int axc_poll(axc_ctx *ctx, uint64_t job_id, uint32_t *out_part, axc_stats *stats, int timeout_ms) {
    if (!ctx) return AXC_EINVAL;
    BatchState *s = state_for(ctx);
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return AXC_ENOTFOUND;
    Job *j = it->second.get();
    auto ready = [&] { return j->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return AXC_ETIMEDOUT;
    int rc = j->rc;
    if (out_part && j->g.n) std::memcpy(out_part, j->part.data(), (size_t)j->g.n * 4);
    if (stats) *stats = j->st;
    s->jobs.erase(it);
    return rc;
}

extern "C" int axc_partition_batch(axc_ctx *ctx, uint32_t count, const axc_hgraph *g, const axc_params *p,
                                   uint32_t *const *out_parts, axc_stats *stats) {
    if (!ctx || (count && (!g || !p || !out_parts))) return AXC_EINVAL;
    for (uint32_t i = 0; i < count; ++i) {
        int rc = axc_partition(ctx, &g[i], &p[i], out_parts[i], stats ? &stats[i] : nullptr);
        if (rc) return rc;
    }
    return AXC_OK;
}
