// Context, the multilevel driver and the C ABI (include/axc.h).
//
// The driver restates main()'s recursion (sources/main.cu:282-800) as an explicit level stack in
// one device arena: level l+1 is allocated on top of level l, so uncoarsening pops levels in LIFO
// order. Stop rules follow sources/main.cu:358, 448, 495-500 and headers/defines.cuh:28-37.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "axc_host.h"

struct axc_ctx {
    axc::Ctx c;
    std::mutex mu;
    void *batch = nullptr;  // batching / serving state (batch.cpp)
};

namespace axc {

struct Resolved {
    bool kway;
    u32 omega, delta, max_parts, k, target, omega_c, cnc, rfr;
    int ipm;
    u64 seed;
    int verbose;
};

// Phase log on stderr (-v 1 and up): synchronizes the stream, so it perturbs timing.
struct PhaseLog {
    Ctx &c;
    int on;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double ms() {
        cudaStreamSynchronize(c.stream);
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    template <class... A>
    void operator()(const char *fmt, A... a) {
        if (!on) return;
        const double t = ms();
        std::fprintf(stderr, "[axc %9.2f ms] ", t);
        std::fprintf(stderr, fmt, a...);
        std::fprintf(stderr, "  (arena %.2f GB, peak %.2f GB)\n", c.arena.top / 1e9, c.arena.peak / 1e9);
    }
};

static int resolve(const axc_params *p, u32 n, Resolved &r) {
    if (!p) return AXC_EINVAL;
    r.kway = p->mode == AXC_MODE_KWAY;
    r.cnc = p->cnc ? p->cnc : 1;
    if (r.cnc > AXC_MAX_CANDIDATES) return AXC_EINVAL;
    r.rfr = p->rfr;
    r.ipm = p->ipm;
    r.seed = p->seed;
    r.verbose = p->verbose;
    if (r.kway) {
        if (p->k == 0 || !(p->eps >= 0.0f)) return AXC_EINVAL;
        r.k = p->k;
        r.omega = axc_kway_omega(n, p->k, p->eps);
        r.delta = 0x7FFFFFFFu;  // sources/runconfig.cpp:191
        r.max_parts = p->k;
        // clusters stay below the balance slack so that weight chunks of the coarsest level fit
        double slack = std::floor((double)p->eps * (double)n / (double)p->k);
        r.omega_c = (u32)std::max(1.0, std::min<double>(slack, (double)r.omega));
    } else {
        if (p->omega == 0 || p->delta == 0 || p->max_parts == 0) return AXC_EINVAL;
        r.k = 0;
        r.omega = p->omega;
        r.delta = p->delta;
        r.max_parts = p->max_parts;
        r.omega_c = p->omega;
    }
    r.target = std::min<u32>(r.max_parts, (u32)(((u64)n + r.omega - 1) / r.omega));
    return AXC_OK;
}

// Allocate and build level 0 from a raw device hypergraph (dedupe + incidence CSR).
static DLevel build_level0(Ctx &c, u32 n, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc, u64 P_in) {
    DLevel L;
    check_input(c, n, e, off, pins, nsrc);
    L.arena_mark = c.arena.mark();
    L.n = n;
    L.e = e;
    L.off = c.arena.alloc<u64>((u64)e + 1);
    L.nsrc = c.arena.alloc<u32>(e ? e : 1);
    L.pins = c.arena.alloc<u32>(P_in ? P_in : 1);
    L.P = hedge_unique(c, e, off, pins, nsrc, nullptr, false, L.off, L.pins, L.nsrc, P_in);
    L.toff = c.arena.alloc<u64>((u64)n + 1);
    L.touch = c.arena.alloc<u32>(L.P ? L.P : 1);
    L.nin = c.arena.alloc<u32>(n ? n : 1);
    build_touching(c, n, e, L.off, L.pins, L.nsrc, L.P, L.toff, L.touch, L.nin);
    L.nsize = c.arena.alloc<u32>(n ? n : 1);
    fill_u32(c, L.nsize, 1u, n);
    L.groups = c.arena.alloc<u32>(n ? n : 1);
    return L;
}

static DLevel build_coarse(Ctx &c, const DLevel &F) {
    DLevel L;
    L.arena_mark = c.arena.mark();
    L.n = F.ngroups;
    L.e = F.e;
    L.off = c.arena.alloc<u64>((u64)F.e + 1);
    L.nsrc = c.arena.alloc<u32>(F.e ? F.e : 1);
    // the coarse pin count is bounded by the fine one; trim after the count is known
    const size_t before_pins = c.arena.mark();
    L.pins = c.arena.alloc<u32>(F.P ? F.P : 1);
    L.P = hedge_unique(c, F.e, F.off, F.pins, F.nsrc, F.groups, true, L.off, L.pins, L.nsrc, F.P);
    c.arena.release(before_pins);
    L.pins = c.arena.alloc<u32>(L.P ? L.P : 1);  // same address, tighter size
    L.toff = c.arena.alloc<u64>((u64)L.n + 1);
    L.touch = c.arena.alloc<u32>(L.P ? L.P : 1);
    L.nin = c.arena.alloc<u32>(L.n ? L.n : 1);
    build_touching(c, L.n, L.e, L.off, L.pins, L.nsrc, L.P, L.toff, L.touch, L.nin);
    L.nsize = c.arena.alloc<u32>(L.n ? L.n : 1);
    group_sizes(c, F.n, F.groups, F.nsize, L.nsize, L.n);
    L.groups = c.arena.alloc<u32>(L.n ? L.n : 1);
    return L;
}

// The multilevel core on a raw hypergraph in device memory; writes d_out[n]. Returns K'.
static u32 partition_core(Ctx &c, u32 n, u32 e, const u64 *d_off, const u32 *d_pins, const u32 *d_nsrc,
                          const float *d_w, u64 P_in, const Resolved &R, u32 *d_out, axc_stats *st,
                          cudaEvent_t ev_core) {
    const size_t base = c.arena.mark();
    PhaseLog log{c, R.verbose};
    u32 *wfx = c.arena.alloc<u32>(e ? e : 1);
    compute_wfx(c, d_w, wfx, e);
    std::vector<DLevel> lv;
    lv.push_back(build_level0(c, n, e, d_off, d_pins, d_nsrc, P_in));
    log("level 0 built: n %u, e %u, pins %llu", n, e, (unsigned long long)lv[0].P);
    if (st) st->pins = lv[0].P;
    if (ev_core) AXC_CUDA(cudaEventRecord(ev_core, c.stream));
    u32 K = 0;
    bool refine_deepest = false;
    u32 *deep_part = nullptr;
    for (u32 l = 0;; ++l) {
        DLevel &cur = lv.back();
        if (st && l < 64) { st->level_pins[l] = cur.P; st->level_nodes[l] = cur.n; }
        if (R.kway && cur.n < 8192) {  // KWAY_INIT_UPPER_THREASHOLD (headers/defines.cuh:35)
            deep_part = c.arena.alloc<u32>(cur.n ? cur.n : 1);
            kway_initial(c, cur, R.k, deep_part);
            K = R.k;
            refine_deepest = !kway_multistart(c, cur, wfx, R.k, R.omega, R.seed, deep_part);
            break;
        }
        const size_t tmp = c.arena.mark();
        u32 *pairs = c.arena.alloc<u32>((u64)cur.n * R.cnc), *scores = c.arena.alloc<u32>((u64)cur.n * R.cnc);
        u64 visits = 0;
        rating(c, cur, wfx, R.kway ? R.omega_c : R.omega, R.delta, R.cnc, pairs, scores, st ? &visits : nullptr);
        if (st) st->rating_pin_visits += visits;
        log("level %u rated", l);
        u32 ng = matching(c, cur.n, R.cnc, pairs, scores, cur.nsize, cur.nin, R.kway ? R.omega_c : R.omega, R.delta, 32,
                          cur.groups);
        c.arena.release(tmp);
        log("level %u matched: %u -> %u groups", l, cur.n, ng);
        const float ratio = (float)ng / (float)cur.n;
        if (R.kway && (ratio > 0.95f || ng < 1024)) {  // headers/defines.cuh:36-37
            deep_part = c.arena.alloc<u32>(cur.n ? cur.n : 1);
            kway_initial(c, cur, R.k, deep_part);
            K = R.k;
            refine_deepest = !kway_multistart(c, cur, wfx, R.k, R.omega, R.seed, deep_part);
            break;
        }
        if (!R.kway && (ng <= R.target || ng == cur.n || (l >= 32 && ratio > 0.95f))) {
            if (R.ipm) ng = greedy_merge_groups(c, cur.n, cur.nsize, cur.nin, cur.groups, ng, R.omega, R.delta);
            deep_part = cur.groups;
            K = ng;
            break;
        }
        cur.ngroups = ng;
        DLevel nx = build_coarse(c, lv.back());
        lv.push_back(nx);
        log("level %u built: n %u, pins %llu", l + 1, nx.n, (unsigned long long)nx.P);
    }
    log("initial partition: %u parts at level %zu", K, lv.size() - 1);
    if (st) st->levels = (u32)lv.size();
    // uncoarsen and refine, popping levels
    RefineParams rp{K, R.omega, R.delta, !R.kway, R.rfr, R.seed};
    const int deepest = (int)lv.size() - 1;
    u32 *upper = deep_part;  // partition of the level above the one being processed
    for (int l = deepest; l >= 0; --l) {
        DLevel &L = lv[l];
        u32 *part;
        if (l == deepest) {
            part = deep_part;
        } else {
            part = c.arena.alloc<u32>(L.n ? L.n : 1);  // above level l+1's arrays; copied below
            uncoarsen(c, L.n, L.groups, upper, part);
            // drop level l+1 (and everything above it), keeping `part` by moving it down
            const size_t keep_at = lv[l + 1].arena_mark;
            c.arena.release(keep_at);
            u32 *moved = c.arena.alloc<u32>(L.n ? L.n : 1);
            if (moved != part)
                AXC_CUDA(cudaMemcpyAsync(moved, part, (size_t)L.n * 4, cudaMemcpyDeviceToDevice, c.stream));
            part = moved;
        }
        if (l < deepest || refine_deepest) {
            u32 rr = refine_level(c, L, wfx, rp, part);
            if (st && l < 64) st->refine_rounds[l] = rr;
            log("level %d refined: %u rounds", l, rr);
        }
        upper = part;
    }
    u32 *final_part = upper;
    if (!R.kway) merge_small_partitions(c, lv[0], final_part, K, R.omega, R.delta);
    const u32 Kp = zero_base(c, n, final_part, K);
    AXC_CUDA(cudaMemcpyAsync(d_out, final_part, (size_t)n * 4, cudaMemcpyDeviceToDevice, c.stream));
    log("done: %u parts", Kp);
    c.arena.release(base);
    return Kp;
}

static int guard(axc_ctx *ctx, const std::exception &e) {
    if (auto *x = dynamic_cast<const Error *>(&e)) {
        if (ctx) ctx->c.last_error = x->what();
        return x->code;
    }
    if (ctx) ctx->c.last_error = e.what();
    return AXC_EINTERNAL;
}

}  // namespace axc

using namespace axc;

extern "C" {

const char *axc_strerror(int s) {
    switch (s) {
        case AXC_OK: return "ok";
        case AXC_EINVAL: return "invalid argument";
        case AXC_ENOMEM: return "out of device memory";
        case AXC_ECUDA: return "CUDA error";
        case AXC_EIO: return "I/O error";
        case AXC_EFORMAT: return "malformed input";
        case AXC_EINFEASIBLE: return "partition violates the constraints";
        case AXC_ETIMEDOUT: return "timed out";
        case AXC_ENOTFOUND: return "unknown job";
        case AXC_EBUSY: return "admission refused by the memory budget";
        case AXC_EINTERNAL: return "internal device check failed";
        case AXC_EOVERFLOW: return "size exceeds the limit of this call";
        case AXC_ECANCELED: return "the context shut down before the job ran";
        default: return "unknown status";
    }
}

const char *axc_last_error(axc_ctx *ctx) { return ctx ? ctx->c.last_error.c_str() : ""; }

void axc_params_default(axc_params *p, int mode) {
    std::memset(p, 0, sizeof(*p));
    p->mode = mode;
    p->cnc = AXC_MAX_CANDIDATES;   // MAX_CANDIDATES (headers/defines.cuh:49)
    p->rfr = 16;                   // REFINE_REPEATS (headers/defines.cuh:54)
    p->smh = 2;                    // SAVE_MEMORY_UP_TO_LEVEL (headers/defines.cuh:31)
    p->om = 1.5f;                  // OVERSIZED_SIZE_MULTIPLIER (headers/defines.cuh:26)
    p->omega = 1024; p->delta = 4096; p->max_parts = 4096;  // loihi64, the CLI default
    p->k = 2;
    p->eps = 0.03f;
}

int axc_params_preset(axc_params *p, const char *name) {
    if (!p || !name) return AXC_EINVAL;
    struct { const char *n; u32 o, d, k; } t[] = {
        {"loihi64", 1024, 4096, 4096}, {"loihi84", 4096, 1024 * 64, 7056},
        {"loihi1024", 4096, 1024 * 64, 1048576}, {"truenorth", 256, 256, 4096}};
    for (auto &x : t)
        if (!std::strcmp(x.n, name)) {
            p->mode = AXC_MODE_INCC;
            p->omega = x.o; p->delta = x.d; p->max_parts = x.k;
            return AXC_OK;
        }
    return AXC_EINVAL;
}

uint32_t axc_kway_omega(uint32_t n, uint32_t k, float eps) {
    return (uint32_t)std::ceil((1 + eps) * (float)n / k);  // sources/runconfig.cpp:190
}

int axc_create(int device, size_t arena_bytes, axc_ctx **out) {
    if (!out) return AXC_EINVAL;
    auto *x = new axc_ctx();
    try {
        Ctx &c = x->c;
        c.device = device;
        AXC_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        AXC_CUDA(cudaGetDeviceProperties(&prop, device));
        c.sms = prop.multiProcessorCount;
        c.smem_optin = prop.sharedMemPerBlockOptin;
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
        c.coop_supported = coop;
        AXC_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        if (arena_bytes == 0) {
            size_t fr = 0, tot = 0;
            AXC_CUDA(cudaMemGetInfo(&fr, &tot));
            arena_bytes = (size_t)((double)fr * 0.6);
        }
        AXC_CUDA(cudaMalloc(&c.arena.base, arena_bytes));
        c.arena.cap = arena_bytes;
        AXC_CUDA(cudaMalloc(&c.d_status, STATUS_BYTES));
        AXC_CUDA(cudaMemset(c.d_status, 0, STATUS_BYTES));
        AXC_CUDA(cudaHostAlloc((void **)&c.h_pinned, 4096, cudaHostAllocDefault));
        setup_construct_kernels();
        setup_prim_kernels();
        setup_coarsen_kernels(c);
        setup_refine_kernels(c);
        scan_state_create(c, 1u << 18);  // single-pass scans of up to 2^29 elements
        AXC_CUDA(cudaDeviceSynchronize());
    } catch (const std::exception &e) {
        int rc = guard(x, e);
        axc_destroy(x);
        return rc;
    }
    *out = x;
    return AXC_OK;
}

int axc_profile_kernel(axc_ctx *ctx, const char *kernel) {
    if (!ctx) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    c.prof_on = kernel != nullptr;
    c.prof_name = kernel ? kernel : "";
    c.prof_used = 0;
    c.prof_bytes = 0;
    c.prof_ms = 0;
    c.prof_launches = 0;
    if (c.d_status && cudaMemset(c.d_prof_bytes(), 0, 8ull * PROF_SLOTS * PROF_STRIDE) != cudaSuccess)
        return AXC_ECUDA;
    return AXC_OK;
}

int axc_profile_read(axc_ctx *ctx, axc_kernel_timing *out) {
    if (!ctx || !out) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        c.prof_collect(0, c.prof_used);
        unsigned long long slots[PROF_SLOTS * PROF_STRIDE], dev_bytes = 0;  // bytes the profiled kernel counted
        AXC_CUDA(cudaMemcpy(slots, c.d_prof_bytes(), sizeof slots, cudaMemcpyDeviceToHost));
        AXC_CUDA(cudaMemset(c.d_prof_bytes(), 0, sizeof slots));
        for (unsigned i = 0; i < PROF_SLOTS; ++i) dev_bytes += slots[i * PROF_STRIDE];
        out->launches = c.prof_launches;
        out->ms_total = c.prof_ms;
        out->bytes = c.prof_bytes + dev_bytes;
        c.prof_used = 0;
        c.prof_bytes = 0;
        c.prof_ms = 0;
        c.prof_launches = 0;
    } catch (const std::exception &e) {
        return guard(ctx, e);
    }
    return AXC_OK;
}

void axc_destroy(axc_ctx *ctx) {
    if (!ctx) return;
    Ctx &c = ctx->c;
    extern void axc_batch_free(axc_ctx *);
    axc_batch_free(ctx);
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (cudaEvent_t e : c.prof_ev) cudaEventDestroy(e);
    if (c.arena.base) cudaFree(c.arena.base);
    if (c.d_status) cudaFree(c.d_status);
    scan_state_destroy(c);
    if (c.h_pinned) cudaFreeHost(c.h_pinned);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete ctx;
}

static int check_graph(const axc_hgraph *g) {
    if (!g || (g->e && (!g->hedge_off || !g->src_count)) || (!g->pins && g->e && g->hedge_off && g->hedge_off[g->e]))
        return AXC_EINVAL;
    return AXC_OK;
}

int axc_partition_device(axc_ctx *ctx, const axc_hgraph *d_g, const axc_params *p, uint32_t *d_out_part,
                         axc_stats *stats) {
    if (!ctx || !d_g || !p || !d_out_part) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        Resolved R;
        int rc = resolve(p, d_g->n, R);
        if (rc) return rc;
        if (d_g->n == 0) return AXC_OK;
        u64 P = 0;
        if (d_g->e) AXC_CUDA(cudaMemcpy(&P, d_g->hedge_off + d_g->e, 8, cudaMemcpyDeviceToHost));
        axc_stats local;
        std::memset(&local, 0, sizeof local);
        axc_stats *st = stats ? stats : &local;
        std::memset(st, 0, sizeof *st);
        c.launches = 0;
        const size_t top0 = c.arena.top;
        c.arena.peak = top0;
        cudaEvent_t e0, e1, ec;
        AXC_CUDA(cudaEventCreate(&e0));
        AXC_CUDA(cudaEventCreate(&e1));
        AXC_CUDA(cudaEventCreate(&ec));
        AXC_CUDA(cudaEventRecord(e0, c.stream));
        const u32 Kp = partition_core(c, d_g->n, d_g->e, d_g->hedge_off, d_g->pins, d_g->src_count, d_g->hedge_w, P, R,
                                      d_out_part, st, ec);
        AXC_CUDA(cudaEventRecord(e1, c.stream));
        AXC_CUDA(cudaEventSynchronize(e1));
        float ms = 0, mc = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventElapsedTime(&mc, ec, e1);
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(ec);
        st->ms_device = ms;
        st->ms_core = mc;
        st->num_parts = Kp;
        st->kernel_launches = c.launches;
        st->device_bytes_peak = c.arena.peak - top0;
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

// Upload a host hypergraph into the arena (raw, as given). Returns the device view.
static axc_hgraph upload(Ctx &c, const axc_hgraph *g, u64 &P) {
    P = g->e ? g->hedge_off[g->e] : 0;
    axc_hgraph d{};
    d.n = g->n;
    d.e = g->e;
    u64 *off = c.arena.alloc<u64>((u64)g->e + 1);
    u32 *pins = c.arena.alloc<u32>(P ? P : 1), *ns = c.arena.alloc<u32>(g->e ? g->e : 1);
    float *w = g->hedge_w ? c.arena.alloc<float>(g->e ? g->e : 1) : nullptr;
    if (g->e) {
        AXC_CUDA(cudaMemcpyAsync(off, g->hedge_off, ((size_t)g->e + 1) * 8, cudaMemcpyHostToDevice, c.stream));
        AXC_CUDA(cudaMemcpyAsync(ns, g->src_count, (size_t)g->e * 4, cudaMemcpyHostToDevice, c.stream));
        if (w) AXC_CUDA(cudaMemcpyAsync(w, g->hedge_w, (size_t)g->e * 4, cudaMemcpyHostToDevice, c.stream));
    } else {
        AXC_CUDA(cudaMemsetAsync(off, 0, 8, c.stream));
    }
    if (P) AXC_CUDA(cudaMemcpyAsync(pins, g->pins, (size_t)P * 4, cudaMemcpyHostToDevice, c.stream));
    d.hedge_off = off;
    d.pins = pins;
    d.src_count = ns;
    d.hedge_w = w;
    check_input(c, g->n, g->e, off, pins, ns);
    return d;
}

static int validate_ids(const axc_hgraph *g) {
    const u64 P = g->e ? g->hedge_off[g->e] : 0;
    for (u32 h = 0; h < g->e; ++h) {
        if (g->hedge_off[h + 1] < g->hedge_off[h]) return AXC_EINVAL;
        if (g->src_count[h] > g->hedge_off[h + 1] - g->hedge_off[h]) return AXC_EINVAL;
    }
    (void)P;
    return AXC_OK;
}

}  // extern "C"

namespace axc {
// axc_partition on a given context (the caller serializes calls on it): upload, partition,
// download and, when stats are wanted, the metrics of the result.
int partition_host(Ctx &c, const axc_hgraph *g, const axc_params *p, uint32_t *out_part, axc_stats *stats) {
    if (check_graph(g) || !p || (!out_part && g->n)) return AXC_EINVAL;
    if (int rc = validate_ids(g)) return rc;
    try {
        Resolved R;
        int rc = resolve(p, g->n, R);
        if (rc) return rc;
        if (g->n == 0) return AXC_OK;
        axc_stats local;
        axc_stats *st = stats ? stats : &local;
        std::memset(st, 0, sizeof *st);
        c.launches = 0;
        const size_t top0 = c.arena.top;
        c.arena.peak = top0;
        cudaEvent_t e0, e1, ec;
        AXC_CUDA(cudaEventCreate(&e0));
        AXC_CUDA(cudaEventCreate(&e1));
        AXC_CUDA(cudaEventCreate(&ec));
        AXC_CUDA(cudaEventRecord(e0, c.stream));
        const size_t m = c.arena.mark();
        u64 P = 0;
        axc_hgraph d = upload(c, g, P);
        u32 *d_out = c.arena.alloc<u32>(g->n);
        const u32 Kp = partition_core(c, g->n, g->e, d.hedge_off, d.pins, d.src_count, d.hedge_w, P, R, d_out, st, ec);
        AXC_CUDA(cudaMemcpyAsync(out_part, d_out, (size_t)g->n * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaEventRecord(e1, c.stream));
        AXC_CUDA(cudaEventSynchronize(e1));
        float ms = 0, mc = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventElapsedTime(&mc, ec, e1);
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(ec);
        st->ms_device = ms;
        st->ms_core = mc;
        st->num_parts = Kp;
        st->kernel_launches = c.launches;
        st->device_bytes_peak = c.arena.peak - top0;
        if (stats) {
            // metrics of the result on the deduplicated graph (untimed, like sources/main.cu:917-928)
            DLevel L0 = build_level0(c, g->n, g->e, d.hedge_off, d.pins, d.src_count, P);
            u32 *wfx = c.arena.alloc<u32>(g->e ? g->e : 1);
            compute_wfx(c, d.hedge_w, wfx, g->e);
            axc_stats ev;
            std::memset(&ev, 0, sizeof ev);
            evaluate(c, L0, wfx, d_out, R.omega, R.delta, R.max_parts, &ev);
            st->connectivity_fx = ev.connectivity_fx; st->cutnet_fx = ev.cutnet_fx; st->soed_fx = ev.soed_fx;
            st->connectivity = ev.connectivity; st->cutnet = ev.cutnet; st->soed = ev.soed;
            st->max_part_size = ev.max_part_size; st->max_part_inbound = ev.max_part_inbound;
            st->valid = ev.valid;
        }
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        if (auto *x = dynamic_cast<const Error *>(&e)) {
            c.last_error = x->what();
            return x->code;
        }
        c.last_error = e.what();
        return AXC_EINTERNAL;
    }
}

// ---------------------------------------------------------------- lanes (batching and serving)
// A lane is a context without an arena of its own: a stream, a status word, a pinned staging
// buffer and a scan state. Each job gets a device arena from the stream-ordered allocator on the
// lane's stream, sized by the caller, and returns it when it finishes.
struct Lane {
    Ctx c;
};

int ctx_device(axc_ctx *ctx) { return ctx ? ctx->c.device : 0; }

size_t device_free_bytes(int device) {
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 0;
    return fr;
}

void lane_destroy(Lane *l) {
    if (!l) return;
    Ctx &c = l->c;
    if (c.stream) cudaStreamSynchronize(c.stream);
    if (c.d_status) cudaFree(c.d_status);
    if (c.h_pinned) cudaFreeHost(c.h_pinned);
    scan_state_destroy(c);
    if (c.stream) cudaStreamDestroy(c.stream);
    for (cudaEvent_t e : c.prof_ev) cudaEventDestroy(e);
    delete l;
}

Lane *lane_create(int device, int *rc) {
    auto *l = new Lane();
    Ctx &c = l->c;
    try {
        c.device = device;
        AXC_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        AXC_CUDA(cudaGetDeviceProperties(&prop, device));
        c.sms = prop.multiProcessorCount;
        c.smem_optin = prop.sharedMemPerBlockOptin;
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
        c.coop_supported = coop;
        AXC_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        AXC_CUDA(cudaMalloc(&c.d_status, STATUS_BYTES));
        AXC_CUDA(cudaMemset(c.d_status, 0, STATUS_BYTES));
        AXC_CUDA(cudaHostAlloc((void **)&c.h_pinned, 4096, cudaHostAllocDefault));
        scan_state_create(c, 1u << 18);
        // freed job arenas stay in the pool for the next job instead of going back to the driver
        cudaMemPool_t pool;
        AXC_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        u64 keep = ~0ull;
        AXC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        *rc = AXC_OK;
    } catch (const std::exception &e) {
        auto *x = dynamic_cast<const Error *>(&e);
        *rc = x ? x->code : AXC_ECUDA;
        lane_destroy(l);
        return nullptr;
    }
    return l;
}

void lane_tune(Lane *l, uint32_t rate_try, uint32_t rate_mid, uint32_t cascade_movers) {
    l->c.tune.rate_try = rate_try;
    l->c.tune.rate_mid = rate_mid;
    l->c.tune.cascade_movers = cascade_movers;
}

void ctx_tune_get(axc_ctx *ctx, uint32_t out[3]) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    out[0] = ctx->c.tune.rate_try;
    out[1] = ctx->c.tune.rate_mid;
    out[2] = ctx->c.tune.cascade_movers;
}

bool tune_pow2_in(uint64_t v, uint64_t lo, uint64_t hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

// The context's own tile and table sizes (include/axc.h axc_tune_set); AXC_ENOTFOUND for other keys.
int ctx_tune_set(axc_ctx *ctx, const std::string &key, uint64_t v) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    Tune &t = ctx->c.tune;
    if (key == "rate.try_slots") {
        if (!tune_pow2_in(v, 64, 16384)) return AXC_EINVAL;
        t.rate_try = (u32)v;
    } else if (key == "rate.mid_slots") {
        if (!tune_pow2_in(v, 64, 16384)) return AXC_EINVAL;
        t.rate_mid = (u32)v;
    } else if (key == "cascade.block_movers") {
        if (v != 0 && !tune_pow2_in(v, 128, 2048)) return AXC_EINVAL;
        t.cascade_movers = (u32)v;
    } else {
        return AXC_ENOTFOUND;
    }
    return AXC_OK;
}

// One job on the lane in a fresh arena of `arena_bytes`. AXC_ENOMEM when the arena cannot be had
// or turns out too small.
int lane_partition(Lane *l, size_t arena_bytes, const axc_hgraph *g, const axc_params *p, uint32_t *out_part,
                   axc_stats *stats, std::string *err) {
    Ctx &c = l->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return AXC_ECUDA;
    void *mem = nullptr;
    if (cudaMallocAsync(&mem, arena_bytes, c.stream) != cudaSuccess) {
        cudaGetLastError();
        if (err) *err = "device arena of " + std::to_string(arena_bytes) + " bytes not available";
        return AXC_ENOMEM;
    }
    c.arena.base = (char *)mem;
    c.arena.cap = arena_bytes;
    c.arena.top = 0;
    c.arena.peak = 0;
    const int rc = partition_host(c, g, p, out_part, stats);
    if (rc && err) *err = c.last_error;
    cudaFreeAsync(mem, c.stream);
    cudaStreamSynchronize(c.stream);
    c.arena = Arena();
    return rc;
}

}  // namespace axc

extern "C" {

int axc_partition(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, uint32_t *out_part, axc_stats *stats) {
    if (!ctx) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    return partition_host(ctx->c, g, p, out_part, stats);
}

int axc_evaluate(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, const uint32_t *part, axc_stats *stats) {
    if (!ctx || check_graph(g) || !p || !stats || (!part && g->n)) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        Resolved R;
        int rc = resolve(p, g->n, R);
        if (rc) return rc;
        std::memset(stats, 0, sizeof *stats);
        const size_t m = c.arena.mark();
        u64 P = 0;
        axc_hgraph d = upload(c, g, P);
        DLevel L;
        L.n = g->n; L.e = g->e; L.P = P;
        L.off = (u64 *)d.hedge_off; L.pins = (u32 *)d.pins; L.nsrc = (u32 *)d.src_count;
        u32 *dp = c.arena.alloc<u32>(g->n ? g->n : 1);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(dp, part, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
        u32 *wfx = c.arena.alloc<u32>(g->e ? g->e : 1);
        compute_wfx(c, d.hedge_w, wfx, g->e);
        evaluate(c, L, wfx, dp, R.omega, R.delta, R.max_parts, stats);
        stats->pins = P;
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_quotient_hgraph_device(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, axc_hgraph *out) {
    if (!ctx || check_graph(g) || !out || (!part && g->n)) return AXC_EINVAL;
    uint32_t K = 0;
    for (uint32_t v = 0; v < g->n; ++v) K = std::max(K, part[v] + 1);
    if (g->n && K == 0) return AXC_EOVERFLOW;  // an id of 2^32 - 1
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u64 P = 0;
        axc_hgraph d = upload(c, g, P);
        u32 *dp = c.arena.alloc<u32>(g->n ? g->n : 1);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(dp, part, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
        std::vector<u32> qcnt, qsrc, qpins;
        quotient_extract(c, g->e, P, d.hedge_off, d.pins, d.src_count, dp, K, qcnt, qsrc, qpins);
        c.arena.release(m);
        publish(quotient_merge(K, g->e, qcnt, qsrc, qpins, g->hedge_w), out);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

// ---------------------------------------------------------------- stage entry points
int axc_stage_construct(axc_ctx *ctx, const axc_hgraph *g, uint64_t *out_hedge_off, uint32_t *out_pins,
                        uint32_t *out_src_count, uint64_t *out_touch_off, uint32_t *out_touch, uint32_t *out_inbound,
                        uint64_t *out_pins_after) {
    if (!ctx || check_graph(g)) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u64 P = 0;
        axc_hgraph d = upload(c, g, P);
        DLevel L = build_level0(c, g->n, g->e, d.hedge_off, d.pins, d.src_count, P);
        AXC_CUDA(cudaMemcpyAsync(out_hedge_off, L.off, ((size_t)g->e + 1) * 8, cudaMemcpyDeviceToHost, c.stream));
        if (L.P) AXC_CUDA(cudaMemcpyAsync(out_pins, L.pins, L.P * 4, cudaMemcpyDeviceToHost, c.stream));
        if (g->e) AXC_CUDA(cudaMemcpyAsync(out_src_count, L.nsrc, (size_t)g->e * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaMemcpyAsync(out_touch_off, L.toff, ((size_t)g->n + 1) * 8, cudaMemcpyDeviceToHost, c.stream));
        if (L.P) AXC_CUDA(cudaMemcpyAsync(out_touch, L.touch, L.P * 4, cudaMemcpyDeviceToHost, c.stream));
        if (g->n) AXC_CUDA(cudaMemcpyAsync(out_inbound, L.nin, (size_t)g->n * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        if (out_pins_after) *out_pins_after = L.P;
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

// Level graph as given (already deduplicated) + incidence CSR.
static DLevel upload_level(Ctx &c, const axc_hgraph *g, const uint32_t *node_size, u32 **wfx_out) {
    u64 P = 0;
    axc_hgraph d = upload(c, g, P);
    DLevel L;
    L.n = g->n; L.e = g->e; L.P = P;
    L.off = (u64 *)d.hedge_off; L.pins = (u32 *)d.pins; L.nsrc = (u32 *)d.src_count;
    L.toff = c.arena.alloc<u64>((u64)g->n + 1);
    L.touch = c.arena.alloc<u32>(P ? P : 1);
    L.nin = c.arena.alloc<u32>(g->n ? g->n : 1);
    build_touching(c, L.n, L.e, L.off, L.pins, L.nsrc, L.P, L.toff, L.touch, L.nin);
    L.nsize = c.arena.alloc<u32>(g->n ? g->n : 1);
    if (node_size) {
        if (g->n) AXC_CUDA(cudaMemcpyAsync(L.nsize, node_size, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
    } else {
        fill_u32(c, L.nsize, 1u, g->n);
    }
    u32 *wfx = c.arena.alloc<u32>(g->e ? g->e : 1);
    compute_wfx(c, d.hedge_w, wfx, g->e);
    *wfx_out = wfx;
    return L;
}

int axc_stage_rating(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *node_size, uint32_t omega, uint32_t delta,
                     uint32_t cnc, uint64_t seed, uint32_t *out_pairs, uint32_t *out_scores) {
    (void)seed;
    if (!ctx || check_graph(g) || cnc == 0 || cnc > AXC_MAX_CANDIDATES) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u32 *wfx;
        DLevel L = upload_level(c, g, node_size, &wfx);
        u32 *pairs = c.arena.alloc<u32>((u64)g->n * cnc + 1), *scores = c.arena.alloc<u32>((u64)g->n * cnc + 1);
        rating(c, L, wfx, omega, delta, cnc, pairs, scores, nullptr);
        if (g->n) {
            AXC_CUDA(cudaMemcpyAsync(out_pairs, pairs, (size_t)g->n * cnc * 4, cudaMemcpyDeviceToHost, c.stream));
            AXC_CUDA(cudaMemcpyAsync(out_scores, scores, (size_t)g->n * cnc * 4, cudaMemcpyDeviceToHost, c.stream));
        }
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_stage_matching(axc_ctx *ctx, uint32_t n, uint32_t cnc, const uint32_t *pairs, const uint32_t *scores,
                       const uint32_t *node_size, const uint32_t *inbound, uint32_t omega, uint32_t delta,
                       uint32_t *out_groups, uint32_t *out_num_groups) {
    if (!ctx || !pairs || !scores || !node_size || !inbound || !out_groups || !out_num_groups || cnc == 0)
        return AXC_EINVAL;
    for (u64 i = 0; i < (u64)n * cnc; ++i)
        if (pairs[i] != NONE && pairs[i] >= n) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u32 *dp = c.arena.alloc<u32>((u64)n * cnc + 1), *ds = c.arena.alloc<u32>(n + 1), *di = c.arena.alloc<u32>(n + 1);
        u32 *dsc = c.arena.alloc<u32>((u64)n * cnc + 1);
        u32 *dg = c.arena.alloc<u32>(n + 1);
        if (n) {
            AXC_CUDA(cudaMemcpyAsync(dp, pairs, (size_t)n * cnc * 4, cudaMemcpyHostToDevice, c.stream));
            AXC_CUDA(cudaMemcpyAsync(dsc, scores, (size_t)n * cnc * 4, cudaMemcpyHostToDevice, c.stream));
            AXC_CUDA(cudaMemcpyAsync(ds, node_size, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
            AXC_CUDA(cudaMemcpyAsync(di, inbound, (size_t)n * 4, cudaMemcpyHostToDevice, c.stream));
        }
        u32 ng = matching(c, n, cnc, dp, dsc, ds, di, omega, delta, 32, dg);
        if (n) AXC_CUDA(cudaMemcpyAsync(out_groups, dg, (size_t)n * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        *out_num_groups = ng;
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_stage_contract(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *groups, uint32_t num_groups,
                       uint64_t *out_hedge_off, uint32_t *out_pins, uint32_t *out_src_count, uint64_t *out_pins_after) {
    (void)num_groups;
    if (!ctx || check_graph(g) || (!groups && g->n)) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u64 P = 0;
        axc_hgraph d = upload(c, g, P);
        u32 *dg = c.arena.alloc<u32>(g->n ? g->n : 1);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(dg, groups, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
        u64 *off = c.arena.alloc<u64>((u64)g->e + 1);
        u32 *pins = c.arena.alloc<u32>(P ? P : 1), *ns = c.arena.alloc<u32>(g->e ? g->e : 1);
        u64 Pc = hedge_unique(c, g->e, d.hedge_off, d.pins, d.src_count, dg, true, off, pins, ns, P);
        AXC_CUDA(cudaMemcpyAsync(out_hedge_off, off, ((size_t)g->e + 1) * 8, cudaMemcpyDeviceToHost, c.stream));
        if (Pc) AXC_CUDA(cudaMemcpyAsync(out_pins, pins, Pc * 4, cudaMemcpyDeviceToHost, c.stream));
        if (g->e) AXC_CUDA(cudaMemcpyAsync(out_src_count, ns, (size_t)g->e * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        if (out_pins_after) *out_pins_after = Pc;
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_stage_gains(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, uint32_t num_parts,
                    const uint32_t *node_size, uint32_t omega, uint32_t delta, int encourage, uint32_t discount,
                    uint32_t *out_target, int64_t *out_gain) {
    if (!ctx || check_graph(g) || !part || num_parts == 0 || discount == 0) return AXC_EINVAL;
    for (u32 v = 0; v < g->n; ++v)
        if (part[v] >= num_parts) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u32 *wfx;
        DLevel L = upload_level(c, g, node_size, &wfx);
        u32 *dp = c.arena.alloc<u32>(g->n ? g->n : 1), *dt = c.arena.alloc<u32>(g->n ? g->n : 1);
        i64 *dgn = c.arena.alloc<i64>(g->n ? g->n : 1);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(dp, part, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
        RefineParams rp{num_parts, omega, delta, encourage != 0, 1, 0};
        refine_gains_only(c, L, wfx, rp, dp, discount, 0, dt, dgn);
        if (g->n) {
            AXC_CUDA(cudaMemcpyAsync(out_target, dt, (size_t)g->n * 4, cudaMemcpyDeviceToHost, c.stream));
            AXC_CUDA(cudaMemcpyAsync(out_gain, dgn, (size_t)g->n * 8, cudaMemcpyDeviceToHost, c.stream));
        }
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_stage_refine(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, uint32_t num_parts,
                     const uint32_t *node_size, uint32_t omega, uint32_t delta, int encourage, uint32_t rounds,
                     uint64_t seed, uint32_t *out_part, uint32_t *out_rounds) {
    if (!ctx || check_graph(g) || !part || !out_part || num_parts == 0) return AXC_EINVAL;
    for (u32 v = 0; v < g->n; ++v)
        if (part[v] >= num_parts) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        const size_t m = c.arena.mark();
        u32 *wfx;
        DLevel L = upload_level(c, g, node_size, &wfx);
        u32 *dp = c.arena.alloc<u32>(g->n ? g->n : 1);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(dp, part, (size_t)g->n * 4, cudaMemcpyHostToDevice, c.stream));
        RefineParams rp{num_parts, omega, delta, encourage != 0, rounds, seed};
        const u32 ran = refine_level(c, L, wfx, rp, dp);
        if (g->n) AXC_CUDA(cudaMemcpyAsync(out_part, dp, (size_t)g->n * 4, cudaMemcpyDeviceToHost, c.stream));
        AXC_CUDA(cudaStreamSynchronize(c.stream));
        if (out_rounds) *out_rounds = ran;
        c.arena.release(m);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        c.arena.release(0);
        return guard(ctx, e);
    }
}

int axc_selftest_bounded_wait(axc_ctx *ctx, uint32_t spin_limit) {
    if (!ctx || spin_limit == 0) return AXC_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Ctx &c = ctx->c;
    try {
        lookback_selftest(c, spin_limit);
        return AXC_OK;
    } catch (const std::exception &e) {
        cudaStreamSynchronize(c.stream);
        return guard(ctx, e);
    }
}

}  // extern "C"
