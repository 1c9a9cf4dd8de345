// Seeded synthetic hypergraph generators. They stand in for the public SNN (Zenodo) and
// ISPD98 suites the reference benchmarks on (hgraphs/procure_hgraphs.sh), which are not
// available offline; only shapes, sizes and value distributions follow the workload specs.
// Every hyperedge draws from its own xoshiro stream seeded by (seed, hyperedge index), so the
// output is identical for any OpenMP thread count.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "axc_host.h"

using namespace axc;

// Small open-addressing set used to draw distinct ids.
namespace {
struct DistinctSet {
    std::vector<uint32_t> slots;
    uint32_t mask = 0;
    void reset(uint32_t want) {
        uint32_t cap = 16;
        while (cap < 2 * want + 2) cap <<= 1;
        if (slots.size() < cap) slots.resize(cap);
        mask = cap - 1;
        std::fill(slots.begin(), slots.begin() + cap, 0xFFFFFFFFu);
    }
    bool insert(uint32_t v) {
        uint32_t h = (v * 0x9E3779B1u) & mask;
        while (true) {
            if (slots[h] == v) return false;
            if (slots[h] == 0xFFFFFFFFu) { slots[h] = v; return true; }
            h = (h + 1) & mask;
        }
    }
};
}  // namespace

// Normal deviate by the Box-Muller transform.
static double normal01(Rng &r) {
    double u1 = r.uniform(), u2 = r.uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

extern "C" int axc_gen_snn(uint32_t layers, uint32_t width, double fanout, double sigma, uint32_t cap,
                           double p_next, uint64_t seed, axc_hgraph *out) {
    if (!out || layers < 2 || width == 0 || fanout < 1) return AXC_EINVAL;
    const uint64_t n64 = (uint64_t)layers * width;
    if (n64 > 0xFFFFFFFEull) return AXC_EOVERFLOW;
    const uint32_t n = (uint32_t)n64;
    const uint32_t E = (layers - 1) * width;  // the last layer owns no hedge
    // pass 1: fan-out per hedge
    std::vector<uint32_t> fan(E);
#pragma omp parallel for schedule(static)
    for (int64_t h = 0; h < (int64_t)E; ++h) {
        Rng r(seed, 2 * (uint64_t)h);
        uint32_t layer = (uint32_t)(h / width);
        uint64_t avail = (uint64_t)(layers - 1 - layer) * width;  // later neurons
        uint32_t f;
        if (sigma <= 0) {
            f = (uint32_t)fanout;
        } else {
            double x = std::exp(std::log(fanout) + sigma * normal01(r));
            f = (uint32_t)std::llround(x);
            if (f < 1) f = 1;
            if (cap && f > cap) f = cap;
        }
        if (f > avail) f = (uint32_t)avail;
        fan[h] = f;
    }
    auto *hg = new HostGraph();
    hg->n = n;
    hg->off.resize((size_t)E + 1);
    hg->off[0] = 0;
    for (uint32_t h = 0; h < E; ++h) hg->off[h + 1] = hg->off[h] + 1 + fan[h];
    hg->pins.resize(hg->off[E]);
    hg->nsrc.assign(E, 1);
    hg->w.assign(E, 1.0f);
    // pass 2: destinations, without replacement
#pragma omp parallel
    {
        DistinctSet ds;
#pragma omp for schedule(dynamic, 256)
        for (int64_t h = 0; h < (int64_t)E; ++h) {
            Rng r(seed, 2 * (uint64_t)h + 1);
            const uint32_t layer = (uint32_t)(h / width);
            uint32_t *dst = hg->pins.data() + hg->off[h];
            dst[0] = (uint32_t)h;  // neuron h owns hedge h (ids are layer-major)
            const uint32_t f = fan[h];
            const uint32_t next0 = (layer + 1) * width;
            const uint32_t later = (layers - 1 - layer) * width;  // ids [next0, next0 + later)
            const bool only_next = (layer + 2 == layers);
            // when the next layer alone cannot host the draws, fall back to all later layers
            ds.reset(f);
            uint32_t got = 0;
            uint64_t guard = 0;
            while (got < f) {
                uint32_t v;
                bool from_next = only_next || r.uniform() < p_next;
                if (from_next && f <= width / 2 + 1)
                    v = next0 + r.below(width);
                else
                    v = next0 + r.below(later);
                if (ds.insert(v)) dst[1 + got++] = v;
                if (++guard > 64ull * f + 4096) {  // dense fan-out: fill the rest in order
                    for (uint32_t c = 0; got < f && c < later; ++c)
                        if (ds.insert(next0 + c)) dst[1 + got++] = next0 + c;
                }
            }
        }
    }
    publish(hg, out);
    return AXC_OK;
}

extern "C" int axc_gen_circuit(uint32_t n, uint32_t e, uint32_t smin, uint32_t smax, double alpha,
                               double p_local, double local_frac, uint64_t seed, axc_hgraph *out) {
    if (!out || n < 2 || smin < 2 || smax < smin || smax > n) return AXC_EINVAL;
    // truncated discrete power law P(s) ~ s^-alpha on [smin, smax], sampled by inverse CDF
    std::vector<double> cdf(smax - smin + 1);
    double acc = 0;
    for (uint32_t s = smin; s <= smax; ++s) {
        acc += std::pow((double)s, -alpha);
        cdf[s - smin] = acc;
    }
    for (auto &c : cdf) c /= acc;
    std::vector<uint32_t> sz(e);
#pragma omp parallel for schedule(static)
    for (int64_t h = 0; h < (int64_t)e; ++h) {
        Rng r(seed, 2 * (uint64_t)h);
        double u = r.uniform();
        uint32_t idx = (uint32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (idx >= cdf.size()) idx = (uint32_t)cdf.size() - 1;
        sz[h] = smin + idx;
    }
    auto *hg = new HostGraph();
    hg->n = n;
    hg->off.resize((size_t)e + 1);
    hg->off[0] = 0;
    for (uint32_t h = 0; h < e; ++h) hg->off[h + 1] = hg->off[h] + sz[h];
    hg->pins.resize(hg->off[e]);
    hg->nsrc.assign(e, 0);
    hg->w.assign(e, 1.0f);
    const uint32_t radius = std::max<uint32_t>(1, (uint32_t)std::llround(local_frac * (double)n));
#pragma omp parallel
    {
        DistinctSet ds;
#pragma omp for schedule(static)
        for (int64_t h = 0; h < (int64_t)e; ++h) {
            Rng r(seed, 2 * (uint64_t)h + 1);
            uint32_t *p = hg->pins.data() + hg->off[h];
            const uint32_t s = sz[h];
            const uint32_t anchor = r.below(n);
            const uint32_t lo = anchor > radius ? anchor - radius : 0;
            const uint32_t hi = std::min<uint64_t>((uint64_t)anchor + radius, (uint64_t)n - 1);
            ds.reset(s);
            uint32_t got = 0;
            while (got < s) {  // duplicates are redrawn, so every net keeps s distinct pins
                uint32_t v = (r.uniform() < p_local) ? lo + r.below(hi - lo + 1) : r.below(n);
                if (ds.insert(v)) p[got++] = v;
            }
        }
    }
    publish(hg, out);
    return AXC_OK;
}
