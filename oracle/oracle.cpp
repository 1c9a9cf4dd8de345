// oracle.cpp — CPU restatement of every stage of the partitioner. TEST INFRASTRUCTURE ONLY:
// used by tests/ and __graft_entry__.smoke() as the checker, and by bench.py as the timed CPU
// port; never by the product path.
//
// Parity status: the readers, rule-2 dedupe, incidence CSR and the metrics/validity functions are
// pinned against the reference's own code compiled here (oracle/_ref/refharness.exe and
// oracle/_ref/hgrade.exe) by tests/test_oracle_pins.py. The rating restates
// kernels/coarsening.cu:76-212 exactly (same score, noise, filters and (score, id) order). The
// matching, the refinement's move selection and the k-way initial partition are this build's own
// deterministic algorithms (the reference's grouping_kernel and event pipeline are
// nondeterministic under atomics, and its k-way initial partition is the external Mt-KaHyPar);
// for those the oracle is the specification the GPU path must reproduce bit for bit.
#include "oracle.h"
#include "../include/axc.h"  // public constants the restatement shares (AXC_RATE_MAX_LEN)

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
const u32 NONE = 0xFFFFFFFFu;
const u64 RATE_MAX_LEN = AXC_RATE_MAX_LEN;  // the rating's hyperedge length limit (include/axc.h)
const u32 PAIR_RANK_MAX_K = AXC_PAIR_RANK_MAX_K;  // k-way pair ranking needs (a*K + b) * 2 < 2^32

struct G {
    u32 n = 0, e = 0;
    std::vector<u64> off;
    std::vector<u32> pins, nsrc;
};
struct T {
    std::vector<u64> toff;
    std::vector<u32> touch, nin;
};

// headers/utils.cuh:159-171: symmetric deterministic noise in [0, 63] of an unordered id pair.
u32 noise64(u32 a, u32 b) {
    u32 lo = a < b ? a : b, hi = a < b ? b : a;
    u32 x = lo * 0x9E3779B1u;
    x ^= hi + 0x85EBCA6Bu + (x << 6) + (x >> 2);
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 13;
    x *= 0x9E3779B1u;
    x ^= x >> 16;
    return x & 63u;
}

// headers/utils.cuh:252-261: 32-bit integer mixer used for refinement tie-breaks.
u32 mix32(u32 x) {
    x ^= x >> 17;
    x *= 0xED5AD4BBu;
    x ^= x >> 11;
    x *= 0xAC4C1B51u;
    x ^= x >> 15;
    x *= 0x31848BABu;
    x ^= x >> 14;
    return x;
}

G dedupe(const G &in) {
    G out;
    out.n = in.n;
    out.e = in.e;
    out.off.assign(in.e + 1, 0);
    out.nsrc.assign(in.e, 0);
    out.pins.reserve(in.pins.size());
    std::vector<u32> seen;
    for (u32 h = 0; h < in.e; ++h) {
        seen.clear();
        u64 a = in.off[h], b = in.off[h + 1];
        u32 ns = 0;
        for (u64 k = a; k < b; ++k) {
            u32 v = in.pins[k];
            if (std::find(seen.begin(), seen.end(), v) != seen.end()) continue;
            seen.push_back(v);
            out.pins.push_back(v);
            if (k < a + in.nsrc[h]) ++ns;
        }
        out.nsrc[h] = ns;
        out.off[h + 1] = out.pins.size();
    }
    return out;
}

T touching(const G &g) {
    T t;
    std::vector<u32> din(g.n, 0), dout(g.n, 0);
    for (u32 h = 0; h < g.e; ++h)
        for (u64 k = g.off[h]; k < g.off[h + 1]; ++k)
            (k < g.off[h] + g.nsrc[h] ? dout : din)[g.pins[k]]++;
    t.toff.assign(g.n + 1, 0);
    for (u32 v = 0; v < g.n; ++v) t.toff[v + 1] = t.toff[v] + din[v] + dout[v];
    t.touch.assign(t.toff[g.n], 0);
    t.nin = din;
    std::vector<u64> ci(g.n), co(g.n);
    for (u32 v = 0; v < g.n; ++v) { ci[v] = t.toff[v]; co[v] = t.toff[v] + din[v]; }
    for (u32 h = 0; h < g.e; ++h)  // hedges in ascending order => each part ascending
        for (u64 k = g.off[h]; k < g.off[h + 1]; ++k) {
            u32 v = g.pins[k];
            if (k < g.off[h] + g.nsrc[h]) t.touch[co[v]++] = h; else t.touch[ci[v]++] = h;
        }
    return t;
}

// kernels/coarsening.cu:76-212. For node u every neighbour v (v != u, sharing a hyperedge) with
// size_u + size_v <= omega scores noise(u,v) + sum over hyperedges e incident to u that contain v
// of floor(w_fx(e) / |e|) (uint32, wrapping). v is dropped when
// |in(u)| + |in(v)| - |in(u) cap in(v)| > delta, where the intersection counts hyperedges inbound
// to u in which v is a destination. The top cnc by (score desc, id desc) with score > 0 are kept.
// This build's one departure: hyperedges of more than RATE_MAX_LEN pins take no part in the rating
// (their pair visits grow as |e|^2 while each pair gains only floor(w/|e|)); leaving them out of
// the shared-inbound count only makes the delta filter stricter.
void rating(const G &g, const std::vector<u32> &wfx, const T &t, const u32 *nsize, u32 omega,
            u32 delta, u32 cnc, u32 *pairs, u32 *scores, u64 max_len = RATE_MAX_LEN) {
    std::vector<u32> sc(g.n, 0), cm(g.n, 0), mark(g.n, NONE);
    std::vector<u32> touched;
    std::vector<std::pair<u32, u32>> cand;
    for (u32 u = 0; u < g.n; ++u) {
        touched.clear();
        const u64 t0 = t.toff[u], t1 = t.toff[u + 1];
        for (u64 j = t0; j < t1; ++j) {
            const u32 h = t.touch[j];
            const bool inb = (j - t0) < t.nin[u];
            const u64 a = g.off[h], b = g.off[h + 1];
            if (b - a > max_len) continue;
            const u32 c = wfx[h] / (u32)(b - a);
            for (u64 k = a; k < b; ++k) {
                const u32 v = g.pins[k];
                if (v == u) continue;
                if (mark[v] != u) { mark[v] = u; sc[v] = 0; cm[v] = 0; touched.push_back(v); }
                sc[v] += c;
                if (inb && k >= a + g.nsrc[h]) cm[v]++;
            }
        }
        cand.clear();
        for (u32 v : touched) {
            if ((u64)nsize[u] + nsize[v] > omega) continue;
            if ((u64)t.nin[u] + t.nin[v] - cm[v] > delta) continue;
            u32 s = sc[v] + noise64(u, v);
            if (s == 0) continue;
            cand.push_back({s, v});
        }
        std::sort(cand.begin(), cand.end(), [](auto &x, auto &y) {
            return x.first != y.first ? x.first > y.first : x.second > y.second;
        });
        for (u32 i = 0; i < cnc; ++i) {
            pairs[(u64)u * cnc + i] = i < cand.size() ? cand[i].second : NONE;
            scores[(u64)u * cnc + i] = i < cand.size() ? cand[i].first : 0;
        }
    }
}

// Deterministic matching by rounds of proposals (this build's rule; the reference's
// grouping_kernel, kernels/coarsening.cu:241-505, resolves its candidate forests with atomics).
// Each round, on the previous round's state:
//  A. every unmatched node u proposes to its best still-unmatched candidate p(u) (candidate lists
//     are in (score desc, id desc) order);
//  B. every node v accepts its best proposer best(v) by (score, id);
//  C. with acc(u) = [best(p(u)) == u]: u and p(u) match when acc(u) and not acc(p(u)) (p(u)'s own
//     proposal was refused, so it is free), or when they propose to and accept each other.
// Each node is matched at most once per round. Stops at a fixed point or after `rounds`.
// Orphans (nodes without any candidate) are then paired k-th smallest with k-th largest by
// (size, id) when size and inbound-count sums fit (sources/chaining.cu:260-329,
// kernels/chaining.cu:237-270). Groups are relabelled 0.. in order of their smallest member.
u32 matching(u32 n, u32 cnc, const u32 *pairs, const u32 *scores, const u32 *nsize, const u32 *nin,
             u32 omega, u32 delta, u32 rounds, u32 *groups) {
    std::vector<u32> mate(n, NONE), ptr(n, 0), prop(n, NONE);
    std::vector<u64> best(n, 0);
    for (u32 r = 0; r < rounds; ++r) {
        for (u32 v = 0; v < n; ++v) {
            prop[v] = NONE;
            best[v] = 0;
            if (mate[v] != NONE) continue;
            u32 p = ptr[v];
            while (p < cnc) {
                u32 w = pairs[(u64)v * cnc + p];
                if (w == NONE) { p = cnc; break; }
                if (mate[w] == NONE) break;
                ++p;
            }
            ptr[v] = p;
            if (p < cnc) prop[v] = pairs[(u64)v * cnc + p];
        }
        for (u32 u = 0; u < n; ++u)
            if (prop[u] != NONE) {
                u64 key = ((u64)scores[(u64)u * cnc + ptr[u]] << 32) | u;
                best[prop[u]] = std::max(best[prop[u]], key);
            }
        // candidate scores are > 0, so a node with proposers has best != 0
        auto acc = [&](u32 u) { return prop[u] != NONE && best[prop[u]] != 0 && (u32)best[prop[u]] == u; };
        bool changed = false;
        std::vector<std::pair<u32, u32>> mk;
        for (u32 u = 0; u < n; ++u) {
            const u32 v = prop[u];
            if (v == NONE || !acc(u)) continue;
            const bool av = acc(v);
            if (!av || (prop[v] == u && u < v)) mk.push_back({u, v});
        }
        for (auto &x : mk) { mate[x.first] = x.second; mate[x.second] = x.first; changed = true; }
        if (!changed) break;
    }
    // Two-hop pass: still-unmatched nodes that have candidates are bucketed by their best
    // candidate; within a bucket (ascending ids) positions 2i and 2i+1 pair up when their size sum
    // fits omega and their inbound-count sum fits delta.
    {
        std::vector<std::pair<u32, u32>> hop;  // (best candidate, node)
        for (u32 v = 0; v < n; ++v)
            if (mate[v] == NONE && pairs[(u64)v * cnc] != NONE) hop.push_back({pairs[(u64)v * cnc], v});
        std::sort(hop.begin(), hop.end());
        size_t i = 0;
        while (i < hop.size()) {
            size_t j = i;
            while (j < hop.size() && hop[j].first == hop[i].first) ++j;
            for (size_t a = i; a + 1 < j; a += 2) {
                const u32 x = hop[a].second, y = hop[a + 1].second;
                if ((u64)nsize[x] + nsize[y] > omega || (u64)nin[x] + nin[y] > delta) continue;
                mate[x] = y;
                mate[y] = x;
            }
            i = j;
        }
    }
    std::vector<u32> orph;
    for (u32 v = 0; v < n; ++v)
        if (pairs[(u64)v * cnc] == NONE) orph.push_back(v);
    std::stable_sort(orph.begin(), orph.end(), [&](u32 a, u32 b) { return nsize[a] < nsize[b]; });
    const u32 m = (u32)orph.size();
    for (u32 k = 0; k < m / 2; ++k) {
        u32 L = orph[k], R = orph[m - 1 - k];
        if ((u64)nsize[L] + nsize[R] > omega) continue;
        if ((u64)nin[L] + nin[R] > delta) continue;
        mate[L] = R; mate[R] = L;
    }
    std::vector<u32> gid(n, 0);
    u32 ng = 0;
    for (u32 v = 0; v < n; ++v)
        if (mate[v] == NONE || v < mate[v]) gid[v] = ng++;
    for (u32 v = 0; v < n; ++v) groups[v] = gid[mate[v] == NONE || v < mate[v] ? v : mate[v]];
    return ng;
}

// kernels/construction.cu:304-489: coarse pins are the distinct groups; a group that is both a
// source and a destination stays a destination only; hyperedges keep their ids (size-1 coarse
// hyperedges stay). Order: sources then destinations, each in first-occurrence order.
G contract(const G &g, const u32 *groups, u32 ng) {
    G c;
    c.n = ng;
    c.e = g.e;
    c.off.assign(g.e + 1, 0);
    c.nsrc.assign(g.e, 0);
    c.pins.reserve(g.pins.size());
    std::vector<u32> mark(ng, NONE), dl, sl;
    for (u32 h = 0; h < g.e; ++h) {
        dl.clear(); sl.clear();
        const u64 a = g.off[h], b = g.off[h + 1], s = a + g.nsrc[h];
        for (u64 k = s; k < b; ++k) {
            u32 x = groups[g.pins[k]];
            if (mark[x] != 2 * h) { mark[x] = 2 * h; dl.push_back(x); }
        }
        for (u64 k = a; k < s; ++k) {
            u32 x = groups[g.pins[k]];
            if (mark[x] == 2 * h || mark[x] == 2 * h + 1) continue;
            mark[x] = 2 * h + 1;
            sl.push_back(x);
        }
        c.pins.insert(c.pins.end(), sl.begin(), sl.end());
        c.pins.insert(c.pins.end(), dl.begin(), dl.end());
        c.nsrc[h] = (u32)sl.size();
        c.off[h + 1] = c.pins.size();
    }
    return c;
}

// Per-hyperedge partition census: for hyperedge h, entries [cbeg[h], cbeg[h+1]) of (part, pins in
// part, destination pins in part), in first-occurrence order over h's pins.
struct Census {
    std::vector<u64> beg;
    std::vector<u32> part, cnt, dcnt;
};
Census census(const G &g, const std::vector<u32> &part) {
    Census cs;
    cs.beg.assign(g.e + 1, 0);
    std::vector<u32> slot(0);
    for (u32 h = 0; h < g.e; ++h) {
        const u64 a = g.off[h], b = g.off[h + 1], s = a + g.nsrc[h];
        const u64 base = cs.part.size();
        for (u64 k = a; k < b; ++k) {
            u32 p = part[g.pins[k]];
            u64 j = base;
            while (j < cs.part.size() && cs.part[j] != p) ++j;
            if (j == cs.part.size()) { cs.part.push_back(p); cs.cnt.push_back(0); cs.dcnt.push_back(0); }
            cs.cnt[j]++;
            if (k >= s) cs.dcnt[j]++;
        }
        cs.beg[h + 1] = cs.part.size();
    }
    return cs;
}
u32 census_get(const Census &cs, u32 h, u32 p, u32 *dc = nullptr) {
    for (u64 j = cs.beg[h]; j < cs.beg[h + 1]; ++j)
        if (cs.part[j] == p) { if (dc) *dc = cs.dcnt[j]; return cs.cnt[j]; }
    if (dc) *dc = 0;
    return 0;
}

struct RefineCtx {
    const G *g;
    const T *t;
    const std::vector<u32> *wfx;
    const u32 *nsize;
    u32 K, omega, delta;
    bool encourage;
    u64 seed;
    // copies > 1: the level is that many disjoint copies of copy_n nodes each (the k-way
    // multi-start); moves are ranked copy by copy and every copy takes its own best prefix
    u32 copies = 1, copy_n = 0;
};

inline i64 leave_gain(bool encourage, u32 w, u32 c) {
    if (encourage) return c >= 1 ? (i64)(w / ((u64)c * c)) : 0;
    return c == 1 ? (i64)w : 0;
}

// kernels/refinement.cu:82-209 with integer gains: every node's best target among the partitions
// adjacent to it (loss(q) = sum of w over incident hyperedges without a pin in q), feasible when
// size(q) + s - floor(s/discount) <= omega and (this build) size_in(q) + new inbound <= delta;
// ties go to the larger mix32(q + round + seed), then the smaller id. Only positive gains move.
// With more than AXC_SPARSE_GAIN_K partitions, a node whose incidences hold more census entries
// than AXC_SPARSE_GAIN_SAMPLE takes the sampled rule of sampled_target (include/axc.h).
bool sampled_target(const RefineCtx &rc, const std::vector<u32> &part, const Census &cs,
                    const std::vector<u64> &psize, const std::vector<u64> &pinb, u32 discount, u32 round,
                    u32 u, u32 *target, i64 *gain);

void gains(const RefineCtx &rc, const std::vector<u32> &part, const Census &cs,
           const std::vector<u64> &psize, const std::vector<u64> &pinb, u32 discount, u32 round,
           u32 *target, i64 *gain) {
    const G &g = *rc.g;
    const T &t = *rc.t;
    std::vector<i64> conn(rc.K, 0);
    std::vector<u32> dconn(rc.K, 0), mark(rc.K, NONE), touched;
    for (u32 u = 0; u < g.n; ++u) {
        if (rc.K > AXC_SPARSE_GAIN_K && sampled_target(rc, part, cs, psize, pinb, discount, round, u, target, gain))
            continue;
        const u32 p = part[u];
        const u64 s = rc.nsize[u];
        i64 saving = 0, wtot = 0;
        touched.clear();
        const u64 t0 = t.toff[u], t1 = t.toff[u + 1];
        for (u64 j = t0; j < t1; ++j) {
            const u32 h = t.touch[j];
            const u32 w = (*rc.wfx)[h];
            const bool inb = (j - t0) < t.nin[u];
            saving += leave_gain(rc.encourage, w, census_get(cs, h, p));
            wtot += w;
            for (u64 k = cs.beg[h]; k < cs.beg[h + 1]; ++k) {
                const u32 q = cs.part[k];
                if (q == p) continue;
                if (mark[q] != u) { mark[q] = u; conn[q] = 0; dconn[q] = 0; touched.push_back(q); }
                conn[q] += w;
                if (inb && cs.dcnt[k] > 0) dconn[q]++;
            }
        }
        u32 best = NONE;
        i64 bg = 0;
        u32 bh = 0;
        for (u32 q : touched) {
            if (psize[q] + s - s / discount > rc.omega) continue;
            if (pinb[q] + (u64)(t.nin[u] - dconn[q]) > rc.delta) continue;
            const i64 gq = saving - (wtot - conn[q]);
            const u32 hq = mix32(q + round + (u32)rc.seed);
            if (best == NONE || gq > bg || (gq == bg && (hq > bh || (hq == bh && q < best)))) {
                best = q; bg = gq; bh = hq;
            }
        }
        if (best != NONE && bg > 0) { target[u] = best; gain[u] = bg; }
        else { target[u] = NONE; gain[u] = 0; }
    }
}

// The sampled rule for node u (include/axc.h AXC_SPARSE_GAIN_*). Returns false when u's sample
// is all of its incidences (the exact rule of gains() then applies, with the same result);
// otherwise writes u's target and gain.
//  1. The sample: the longest prefix j < m of u's incidences (touching order: inbound ascending,
//     then outbound ascending) whose census entries number at most AXC_SPARSE_GAIN_SAMPLE.
//  2. Sampled connectivity sconn[q] = sum of w over the sample's hyperedges holding q (q != p),
//     sdc[q] = the sample's inbound hyperedges with destination pins in q.
//  3. q is ruled out when size(q) + s - floor(s/discount) > omega, or when even the inbound
//     hyperedges outside the sample all shared with q could not make room:
//     pinb[q] + min(m, nin_u) - sdc[q] > delta.
//  4. The first AXC_SPARSE_GAIN_CANDIDATES of the others by (sconn desc, mix32(q + round + seed)
//     desc, q asc) are evaluated exactly over all incidences, as gains() would; the best feasible
//     one by (gain desc, hash desc, q asc) is the target when its gain is positive.
bool sampled_target(const RefineCtx &rc, const std::vector<u32> &part, const Census &cs,
                    const std::vector<u64> &psize, const std::vector<u64> &pinb, u32 discount, u32 round,
                    u32 u, u32 *target, i64 *gain) {
    const T &t = *rc.t;
    const u64 t0 = t.toff[u], deg = t.toff[u + 1] - t0;
    const u32 nin = t.nin[u], p = part[u];
    u64 m = 0, acc = 0;
    while (m < deg) {
        const u32 h = t.touch[t0 + m];
        const u64 lam = cs.beg[h + 1] - cs.beg[h];
        if (acc + lam > AXC_SPARSE_GAIN_SAMPLE) break;
        acc += lam;
        ++m;
    }
    if (m == deg) return false;
    struct Acc { u64 conn = 0; u32 dc = 0; };
    std::unordered_map<u32, Acc> tab;  // at most AXC_SPARSE_GAIN_SAMPLE entries
    auto find = [&](u32 q) -> Acc & { return tab[q]; };
    for (u64 j = 0; j < m; ++j) {
        const u32 h = t.touch[t0 + j];
        const u32 w = (*rc.wfx)[h];
        for (u64 k = cs.beg[h]; k < cs.beg[h + 1]; ++k) {
            const u32 q = cs.part[k];
            if (q == p) continue;
            Acc &a = find(q);
            a.conn += w;
            if (j < nin && cs.dcnt[k] > 0) a.dc++;
        }
    }
    const u64 s = rc.nsize[u];
    const u64 in_sample = std::min<u64>(m, nin);
    struct Key { u64 conn; u32 hash; u32 q; };
    std::vector<Key> keys;
    for (auto &x : tab) {
        const u32 q = x.first;
        if (psize[q] + s - s / discount > rc.omega) continue;
        if (pinb[q] + in_sample - x.second.dc > rc.delta) continue;
        keys.push_back({x.second.conn, mix32(q + round + (u32)rc.seed), q});
    }
    std::sort(keys.begin(), keys.end(), [](const Key &a, const Key &b) {
        if (a.conn != b.conn) return a.conn > b.conn;
        if (a.hash != b.hash) return a.hash > b.hash;
        return a.q < b.q;
    });
    if (keys.size() > AXC_SPARSE_GAIN_CANDIDATES) keys.resize(AXC_SPARSE_GAIN_CANDIDATES);
    const size_t nc = keys.size();
    std::vector<i64> conn(nc, 0);
    std::vector<u32> dconn(nc, 0);
    i64 saving = 0, wtot = 0;
    for (u64 j = 0; j < deg; ++j) {
        const u32 h = t.touch[t0 + j];
        const u32 w = (*rc.wfx)[h];
        wtot += w;
        for (u64 k = cs.beg[h]; k < cs.beg[h + 1]; ++k) {
            const u32 q = cs.part[k];
            if (q == p) { saving += leave_gain(rc.encourage, w, cs.cnt[k]); continue; }
            for (size_t i = 0; i < nc; ++i)
                if (keys[i].q == q) {
                    conn[i] += w;
                    if (j < nin && cs.dcnt[k] > 0) dconn[i]++;
                }
        }
    }
    u32 best = NONE, bh = 0;
    i64 bg = 0;
    for (size_t i = 0; i < nc; ++i) {
        const u32 q = keys[i].q;
        if (psize[q] + s - s / discount > rc.omega) continue;
        if (pinb[q] + (u64)(nin - dconn[i]) > rc.delta) continue;
        const i64 gq = saving - (wtot - conn[i]);
        const u32 hq = keys[i].hash;
        if (best == NONE || gq > bg || (gq == bg && (hq > bh || (hq == bh && q < best)))) {
            best = q; bg = gq; bh = hq;
        }
    }
    if (best != NONE && bg > 0) { target[u] = best; gain[u] = bg; }
    else { target[u] = NONE; gain[u] = 0; }
    return true;
}

std::vector<u64> part_sizes(const std::vector<u32> &part, const u32 *nsize, u32 K) {
    std::vector<u64> ps(K, 0);
    for (size_t v = 0; v < part.size(); ++v) ps[part[v]] += nsize[v];
    return ps;
}
std::vector<u64> part_inbound(const Census &cs, u32 e, u32 K) {
    std::vector<u64> pi(K, 0);
    for (u32 h = 0; h < e; ++h)
        for (u64 k = cs.beg[h]; k < cs.beg[h + 1]; ++k)
            if (cs.dcnt[k] > 0) pi[cs.part[k]]++;
    return pi;
}

// k-way move order (this build's deterministic stand-in for the reference's chaining,
// sources/chaining.cu:19-254, which links a move into partition q with a move out of q so that
// prefixes stay balanced). mv arrives in (gain desc, id asc) order. Moves between the same two
// partitions a < b are split by direction d (0: a -> b, 1: b -> a); the i-th move of one
// direction (in that order) pairs with the i-th of the other. A pair is ranked by the sum of its
// two gains, a single by its own gain; ties by the pair's position (a, b, i), and d = 0 first,
// so the two moves of a pair are adjacent and every even prefix of a pair chain is balanced.
void pair_rank(const std::vector<u32> &part, const std::vector<u32> &target, const std::vector<i64> &gain,
               std::vector<u32> &mv, u32 K) {
    const size_t M = mv.size();
    std::vector<u32> gk(M), ord(M);
    for (size_t i = 0; i < M; ++i) {
        const u32 p = part[mv[i]], q = target[mv[i]];
        gk[i] = ((std::min(p, q) * K + std::max(p, q)) << 1) | (p < q ? 0u : 1u);
    }
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](u32 x, u32 y) { return gk[x] < gk[y]; });
    std::vector<u32> sk(M);
    for (size_t j = 0; j < M; ++j) sk[j] = gk[ord[j]];
    struct Key { i64 ps; u64 pk; u32 u; };
    std::vector<Key> keys(M);
    for (size_t j = 0; j < M; ++j) {
        const u32 g = sk[j], d = g & 1u;
        const size_t s = std::lower_bound(sk.begin(), sk.end(), g) - sk.begin(), i = j - s;
        const size_t s2 = std::lower_bound(sk.begin(), sk.end(), g ^ 1u) - sk.begin();
        const size_t e2 = std::upper_bound(sk.begin(), sk.end(), g ^ 1u) - sk.begin();
        const u32 u = mv[ord[j]];
        i64 ps = gain[u];
        u64 pk = j;
        if (i < e2 - s2) {
            ps += gain[mv[ord[s2 + i]]];
            if (d == 1) pk = s2 + i;
        }
        keys[j] = {ps, (pk << 1) | d, u};
    }
    std::stable_sort(keys.begin(), keys.end(), [](const Key &x, const Key &y) {
        return x.ps != y.ps ? x.ps > y.ps : x.pk < y.pk;
    });
    for (size_t j = 0; j < M; ++j) mv[j] = keys[j].u;
}

// One refinement round (sources/refinement.cu:82-543 restated with exact integers):
// proposals -> rank by (gain desc, id asc) -> cascaded gain of each move assuming every
// better-ranked move is applied (per hyperedge sweep) -> prefix sums -> size excess and inbound
// validity of every prefix -> best prefix by best_move_functor (headers/data_types.cuh:113-136)
// -> apply when valid with prefix gain >= 0. Returns whether moves were applied.
bool refine_round(const RefineCtx &rc, std::vector<u32> &part, u32 discount, u32 round) {
    const G &g = *rc.g;
    const T &t = *rc.t;
    Census cs = census(g, part);
    std::vector<u64> psize = part_sizes(part, rc.nsize, rc.K);
    std::vector<u64> pinb = part_inbound(cs, g.e, rc.K);
    std::vector<u32> target(g.n);
    std::vector<i64> gain(g.n);
    gains(rc, part, cs, psize, pinb, discount, round, target.data(), gain.data());
    std::vector<u32> mv;
    for (u32 u = 0; u < g.n; ++u)
        if (target[u] != NONE) mv.push_back(u);
    if (mv.empty()) return false;
    std::stable_sort(mv.begin(), mv.end(), [&](u32 a, u32 b) { return gain[a] > gain[b]; });
    if (!rc.encourage && rc.K <= PAIR_RANK_MAX_K) pair_rank(part, target, gain, mv, rc.K);
    if (rc.copies > 1)
        std::stable_sort(mv.begin(), mv.end(), [&](u32 a, u32 b) { return a / rc.copy_n < b / rc.copy_n; });
    const u32 M = (u32)mv.size();
    std::vector<u32> rank(g.n, NONE);
    for (u32 r = 0; r < M; ++r) rank[mv[r]] = r;
    // cascade
    std::vector<i64> g2(g.n, 0);
    std::vector<std::pair<u32, u32>> ms;  // (rank, node)
    std::vector<u32> cp, cc;              // local census copy (part, count)
    for (u32 h = 0; h < g.e; ++h) {
        ms.clear();
        for (u64 k = g.off[h]; k < g.off[h + 1]; ++k)
            if (rank[g.pins[k]] != NONE) ms.push_back({rank[g.pins[k]], g.pins[k]});
        if (ms.empty()) continue;
        std::sort(ms.begin(), ms.end());
        cp.assign(cs.part.begin() + cs.beg[h], cs.part.begin() + cs.beg[h + 1]);
        cc.assign(cs.cnt.begin() + cs.beg[h], cs.cnt.begin() + cs.beg[h + 1]);
        auto at = [&](u32 p) -> u32 & {
            for (size_t j = 0; j < cp.size(); ++j) if (cp[j] == p) return cc[j];
            cp.push_back(p); cc.push_back(0);
            return cc.back();
        };
        const u32 w = (*rc.wfx)[h];
        for (auto &x : ms) {
            const u32 u = x.second, p = part[u], q = target[u];
            const u32 cpv = at(p), cqv = at(q);
            g2[u] += leave_gain(rc.encourage, w, cpv) - (cqv == 0 ? (i64)w : 0);
            at(p)--;
            at(q)++;
        }
    }
    std::vector<i64> G2(M);
    i64 acc = 0;
    for (u32 r = 0; r < M; ++r) { acc += g2[mv[r]]; G2[r] = acc; }
    // size validity: V[r] = sum_p (excess_p after prefix r - excess_p initially)
    std::vector<i64> Vs(M), Vi(M, 0);
    {
        std::vector<u64> cur = psize;
        i64 v = 0;
        auto ex = [&](u64 x) -> i64 { return x > rc.omega ? (i64)(x - rc.omega) : 0; };
        for (u32 r = 0; r < M; ++r) {
            const u32 u = mv[r], p = part[u], q = target[u];
            const u64 s = rc.nsize[u];
            v -= ex(cur[p]); cur[p] -= s; v += ex(cur[p]);
            v -= ex(cur[q]); cur[q] += s; v += ex(cur[q]);
            Vs[r] = v;
        }
    }
    // inbound validity: V[r] = partitions whose inbound set changed by rank r and exceeds delta
    if (rc.delta < 0x7FFFFFFFu) {
        std::vector<u64> cur = pinb;
        std::vector<char> touchedp(rc.K, 0);
        // running destination counts of (hyperedge, partition) touched by moves
        std::vector<std::vector<std::pair<u32, i64>>> dc(g.e);
        auto dget = [&](u32 h, u32 p) -> i64 & {
            for (auto &x : dc[h]) if (x.first == p) return x.second;
            u32 d0 = 0;
            census_get(cs, h, p, &d0);
            dc[h].push_back({p, (i64)d0});
            return dc[h].back().second;
        };
        i64 v = 0;
        for (u32 r = 0; r < M; ++r) {
            const u32 u = mv[r], p = part[u], q = target[u];
            for (u64 j = t.toff[u]; j < t.toff[u] + t.nin[u]; ++j) {
                const u32 h = t.touch[j];
                i64 &a = dget(h, p);
                if (a-- == 1) {
                    bool was = touchedp[p] ? cur[p] > rc.delta : false;
                    cur[p]--; touchedp[p] = 1;
                    v += (i64)(cur[p] > rc.delta) - (i64)was;
                }
                i64 &b = dget(h, q);
                if (b++ == 0) {
                    bool was = touchedp[q] ? cur[q] > rc.delta : false;
                    cur[q]++; touchedp[q] = 1;
                    v += (i64)(cur[q] > rc.delta) - (i64)was;
                }
            }
            Vi[r] = v;
        }
    }
    // best prefix of every copy's rank segment [s, e) (one segment without copies), prefix values
    // relative to the segment start
    bool any = false;
    for (u32 s = 0; s < M;) {
        u32 e = s + 1;
        if (rc.copies > 1)
            while (e < M && mv[e] / rc.copy_n == mv[s] / rc.copy_n) ++e;
        else
            e = M;
        auto rel = [&](const std::vector<i64> &X, u32 r) { return X[r] - (s ? X[s - 1] : 0); };
        u32 best = s;
        for (u32 r = s + 1; r < e; ++r) {
            const u32 a = best, b = r;
            const bool aok = rel(Vi, a) == 0, bok = rel(Vi, b) == 0;
            bool take;
            if (aok != bok) take = bok;
            else if (!aok) take = false;
            else if (rel(Vs, a) != rel(Vs, b)) take = rel(Vs, a) > rel(Vs, b);
            else if (rel(G2, a) != rel(G2, b)) take = rel(G2, a) < rel(G2, b);
            else take = false;
            if (take) best = b;
        }
        if (rel(Vs, best) <= 0 && rel(Vi, best) <= 0 && rel(G2, best) >= 0) {
            for (u32 r = s; r <= best; ++r) part[mv[r]] = target[mv[r]];
            any = true;
        }
        s = e;
    }
    return any;
}

void refine_level(const RefineCtx &rc, std::vector<u32> &part, u32 R) {
    for (u32 r = 0; r < R; ++r) {
        const u32 discount = r < R / 3 ? 1u : (r < 2 * R / 3 ? 2u : 0xFFFFFFFFu);
        if (!refine_round(rc, part, discount, r)) {
            if (r < R / 3) r = R / 2;
            else if (r < 2 * R / 3) r = 2 * R / 3;
            else r = R;
        }
    }
}

// Greedy contiguous packing of items sorted by (size, inbound, id) under sum(size) <= omega and
// sum(inbound) <= delta (sources/postprocess.cu:16-245 and 247-420). Returns, per sorted
// position, its pack index.
std::vector<u32> greedy_packs(const std::vector<u64> &sz, const std::vector<u64> &inb, u64 omega,
                              u64 delta) {
    const size_t m = sz.size();
    std::vector<u64> ps(m + 1, 0), pi(m + 1, 0);
    for (size_t i = 0; i < m; ++i) { ps[i + 1] = ps[i] + sz[i]; pi[i + 1] = pi[i] + inb[i]; }
    std::vector<u32> pack(m, 0);
    size_t pos = 0;
    u32 id = 0;
    while (pos < m) {
        size_t js = std::upper_bound(ps.begin(), ps.end(), ps[pos] + omega) - ps.begin();
        size_t ji = std::upper_bound(pi.begin(), pi.end(), pi[pos] + delta) - pi.begin();
        size_t nxt = std::max(pos + 1, std::min(js, ji) - 1);
        for (size_t i = pos; i < nxt && i < m; ++i) pack[i] = id;
        ++id;
        pos = nxt;
    }
    return pack;
}

// Level-synchronous BFS distances over hyperedges from `root` (NONE = unreached).
std::vector<u32> bfs(const G &g, const T &t, u32 root) {
    std::vector<u32> d(g.n, NONE), fr{root}, nx;
    std::vector<char> hd(g.e, 0);
    d[root] = 0;
    u32 L = 0;
    while (!fr.empty()) {
        nx.clear();
        for (u32 u : fr)
            for (u64 j = t.toff[u]; j < t.toff[u + 1]; ++j) {
                u32 h = t.touch[j];
                if (hd[h]) continue;
                hd[h] = 1;
                for (u64 k = g.off[h]; k < g.off[h + 1]; ++k)
                    if (d[g.pins[k]] == NONE) { d[g.pins[k]] = L + 1; nx.push_back(g.pins[k]); }
            }
        std::swap(fr, nx);
        ++L;
    }
    return d;
}

// This build's k-way initial partition: BFS from node 0, re-rooted at the farthest node
// (largest distance, then largest id); nodes ordered by (distance, id) with unreached nodes last;
// consecutive chunks of equal node weight: node i goes to floor((2*W_before + s_i) * k / (2*W)).
std::vector<u32> kway_initial(const G &g, const T &t, const u32 *nsize, u32 k) {
    std::vector<u32> part(g.n, 0);
    if (g.n == 0) return part;
    std::vector<u32> d0 = bfs(g, t, 0);
    u32 far = 0;
    for (u32 v = 0; v < g.n; ++v)
        if (d0[v] != NONE && (d0[v] > d0[far] || (d0[v] == d0[far] && v > far))) far = v;
    std::vector<u32> d = bfs(g, t, far);
    std::vector<u32> ord(g.n);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](u32 a, u32 b) { return d[a] < d[b]; });
    u64 W = 0;
    for (u32 v = 0; v < g.n; ++v) W += nsize[v];
    u64 before = 0;
    for (u32 i = 0; i < g.n; ++i) {
        u32 v = ord[i];
        u64 x = (2 * before + nsize[v]) * (u64)k / (2 * W);
        part[v] = (u32)std::min<u64>(x, k - 1);
        before += nsize[v];
    }
    return part;
}

// A random balanced start of the k-way multi-start: nodes ordered by
// (mix32(v ^ mix32(t * 0x9E3779B9 + seed)), v), cut into weight chunks as kway_initial does.
std::vector<u32> kway_random(const G &g, const u32 *nsize, u32 k, u32 t, u64 seed) {
    const u32 salt = mix32(t * 0x9E3779B9u + (u32)seed);
    std::vector<u32> ord(g.n), key(g.n), part(g.n, 0);
    for (u32 v = 0; v < g.n; ++v) key[v] = mix32(v ^ salt);
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](u32 a, u32 b) { return key[a] < key[b]; });
    u64 W = 0;
    for (u32 v = 0; v < g.n; ++v) W += nsize[v];
    u64 before = 0;
    for (u32 i = 0; i < g.n; ++i) {
        const u32 v = ord[i];
        const u64 x = (2 * before + nsize[v]) * (u64)k / (2 * (W ? W : 1));
        part[v] = (u32)std::min<u64>(x, k - 1);
        before += nsize[v];
    }
    return part;
}

// The k-way multi-start on the coarsest level (include/axc.h AXC_KWAY_TRIES): T copies of the
// level without its hyperedges of fewer than 2 pins (they never change a k-way gain), copy 0
// starting from `part`, copy t >= 1 from kway_random(t); all refined together for
// AXC_KWAY_TRY_ROUNDS rounds (each copy takes its own best prefix); the copy of least
// connectivity (the first on ties) replaces `part`. Returns false when fewer than 2 copies fit.
bool kway_multistart(const G &g, const std::vector<u32> &wfx, const u32 *nsize, u32 k, u32 omega, u64 seed,
                     std::vector<u32> &part) {
    std::vector<u32> keep;
    u64 P2 = 0;
    for (u32 h = 0; h < g.e; ++h) {
        const u64 len = g.off[h + 1] - g.off[h];
        if (len >= 2) { keep.push_back(h); P2 += len; }
    }
    const u64 NC = P2 ? std::min<u64>(AXC_KWAY_TRIES, AXC_KWAY_TRY_PINS / P2) : 0;
    if (NC < 2) return false;
    const u32 n = g.n, e2 = (u32)keep.size();
    G S;
    S.n = (u32)(NC * n);
    S.e = (u32)(NC * e2);
    S.off.assign(1, 0);
    std::vector<u32> wS;
    for (u32 t = 0; t < NC; ++t)
        for (u32 h : keep) {
            for (u64 i = g.off[h]; i < g.off[h + 1]; ++i) S.pins.push_back(g.pins[i] + t * n);
            S.off.push_back(S.pins.size());
            S.nsrc.push_back(g.nsrc[h]);
            wS.push_back(wfx[h]);
        }
    T tS = touching(S);
    std::vector<u32> nsS((size_t)NC * n), pS((size_t)NC * n);
    for (u32 t = 0; t < NC; ++t) {
        std::vector<u32> p0 = t == 0 ? part : kway_random(g, nsize, k, t, seed);
        for (u32 v = 0; v < n; ++v) { nsS[(size_t)t * n + v] = nsize[v]; pS[(size_t)t * n + v] = p0[v] + t * k; }
    }
    RefineCtx rc{&S, &tS, &wS, nsS.data(), (u32)(NC * k), omega, 0x7FFFFFFFu, false, seed};
    rc.copies = (u32)NC;
    rc.copy_n = n;
    refine_level(rc, pS, AXC_KWAY_TRY_ROUNDS);
    Census cs = census(S, pS);
    std::vector<i64> conn(NC, 0);
    for (u32 h = 0; h < S.e; ++h) conn[h / e2] += (i64)wS[h] * (i64)(cs.beg[h + 1] - cs.beg[h] - 1);
    u32 best = 0;
    for (u32 t = 1; t < NC; ++t)
        if (conn[t] < conn[best]) best = t;
    for (u32 v = 0; v < n; ++v) part[v] = pS[(size_t)best * n + v] - best * k;
    return true;
}

struct Level {
    G g;
    T t;
    std::vector<u32> nsize;
    std::vector<u32> groups;  // map to the next level
};

}  // namespace

extern "C" {

uint32_t or_wfx(float w) {
    if (!(w > 0.0f)) return 0;
    double x = std::floor((double)w * 262144.0);
    return x >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)x;
}

int or_read(const char *path, uint32_t *n, uint32_t *e, uint64_t *p, uint64_t *off, uint32_t *pins,
            uint32_t *nsrc, float *w) {
    std::string s(path);
    std::vector<u64> O{0};
    std::vector<u32> P, S;
    std::vector<float> W;
    u32 N = 0;
    auto ext = s.size() >= 4 ? s.substr(s.size() - 4) : std::string();
    if (ext == ".snn" || ext == ".axh") {
        std::ifstream f(path, std::ios::binary);
        if (!f) return 4;
        auto r32 = [&](u32 &v) { f.read((char *)&v, 4); return (bool)f; };
        u32 E;
        if (!r32(N) || !r32(E)) return 5;
        for (u32 i = 0; i < E; ++i) {
            u32 a, b;
            if (!r32(a) || !r32(b)) return 5;
            u32 cnt, ns;
            if (ext == ".snn") {
                if (a < 1 || b >= N) return 5;
                P.push_back(b); cnt = a; ns = 1;
            } else {
                if (b == 0 || a <= b) return 5;
                cnt = a; ns = b;
            }
            for (u32 k = 0; k < cnt; ++k) { u32 v; if (!r32(v) || v >= N) return 5; P.push_back(v); }
            float x; f.read((char *)&x, 4); if (!f) return 5;
            S.push_back(ns); W.push_back(x); O.push_back(P.size());
        }
    } else if (ext == ".hgr") {
        std::ifstream f(path);
        if (!f) return 4;
        std::string line;
        auto next = [&]() -> bool {
            while (std::getline(f, line)) {
                if (!line.empty() && line.back() == '\r') line.pop_back();
                size_t i = line.find_first_not_of(" \t");
                if (i == std::string::npos || line[i] == '%') continue;
                line = line.substr(i);
                return true;
            }
            return false;
        };
        if (!next()) return 5;
        unsigned long long E = 0, V = 0, fmt = 0;
        int got = std::sscanf(line.c_str(), "%llu %llu %llu", &E, &V, &fmt);
        if (got < 2) return 5;
        if (got < 3) fmt = 0;
        N = (u32)V;
        bool ew = fmt == 1 || fmt == 11;
        for (unsigned long long i = 0; i < E; ++i) {
            if (!next()) return 5;
            const char *c = line.c_str();
            char *endp;
            float x = 1.0f;
            if (ew) { x = std::strtof(c, &endp); c = endp; }
            std::vector<u32> nodes;
            while (true) {
                while (*c == ' ' || *c == '\t') ++c;
                if (*c < '0' || *c > '9') break;
                unsigned long long v = std::strtoull(c, &endp, 10);
                c = endp;
                if (v == 0 || v > V) return 5;
                nodes.push_back((u32)(v - 1));
            }
            if (nodes.empty()) return 5;
            if (nodes.size() == 1) continue;
            P.insert(P.end(), nodes.begin(), nodes.end());
            S.push_back(0); W.push_back(x); O.push_back(P.size());
        }
    } else {
        return 5;
    }
    *n = N; *e = (u32)S.size(); *p = P.size();
    if (off) std::copy(O.begin(), O.end(), off);
    if (pins) std::copy(P.begin(), P.end(), pins);
    if (nsrc) std::copy(S.begin(), S.end(), nsrc);
    if (w) std::copy(W.begin(), W.end(), w);
    return 0;
}

static G mkG(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc) {
    G g;
    g.n = n; g.e = e;
    g.off.assign(off, off + e + 1);
    g.pins.assign(pins, pins + off[e]);
    g.nsrc.assign(nsrc, nsrc + e);
    return g;
}

uint64_t or_dedupe(uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
                   uint64_t *out_off, uint32_t *out_pins, uint32_t *out_nsrc) {
    G d = dedupe(mkG(0, e, off, pins, nsrc));
    std::copy(d.off.begin(), d.off.end(), out_off);
    std::copy(d.pins.begin(), d.pins.end(), out_pins);
    std::copy(d.nsrc.begin(), d.nsrc.end(), out_nsrc);
    return d.pins.size();
}

void or_touching(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                 const uint32_t *nsrc, uint64_t *toff, uint32_t *touch, uint32_t *inbound) {
    T t = touching(mkG(n, e, off, pins, nsrc));
    std::copy(t.toff.begin(), t.toff.end(), toff);
    std::copy(t.touch.begin(), t.touch.end(), touch);
    std::copy(t.nin.begin(), t.nin.end(), inbound);
}

void or_rating(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
               const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
               const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
               uint32_t omega, uint32_t delta, uint32_t cnc, uint32_t *pairs, uint32_t *scores) {
    or_rating_len(n, e, off, pins, nsrc, wfx, toff, touch, inbound, node_size, omega, delta, cnc, RATE_MAX_LEN,
                  pairs, scores);
}

void or_rating_len(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                   const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
                   const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
                   uint32_t omega, uint32_t delta, uint32_t cnc, uint64_t max_len, uint32_t *pairs,
                   uint32_t *scores) {
    G g = mkG(n, e, off, pins, nsrc);
    T t;
    t.toff.assign(toff, toff + n + 1);
    t.touch.assign(touch, touch + toff[n]);
    t.nin.assign(inbound, inbound + n);
    std::vector<u32> w(wfx, wfx + e);
    rating(g, w, t, node_size, omega, delta, cnc, pairs, scores, max_len);
}

uint32_t or_matching(uint32_t n, uint32_t cnc, const uint32_t *pairs, const uint32_t *scores,
                     const uint32_t *node_size, const uint32_t *inbound, uint32_t omega, uint32_t delta,
                     uint32_t rounds, uint32_t *groups) {
    return matching(n, cnc, pairs, scores, node_size, inbound, omega, delta, rounds, groups);
}

uint64_t or_contract(uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
                     const uint32_t *groups, uint64_t *out_off, uint32_t *out_pins,
                     uint32_t *out_nsrc) {
    G g = mkG(0, e, off, pins, nsrc);
    u32 ng = 0;
    for (u64 k = 0; k < g.pins.size(); ++k) ng = std::max(ng, groups[g.pins[k]] + 1);
    G c = contract(g, groups, ng);
    std::copy(c.off.begin(), c.off.end(), out_off);
    std::copy(c.pins.begin(), c.pins.end(), out_pins);
    std::copy(c.nsrc.begin(), c.nsrc.end(), out_nsrc);
    return c.pins.size();
}

void or_gains(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
              const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
              const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
              const uint32_t *part, uint32_t num_parts, uint32_t omega, uint32_t delta,
              int encourage, uint32_t discount, uint32_t round, uint64_t seed, uint32_t *target,
              int64_t *gain) {
    G g = mkG(n, e, off, pins, nsrc);
    T t;
    t.toff.assign(toff, toff + n + 1);
    t.touch.assign(touch, touch + toff[n]);
    t.nin.assign(inbound, inbound + n);
    std::vector<u32> w(wfx, wfx + e), pv(part, part + n);
    RefineCtx rc{&g, &t, &w, node_size, num_parts, omega, delta, encourage != 0, seed};
    Census cs = census(g, pv);
    std::vector<u64> ps = part_sizes(pv, node_size, num_parts), pi = part_inbound(cs, e, num_parts);
    gains(rc, pv, cs, ps, pi, discount, round, target, gain);
}

void or_refine(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
               const uint32_t *wfx, const uint64_t *toff, const uint32_t *touch, const uint32_t *inbound,
               const uint32_t *node_size, uint32_t *part, uint32_t num_parts, uint32_t omega, uint32_t delta,
               int encourage, uint32_t rounds, uint64_t seed) {
    G g = mkG(n, e, off, pins, nsrc);
    T t;
    t.toff.assign(toff, toff + n + 1);
    t.touch.assign(touch, touch + toff[n]);
    t.nin.assign(inbound, inbound + n);
    std::vector<u32> w(wfx, wfx + e), pv(part, part + n);
    RefineCtx rc{&g, &t, &w, node_size, num_parts, omega, delta, encourage != 0, seed};
    refine_level(rc, pv, rounds);
    std::copy(pv.begin(), pv.end(), part);
}

void or_evaluate(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                 const uint32_t *nsrc, const float *w, const uint32_t *part, uint32_t omega,
                 uint32_t delta, uint32_t max_parts, int64_t *out) {
    u32 K = 0;
    for (u32 v = 0; v < n; ++v) K = std::max(K, part[v] + 1);
    std::vector<u64> cnt(K, 0), inb(K, 0);
    for (u32 v = 0; v < n; ++v) cnt[part[v]]++;
    u32 used = 0;
    u64 mx = 0;
    for (u32 p = 0; p < K; ++p) { used += cnt[p] > 0; mx = std::max(mx, cnt[p]); }
    i64 conn = 0, cut = 0, soed = 0;
    std::vector<u32> mk(K, NONE), mkd(K, NONE);
    for (u32 h = 0; h < e; ++h) {
        const u64 a = off[h], b = off[h + 1], s = a + nsrc[h];
        u32 lam = 0;
        for (u64 k = a; k < b; ++k) {
            u32 p = part[pins[k]];
            if (mk[p] != h) { mk[p] = h; ++lam; }
            if (k >= s && mkd[p] != h) { mkd[p] = h; inb[p]++; }
        }
        const i64 wf = (i64)or_wfx(w ? w[h] : 1.0f);
        const i64 l1 = lam ? (i64)lam - 1 : 0;  // an empty hyperedge connects nothing
        conn += wf * l1;
        cut += lam > 1 ? wf : 0;
        soed += wf * l1 * (i64)(b - a);
    }
    u64 mi = 0;
    for (u32 p = 0; p < K; ++p) mi = std::max(mi, inb[p]);
    const bool dense = used == K;
    const bool valid = dense && used <= max_parts && mx <= omega && mi <= delta;
    out[0] = conn; out[1] = cut; out[2] = soed; out[3] = used; out[4] = (i64)mx;
    out[5] = (i64)mi; out[6] = valid; out[7] = dense;
}

uint32_t or_partition(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                      const uint32_t *nsrc, const float *w, int mode, uint32_t omega,
                      uint32_t delta, uint32_t max_parts, uint32_t k, float eps, uint32_t cnc,
                      uint32_t rfr, int ipm, uint64_t seed, uint32_t *part, uint64_t *stats) {
    const bool kway = mode == 1;
    if (kway) {
        omega = (u32)std::ceil((1 + eps) * (float)n / k);  // sources/runconfig.cpp:190
        delta = 0x7FFFFFFFu;
        max_parts = k;
    }
    const u32 target = std::min<u32>(max_parts, (n + omega - 1) / omega);
    // k-way clusters stay below the balance slack, so weight-chunking stays within omega
    u32 omega_c = omega;
    if (kway) {
        double slack = std::floor((double)eps * (double)n / (double)k);
        omega_c = (u32)std::max(1.0, std::min<double>(slack, omega));
    }
    std::vector<Level> L(1);
    L[0].g = dedupe(mkG(n, e, off, pins, nsrc));
    L[0].t = touching(L[0].g);
    L[0].nsize.assign(n, 1);
    std::vector<u32> wfx(e);
    for (u32 h = 0; h < e; ++h) wfx[h] = or_wfx(w ? w[h] : 1.0f);
    if (stats) { stats[1] = L[0].g.pins.size(); }
    std::vector<u32> cpart;  // partition of the deepest level's nodes
    u32 K = 0;
    bool refine_deepest = false;
    for (u32 lv = 0;; ++lv) {
        Level &cur = L[lv];
        const u32 cn = cur.g.n;
        if (kway && cn < 8192) {
            cpart = kway_initial(cur.g, cur.t, cur.nsize.data(), k);
            K = k;
            refine_deepest = !kway_multistart(cur.g, wfx, cur.nsize.data(), k, omega, seed, cpart);
            break;
        }
        std::vector<u32> pairs((size_t)cn * cnc), scores((size_t)cn * cnc), groups(cn);
        rating(cur.g, wfx, cur.t, cur.nsize.data(), kway ? omega_c : omega, delta, cnc,
               pairs.data(), scores.data());
        u32 ng = matching(cn, cnc, pairs.data(), scores.data(), cur.nsize.data(), cur.t.nin.data(),
                          kway ? omega_c : omega, delta, 32, groups.data());
        const float ratio = (float)ng / (float)cn;
        if (kway && (ratio > 0.95f || ng < 1024)) {
            cpart = kway_initial(cur.g, cur.t, cur.nsize.data(), k);
            K = k;
            refine_deepest = !kway_multistart(cur.g, wfx, cur.nsize.data(), k, omega, seed, cpart);
            break;
        }
        if (!kway && (ng <= target || ng == cn || (lv >= 32 && ratio > 0.95f))) {
            if (ipm && ng >= 2) {
                std::vector<u64> gs(ng, 0), gi(ng, 0);
                for (u32 v = 0; v < cn; ++v) { gs[groups[v]] += cur.nsize[v]; gi[groups[v]] += cur.t.nin[v]; }
                std::vector<u32> ord(ng);
                std::iota(ord.begin(), ord.end(), 0u);
                std::stable_sort(ord.begin(), ord.end(), [&](u32 a, u32 b) {
                    return gs[a] != gs[b] ? gs[a] < gs[b] : gi[a] < gi[b];
                });
                std::vector<u64> ss(ng), si(ng);
                for (u32 i = 0; i < ng; ++i) { ss[i] = gs[ord[i]]; si[i] = gi[ord[i]]; }
                std::vector<u32> pk = greedy_packs(ss, si, omega, delta);
                std::vector<u32> rep(ng, NONE), gmap(ng);
                for (u32 i = 0; i < ng; ++i) rep[pk[i]] = std::min(rep[pk[i]], ord[i]);
                for (u32 i = 0; i < ng; ++i) gmap[ord[i]] = rep[pk[i]];
                std::vector<u32> nid(ng, NONE);
                u32 c = 0;
                for (u32 x = 0; x < ng; ++x) if (gmap[x] == x) nid[x] = c++;
                for (u32 v = 0; v < cn; ++v) groups[v] = nid[gmap[groups[v]]];
                ng = c;
            }
            cpart = groups;
            K = ng;
            break;
        }
        cur.groups = groups;
        Level nx;
        nx.g = contract(cur.g, groups.data(), ng);
        nx.t = touching(nx.g);
        nx.nsize.assign(ng, 0);
        for (u32 v = 0; v < cn; ++v) nx.nsize[groups[v]] += cur.nsize[v];
        L.push_back(std::move(nx));
    }
    if (stats) stats[0] = L.size();
    // uncoarsen and refine
    int deepest = (int)L.size() - 1;
    std::vector<u32> pcur = cpart;
    for (int lv = deepest; lv >= 0; --lv) {
        if (lv < deepest) {
            std::vector<u32> fine(L[lv].g.n);
            for (u32 v = 0; v < L[lv].g.n; ++v) fine[v] = pcur[L[lv].groups[v]];
            pcur.swap(fine);
        }
        if (lv == deepest && !refine_deepest) continue;
        RefineCtx rc{&L[lv].g, &L[lv].t, &wfx, L[lv].nsize.data(), K, omega, delta, !kway, seed};
        refine_level(rc, pcur, rfr);
    }
    // INCC: merge small partitions (sources/postprocess.cu:247-420)
    if (!kway) {
        Census cs = census(L[0].g, pcur);
        std::vector<u64> ps = part_sizes(pcur, L[0].nsize.data(), K), pi = part_inbound(cs, L[0].g.e, K);
        std::vector<u32> small;
        for (u32 p = 0; p < K; ++p) if (ps[p] < 16) small.push_back(p);
        if (!small.empty()) {
            std::stable_sort(small.begin(), small.end(), [&](u32 a, u32 b) {
                return ps[a] != ps[b] ? ps[a] < ps[b] : pi[a] < pi[b];
            });
            std::vector<u64> ss, si;
            for (u32 p : small) { ss.push_back(ps[p]); si.push_back(pi[p]); }
            std::vector<u32> pk = greedy_packs(ss, si, omega, delta);
            std::vector<u32> rep(small.size(), NONE), pmap(K);
            std::iota(pmap.begin(), pmap.end(), 0u);
            for (size_t i = 0; i < small.size(); ++i) rep[pk[i]] = std::min(rep[pk[i]], small[i]);
            for (size_t i = 0; i < small.size(); ++i) pmap[small[i]] = rep[pk[i]];
            for (auto &x : pcur) x = pmap[x];
        }
    }
    // zero-base in order of old id (sources/main.cu:817-830)
    std::vector<u32> used(K, 0), nid(K, NONE);
    for (u32 x : pcur) used[x] = 1;
    u32 c = 0;
    for (u32 p = 0; p < K; ++p) if (used[p]) nid[p] = c++;
    for (u32 v = 0; v < n; ++v) part[v] = nid[pcur[v]];
    return c;
}

}  // extern "C"
