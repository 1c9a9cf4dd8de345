// Host side of the C ABI: hypergraph readers and writers, partition files, the quotient
// hypergraph used by `-s`, and the seeded synthetic generators.
//
// Readers follow the reference's HyperGraph loaders (includes/hgraph.hpp:707-743 .snn,
// 805-854 .axh, 936-1013 .hgr) including their quirks: .hgr nets have no sources, singleton
// nets are skipped, vertex weights are ignored, ids are 1-based in the file. Unlike the
// reference (which reads 4 bytes per call through std::ifstream) the binary formats are read
// with one bulk read and parsed in memory.
#include "axc_host.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <omp.h>
#include <string>
#include <vector>

namespace axc {

static bool read_file(const char *path, std::vector<char> &buf) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    if (std::fseek(f, 0, SEEK_END) != 0) { std::fclose(f); return false; }
    long sz = std::ftell(f);
    if (sz < 0) { std::fclose(f); return false; }
    std::rewind(f);
    buf.resize((size_t)sz);
    size_t got = sz ? std::fread(buf.data(), 1, (size_t)sz, f) : 0;
    std::fclose(f);
    return got == (size_t)sz;
}

void publish(HostGraph *hg, axc_hgraph *out) {
    out->n = hg->n;
    out->e = (uint32_t)hg->nsrc.size();
    out->hedge_off = hg->off.data();
    out->pins = hg->pins.data();
    out->src_count = hg->nsrc.data();
    out->hedge_w = hg->w.data();
    out->_owner = hg;
}

}  // namespace axc

using namespace axc;

extern "C" void axc_free_hgraph(axc_hgraph *g) {
    if (!g) return;
    delete static_cast<HostGraph *>(g->_owner);
    std::memset(g, 0, sizeof(*g));
}

// .snn: u32 n, u32 E, then per hedge {u32 dst_count, u32 src, u32 dst[dst_count], f32 w}
extern "C" int axc_read_snn(const char *path, axc_hgraph *out) {
    if (!path || !out) return AXC_EINVAL;
    std::vector<char> buf;
    if (!read_file(path, buf)) return AXC_EIO;
    if (buf.size() < 8) return AXC_EFORMAT;
    const uint8_t *p = (const uint8_t *)buf.data(), *end = p + buf.size();
    auto r32 = [&](uint32_t &v) -> bool {
        if (end - p < 4) return false;
        std::memcpy(&v, p, 4); p += 4; return true;
    };
    uint32_t n, E;
    if (!r32(n) || !r32(E)) return AXC_EFORMAT;
    auto *hg = new HostGraph();
    hg->n = n;
    hg->off.reserve((size_t)E + 1);
    hg->nsrc.reserve(E);
    hg->w.reserve(E);
    hg->off.push_back(0);
    hg->pins.reserve((buf.size() - 8) / 4);
    for (uint32_t i = 0; i < E; ++i) {
        uint32_t dstc, src;
        if (!r32(dstc) || !r32(src)) { delete hg; return AXC_EFORMAT; }
        if (dstc < 1 || src >= n) { delete hg; return AXC_EFORMAT; }  // hgraph.hpp:145 needs >= 1 destination
        if ((size_t)(end - p) < (size_t)dstc * 4 + 4) { delete hg; return AXC_EFORMAT; }
        hg->pins.push_back(src);
        size_t base = hg->pins.size();
        hg->pins.resize(base + dstc);
        std::memcpy(hg->pins.data() + base, p, (size_t)dstc * 4);
        p += (size_t)dstc * 4;
        for (size_t k = base; k < base + dstc; ++k)
            if (hg->pins[k] >= n) { delete hg; return AXC_EFORMAT; }
        float w; std::memcpy(&w, p, 4); p += 4;
        hg->nsrc.push_back(1);
        hg->w.push_back(w);
        hg->off.push_back(hg->pins.size());
    }
    publish(hg, out);
    return AXC_OK;
}

// .axh: u32 n, u32 E, then per hedge {u32 pin_count, u32 src_count, u32 pins[], f32 w}
extern "C" int axc_read_axh(const char *path, axc_hgraph *out) {
    if (!path || !out) return AXC_EINVAL;
    std::vector<char> buf;
    if (!read_file(path, buf)) return AXC_EIO;
    if (buf.size() < 8) return AXC_EFORMAT;
    const uint8_t *p = (const uint8_t *)buf.data(), *end = p + buf.size();
    auto r32 = [&](uint32_t &v) -> bool {
        if (end - p < 4) return false;
        std::memcpy(&v, p, 4); p += 4; return true;
    };
    uint32_t n, E;
    if (!r32(n) || !r32(E)) return AXC_EFORMAT;
    auto *hg = new HostGraph();
    hg->n = n;
    hg->off.push_back(0);
    for (uint32_t i = 0; i < E; ++i) {
        uint32_t pc, sc;
        if (!r32(pc) || !r32(sc)) { delete hg; return AXC_EFORMAT; }
        // hgraph.hpp:826-827 (src_count >= 1, pin_count >= src_count) and :145 (>= 1 destination)
        if (sc == 0 || pc < sc || pc == sc) { delete hg; return AXC_EFORMAT; }
        if ((size_t)(end - p) < (size_t)pc * 4 + 4) { delete hg; return AXC_EFORMAT; }
        size_t base = hg->pins.size();
        hg->pins.resize(base + pc);
        std::memcpy(hg->pins.data() + base, p, (size_t)pc * 4);
        p += (size_t)pc * 4;
        for (size_t k = base; k < base + pc; ++k)
            if (hg->pins[k] >= n) { delete hg; return AXC_EFORMAT; }
        float w; std::memcpy(&w, p, 4); p += 4;
        hg->nsrc.push_back(sc);
        hg->w.push_back(w);
        hg->off.push_back(hg->pins.size());
    }
    publish(hg, out);
    return AXC_OK;
}

// .hgr (hMETIS): "E V [fmt]" header, E net lines "[w] v1 v2 ...", '%' comments.
//
// Parsed in parallel (OpenMP): the line breaks are found per chunk of the buffer, the lines are
// classified (blank and '%' lines are not data), and the net lines are parsed twice, once to
// count and check each net and once, after a prefix sum over the kept nets, to write its pins.
// The result, and which inputs fail, are those of a line-by-line reading.
namespace {

bool hgr_u64(const char *&q, const char *le, uint64_t &v) {
    while (q < le && (*q == ' ' || *q == '\t')) ++q;
    if (q >= le || *q < '0' || *q > '9') return false;
    uint64_t x = 0;
    while (q < le && *q >= '0' && *q <= '9') {
        x = x * 10 + (uint64_t)(*q - '0');
        if (x > 0xFFFFFFFFFFull) return false;
        ++q;
    }
    v = x;
    return true;
}

// One net line: its weight and pins (1-based ids in the file, 0-based out). Counts the pins and
// writes them when `pins` is set. Returns false for a malformed line ("Invalid node
// encountered", a missing weight or no node at all).
bool hgr_net(const char *q, const char *le, bool edge_w, uint64_t V, float &w, uint64_t &cnt, uint32_t *pins) {
    w = 1.0f;
    if (edge_w) {
        char tmp[64];
        while (q < le && (*q == ' ' || *q == '\t')) ++q;
        size_t k = 0;
        while (q < le && *q != ' ' && *q != '\t' && k < 63) tmp[k++] = *q++;
        tmp[k] = 0;
        char *ep = nullptr;
        w = std::strtof(tmp, &ep);
        if (ep == tmp) return false;
    }
    cnt = 0;
    uint64_t v;
    while (hgr_u64(q, le, v)) {
        if (v == 0 || v > V) return false;
        if (pins) pins[cnt] = (uint32_t)(v - 1);
        ++cnt;
    }
    return cnt > 0;
}

}  // namespace

extern "C" int axc_read_hgr(const char *path, axc_hgraph *out) {
    if (!path || !out) return AXC_EINVAL;
    std::vector<char> buf;
    if (!read_file(path, buf)) return AXC_EIO;
    buf.push_back('\n');
    const char *base = buf.data();
    const size_t N = buf.size();
    // line ends ('\n' positions), found per chunk
    const int T = std::max(1, omp_get_max_threads());
    const size_t chunk = (N + (size_t)T - 1) / (size_t)T;
    std::vector<size_t> ccount((size_t)T + 1, 0);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; ++t) {
        const size_t a = std::min(N, (size_t)t * chunk), b = std::min(N, a + chunk);
        size_t c = 0;
        for (const char *x = base + a, *e = base + b; x < e; ++c) {
            x = (const char *)std::memchr(x, '\n', (size_t)(e - x));
            if (!x) break;
            ++x;
        }
        ccount[(size_t)t + 1] = c;
    }
    for (int t = 0; t < T; ++t) ccount[(size_t)t + 1] += ccount[(size_t)t];
    const size_t L = ccount[(size_t)T];
    std::vector<size_t> lend(L);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; ++t) {
        const size_t a = std::min(N, (size_t)t * chunk), b = std::min(N, a + chunk);
        size_t i = ccount[(size_t)t];
        for (const char *x = base + a, *e = base + b; x < e;) {
            x = (const char *)std::memchr(x, '\n', (size_t)(e - x));
            if (!x) break;
            lend[i++] = (size_t)(x - base);
            ++x;
        }
    }
    // data lines: trimmed of leading blanks and a trailing '\r'; blank and '%' lines skipped
    // (hgraph.hpp:940-950)
    std::vector<uint32_t> isdata(L);
    std::vector<size_t> lbeg(L), lfin(L);
#pragma omp parallel for num_threads(T) schedule(static)
    for (size_t i = 0; i < L; ++i) {
        const size_t s0 = i ? lend[i - 1] + 1 : 0;
        const char *q = base + s0, *e = base + lend[i];
        while (q < e && (*q == ' ' || *q == '\t')) ++q;
        const char *ee = e;
        if (ee > q && ee[-1] == '\r') --ee;
        isdata[i] = (q == ee || *q == '%') ? 0u : 1u;
        lbeg[i] = (size_t)(q - base);
        lfin[i] = (size_t)(ee - base);
    }
    std::vector<size_t> data;
    data.reserve(L);
    for (size_t i = 0; i < L; ++i)
        if (isdata[i]) data.push_back(i);
    if (data.empty()) return AXC_EFORMAT;  // "Empty .hgr file"
    uint64_t E64, V64, fmt = 0;
    {
        const char *q = base + lbeg[data[0]], *le = base + lfin[data[0]];
        if (!hgr_u64(q, le, E64) || !hgr_u64(q, le, V64)) return AXC_EFORMAT;
        if (E64 > 0xFFFFFFFFull || V64 > 0xFFFFFFFFull) return AXC_EFORMAT;
        if (!hgr_u64(q, le, fmt)) fmt = 0;
    }
    if (data.size() - 1 < E64) return AXC_EFORMAT;  // unexpected end of file
    const bool edge_w = (fmt == 1 || fmt == 11);
    // pass 1: count and check every net; singleton nets are skipped (hgraph.hpp:989-992)
    std::vector<uint64_t> cnt(E64 + 1, 0);
    std::vector<float> wv(E64);
    int bad = 0;
#pragma omp parallel for num_threads(T) schedule(dynamic, 4096) reduction(| : bad)
    for (int64_t i = 0; i < (int64_t)E64; ++i) {
        const size_t l = data[(size_t)i + 1];
        uint64_t c = 0;
        if (!hgr_net(base + lbeg[l], base + lfin[l], edge_w, V64, wv[(size_t)i], c, nullptr)) bad |= 1;
        cnt[(size_t)i] = c == 1 ? 0 : c;
    }
    if (bad) return AXC_EFORMAT;
    auto *hg = new HostGraph();
    hg->n = (uint32_t)V64;
    std::vector<uint64_t> poff(E64 + 1, 0);
    for (uint64_t i = 0; i < E64; ++i) poff[i + 1] = poff[i] + cnt[i];
    hg->pins.resize(poff[E64]);
    // pass 2: write the kept nets' pins
#pragma omp parallel for num_threads(T) schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)E64; ++i) {
        if (!cnt[(size_t)i]) continue;
        const size_t l = data[(size_t)i + 1];
        float w;
        uint64_t c;
        hgr_net(base + lbeg[l], base + lfin[l], edge_w, V64, w, c, hg->pins.data() + poff[(size_t)i]);
    }
    hg->off.reserve(E64 + 1);
    hg->off.push_back(0);
    for (uint64_t i = 0; i < E64; ++i) {
        if (!cnt[i]) continue;
        hg->nsrc.push_back(0);
        hg->w.push_back(wv[i]);
        hg->off.push_back(poff[i + 1]);
    }
    publish(hg, out);
    return AXC_OK;
}

extern "C" int axc_read_auto(const char *path, axc_hgraph *out) {
    if (!path) return AXC_EINVAL;
    std::string s(path);
    auto ends = [&](const char *x) {
        size_t l = std::strlen(x);
        return s.size() >= l && s.compare(s.size() - l, l, x) == 0;
    };
    if (ends(".hgr")) return axc_read_hgr(path, out);
    if (ends(".snn")) return axc_read_snn(path, out);
    if (ends(".axh")) return axc_read_axh(path, out);
    return AXC_EFORMAT;  // runconfig.cpp:171-173
}

static int write_snn(const char *path, const axc_hgraph *g) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return AXC_EIO;
    std::vector<uint32_t> rec;
    uint32_t hdr[2] = {g->n, g->e};
    std::fwrite(hdr, 4, 2, f);
    for (uint32_t i = 0; i < g->e; ++i) {
        uint64_t a = g->hedge_off[i], b = g->hedge_off[i + 1];
        uint32_t dstc = (uint32_t)(b - a - 1);  // saveSNN keeps the first pin as the source
        std::fwrite(&dstc, 4, 1, f);
        std::fwrite(g->pins + a, 4, (size_t)(b - a), f);
        float w = g->hedge_w ? g->hedge_w[i] : 1.0f;
        std::fwrite(&w, 4, 1, f);
    }
    return std::fclose(f) == 0 ? AXC_OK : AXC_EIO;
}

static int write_axh(const char *path, const axc_hgraph *g) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return AXC_EIO;
    uint32_t hdr[2] = {g->n, g->e};
    std::fwrite(hdr, 4, 2, f);
    for (uint32_t i = 0; i < g->e; ++i) {
        uint64_t a = g->hedge_off[i], b = g->hedge_off[i + 1];
        uint32_t rec[2] = {(uint32_t)(b - a), g->src_count[i]};
        if (rec[1] == 0 || rec[0] < rec[1]) { std::fclose(f); return AXC_EINVAL; }
        std::fwrite(rec, 4, 2, f);
        std::fwrite(g->pins + a, 4, (size_t)(b - a), f);
        float w = g->hedge_w ? g->hedge_w[i] : 1.0f;
        std::fwrite(&w, 4, 1, f);
    }
    return std::fclose(f) == 0 ? AXC_OK : AXC_EIO;
}

static int write_hgr(const char *path, const axc_hgraph *g) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return AXC_EIO;
    bool emit_w = false;
    for (uint32_t i = 0; g->hedge_w && i < g->e; ++i)
        if (g->hedge_w[i] != 1.0f) { emit_w = true; break; }
    std::fprintf(f, emit_w ? "%u %u 01\n" : "%u %u\n", g->e, g->n);
    std::string line;
    char tmp[32];
    for (uint32_t i = 0; i < g->e; ++i) {
        line.clear();
        if (emit_w) {
            // savehMETIS writes uint32(w * 1024) (hgraph.hpp:1040)
            std::snprintf(tmp, sizeof tmp, "%u ", (uint32_t)(g->hedge_w[i] * 1024.0f));
            line += tmp;
        }
        for (uint64_t k = g->hedge_off[i]; k < g->hedge_off[i + 1]; ++k) {
            std::snprintf(tmp, sizeof tmp, k + 1 < g->hedge_off[i + 1] ? "%u " : "%u", g->pins[k] + 1);
            line += tmp;
        }
        line += '\n';
        std::fwrite(line.data(), 1, line.size(), f);
    }
    return std::fclose(f) == 0 ? AXC_OK : AXC_EIO;
}

extern "C" int axc_write_hgraph(const char *path, const axc_hgraph *g) {
    if (!path || !g) return AXC_EINVAL;
    std::string s(path);
    auto ends = [&](const char *x) {
        size_t l = std::strlen(x);
        return s.size() >= l && s.compare(s.size() - l, l, x) == 0;
    };
    if (ends(".snn")) return write_snn(path, g);
    if (ends(".axh")) return write_axh(path, g);
    if (ends(".hgr")) return write_hgr(path, g);
    return AXC_EFORMAT;
}

extern "C" int axc_write_partition(const char *path, const uint32_t *part, uint32_t n) {
    if (!path || (!part && n)) return AXC_EINVAL;
    FILE *f = std::fopen(path, "wb");
    if (!f) return AXC_EIO;
    std::string out;
    out.reserve((size_t)n * 7);
    char tmp[16];
    for (uint32_t i = 0; i < n; ++i) {
        int l = std::snprintf(tmp, sizeof tmp, "%u\n", part[i]);
        out.append(tmp, (size_t)l);
    }
    size_t w = std::fwrite(out.data(), 1, out.size(), f);
    int rc = std::fclose(f);
    return (w == out.size() && rc == 0) ? AXC_OK : AXC_EIO;
}

extern "C" int axc_read_partition(const char *path, uint32_t n, uint32_t *out) {
    if (!path || (!out && n)) return AXC_EINVAL;
    std::vector<char> buf;
    if (!read_file(path, buf)) return AXC_EIO;
    buf.push_back('\n');
    const char *p = buf.data(), *end = p + buf.size() - 1;
    uint32_t idx = 0;
    while (p < end) {
        const char *e = (const char *)std::memchr(p, '\n', (size_t)(end + 1 - p));
        const char *q = p, *le = e;
        if (le > q && le[-1] == '\r') --le;
        while (q < le && (*q == ' ' || *q == '\t')) ++q;
        if (idx >= n) return AXC_EFORMAT;  // more entries than nodes (hgraph.hpp:1070)
        uint64_t v = 0;
        if (q >= le || *q < '0' || *q > '9') return AXC_EFORMAT;
        while (q < le && *q >= '0' && *q <= '9') {
            v = v * 10 + (uint64_t)(*q - '0');
            if (v > 0xFFFFFFFFull) return AXC_EFORMAT;
            ++q;
        }
        while (q < le && (*q == ' ' || *q == '\t')) ++q;
        if (q != le) return AXC_EFORMAT;  // trailing data (hgraph.hpp:1075)
        out[idx++] = (uint32_t)v;
        p = e + 1;
    }
    return idx == n ? AXC_OK : AXC_EFORMAT;
}

namespace axc {

HostGraph *quotient_merge(uint32_t K, uint32_t e, const std::vector<uint32_t> &qcnt, const std::vector<uint32_t> &qsrc,
                          const std::vector<uint32_t> &qpins, const float *w) {
    struct Item {
        uint64_t at;  // first entry in qpins
        uint32_t ns, nd, h;
    };
    std::vector<Item> items;
    uint64_t at = 0;
    for (uint32_t h = 0; h < e; ++h) {
        if (!qcnt[h]) continue;
        items.push_back({at, qsrc[h], qcnt[h] - qsrc[h], h});
        at += qcnt[h];
    }
    const uint32_t *q = qpins.data();
    auto less = [&](const Item &x, const Item &y) {  // std::pair<std::vector, std::vector> order
        const uint32_t *xs = q + x.at, *ys = q + y.at;
        if (std::lexicographical_compare(xs, xs + x.ns, ys, ys + y.ns)) return true;
        if (std::lexicographical_compare(ys, ys + y.ns, xs, xs + x.ns)) return false;
        return std::lexicographical_compare(xs + x.ns, xs + x.ns + x.nd, ys + y.ns, ys + y.ns + y.nd);
    };
    auto same = [&](const Item &x, const Item &y) {
        return x.ns == y.ns && x.nd == y.nd && std::equal(q + x.at, q + x.at + x.ns + x.nd, q + y.at);
    };
    std::stable_sort(items.begin(), items.end(), less);  // equal keys stay in hyperedge order
    auto *hg = new HostGraph();
    hg->n = K;
    hg->off.push_back(0);
    for (size_t i = 0; i < items.size();) {
        size_t j = i;
        double sum = 0.0;
        for (; j < items.size() && same(items[i], items[j]); ++j) sum += w ? (double)w[items[j].h] : 1.0;
        const Item &it = items[i];
        hg->pins.insert(hg->pins.end(), q + it.at, q + it.at + it.ns + it.nd);
        hg->nsrc.push_back(it.ns);
        hg->w.push_back((float)sum);
        hg->off.push_back(hg->pins.size());
        i = j;
    }
    return hg;
}

}  // namespace axc

// Quotient hypergraph of getPartitionsHypergraph(part, remove_self_cycles=2, squish=true)
// (includes/hgraph.hpp:286-376): per hedge the distinct source partitions and the distinct
// destination partitions minus the source ones; hedges with <= 1 source partition and no
// destination partition vanish; identical (sources, destinations) pairs merge with summed weight.
// The reference merges by a 64-bit hash of the pair; this version merges by the exact pair and
// emits hedges in ascending (sources, destinations) order.
extern "C" int axc_quotient_hgraph(const axc_hgraph *g, const uint32_t *part, axc_hgraph *out) {
    if (!g || !part || !out) return AXC_EINVAL;
    uint32_t K = 0;
    for (uint32_t v = 0; v < g->n; ++v) K = std::max(K, part[v] + 1);
    std::map<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>, double> acc;
    std::vector<uint32_t> sp, dp;
    for (uint32_t i = 0; i < g->e; ++i) {
        uint64_t a = g->hedge_off[i], b = g->hedge_off[i + 1];
        sp.clear(); dp.clear();
        for (uint64_t k = a; k < b; ++k) {
            uint32_t pp = part[g->pins[k]];
            if (k < a + g->src_count[i]) sp.push_back(pp); else dp.push_back(pp);
        }
        std::sort(sp.begin(), sp.end()); sp.erase(std::unique(sp.begin(), sp.end()), sp.end());
        std::sort(dp.begin(), dp.end()); dp.erase(std::unique(dp.begin(), dp.end()), dp.end());
        std::vector<uint32_t> d2;
        std::set_difference(dp.begin(), dp.end(), sp.begin(), sp.end(), std::back_inserter(d2));
        if (sp.size() <= 1 && d2.empty()) continue;
        acc[{sp, d2}] += g->hedge_w ? (double)g->hedge_w[i] : 1.0;
    }
    auto *hg = new HostGraph();
    hg->n = K;
    hg->off.push_back(0);
    for (auto &kv : acc) {
        hg->pins.insert(hg->pins.end(), kv.first.first.begin(), kv.first.first.end());
        hg->pins.insert(hg->pins.end(), kv.first.second.begin(), kv.first.second.end());
        hg->nsrc.push_back((uint32_t)kv.first.first.size());
        hg->w.push_back((float)kv.second);
        hg->off.push_back(hg->pins.size());
    }
    publish(hg, out);
    return AXC_OK;
}
