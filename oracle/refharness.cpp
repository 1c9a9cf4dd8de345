// refharness.cpp — runs the reference's own host code (includes/hgraph.hpp, compiled here from
// the reference sources by oracle/Makefile) and dumps what it computes, so the oracle's
// restatements can be pinned against the reference itself. TEST INFRASTRUCTURE ONLY.
//
//   refharness.exe dump <hypergraph> <out.bin>
//
// out.bin (little-endian):
//   section A, as loaded (HyperGraph::loadhMETIS/loadSNN/loadAXH):
//     u32 n, u32 e, u64 P, u64 off[e+1], u32 pins[P], u32 nsrc[e], f32 w[e]
//   section B, after deduplicateHyperedges(2, false) (sources/main.cu:125): same layout
//   section C, incidence sets of the deduplicated graph (buildIncidenceSets + inboundSortedIds /
//     outboundSortedIds, the layout of sources/construction.cu:17-62):
//     u64 toff[n+1], u32 touch[toff[n]], u32 inbound[n]
#include <cstdio>
#include <string>
#include <vector>

#include "constr.hpp"
#include "hgraph.hpp"

using namespace hgraph;

static void put_graph(FILE *f, const HyperGraph &hg) {
    uint32_t n = hg.nodes(), e = (uint32_t)hg.hedges().size();
    uint64_t P = hg.hedgesFlat().size();
    std::fwrite(&n, 4, 1, f);
    std::fwrite(&e, 4, 1, f);
    std::fwrite(&P, 8, 1, f);
    std::vector<uint64_t> off(e + 1);
    std::vector<uint32_t> ns(e);
    std::vector<float> w(e);
    for (uint32_t i = 0; i < e; ++i) {
        off[i] = hg.hedges()[i].offset();
        ns[i] = hg.hedges()[i].src_count();
        w[i] = hg.hedges()[i].weight();
    }
    off[e] = P;
    std::fwrite(off.data(), 8, off.size(), f);
    std::fwrite(hg.hedgesFlat().data(), 4, P, f);
    std::fwrite(ns.data(), 4, e, f);
    std::fwrite(w.data(), 4, e, f);
}

int main(int argc, char **argv) {
    if (argc != 4 || std::string(argv[1]) != "dump") {
        std::fprintf(stderr, "usage: refharness.exe dump <hypergraph> <out.bin>\n");
        return 2;
    }
    std::string in = argv[2];
    auto ends = [&](const char *x) { return in.size() >= 4 && in.substr(in.size() - 4) == x; };
    HyperGraph hg(0, {}, {}, false);
    try {
        if (ends(".hgr")) hg = HyperGraph::loadhMETIS(in, false);
        else if (ends(".snn")) hg = HyperGraph::loadSNN(in, false);
        else if (ends(".axh")) hg = HyperGraph::loadAXH(in, false);
        else { std::fprintf(stderr, "unsupported extension\n"); return 2; }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "load error: %s\n", e.what());
        return 1;
    }
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    put_graph(f, hg);
    hg.deduplicateHyperedges(2, false);
    put_graph(f, hg);
    hg.buildIncidenceSets();
    uint32_t n = hg.nodes();
    std::vector<uint64_t> toff(n + 1, 0);
    std::vector<uint32_t> touch, inb(n);
    for (uint32_t v = 0; v < n; ++v) {
        toff[v] = touch.size();
        for (uint32_t h : hg.inboundSortedIds(v)) touch.push_back(h);
        inb[v] = (uint32_t)(touch.size() - toff[v]);
        for (uint32_t h : hg.outboundSortedIds(v)) touch.push_back(h);
    }
    toff[n] = touch.size();
    std::fwrite(toff.data(), 8, toff.size(), f);
    std::fwrite(touch.data(), 4, touch.size(), f);
    std::fwrite(inb.data(), 4, inb.size(), f);
    std::fclose(f);
    return 0;
}
