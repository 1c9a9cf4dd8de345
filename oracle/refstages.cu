// refstages.cu — runs the reference's own coarsening stages on the GPU and dumps what they compute,
// so the oracle's rating and contraction can be pinned against the reference itself. TEST
// INFRASTRUCTURE ONLY: oracle/Makefile links it with the reference's objects compiled from the
// reference sources (everything but sources/main.cu), and tests/golden/make_refstages.py turns its
// output into committed fixtures.
//
//   refstages.exe <hypergraph> <omega> <delta> <cnc> <out.bin>
//
// It follows the set-up of sources/main.cu:117-248 for level 0 (rule-2 dedupe, upload, unit node
// sizes, the two constraint constants, device touching construction, sampled neighbourhood bound,
// neighbour lists), then calls, once each:
//   candidatesProposal (sources/coarsening.cu:17-68)       -> pairs, scores   [n * cnc]
//   groupNodes         (sources/coarsening.cu:70-210)      -> groups [n], their count
//   coarsenHedges      (sources/construction.cu:563-676)   -> coarse hyperedges of those groups
//   coarsenTouching    (sources/construction.cu:678-789)   -> coarse incidence sets
//
// out.bin (little-endian):
//   u32 n, u32 e, u64 P, u32 cnc
//   u32 pairs[n*cnc], u32 scores[n*cnc]
//   u32 ngroups, u32 groups[n]
//   u64 cP, u64 coff[e+1], u32 cpins[cP], u32 cnsrc[e]
//   u64 ctoff[ngroups+1], u32 ctouch[ctoff[ngroups]], u32 cinb[ngroups]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hgraph.hpp"
#include "constr.hpp"
#include "runconfig.hpp"

#include "utils.cuh"
#include "defines.cuh"
#include "constants.cuh"
#include "data_types.cuh"
#include "coarsening.cuh"
#include "construction.cuh"

using namespace hgraph;
using namespace config;

template <typename T>
static std::vector<T> down(const T *d, size_t count) {
    std::vector<T> h(count);
    if (count) CUDA_CHECK(cudaMemcpy(h.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}
template <typename T>
static T *up(const std::vector<T> &h) {
    T *d = nullptr;
    CUDA_CHECK(cudaMalloc(&d, (h.size() ? h.size() : 1) * sizeof(T)));
    if (!h.empty()) CUDA_CHECK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}
template <typename T>
static void put(FILE *f, const std::vector<T> &v) {
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
}
template <typename T>
static void put1(FILE *f, T x) {
    std::fwrite(&x, sizeof(T), 1, f);
}

int main(int argc, char **argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: refstages.exe <hypergraph> <omega> <delta> <cnc> <out.bin>\n");
        return 2;
    }
    const std::string in = argv[1];
    const uint32_t omega = (uint32_t)std::strtoul(argv[2], nullptr, 10);
    const uint32_t delta = (uint32_t)std::strtoul(argv[3], nullptr, 10);
    const uint32_t cnc = (uint32_t)std::strtoul(argv[4], nullptr, 10);
    if (cnc < 1 || cnc > MAX_CANDIDATES) {
        std::fprintf(stderr, "cnc must be in [1, %u]\n", MAX_CANDIDATES);
        return 2;
    }
    auto ends = [&](const char *x) { return in.size() >= 4 && in.substr(in.size() - 4) == x; };
    HyperGraph hg(0, {}, {}, false);
    try {
        if (ends(".hgr")) hg = HyperGraph::loadhMETIS(in, false);
        else if (ends(".snn")) hg = HyperGraph::loadSNN(in, false);
        else if (ends(".axh")) hg = HyperGraph::loadAXH(in, false);
        else { std::fprintf(stderr, "unsupported extension\n"); return 2; }
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "load error: %s\n", ex.what());
        return 1;
    }

    runconfig cfg{};
    cfg.mode = Mode::INCC;
    cfg.constr_type = ConstrType::MANL;
    cfg.oversized_multiplier = OVERSIZED_SIZE_MULTIPLIER;
    cfg.candidates_count = cnc;
    cfg.refine_repeats = REFINE_REPEATS;
    cfg.save_memory_up_to_level = 0;
    cfg.device_touching_construction = true;
    cfg.initial_partitions_merge = false;
    cfg.verbose_logs = false;
    cfg.verbose_info = false;
    cfg.verbose_errs_and_warns = true;
    cfg.verbose_kernel_launches = false;

    // sources/main.cu:117-136: rule-2 dedupe, offsets, source counts, weights
    hg.deduplicateHyperedges(2, false);
    const uint32_t n = hg.nodes(), e = (uint32_t)hg.hedges().size();
    const dim_t P = hg.hedgesFlat().size();
    std::vector<dim_t> off(e + 1);
    std::vector<uint32_t> nsrc(e);
    std::vector<float> w(e);
    for (uint32_t i = 0; i < e; ++i) {
        off[i] = hg.hedges()[i].offset();
        nsrc[i] = hg.hedges()[i].src_count();
        w[i] = hg.hedges()[i].weight();
    }
    off[e] = P;

    // sources/main.cu:196-241: device copies, unit node sizes, constraint constants
    uint32_t *d_hedges = up(hg.hedgesFlat());
    dim_t *d_off = up(off);
    uint32_t *d_nsrc = up(nsrc);
    float *d_w = up(w);
    uint32_t *d_nsizes = up(std::vector<uint32_t>(n, 1u));
    uint32_t *d_pairs = nullptr, *d_scores = nullptr;
    CUDA_CHECK(cudaMalloc(&d_pairs, (size_t)n * cnc * sizeof(uint32_t)));
    CUDA_CHECK(cudaMalloc(&d_scores, (size_t)n * cnc * sizeof(uint32_t)));
    slot *d_slots = nullptr;
    dp_score *d_dp = nullptr;
    CUDA_CHECK(cudaMalloc(&d_slots, (size_t)n * sizeof(slot)));
    CUDA_CHECK(cudaMalloc(&d_dp, (size_t)n * sizeof(dp_score)));
    CUDA_CHECK(cudaMemcpyToSymbol(max_nodes_per_part, &omega, sizeof(uint32_t)));
    CUDA_CHECK(cudaMemcpyToSymbol(max_inbound_per_part, &delta, sizeof(uint32_t)));
    CUDA_CHECK(cudaDeviceSynchronize());
    cudaDeviceProp props;
    CUDA_CHECK(cudaGetDeviceProperties(&props, 0));

    // sources/main.cu:244-289: touching sets, neighbourhood bound, neighbour lists
    auto [tsize, d_touch, d_toff, d_inb] = buildTouching(cfg, d_hedges, d_off, d_nsrc, n, e);
    const dim_t max_nb = sampleMaxNeighborhoodSize(cfg, d_hedges, d_off, d_touch, d_toff, n, NEIGHBORS_SAMPLE_SIZE);
    uint32_t *d_nb = nullptr;
    dim_t *d_nboff = nullptr;
    dim_t nbsize;
    std::tie(nbsize, d_nb, d_nboff) = buildNeighbors(cfg, d_hedges, d_off, d_touch, d_toff, n, (uint32_t)max_nb,
                                                     d_nb, d_nboff);

    // one coarsening level (sources/main.cu:394-433, 611-638)
    candidatesProposal(cfg, d_hedges, d_off, d_nsrc, d_nb, d_nboff, d_touch, d_toff, d_inb, d_w, d_nsizes, n, d_pairs,
                       d_scores);
    auto [ngroups, d_groups, d_gsizes, d_ungroups, d_ungroups_off] =
        groupNodes(cfg, props, d_inb, d_pairs, d_scores, d_nsizes, n, omega, delta, d_slots, d_dp);
    auto [cP, d_cpins, d_coff, d_cnsrc] = coarsenHedges(cfg, d_hedges, d_off, d_nsrc, d_groups, e, P);
    auto [ctsize, d_ctouch, d_ctoff, d_cinb] =
        coarsenTouching(cfg, d_cpins, d_coff, d_touch, d_toff, d_inb, d_ungroups, d_ungroups_off, ngroups, e);
    CUDA_CHECK(cudaDeviceSynchronize());

    FILE *f = std::fopen(argv[5], "wb");
    if (!f) return 1;
    put1<uint32_t>(f, n);
    put1<uint32_t>(f, e);
    put1<uint64_t>(f, P);
    put1<uint32_t>(f, cnc);
    put(f, down(d_pairs, (size_t)n * cnc));
    put(f, down(d_scores, (size_t)n * cnc));
    put1<uint32_t>(f, ngroups);
    put(f, down(d_groups, n));
    put1<uint64_t>(f, cP);
    put(f, down(d_coff, (size_t)e + 1));
    put(f, down(d_cpins, cP));
    put(f, down(d_cnsrc, e));
    std::vector<dim_t> ctoff = down(d_ctoff, (size_t)ngroups + 1);
    put(f, ctoff);
    put(f, down(d_ctouch, ngroups ? ctoff[ngroups] : 0));
    put(f, down(d_cinb, ngroups));
    std::fclose(f);
    std::printf("refstages: n=%u e=%u P=%llu groups=%u coarse pins=%llu\n", n, e, (unsigned long long)P, ngroups,
                (unsigned long long)cP);
    return 0;
}
