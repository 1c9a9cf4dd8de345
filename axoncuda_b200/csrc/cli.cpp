// axc_hgraph_gpu — drop-in for the reference's hgraph_gpu.exe command line
// (flags of sources/runconfig.cpp:25-46, result lines of sources/main.cu:54-70 and 908-928).
// A thin client of include/axc.h: all partitioning runs on the GPU behind the C ABI.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/axc.h"

static void help() {
    std::printf(
        "Usage:\n"
        "  prog -r <input_file> [-c <constr>] [-s <output_file>] [-p <part_file>]\n"
        "  prog -r <input_file> [-k <k> <eps>] [-s <output_file>] [-p <part_file>]\n"
        "  prog -h\n\n"
        "Options:\n"
        "  -r <file>   Read hypergraph from file (.hgr, .snn, .axh)\n"
        "  -s <file>   Save partitioned hypergraph to file\n"
        "  -p <file>   Save the partitioning to file (one line per node, its partition id)\n"
        "  -c <name>   Preset constraints: truenorth, loihi64, loihi84, loihi1024 (default loihi64)\n"
        "  -m <> <> <> Constraints: max part. size, max part. distinct inbound hedges, max num. of part.s\n"
        "  -k <k> <e>  K-way balanced constraints (overrides -c and -m)\n"
        "  -om <mult>  Accepted for compatibility (no oversized buffers are used)\n"
        "  -cnc <num>  Candidates proposed per node during coarsening (<= 16)\n"
        "  -rfr <num>  Refinement repetitions per level\n"
        "  -smh <lvl>  Accepted for compatibility (level hierarchies stay on the device)\n"
        "  -dtc        Accepted for compatibility (incidence sets are always built on the device)\n"
        "  -ipm        Greedily merge the initial partitions\n"
        "  -seed <n>   Seed for tie-breaks (same seed, same partition)\n"
        "  -v <lvl>    Verbosity 0..3\n"
        "  -h          Show this help message\n");
}

static void die(const char *m) {
    std::fprintf(stderr, "%s\n", m);
    std::exit(1);
}

int main(int argc, char **argv) {
    if (argc == 1) { help(); return 0; }
    std::string load, save, partf, cname;
    axc_params p;
    axc_params_default(&p, AXC_MODE_INCC);
    bool have_m = false, have_k = false, have_c = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto need = [&](int k, const char *m) { if (i + k >= argc) die(m); };
        if (a == "-h") { help(); return 0; }
        else if (a == "-r") { need(1, "Error: -r requires a file path"); load = argv[++i]; }
        else if (a == "-s") { need(1, "Error: -s requires a file path"); save = argv[++i]; }
        else if (a == "-p") { need(1, "Error: -p requires a file path"); partf = argv[++i]; }
        else if (a == "-c") { need(1, "Error: -c requires a config name"); cname = argv[++i]; have_c = true; }
        else if (a == "-m") {
            need(3, "Error: -m requires integer values for the three constraints");
            p.omega = (uint32_t)std::stoul(argv[++i]);
            p.delta = (uint32_t)std::stoul(argv[++i]);
            p.max_parts = (uint32_t)std::stoul(argv[++i]);
            have_m = true;
        } else if (a == "-k") {
            need(2, "Error: -k requires values for 'k' and 'eps'");
            p.k = (uint32_t)std::stoul(argv[++i]);
            p.eps = std::stof(argv[++i]);
            have_k = true;
        } else if (a == "-om") { need(1, "Error: -om requires a float value"); p.om = std::stof(argv[++i]); }
        else if (a == "-cnc") {
            need(1, "Error: -cnc requires a positive integer value");
            p.cnc = (uint32_t)std::stoul(argv[++i]);
            if (p.cnc == 0 || p.cnc > AXC_MAX_CANDIDATES) die("Error: -cnc must be between 1 and 16");
        } else if (a == "-rfr") { need(1, "Error: -rfr requires a positive integer value"); p.rfr = (uint32_t)std::stoul(argv[++i]); }
        else if (a == "-smh") { need(1, "Error: -smh requires a positive integer value"); p.smh = (uint32_t)std::stoul(argv[++i]); }
        else if (a == "-dtc") {}
        else if (a == "-ipm") { p.ipm = 1; }
        else if (a == "-seed") { need(1, "Error: -seed requires a value"); p.seed = std::stoull(argv[++i]); }
        else if (a == "-v") {
            need(1, "Error: -v requires a positive value between 0 and 3");
            p.verbose = std::stoi(argv[++i]);
            if (p.verbose < 0 || p.verbose > 3) die("Error: -v must be between 0 and 3 (extremes included)");
        } else {
            std::fprintf(stderr, "Unknown option: %s\n", a.c_str());
            return 1;
        }
    }
    if (load.empty()) die("Error: -r is required");
    axc_hgraph g;
    std::memset(&g, 0, sizeof g);
    std::printf("Loading hypergraph from: %s ...\n", load.c_str());
    int rc = axc_read_auto(load.c_str(), &g);
    if (rc) { std::fprintf(stderr, "Error loading file: %s\n", axc_strerror(rc)); return 1; }
    if (have_k) {
        p.mode = AXC_MODE_KWAY;
    } else if (have_m) {
        p.mode = AXC_MODE_INCC;
        if (!p.omega || !p.delta || !p.max_parts) die("Error: constraints must be positive integers");
    } else {
        if (!have_c) std::fprintf(stderr, "WARNING, no constraints provided (-c, -m, -k), using loihi64 !!\n");
        if (axc_params_preset(&p, have_c ? cname.c_str() : "loihi64")) {
            std::fprintf(stderr, "WARNING, constraints name (-c %s) not recognized, using loihi64 !!\n", cname.c_str());
            axc_params_preset(&p, "loihi64");
        }
    }
    const uint64_t P = g.e ? g.hedge_off[g.e] : 0;
    std::printf("Loaded hypergraph:\n  Nodes:      %u\n  Hyperedges: %u\n  Total pins: %llu\n", g.n, g.e,
                (unsigned long long)P);
    uint32_t omega = p.mode == AXC_MODE_KWAY ? axc_kway_omega(g.n, p.k, p.eps) : p.omega;
    std::printf("Using constraints:\n  Nodes per partition:         %u\n", omega);
    std::printf("  Inbound hedge per partition: %u\n", p.mode == AXC_MODE_KWAY ? 0x7FFFFFFFu : p.delta);
    std::printf("  Maximum partitions:          %u\n", p.mode == AXC_MODE_KWAY ? p.k : p.max_parts);
    std::printf("Using settings:\n  Candidates count:            %u\n  Refinement repetitions:      %u\n", p.cnc, p.rfr);

    axc_ctx *ctx = nullptr;
    rc = axc_create(0, 0, &ctx);
    if (rc) { std::fprintf(stderr, "CUDA setup failed: %s\n", axc_strerror(rc)); return 1; }
    std::vector<uint32_t> part(g.n ? g.n : 1);
    axc_stats st;
    auto t0 = std::chrono::high_resolution_clock::now();
    rc = axc_partition(ctx, &g, &p, part.data(), &st);
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rc) {
        std::fprintf(stderr, "partitioning failed: %s (%s)\n", axc_strerror(rc), axc_last_error(ctx));
        return 1;
    }
    const double host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::printf("Total device core execution time: %.3f ms\n", st.ms_core);
    std::printf("Total device execution time: %.3f ms\n", st.ms_device);
    std::printf("Total host execution time: %.3f ms\n", host_ms);
    if (!st.valid) {
        std::fprintf(stderr, "ERROR, invalid partitining !!\n");
        return 1;
    }
    axc_hgraph q;
    std::memset(&q, 0, sizeof q);
    rc = axc_quotient_hgraph_device(ctx, &g, part.data(), &q);
    if (rc) {
        std::fprintf(stderr, "quotient hypergraph failed: %s (%s)\n", axc_strerror(rc), axc_last_error(ctx));
        return 1;
    }
    const uint64_t qP = q.e ? q.hedge_off[q.e] : 0;
    std::printf("Partitioned hypergraph:\n");
    std::printf("  Nodes:         %u\n", st.num_parts);
    std::printf("  Hyperedges:    %u\n", q.e);
    std::printf("  Total pins:    %llu\n", (unsigned long long)qP);
    std::printf("  Cut-net:       %.3f\n", st.cutnet);
    std::printf("  Connectivity:  %.3f\n", st.connectivity);
    std::printf("  SOED:          %.3f\n", st.soed);
    if (!save.empty()) {
        rc = axc_write_hgraph(save.c_str(), &q);
        if (rc) { std::fprintf(stderr, "Error saving file: %s\n", axc_strerror(rc)); return 1; }
        std::printf("Partitioned hypergraph saved to %s\n", save.c_str());
    }
    if (!partf.empty()) {
        rc = axc_write_partition(partf.c_str(), part.data(), g.n);
        if (rc) { std::fprintf(stderr, "Error saving file: %s\n", axc_strerror(rc)); return 1; }
        std::printf("Partitioning saved to %s\n", partf.c_str());
    }
    axc_free_hgraph(&q);
    axc_free_hgraph(&g);
    axc_destroy(ctx);
    return 0;
}
