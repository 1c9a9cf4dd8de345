// axc_gen — writes the seeded synthetic workloads to .snn / .hgr / .axh files.
//   axc_gen snn-layered <out> <seed>   8 layers x 512, fan-out 64 from the next layer
//   axc_gen circuit <out> <seed>       200,000 nodes, 220,000 nets, s^-2.5 on [2,64], 90% within +-2%
//   axc_gen snn-large <out> <seed>     20 layers x 50,000, fan-out lognormal(256, 0.8) <= 2048, 70% next layer
//   axc_gen snn-mid <out> <seed>       the same at 20 layers x 5,000
//   axc_gen snn <out> <layers> <width> <fanout> <sigma> <cap> <p_next> <seed>
//   axc_gen circ <out> <n> <e> <smin> <smax> <alpha> <p_local> <local_frac> <seed>
// Built from the generator and writer sources alone (no libaxc.so, no CUDA), so a process that
// only needs the input files loads none of the library.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/axc.h"

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: axc_gen <snn-layered|circuit|snn-large|snn-mid|snn|circ> <out> ...\n");
        return 2;
    }
    std::string kind = argv[1];
    const char *out = argv[2];
    axc_hgraph g;
    std::memset(&g, 0, sizeof g);
    int rc;
    auto A = [&](int i) { return i < argc ? argv[i] : "0"; };
    if (kind == "snn-layered") rc = axc_gen_snn(8, 512, 64, 0.0, 0, 1.0, std::strtoull(A(3), 0, 10), &g);
    else if (kind == "circuit") rc = axc_gen_circuit(200000, 220000, 2, 64, 2.5, 0.9, 0.02, std::strtoull(A(3), 0, 10), &g);
    else if (kind == "snn-large") rc = axc_gen_snn(20, 50000, 256, 0.8, 2048, 0.7, std::strtoull(A(3), 0, 10), &g);
    else if (kind == "snn-mid") rc = axc_gen_snn(20, 5000, 256, 0.8, 2048, 0.7, std::strtoull(A(3), 0, 10), &g);
    else if (kind == "snn")
        rc = axc_gen_snn(std::atoi(A(3)), std::atoi(A(4)), std::atof(A(5)), std::atof(A(6)), std::atoi(A(7)),
                         std::atof(A(8)), std::strtoull(A(9), 0, 10), &g);
    else if (kind == "circ")
        rc = axc_gen_circuit(std::atoi(A(3)), std::atoi(A(4)), std::atoi(A(5)), std::atoi(A(6)), std::atof(A(7)),
                             std::atof(A(8)), std::atof(A(9)), std::strtoull(A(10), 0, 10), &g);
    else {
        std::fprintf(stderr, "unknown kind %s\n", kind.c_str());
        return 2;
    }
    if (rc) { std::fprintf(stderr, "generation failed: axc status %d\n", rc); return 1; }
    rc = axc_write_hgraph(out, &g);
    if (rc) { std::fprintf(stderr, "write failed: axc status %d\n", rc); return 1; }
    std::printf("%s: %u nodes, %u hyperedges, %llu pins\n", out, g.n, g.e,
                (unsigned long long)(g.e ? g.hedge_off[g.e] : 0));
    axc_free_hgraph(&g);
    return 0;
}
