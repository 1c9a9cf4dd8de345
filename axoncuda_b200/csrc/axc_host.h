// Host-only helpers shared by the readers, writers, generators and the driver.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/axc.h"

namespace axc {

// Owning storage behind an axc_hgraph returned by axc_read_* / axc_gen_* / axc_quotient_hgraph.
struct HostGraph {
    uint32_t n = 0;
    std::vector<uint64_t> off;   // e+1
    std::vector<uint32_t> pins;  // sources first per hedge
    std::vector<uint32_t> nsrc;  // e
    std::vector<float> w;        // e
};

void publish(HostGraph *hg, axc_hgraph *out);

// The quotient hypergraph from per-hyperedge partition lists: qcnt[h] kept partitions of
// hyperedge h (0: the hyperedge vanishes), the first qsrc[h] of them its sources, all in qpins
// in hyperedge order. Identical (sources, destinations) pairs merge with their weights summed in
// hyperedge order (1 each when w is null); the result lists them in ascending lexicographic
// order of (sources, destinations) over K nodes.
HostGraph *quotient_merge(uint32_t K, uint32_t e, const std::vector<uint32_t> &qcnt, const std::vector<uint32_t> &qsrc,
                          const std::vector<uint32_t> &qpins, const float *w);

// Lanes of the batching / serving executor (driver.cu): a stream, status word and scan state of
// their own; each job runs in a fresh device arena of the size the executor grants it.
struct Lane;
int ctx_device(axc_ctx *ctx);
size_t device_free_bytes(int device);
Lane *lane_create(int device, int *rc);
void lane_destroy(Lane *l);
int lane_partition(Lane *l, size_t arena_bytes, const axc_hgraph *g, const axc_params *p, uint32_t *out_part,
                   axc_stats *stats, std::string *err);
// tile and table sizes the lane's next jobs use (axc_tune_set's rate.try_slots, rate.mid_slots,
// cascade.block_movers)
void lane_tune(Lane *l, uint32_t rate_try, uint32_t rate_mid, uint32_t cascade_movers);
// the context's own values of the same three, their setter (AXC_ENOTFOUND for another key), and
// the range check of the power-of-two sizes
void ctx_tune_get(axc_ctx *ctx, uint32_t out[3]);
int ctx_tune_set(axc_ctx *ctx, const std::string &key, uint64_t value);
bool tune_pow2_in(uint64_t v, uint64_t lo, uint64_t hi);

// splitmix64: seeds independent xoshiro streams per (seed, index) so generators are
// deterministic under any thread count.
inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {  // xoshiro256**
    uint64_t s[4];
    explicit Rng(uint64_t seed, uint64_t stream = 0) {
        uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull + 0x8BB84B93962EACC9ull);
        for (auto &v : s) v = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, m) (Lemire's multiply-shift; m < 2^32)
    uint32_t below(uint32_t m) { return (uint32_t)(((next() >> 32) * (uint64_t)m) >> 32); }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace axc
