// Internal host API between the kernel files and the driver. Every function enqueues work on the
// context's stream; functions that return a size synchronise once to read it.
#pragma once
#include "common.cuh"

namespace axc {

// One level of the hierarchy, all arrays in device memory.
struct DLevel {
    u32 n = 0, e = 0;
    u64 P = 0;
    u64 *off = nullptr;   // [e+1]
    u32 *pins = nullptr;  // [P]
    u32 *nsrc = nullptr;  // [e]
    u64 *toff = nullptr;  // [n+1]
    u32 *touch = nullptr; // [P]
    u32 *nin = nullptr;   // [n]
    u32 *nsize = nullptr; // [n]
    u32 *groups = nullptr;  // [n] map into the next level (when built)
    u32 ngroups = 0;
    size_t arena_mark = 0;  // arena position before this level's arrays
};

// construct.cu
void setup_construct_kernels();
void compute_wfx(Ctx &c, const float *d_w, u32 *d_wfx, u32 e);
u64 hedge_unique(Ctx &c, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc, const u32 *groups,
                 bool dst_wins, u64 *new_off, u32 *new_pins, u32 *new_nsrc, u64 pins_in);
void build_touching(Ctx &c, u32 n, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc, u64 P,
                    u64 *toff, u32 *touch, u32 *nin);
void group_sizes(Ctx &c, u32 n, const u32 *groups, const u32 *nsize, u32 *gsize, u32 ng);
// rejects (AXC_EINVAL) offsets that decrease, source counts beyond their hyperedge, pins >= n
void check_input(Ctx &c, u32 n, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc);

// coarsen.cu
void setup_coarsen_kernels(Ctx &c);
void rating(Ctx &c, const DLevel &L, const u32 *wfx, u32 omega, u32 delta, u32 cnc, u32 *pairs,
            u32 *scores, u64 *pin_visits);
u32 matching(Ctx &c, u32 n, u32 cnc, const u32 *pairs, const u32 *scores, const u32 *nsize, const u32 *nin, u32 omega,
             u32 delta, u32 rounds, u32 *groups);
// greedy packing of the groups of level L (sources/postprocess.cu:16-245); rewrites groups and
// returns the new group count
u32 greedy_merge_groups(Ctx &c, u32 n, const u32 *nsize, const u32 *nin, u32 *groups, u32 ng,
                        u32 omega, u32 delta);

// refine.cu
struct RefineParams {
    u32 K, omega, delta;
    bool encourage;
    u32 rounds;
    u64 seed;
    // copies > 1: the level is that many disjoint copies of copy_n nodes each (the k-way
    // multi-start); moves are ranked copy by copy and every copy takes its own best prefix
    u32 copies = 1, copy_n = 0;
};
void setup_refine_kernels(Ctx &c);
// all refinement rounds of one level; part[n] is updated in place; returns rounds applied
u32 refine_level(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, u32 *part);
// one round's proposals only (parity stage)
void refine_gains_only(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, const u32 *part,
                       u32 discount, u32 round, u32 *target, i64 *gain);
// per-hyperedge partition census; returns arrays in the arena (caller releases)
struct Census {
    u64 *beg = nullptr;   // [e+1]
    u32 *part = nullptr;  // [P]
    u32 *cnt = nullptr;   // [P]
    u32 *dcnt = nullptr;  // [P]
    u32 *lam = nullptr;   // [e]
    // Optional, for the refinement's partition-indexed gains (K <= 256): the census also adds to
    // save[v] what each node saves by leaving its partition (needs wfx and encourage), and
    // census_masks writes per-hyperedge bitmasks of the partitions present / with destinations.
    i64 *save = nullptr;  // [n]
    const u32 *wfx = nullptr;
    int encourage = 0;
    u32 *mask = nullptr, *dmask = nullptr;  // [e * mw]
    u32 mw = 0;
};
Census build_census(Ctx &c, const DLevel &L, const u32 *part);
void part_sizes(Ctx &c, u32 n, const u32 *part, const u32 *nsize, u64 *psize, u32 K);
void part_inbound(Ctx &c, const DLevel &L, const Census &cs, u64 *pinb, u32 K);

// initpart.cu
void kway_initial(Ctx &c, const DLevel &L, u32 k, u32 *part);
// the k-way multi-start on the coarsest level (include/axc.h AXC_KWAY_TRIES): refines part[n]
// from its BFS start and random ones, keeps the best; false when fewer than 2 copies fit
bool kway_multistart(Ctx &c, const DLevel &L, const u32 *wfx, u32 k, u32 omega, u64 seed, u32 *part);

// post.cu
u32 greedy_pack(Ctx &c, const u64 *ss, const u64 *si, u32 m, u64 omega, u64 delta, u32 *packid);
void uncoarsen(Ctx &c, u32 n, const u32 *groups, const u32 *coarse_part, u32 *part);
// INCC merge of partitions smaller than 16 (sources/postprocess.cu:247-420)
void merge_small_partitions(Ctx &c, const DLevel &L, u32 *part, u32 K, u32 omega, u32 delta);
// zero-base partition ids in order of old id; returns K'
u32 zero_base(Ctx &c, u32 n, u32 *part, u32 K);
// metrics over a level graph (any graph as given): fills the fx fields of stats
// quotient.cu: the distinct source / destination-only partitions of every hyperedge (device
// input, host output; see axc_quotient_hgraph_device)
void quotient_extract(Ctx &c, u32 e, u64 P, const u64 *off, const u32 *pins, const u32 *nsrc, const u32 *part, u32 K,
                      std::vector<u32> &qcnt, std::vector<u32> &qsrc, std::vector<u32> &qpins);
void evaluate(Ctx &c, const DLevel &L, const u32 *wfx, const u32 *part, u32 omega, u32 delta,
              u32 max_parts, axc_stats *st);

}  // namespace axc
