/*
 * oracle.h — CPU restatement of the partitioner's stages. TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library,
 * and only as the checker (or as the timed CPU port). The product path never calls it.
 *
 * Each function states the reference code it restates (file:line in EMJzero/AxonCUDA) and,
 * where this build deliberately differs from the reference, the rule it follows instead.
 * All arithmetic is integer; hyperedge weights enter as w_fx = floor(w * 2^18).
 */
#ifndef AXC_ORACLE_H
#define AXC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Readers: includes/hgraph.hpp:707-743 (.snn), 805-854 (.axh), 936-1013 (.hgr).
 * Two-call protocol: call with NULL outputs to get sizes, then with buffers. */
int or_read(const char *path, uint32_t *n, uint32_t *e, uint64_t *p, uint64_t *off, uint32_t *pins,
            uint32_t *nsrc, float *w);

/* Fixed-point weight: floor(w * 2^18) clamped to [0, 2^32-1] (headers/defines.cuh:24). */
uint32_t or_wfx(float w);

/* Rule-2 dedupe, includes/hgraph.hpp:518-581: keep first occurrences in flat order (sources
 * first). Outputs sized like the input; returns the kept pin count. */
uint64_t or_dedupe(uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
                   uint64_t *out_off, uint32_t *out_pins, uint32_t *out_nsrc);

/* Incidence CSR, sources/construction.cu:17-62: per node inbound hyperedges ascending, then
 * outbound ascending; inbound[v] = number of inbound ones. */
void or_touching(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                 const uint32_t *nsrc, uint64_t *toff, uint32_t *touch, uint32_t *inbound);

/* Candidate rating, kernels/coarsening.cu:76-212 (see oracle.cpp for the exact rule). */
void or_rating(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
               const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
               const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
               uint32_t omega, uint32_t delta, uint32_t cnc, uint32_t *pairs, uint32_t *scores);
/* The same with the hyperedge length limit given: hyperedges of more than max_len pins take no
 * part (or_rating uses AXC_RATE_MAX_LEN; UINT64_MAX rates through every hyperedge, as the
 * reference does). */
void or_rating_len(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                   const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
                   const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
                   uint32_t omega, uint32_t delta, uint32_t cnc, uint64_t max_len, uint32_t *pairs,
                   uint32_t *scores);

/* Matching + orphan pairing + relabel (this build's deterministic propose/accept matching;
 * orphans as sources/chaining.cu:260-329). Returns the number of groups. */
uint32_t or_matching(uint32_t n, uint32_t cnc, const uint32_t *pairs, const uint32_t *scores,
                     const uint32_t *node_size, const uint32_t *inbound, uint32_t omega, uint32_t delta,
                     uint32_t rounds, uint32_t *groups);

/* Contraction, kernels/construction.cu:304-489. Returns the coarse pin count. */
uint64_t or_contract(uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
                     const uint32_t *groups, uint64_t *out_off, uint32_t *out_pins,
                     uint32_t *out_nsrc);

/* One refinement round's proposals (kernels/refinement.cu:82-209, integer gains). */
void or_gains(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
              const uint32_t *nsrc, const uint32_t *wfx, const uint64_t *toff,
              const uint32_t *touch, const uint32_t *inbound, const uint32_t *node_size,
              const uint32_t *part, uint32_t num_parts, uint32_t omega, uint32_t delta,
              int encourage, uint32_t discount, uint32_t round, uint64_t seed, uint32_t *target,
              int64_t *gain);

/* Metrics over a hypergraph as given (grading/grade.cpp:298-309 via includes/hgraph.hpp:214-376,
 * sources/constr.cpp:90-147), all exact in fixed point.
 * out[0]=connectivity_fx out[1]=cutnet_fx out[2]=soed_fx out[3]=num_parts out[4]=max_size
 * out[5]=max_inbound out[6]=valid(0/1) out[7]=ids_dense(0/1). */
// refine_level (sources/refinement.cu:82-545) on a given partition, updated in place
void or_refine(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins, const uint32_t *nsrc,
               const uint32_t *wfx, const uint64_t *toff, const uint32_t *touch, const uint32_t *inbound,
               const uint32_t *node_size, uint32_t *part, uint32_t num_parts, uint32_t omega, uint32_t delta,
               int encourage, uint32_t rounds, uint64_t seed);
void or_evaluate(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                 const uint32_t *nsrc, const float *w, const uint32_t *part, uint32_t omega,
                 uint32_t delta, uint32_t max_parts, int64_t *out);

/* The whole partitioner, single-threaded (the CPU port timed by bench.py).
 * mode 0 = INCC (omega, delta, max_parts, ipm), 1 = KWAY (k, eps). Returns the number of
 * partitions; part[n]. stats[0]=levels stats[1]=pins after dedupe. */
uint32_t or_partition(uint32_t n, uint32_t e, const uint64_t *off, const uint32_t *pins,
                      const uint32_t *nsrc, const float *w, int mode, uint32_t omega,
                      uint32_t delta, uint32_t max_parts, uint32_t k, float eps, uint32_t cnc,
                      uint32_t rfr, int ipm, uint64_t seed, uint32_t *part, uint64_t *stats);

#ifdef __cplusplus
}
#endif
#endif
