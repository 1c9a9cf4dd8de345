/*
 * axc.h — C ABI of the B200-native multilevel hypergraph partitioner.
 *
 * The reference (AxonCUDA) exposes no library: its surface is the `hgraph_gpu.exe` process
 * (sources/main.cu:38-940, flags in sources/runconfig.cpp:25-46), the .hgr/.snn/.axh readers
 * (includes/hgraph.hpp:707-1013), and the per-node partition file scored by grading/grade.cpp.
 * Every entry point below replaces one piece of that surface; the comment on each names the
 * reference code it stands in for. The drop-in CLI (`axc_hgraph_gpu`) is a thin C++ client of
 * this header.
 *
 * Conventions
 *  - Every call returns an axc_status; nothing exits or aborts (the reference calls exit()/abort(),
 *    headers/utils.cuh:16-22, sources/runconfig.cpp:74-127).
 *  - Plain pointers and sizes only. Unless a parameter says "device", buffers are host memory
 *    owned by the caller. The context owns all device memory.
 *  - Node ids are uint32 and 0-based; pins of one hyperedge are stored sources first
 *    (includes/hgraph.hpp:31-77). Offsets are uint64.
 *  - Hyperedge weights are float in files and in axc_hgraph; on the device they become exact
 *    fixed point w_fx = floor(w * 2^18) (the reference's FIXED_POINT_SCALE, headers/defines.cuh:24),
 *    and every gain, cut and inbound count is integer arithmetic on those.
 *  - Results are deterministic for a given input, parameter set and seed.
 */
#ifndef AXC_H
#define AXC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    AXC_OK = 0,
    AXC_EINVAL = 1,        /* bad argument or parameter */
    AXC_ENOMEM = 2,        /* device arena or host allocation exhausted */
    AXC_ECUDA = 3,         /* a CUDA runtime call failed */
    AXC_EIO = 4,           /* file cannot be opened / read / written */
    AXC_EFORMAT = 5,       /* malformed input file */
    AXC_EINFEASIBLE = 6,   /* the result violates the constraints (reference: "ERROR, invalid partitining") */
    AXC_ETIMEDOUT = 7,     /* a bounded device wait or a poll timed out */
    AXC_ENOTFOUND = 8,     /* unknown job id */
    AXC_EBUSY = 9,         /* admission refused (memory budget) */
    AXC_EINTERNAL = 10,    /* device-side invariant check failed (status word set by a kernel) */
    AXC_EOVERFLOW = 11,    /* a size exceeds the documented limit of the call */
    AXC_ECANCELED = 12     /* the context shut down before the submitted job ran */
} axc_status;

typedef enum { AXC_MODE_INCC = 0, AXC_MODE_KWAY = 1 } axc_mode;

/* Hypergraph in the reference's HyperGraph layout (includes/hgraph.hpp:130-168):
 * hedge i owns pins[hedge_off[i] .. hedge_off[i+1]); the first src_count[i] are sources. */
typedef struct {
    uint32_t n;                 /* nodes */
    uint32_t e;                 /* hyperedges */
    const uint64_t *hedge_off;  /* [e+1] */
    const uint32_t *pins;       /* [hedge_off[e]] */
    const uint32_t *src_count;  /* [e] */
    const float *hedge_w;       /* [e], NULL means every weight is 1 */
    void *_owner;               /* non-NULL when the arrays belong to the library (axc_read_*, axc_gen_*) */
} axc_hgraph;

/* Run parameters: the runconfig of includes/runconfig.hpp:26-45 plus the constraint triple of
 * includes/constr.hpp:14-19. */
typedef struct {
    int mode;              /* axc_mode */
    uint32_t omega;        /* INCC: max nodes per partition (-m 1st) */
    uint32_t delta;        /* INCC: max distinct inbound hyperedges per partition (-m 2nd) */
    uint32_t max_parts;    /* INCC: max number of partitions (-m 3rd) */
    uint32_t k;            /* KWAY: number of parts (-k) */
    float eps;             /* KWAY: imbalance (-k) */
    uint32_t cnc;          /* candidates per node (-cnc), <= AXC_MAX_CANDIDATES */
    uint32_t rfr;          /* refinement rounds per level (-rfr) */
    uint32_t smh;          /* -smh: accepted for CLI compatibility; level hierarchies stay resident */
    int ipm;               /* -ipm: greedily merge the coarsest groups (INCC) */
    float om;              /* -om: accepted for CLI compatibility; no oversized buffers are used */
    uint64_t seed;         /* tie-break / noise seed; same seed => same partition */
    int verbose;           /* -v 0..3 */
} axc_params;

#define AXC_MAX_CANDIDATES 16u   /* headers/defines.cuh:49 */
#define AXC_FIXED_POINT_SCALE 262144u
/* Hyperedges with more pins than this take no part in the coarsening rating (they still count
 * everywhere else). The reference rates through every hyperedge (kernels/coarsening.cu:76-202);
 * its pair visits grow as |e|^2, which at 3e8 pins is what exhausts its neighbour lists. */
#define AXC_RATE_MAX_LEN 128u
/* Refinement with more than AXC_SPARSE_GAIN_K partitions bounds each node's gain work. A node's
 * candidate targets come from a sample: the longest prefix of its incidences (inbound hyperedges
 * first, each part ascending) whose hyperedges hold at most AXC_SPARSE_GAIN_SAMPLE (partition,
 * hyperedge) census entries in all. When that prefix is the whole node the gains are the exact
 * ones over every adjacent partition. Otherwise the AXC_SPARSE_GAIN_CANDIDATES partitions with the
 * largest sampled connectivity that are not already ruled out by the size limit or by an upper
 * bound of their shared inbound hyperedges are evaluated exactly, and the best feasible one is the
 * node's target. The reference's dense gain table needs E x K words, which at K near 1e5 does not
 * fit; its sparse path bounds the work differently (sources/refinement.cu:587-1378). */
#define AXC_SPARSE_GAIN_K 4096u
#define AXC_SPARSE_GAIN_SAMPLE 4096u
#define AXC_SPARSE_GAIN_CANDIDATES 8u
/* k-way refinement orders its moves in pairs: the i-th best move from partition a to b next to the
 * i-th best from b to a, pairs ranked by their summed gain, so that balanced prefixes exist when
 * every partition is near its size limit (the reference's chaining, sources/chaining.cu:19-254,
 * serves the same purpose). Up to this many partitions; above it moves are ranked by gain. */
#define AXC_PAIR_RANK_MAX_K 32768u
/* k-way initial partition: a multi-start on the coarsest level, in place of the reference's
 * Mt-KaHyPar call (sources/init_part.cu:733-953) and in the manner of its dormant GPU routine
 * (32 random starts with refinement, sources/init_part.cu:186-727). Up to AXC_KWAY_TRIES starts
 * (the BFS chunks and random balanced ones), as many as fit AXC_KWAY_TRY_PINS pins in all, are
 * refined together for AXC_KWAY_TRY_ROUNDS rounds as disjoint copies of the level; the one of
 * least connectivity is kept. With fewer than 2 copies the BFS chunks are refined alone. */
#define AXC_KWAY_TRIES 16u
#define AXC_KWAY_TRY_ROUNDS 32u
#define AXC_KWAY_TRY_PINS 8388608ull

typedef struct {
    uint32_t num_parts;        /* K' after zero-basing */
    uint32_t levels;           /* coarsening levels built */
    uint64_t pins;             /* pins after rule-2 deduplication (sources included) */
    int64_t connectivity_fx;   /* sum_e w_fx(e) * (lambda_e - 1), exact */
    int64_t cutnet_fx;         /* sum_e w_fx(e) * [lambda_e > 1] */
    int64_t soed_fx;           /* sum_e w_fx(e) * (lambda_e - 1) * |e| over the input pins */
    double connectivity;       /* connectivity_fx / 2^18 */
    double cutnet;
    double soed;
    uint32_t max_part_size;    /* largest partition (nodes) */
    uint32_t max_part_inbound; /* largest distinct-inbound count over partitions */
    int valid;                 /* 1 iff checkPartitionValidity would accept (sources/constr.cpp:90-147) */
    double ms_device;          /* device time from upload start to partition download end */
    double ms_core;            /* device time of the multilevel core (after construction) */
    uint32_t kernel_launches;  /* kernels this call launched */
    uint64_t level_pins[64];   /* pins per level (for the traffic model) */
    uint32_t level_nodes[64];
    uint32_t refine_rounds[64];
    uint64_t rating_pin_visits;  /* sum over rated nodes of incident pins visited */
    uint64_t device_bytes_peak;  /* arena high-water mark of this call (bytes) */
    double ms_queued;            /* submitted jobs: host time from submit to start on a lane */
    double ms_run;               /* submitted jobs: host time from start to finish */
} axc_stats;

typedef struct axc_ctx axc_ctx;

/* ---- context --------------------------------------------------------------------------------
 * One per device; owns a device arena of `arena_bytes` (0 = a default sized from free memory),
 * one stream and the kernels' status word. Replaces the per-step cudaMalloc/cudaFree of
 * sources/main.cu:196-222 and the host wrappers of sources/construction.cu, coarsening.cu,
 * refinement.cu and postprocess.cu. */
int axc_create(int device, size_t arena_bytes, axc_ctx **out);
void axc_destroy(axc_ctx *ctx);
const char *axc_strerror(int status);
const char *axc_last_error(axc_ctx *ctx);   /* human-readable detail of the last failure */

/* ---- kernel timer (measurement; no reference counterpart: the reference times whole phases
 * with host clocks, sources/main.cu:151-910) ------------------------------------------------------
 * While a kernel name is set, every launch of that kernel on the context stream is bracketed by a
 * pair of CUDA events, and launch sites with a byte model add the launch's algorithmic bytes:
 * k_rate_block and the gain kernels from host-side sizes; k_cascade_warp and k_census_direct_warp
 * counted by the kernels themselves (they depend on each round's movers and census). axc_profile_read synchronizes the stream, returns
 * the totals since the kernel was set and resets them. kernel = NULL switches the timer off. */
typedef struct {
    uint32_t launches;  /* launches of the kernel seen */
    double ms_total;    /* sum of their event-timed durations */
    uint64_t bytes;     /* sum of their algorithmic bytes (0 if the kernel has no byte model) */
} axc_kernel_timing;
int axc_profile_kernel(axc_ctx *ctx, const char *kernel);
int axc_profile_read(axc_ctx *ctx, axc_kernel_timing *out);

/* Defaults of sources/runconfig.cpp:48-70 (cnc=16, rfr=16, smh=2, om=1.5) with the given mode. */
void axc_params_default(axc_params *p, int mode);
/* Preset constraints of sources/constr.cpp:195-229: "loihi64", "loihi84", "loihi1024", "truenorth". */
int axc_params_preset(axc_params *p, const char *name);
/* KWAY constraint derivation of sources/runconfig.cpp:186-194: omega = ceil((1+eps)*n/k). */
uint32_t axc_kway_omega(uint32_t n, uint32_t k, float eps);

/* ---- the hot path -----------------------------------------------------------------------------
 * Partition a host hypergraph end to end on the context's device: upload, rule-2 dedupe,
 * incidence CSR, multilevel coarsening, initial partition, uncoarsening with refinement,
 * INCC small-partition merge, zero-basing, download. Replaces main() from the upload at
 * sources/main.cu:196 to the partition download at sources/main.cu:833-834 (the span the
 * reference times as "Total host execution time", sources/main.cu:151-910).
 * out_part: [g->n] host buffer. stats may be NULL. */
int axc_partition(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, uint32_t *out_part,
                  axc_stats *stats);

/* Same, with the hypergraph already resident in device memory (arrays are device pointers;
 * hedge_w may be NULL) and the partition written to device memory d_out_part[n]. */
int axc_partition_device(axc_ctx *ctx, const axc_hgraph *d_g, const axc_params *p,
                         uint32_t *d_out_part, axc_stats *stats);

/* ---- validity and metrics on the device --------------------------------------------------------
 * Replaces Constraints::checkPartitionValidity (sources/constr.cpp:90-147) and the metrics of
 * includes/hgraph.hpp:214-280 as printed by sources/main.cu:917-928 and grading/grade.cpp:298-309.
 * `part` is host memory [g->n]. The hypergraph is used as given (no dedupe), like grade.cpp. */
int axc_evaluate(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, const uint32_t *part,
                 axc_stats *stats);

/* ---- readers / writers (host) -------------------------------------------------------------------
 * HyperGraph::loadhMETIS/loadSNN/loadAXH (includes/hgraph.hpp:936-1013, 707-743, 805-854) and
 * loadHgraph's dispatch by extension (sources/runconfig.cpp:153-184). */
int axc_read_hgr(const char *path, axc_hgraph *out);
int axc_read_snn(const char *path, axc_hgraph *out);
int axc_read_axh(const char *path, axc_hgraph *out);
int axc_read_auto(const char *path, axc_hgraph *out);
void axc_free_hgraph(axc_hgraph *g);
/* saveSNN / saveAXH / savehMETIS (includes/hgraph.hpp:746-774, 856-883, 1016-1051). */
int axc_write_hgraph(const char *path, const axc_hgraph *g);
/* HyperGraph::savePartitioning (includes/hgraph.hpp:1054-1059): one decimal id per line. */
int axc_write_partition(const char *path, const uint32_t *part, uint32_t n);
/* HyperGraph::loadPartitioning (includes/hgraph.hpp:1062-1083). out: [n]. */
int axc_read_partition(const char *path, uint32_t n, uint32_t *out);
/* getPartitionsHypergraph(part, 2, squish=true) (includes/hgraph.hpp:286-376): the quotient
 * hypergraph written by `-s`; identical (source set, destination set) hyperedges are merged. */
int axc_quotient_hgraph(const axc_hgraph *g, const uint32_t *part, axc_hgraph *out);
/* The same quotient hypergraph with the per-hyperedge work on the context's GPU: one radix sort
 * of (hyperedge, side, partition) keys over all pins; only the distinct partitions come back to
 * the host, which merges identical pairs. The output equals axc_quotient_hgraph's. Partition ids
 * must be below 2^31 and the pins fewer than 2^32 (else AXC_EOVERFLOW). Free `out` with
 * axc_free_hgraph. */
int axc_quotient_hgraph_device(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, axc_hgraph *out);

/* ---- synthetic inputs (seeded; stand-ins for the public SNN / ISPD suites) -----------------------
 * Layered SNN: `layers` x `width` neurons; every neuron of layers 0..layers-2 owns one hyperedge
 * (source = itself). Fan-out: fixed `fanout` when sigma <= 0, else lognormal(median=fanout, sigma)
 * capped at `cap`. Each destination comes from the next layer with probability p_next, else
 * uniformly from any later layer; drawn without replacement. Weights 1. */
int axc_gen_snn(uint32_t layers, uint32_t width, double fanout, double sigma, uint32_t cap,
                double p_next, uint64_t seed, axc_hgraph *out);
/* Circuit-style netlist: n nodes, e nets, net sizes ~ s^-alpha on [smin, smax]; each pin is,
 * with probability p_local, uniform within +-local_frac*n of a random anchor, else uniform;
 * pins of one net are distinct. No sources (hMETIS nets). Weights 1. */
int axc_gen_circuit(uint32_t n, uint32_t e, uint32_t smin, uint32_t smax, double alpha,
                    double p_local, double local_frac, uint64_t seed, axc_hgraph *out);

/* ---- batching and serving -------------------------------------------------------------------------
 * Many independent jobs on one device, continuously batched. There is no reference counterpart:
 * the reference partitions exactly one hypergraph per process (sources/main.cu:38).
 * - The context runs `lanes` workers, each with its own stream, status word, scan state and host
 *   thread, next to the context's own arena and stream.
 * - A job takes a device arena of its estimated size from the stream-ordered allocator on its
 *   lane's stream, and keeps its whole level hierarchy there until it finishes.
 * - Admission: a queued job starts when a lane is free and its estimate fits in `device_budget`
 *   minus what running jobs hold. Smaller jobs may start ahead of a larger one that does not fit
 *   yet. A job larger than the whole budget runs alone.
 * - A job that runs out of its arena is requeued once with twice the estimate.
 * - Concurrent jobs overlap on the device; each result equals the same job run alone.
 * Call axc_serve_configure before the first submit; without it there is 1 lane and a budget of
 * half the free device memory at the first submit. */
int axc_serve_configure(axc_ctx *ctx, uint32_t lanes, size_t device_budget);
int axc_submit(axc_ctx *ctx, const axc_hgraph *g, const axc_params *p, uint64_t *job_id);
/* Tile and table sizes and executor settings (no reference counterpart: the reference's are
 * compile-time constants, headers/defines.cuh). None of them changes a result, only speed; the
 * autotuner axoncuda_b200/tune.py picks them per job-size class. Keys:
 *   rate.try_slots, rate.mid_slots  the block rating's first-try and second-try hash tables (slots, a
 *                                   power of two in [64, 16384]; defaults 2048 and 8192)
 *   cascade.block_movers            movers the cascade's shared-memory block kernel keeps (0 = its
 *                                   default of 2048, else a power of two in [128, 2048])
 *   serve.exclusive_pins            submitted jobs of at least this many pins run alone (0 = none;
 *                                   default 1,000,000)
 *   class.<i>.min_pins, class.<i>.rate.try_slots, class.<i>.rate.mid_slots,
 *   class.<i>.cascade.block_movers  for submitted jobs: size class i (0..7) covers jobs of at least
 *                                   min_pins pins (the largest such class applies) and sets their
 *                                   sizes; jobs below every class use the context's own.
 * The first three apply to the context's own calls at once; serve.* and class.* must come before
 * the first submit (AXC_EBUSY after it). Unknown keys give AXC_ENOTFOUND, bad values AXC_EINVAL. */
int axc_tune_set(axc_ctx *ctx, const char *key, uint64_t value);
/* Wait up to timeout_ms (<0: forever) for a job; copies its partition into out_part[n]. A job
 * still queued when the context is destroyed is answered with AXC_ECANCELED. */
int axc_poll(axc_ctx *ctx, uint64_t job_id, uint32_t *out_part, axc_stats *stats, int timeout_ms);
/* Partition `count` jobs through the same lanes (submit all, then wait for all). out_parts[i]
 * points at a host buffer of g[i].n entries; stats may be NULL. Returns the first failing status. */
int axc_partition_batch(axc_ctx *ctx, uint32_t count, const axc_hgraph *g, const axc_params *p,
                        uint32_t *const *out_parts, axc_stats *stats);

/* ---- stage entry points (host buffers in and out; for parity tests against the oracle) -----------
 * Each runs exactly one stage of the device pipeline on the given level graph. */

/* Rule-2 dedupe (includes/hgraph.hpp:518-581, rule 2: a destination equal to a source is dropped)
 * followed by the per-node incidence CSR with inbound hyperedges first, each part ascending
 * (sources/construction.cu:17-62, -dtc path kernels/construction.cu:9-84).
 * out_hedge_off[e+1], out_pins[P], out_src_count[e]; out_touch_off[n+1], out_touch[P],
 * out_inbound[n]. *out_pins_after receives the deduplicated pin count. */
int axc_stage_construct(axc_ctx *ctx, const axc_hgraph *g, uint64_t *out_hedge_off,
                        uint32_t *out_pins, uint32_t *out_src_count, uint64_t *out_touch_off,
                        uint32_t *out_touch, uint32_t *out_inbound, uint64_t *out_pins_after);

/* Candidate rating of kernels/coarsening.cu:10-213 on an already-deduplicated level graph with
 * node sizes `node_size[n]`: top-`cnc` neighbors by (score desc, id desc), score = symmetric noise
 * + sum over shared hyperedges of floor(w_fx/|e|); pairs violating omega or delta are dropped.
 * out_pairs[n*cnc] (UINT32_MAX = none), out_scores[n*cnc]. */
int axc_stage_rating(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *node_size, uint32_t omega,
                     uint32_t delta, uint32_t cnc, uint64_t seed, uint32_t *out_pairs,
                     uint32_t *out_scores);

/* Matching over candidate lists plus orphan pairing (sources/coarsening.cu:70-210,
 * sources/chaining.cu:260-329): out_groups[n] zero-based group ids ordered by their smallest
 * member; *out_num_groups. */
int axc_stage_matching(axc_ctx *ctx, uint32_t n, uint32_t cnc, const uint32_t *pairs,
                       const uint32_t *scores, const uint32_t *node_size, const uint32_t *inbound,
                       uint32_t omega, uint32_t delta, uint32_t *out_groups,
                       uint32_t *out_num_groups);

/* Contraction of hyperedges by a group map (kernels/construction.cu:304-489): coarse pins are the
 * distinct groups, destinations win over sources, each part ascending, hyperedge count unchanged.
 * out_hedge_off[e+1], out_pins[<= P], out_src_count[e]; *out_pins_after. */
int axc_stage_contract(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *groups,
                       uint32_t num_groups, uint64_t *out_hedge_off, uint32_t *out_pins,
                       uint32_t *out_src_count, uint64_t *out_pins_after);

/* Move gains of one refinement round for a given partition (kernels/refinement.cu:82-209 with
 * exact integer arithmetic): for every node its best feasible target and isolated gain.
 * part[n], part_size[K] (node-size sums), node_size[n]. encourage=1 selects the INCC saving
 * sum floor(w_fx / c^2); 0 the k-way saving sum w_fx*[c == 1]. out_target[n] (UINT32_MAX = no
 * move), out_gain[n]. */
int axc_stage_gains(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, uint32_t num_parts,
                    const uint32_t *node_size, uint32_t omega, uint32_t delta, int encourage,
                    uint32_t discount, uint32_t *out_target, int64_t *out_gain);

/* All refinement rounds of one level for a given partition: the rounds of refinementRepeats
 * (sources/refinement.cu:82-545): gains, cascade, size and inbound validity, best prefix and apply,
 * `rounds` rounds under the skip schedule (discount 1, 2, none by thirds; a round without moves
 * skips ahead, sources/refinement.cu:536-543). Arguments as axc_stage_gains, plus the round count
 * and the seed of the tie hash; out_part[n] receives the refined partition (ids below num_parts)
 * and *out_rounds the rounds that ran. */
int axc_stage_refine(axc_ctx *ctx, const axc_hgraph *g, const uint32_t *part, uint32_t num_parts,
                     const uint32_t *node_size, uint32_t omega, uint32_t delta, int encourage,
                     uint32_t rounds, uint64_t seed, uint32_t *out_part, uint32_t *out_rounds);

/* ---- failure path of the bounded device waits (no reference counterpart: the reference's waits
 * are grid syncs and host synchronizations, which never time out) ------------------------------------
 * Runs one look-back wait of the single-pass scans (the only waits on other blocks' flags in this
 * library) against a tile flag that nothing publishes, polling it spin_limit times (the scans poll
 * 2^24 times). The wait gives up, the kernel sets the status word and returns, and the call reports
 * AXC_EINTERNAL with the status in axc_last_error; the context stays usable. Returns AXC_OK only
 * if the wait did not give up, which would be a defect. */
int axc_selftest_bounded_wait(axc_ctx *ctx, uint32_t spin_limit);

/* ---- connectivity without allocating (no reference counterpart) ---------------------------------
 * out_fx[0..2] = connectivity_fx, cutnet_fx and soed_fx of part[] over a hypergraph already in
 * device memory, equal to what axc_evaluate reports for the same inputs. For callers that may not
 * allocate device memory: a serving loop whose memory is all committed to resident hierarchies
 * under its admission budget, or a host runtime whose pool allocator owns the device and leaves no
 * room for the arena an axc_ctx reserves. It needs no context and calls no allocating routine: its
 * scratch is one fixed 16 MiB array in the library's device image, and it clears the part of that
 * array that must start at zero on every call.
 * - Runs on the current device, on `stream` (a cudaStream_t; NULL = the default stream), and
 *   synchronizes that stream before returning.
 * - Every call looks up the scratch array's address in the current context (a lookup, no
 *   allocation), so it follows cudaDeviceReset and contexts the caller makes current. The first
 *   call in a context may load the library's device code; make that call before any stream
 *   capture.
 * - Hyperedges longer than 16384 pins are refused with AXC_EOVERFLOW; a partition id of
 *   UINT32_MAX gives AXC_EINVAL.
 * - Calls that overlap on the GPU (other streams, other host threads) share the scratch and race:
 *   serialize them on one device.
 * d_hedge_off[e+1], d_pins, d_part[n]: device memory; d_hedge_w may be NULL (unit weights). */
int axc_connectivity_noalloc(uint32_t e, const uint64_t *d_hedge_off, const uint32_t *d_pins,
                             const float *d_hedge_w, const uint32_t *d_part, void *stream,
                             int64_t *out_fx);

#ifdef __cplusplus
}
#endif
#endif /* AXC_H */
