// Coarsening kernels: candidate rating, deterministic matching with orphan pairing, group
// relabelling, and the INCC greedy merge of the coarsest groups.
//
// Rating (kernels/coarsening.cu:76-212 restated, node-parallel, no neighbour CSR): for node u,
// every pin v != u of every hyperedge e incident to u adds floor(w_fx(e)/|e|) to v's score and,
// when e is inbound to u and v is one of e's destinations, 1 to v's shared-inbound count. The
// per-node accumulator is an open-addressing table: in shared memory per warp for light nodes,
// per block for medium ones, in a global scratch region for heavy ones. Candidates failing
// size(u)+size(v) <= omega or |in(u)|+|in(v)|-shared <= delta are dropped, the symmetric noise of
// the pair is added, and the top `cnc` by (score desc, id desc) with score > 0 are written.
#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace axc {
namespace {

// Pins a hyperedge contributes to the rating: all of them up to AXC_RATE_MAX_LEN, none above.
__host__ __device__ __forceinline__ u32 rated_len(u64 len) { return len <= AXC_RATE_MAX_LEN ? (u32)len : 0u; }

constexpr u32 RT_WARP_W = 256;     // work (incident pins) handled by one warp
constexpr u32 RT_BLK1_W = 2048;    // block tier 1: table 4096 slots (48 KiB)
constexpr u32 RT_BLK2_W = 8192;    // block tier 2: table 16384 slots (192 KiB)
// The block tiers' first-try table (c.tune.rate_try slots, 2048 by default: 24 KiB) and the
// second try of the larger tier (c.tune.rate_mid, 8192: 96 KiB, two blocks per SM) are tunable.
constexpr u32 RT_WARPS = 4;
constexpr u32 RT_BLOCK = 256;

__global__ void k_rate_work(u32 n, const u64 *__restrict__ toff, const u32 *__restrict__ touch,
                            const u64 *__restrict__ off, u64 *__restrict__ work) {
    const u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (u >= n) return;
    u64 s = 0;
    for (u64 j = toff[u] + lane; j < toff[u + 1]; j += 32) {
        u32 h = touch[j];
        s += rated_len(off[h + 1] - off[h]);
    }
    s = warp_sum(s);
    if (lane == 0) work[u] = s;
}

__global__ void k_rate_tier(u32 n, const u64 *__restrict__ work, u64 lo, u64 hi, u32 *__restrict__ flag) {
    u32 u = blockIdx.x * blockDim.x + threadIdx.x;
    // the first tier (lo == 0) also takes nodes without incident hyperedges
    if (u < n) flag[u] = ((lo == 0 || work[u] > lo) && work[u] <= hi) ? 1u : 0u;
}

struct RateArgs {
    u32 n, cnc, omega, delta;
    const u64 *off;
    const u32 *pins, *nsrc, *wfx;
    const u64 *toff;
    const u32 *touch, *nin, *nsize;
    u32 *pairs, *scores;
    u32 *status;
    const u64 *work;  // per node: pins visited by its rating (the table bound)
};

// Accumulate node u's neighbour scores into (keys, sc, cm) of size mask+1. Warp-cooperative: the
// calling warp takes u's incidences in batches of 32 starting at `first`, every `stride` entries.
// A batch's hyperedge metadata loads in parallel, then its pins are flattened across the lanes
// (each lane finds its pin's hyperedge by a 5-step search over the prefix of the batch's lengths).
// With `ndist` set, the table is a first try: distinct keys are counted there, and once they pass
// `limit` the node stops (the caller retries it with a larger table).
__device__ void rate_flat(const RateArgs &A, u32 u, u32 *keys, u32 *sc, u32 *cm, u32 mask, u32 first,
                          u32 stride, u32 *ndist = nullptr, u32 limit = 0, u32 *used = nullptr) {
    const u32 lane = threadIdx.x & 31u;
    const u64 t0 = A.toff[u];
    const u32 deg = (u32)(A.toff[u + 1] - t0), nin_u = A.nin[u];
    for (u32 jb = first; jb < deg; jb += stride) {
        const u32 j = jb + lane;
        const bool has = j < deg;
        const u32 h = has ? A.touch[t0 + j] : 0;
        const u64 a = has ? A.off[h] : 0;
        const u32 len = has ? rated_len(A.off[h + 1] - a) : 0;  // 0: not rated
        const u32 c = len ? A.wfx[h] / len : 0;
        const u32 s_end = has ? (u32)A.nsrc[h] : 0;  // sources occupy [0, s_end)
        const u32 inb = (has && j < nin_u) ? 1u : 0u;
        u32 x = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if ((int)lane >= o) x += y;
        }
        const u32 total = __shfl_sync(0xFFFFFFFFu, x, 31), excl = x - len;
        const u32 chunk = (deg - jb) < 32 ? (deg - jb) : 32;
        for (u32 fb = 0; fb < total; fb += 32) {
            const u32 f = fb + lane;
            u32 lo = 0, hi = chunk - 1;  // owner: largest o < chunk with excl_o <= f
            for (int it = 0; it < 5; ++it) {
                const u32 mid = (lo + hi + 1) >> 1;
                const u32 em = __shfl_sync(0xFFFFFFFFu, excl, mid & 31);
                if (lo < hi) { if (em <= f) lo = mid; else hi = mid - 1; }
            }
            const u64 ao = __shfl_sync(0xFFFFFFFFu, a, lo);
            const u32 cc = __shfl_sync(0xFFFFFFFFu, c, lo);
            const u32 ss = __shfl_sync(0xFFFFFFFFu, s_end, lo);
            const u32 ib = __shfl_sync(0xFFFFFFFFu, inb, lo);
            const u32 eo = __shfl_sync(0xFFFFFFFFu, excl, lo);
            if (f >= total) continue;
            const u32 i = f - eo;  // position inside the owner hyperedge
            const u32 v = A.pins[ao + i];
            if (v == u) continue;
            u32 slot;
            if (ndist) {  // counted keys: a first try gives up past `limit`; `used` lists them
                if (*(volatile u32 *)ndist > limit) continue;
                bool fresh = false;
                slot = hash_insert_fresh(keys, mask, v, fresh);
                if (slot == NONE) {  // full: a first try overflows, a sized table is an error
                    if (used) atomicExch(A.status, DEV_HASH_FULL);
                    else atomicExch(ndist, limit + 1);
                    continue;
                }
                if (fresh) {
                    const u32 idx = atomicAdd(ndist, 1u);
                    if (used) used[idx] = slot;
                    if (idx + 1 > limit) continue;
                }
            } else {
                slot = hash_find_or_insert(keys, mask, v);
                if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); continue; }
            }
            atomicAdd(&sc[slot], cc);
            if (ib && i >= ss) atomicAdd(&cm[slot], 1u);
        }
    }
}

__device__ __forceinline__ u64 cand_key(const RateArgs &A, u32 u, u32 v, u32 s, u32 shared_inb) {
    if ((u64)A.nsize[u] + A.nsize[v] > A.omega) return 0;
    if ((u64)A.nin[u] + A.nin[v] - shared_inb > A.delta) return 0;
    const u32 score = s + pair_noise(u, v);
    if (score == 0) return 0;
    return ((u64)score << 32) | v;
}

// Per-thread top-cnc candidate keys of the table slots first, first + step, ... (keys are unique:
// the low word is the neighbour id; 0 is empty). One pass, so each neighbour's size and inbound
// count are read once.
// Inserts key k into the descending list top[0, cnc) (a key not above the last entry drops out).
template <int TC>
__device__ __forceinline__ void top_insert(u64 (&top)[TC], u64 k, u32 cnc) {
#pragma unroll
    for (int i = 0; i < TC; ++i)
        if ((u32)i < cnc && k > top[i]) {
            const u64 t = top[i];
            top[i] = k;
            k = t;
        }
}
// Slots [first, cap) step `step` of the table, or with `used` the listed slots used[first, cap).
template <int TC>
__device__ __forceinline__ void top_collect(const RateArgs &A, u32 u, const u32 *keys, const u32 *sc, const u32 *cm,
                                           u32 cap, u32 first, u32 step, u64 (&top)[TC],
                                           const u32 *used = nullptr) {
#pragma unroll
    for (int i = 0; i < TC; ++i) top[i] = 0;
    const u32 cnc = A.cnc;
    u64 floor = 0;  // the list's last entry: a key must beat it to enter
    for (u32 t = first; t < cap; t += step) {
        const u32 s = used ? used[t] : t;
        const u32 v = keys[s];
        if (v == NONE) continue;
        const u64 k = cand_key(A, u, v, sc[s], cm[s]);
        if (k <= floor) continue;
        top_insert<TC>(top, k, cnc);
#pragma unroll
        for (int i = 0; i < TC; ++i)
            if ((u32)i + 1 == cnc) floor = top[i];
    }
}
template <int TC>
__device__ __forceinline__ void top_pop(u64 (&top)[TC]) {
#pragma unroll
    for (int i = 0; i + 1 < TC; ++i) top[i] = top[i + 1];
    top[TC - 1] = 0;
}

// TC: the length of the per-thread top lists, at least cnc (4 for cnc <= 4, else 16).
template <int TC>
__global__ void __launch_bounds__(RT_WARPS * 32) k_rate_warp(RateArgs A, const u32 *__restrict__ list, u32 nlist) {
    __shared__ u32 tk[RT_WARPS][2 * RT_WARP_W], ts[RT_WARPS][2 * RT_WARP_W], tc[RT_WARPS][2 * RT_WARP_W];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 idx = blockIdx.x * RT_WARPS + w;
    if (idx >= nlist) return;
    const u32 u = list[idx];
    u32 *keys = tk[w], *sc = ts[w], *cm = tc[w];
    const u64 W = A.work[u];  // work bound for the table size (at most RT_WARP_W in this tier)
    u32 cap = 64;
    while (cap < 2 * W) cap <<= 1;
    for (u32 i = lane; i < cap; i += 32) { keys[i] = NONE; sc[i] = 0; cm[i] = 0; }
    __syncwarp();
    rate_flat(A, u, keys, sc, cm, cap - 1, 0, 32);
    __syncwarp();
    u64 top[TC];
    top_collect<TC>(A, u, keys, sc, cm, cap, lane, 32, top);
    for (u32 r = 0; r < A.cnc; ++r) {
        const u64 best = warp_max_u64(top[0]);
        if (lane == 0) {
            A.pairs[(u64)u * A.cnc + r] = best ? (u32)best : NONE;
            A.scores[(u64)u * A.cnc + r] = best ? (u32)(best >> 32) : 0u;
        }
        if (best && top[0] == best) top_pop<TC>(top);
    }
}

constexpr u32 RT_SEL = (RT_BLOCK / 32) * AXC_MAX_CANDIDATES;  // shared slots of the block selection

// The top-cnc candidates of node u from its table (keys, sc, cm) of `cap` slots; block-wide.
// Each warp reduces its lanes' lists to its own top cnc with shuffles into red[warp * cnc ..];
// warp 0 merges those after one barrier. red holds RT_SEL entries.
// With `used`, only the nused listed slots are read.
template <int TC>
__device__ void rate_select(const RateArgs &A, u32 u, const u32 *keys, const u32 *sc, const u32 *cm, u32 cap,
                            u64 *red, const u32 *used = nullptr, u32 nused = 0) {
    const u32 lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5, cnc = A.cnc;
    u64 top[TC];
    top_collect<TC>(A, u, keys, sc, cm, used ? nused : cap, threadIdx.x, blockDim.x, top, used);
    for (u32 r = 0; r < cnc; ++r) {
        const u64 best = warp_max_u64(top[0]);
        if (lane == 0) red[w * cnc + r] = best;
        if (best && top[0] == best) top_pop<TC>(top);
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < TC; ++i) top[i] = 0;
        for (u32 i = lane; i < nw * cnc; i += 32) top_insert<TC>(top, red[i], cnc);
        for (u32 r = 0; r < cnc; ++r) {
            const u64 best = warp_max_u64(top[0]);
            if (lane == 0) {
                A.pairs[(u64)u * cnc + r] = best ? (u32)best : NONE;
                A.scores[(u64)u * cnc + r] = best ? (u32)(best >> 32) : 0u;
            }
            if (best && top[0] == best) top_pop<TC>(top);
        }
    }
    __syncthreads();  // red is reused by the block's next node
}

// Heavy nodes of a level with few of them: `splits` blocks per node share the node's table in
// global scratch (keys | sc | cm planes of nl * cap slots, cleared beforehand); block s of node
// idx takes every splits-th group of its warps' incidence batches.
__global__ void __launch_bounds__(RT_BLOCK) k_rate_split_acc(RateArgs A, const u32 *__restrict__ list, u32 nl,
                                                            u32 cap, u32 splits, u32 *gtab) {
    const u32 idx = blockIdx.x / splits, s = blockIdx.x % splits;
    if (idx >= nl) return;
    const u64 plane = (u64)nl * cap;
    u32 *keys = gtab + (u64)idx * cap, *sc = keys + plane, *cm = sc + plane;
    const u32 nw = blockDim.x >> 5;
    rate_flat(A, list[idx], keys, sc, cm, cap - 1, 32 * (s * nw + (threadIdx.x >> 5)), 32 * nw * splits);
}
template <int TC>
__global__ void __launch_bounds__(RT_BLOCK) k_rate_split_select(RateArgs A, const u32 *__restrict__ list, u32 nl,
                                                               u32 cap, const u32 *gtab) {
    __shared__ u64 red[RT_SEL];
    const u32 idx = blockIdx.x;
    if (idx >= nl) return;
    const u64 plane = (u64)nl * cap;
    const u32 *keys = gtab + (u64)idx * cap, *sc = keys + plane, *cm = sc + plane;
    rate_select<TC>(A, list[idx], keys, sc, cm, cap, red);
}

// One node per block iteration; table in dynamic smem (gtab == nullptr) or in this block's
// slice of a global scratch region. A global slice (keys | sc | cm planes of cap_max slots) is
// emptied once at the start; each node lists the slots it fills in its slice of gused, reads its
// candidates from those and empties them again, so its cost follows its distinct neighbours,
// not the slice size.
// With `retry` set the launch is a first try on tables smaller than the nodes' work bounds: a node
// whose distinct neighbours pass half of its table stops and is appended to retry / *d_retry.
// With `d_nl` set the list length is read from device memory (at most nlist).
template <int TC>
__global__ void __launch_bounds__(RT_BLOCK) k_rate_block(RateArgs A, const u32 *__restrict__ list, u32 nlist,
                                                        u32 cap_max, u32 *gtab, const u32 *__restrict__ d_nl,
                                                        u32 *__restrict__ retry, u32 *__restrict__ d_retry,
                                                        u32 *gused) {
    extern __shared__ u32 dyn[];
    __shared__ u64 red[RT_SEL];
    __shared__ u32 ndist;
    u32 *keys, *sc, *cm, *used = nullptr;
    if (d_nl) nlist = min(nlist, *d_nl);
    if (gtab) {
        keys = gtab + (u64)blockIdx.x * 3 * cap_max;
        sc = keys + cap_max;
        cm = sc + cap_max;
        used = gused + (u64)blockIdx.x * cap_max;
        if (blockIdx.x < nlist)
            for (u32 i = threadIdx.x; i < cap_max; i += blockDim.x) { keys[i] = NONE; sc[i] = 0; cm[i] = 0; }
    } else {
        keys = dyn;
    }
    for (u32 idx = blockIdx.x; idx < nlist; idx += gridDim.x) {
        const u32 u = list[idx];
        // table size from the node's work bound, capped by the node count
        const u64 W = A.work[u] < A.n ? A.work[u] : A.n;
        u32 cap = 64;
        while (cap < 2 * W && cap < cap_max) cap <<= 1;
        if (!gtab) {
            sc = keys + cap;
            cm = sc + cap;
            for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = NONE; sc[i] = 0; cm[i] = 0; }
        }
        if (threadIdx.x == 0) ndist = 0;
        __syncthreads();
        const u32 limit = gtab ? cap : cap / 2;
        rate_flat(A, u, keys, sc, cm, cap - 1, 32 * (threadIdx.x >> 5), blockDim.x,
                  (retry || gtab) ? &ndist : nullptr, limit, used);
        __syncthreads();
        if (retry && ndist > limit) {  // table too small: the retry launch redoes this node
            if (threadIdx.x == 0) retry[atomicAdd(d_retry, 1u)] = u;
        } else {
            rate_select<TC>(A, u, keys, sc, cm, cap, red, used, ndist);
        }
        if (gtab) {  // rate_select ends with a barrier: empty the listed slots
            for (u32 t = threadIdx.x; t < ndist; t += blockDim.x) {
                const u32 s2 = used[t];
                keys[s2] = NONE;
                sc[s2] = 0;
                cm[s2] = 0;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- matching
// Rounds of proposals (the rule of or_matching in the oracle): A. every unmatched node proposes to
// its best still-unmatched candidate; B. every node keeps its best proposer by (score, id) with a
// 64-bit atomicMax (order-independent); C. u and its target v match when v accepted u and v's own
// proposal was refused, or when both accepted each other. Phase C reads only phase A/B state, so
// every node is matched at most once per round and the result is deterministic. One cooperative
// launch runs every round with grid-wide barriers; without cooperative launch each phase is a
// kernel.
struct MatchArgs {
    u32 n, cnc;
    const u32 *pairs, *scores;
    u32 *mate, *ptr, *prop;
    unsigned long long *best;
    u32 *changed;
};
__device__ __forceinline__ void match_propose(const MatchArgs &A, u64 i0, u64 stride) {
    for (u64 v = i0; v < A.n; v += stride) {
        A.best[v] = 0;
        if (A.mate[v] != NONE) { A.prop[v] = NONE; continue; }
        u32 p = A.ptr[v];
        while (p < A.cnc) {
            u32 w = A.pairs[v * A.cnc + p];
            if (w == NONE) { p = A.cnc; break; }
            if (A.mate[w] == NONE) break;
            ++p;
        }
        A.ptr[v] = p;
        A.prop[v] = p < A.cnc ? A.pairs[v * A.cnc + p] : NONE;
    }
}
__device__ __forceinline__ void match_bid(const MatchArgs &A, u64 i0, u64 stride) {
    for (u64 u = i0; u < A.n; u += stride) {
        const u32 v = A.prop[u];
        if (v == NONE) continue;
        const unsigned long long key = ((unsigned long long)A.scores[u * A.cnc + A.ptr[u]] << 32) | u;
        atomicMax(&A.best[v], key);
    }
}
__device__ __forceinline__ bool match_acc(const MatchArgs &A, u32 u) {
    const u32 v = A.prop[u];
    if (v == NONE) return false;
    const unsigned long long b = A.best[v];
    return b != 0 && (u32)b == u;
}
__device__ __forceinline__ void match_accept(const MatchArgs &A, u32 *changed, u64 i0, u64 stride) {
    for (u64 u = i0; u < A.n; u += stride) {
        if (!match_acc(A, (u32)u)) continue;
        const u32 v = A.prop[u];
        if (!match_acc(A, v) || (A.prop[v] == u && u < v)) {
            A.mate[u] = v;
            A.mate[v] = (u32)u;
            *changed = 1;
        }
    }
}

__global__ void k_match_coop(MatchArgs A, u32 rounds) {
    cg::grid_group grid = cg::this_grid();
    const u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x, stride = (u64)gridDim.x * blockDim.x;
    for (u32 r = 0; r < rounds; ++r) {
        match_propose(A, i0, stride);
        grid.sync();
        match_bid(A, i0, stride);
        grid.sync();
        match_accept(A, &A.changed[r], i0, stride);
        grid.sync();
        if (((volatile u32 *)A.changed)[r] == 0) break;
    }
}
__global__ void k_match_phase(MatchArgs A, u32 r, int phase) {
    if (r > 0 && A.changed[r - 1] == 0) return;  // a previous round reached the fixed point
    const u64 i0 = (u64)blockIdx.x * blockDim.x + threadIdx.x, stride = (u64)gridDim.x * blockDim.x;
    if (phase == 0) match_propose(A, i0, stride);
    else if (phase == 1) match_bid(A, i0, stride);
    else match_accept(A, &A.changed[r], i0, stride);
}

// Two-hop pass (see or_matching): unmatched nodes with candidates, sorted by (best candidate, id),
// pair at even/odd positions of each bucket when the size and inbound-count sums fit.
__global__ void k_hop_flags(u32 n, u32 cnc, const u32 *__restrict__ pairs, const u32 *__restrict__ mate,
                            u32 *__restrict__ flag) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) flag[v] = (mate[v] == NONE && pairs[(u64)v * cnc] != NONE) ? 1u : 0u;
}
__global__ void k_hop_keys(const u32 *__restrict__ ids, const u32 *__restrict__ dm, u32 cnc,
                           const u32 *__restrict__ pairs, u32 *__restrict__ key) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < *dm) key[i] = pairs[(u64)ids[i] * cnc];
}
__global__ void k_hop_heads(const u32 *__restrict__ key, const u32 *__restrict__ dm, u32 nmax, u32 *__restrict__ head) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmax) return;
    head[i] = (i < *dm && (i == 0 || key[i] != key[i - 1])) ? 1u : 0u;
}
__global__ void k_hop_start(const u32 *__restrict__ head, const u32 *__restrict__ sid, const u32 *__restrict__ dm,
                            u32 *__restrict__ start) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < *dm && head[i]) start[sid[i]] = i;
}
// sid is the exclusive scan of the head flags: the segment of element i is sid[i] + head[i] - 1
__global__ void k_hop_pair(const u32 *__restrict__ ids, const u32 *__restrict__ key, const u32 *__restrict__ head,
                           const u32 *__restrict__ sid, const u32 *__restrict__ start, const u32 *__restrict__ dm,
                           const u32 *__restrict__ nsize, const u32 *__restrict__ nin, u32 omega, u32 delta,
                           u32 *__restrict__ mate) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 m = *dm;
    if (i + 1 >= m) return;
    if (((i - start[sid[i] + head[i] - 1]) & 1u) || key[i + 1] != key[i]) return;
    const u32 x = ids[i], y = ids[i + 1];
    if ((u64)nsize[x] + nsize[y] > omega || (u64)nin[x] + nin[y] > delta) return;
    mate[x] = y;
    mate[y] = x;
}

__global__ void k_orphan_flags(u32 n, u32 cnc, const u32 *__restrict__ pairs, u32 *__restrict__ flag) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) flag[v] = pairs[(u64)v * cnc] == NONE ? 1u : 0u;
}
__global__ void k_gather_size(const u32 *__restrict__ ids, u32 m, const u32 *__restrict__ nsize, u32 *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = nsize[ids[i]];
}
__global__ void k_orphan_pair(const u32 *__restrict__ ord, u32 m, const u32 *__restrict__ nsize,
                              const u32 *__restrict__ nin, u32 omega, u32 delta, u32 *__restrict__ mate) {
    u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m / 2) return;
    u32 L = ord[k], R = ord[m - 1 - k];
    if ((u64)nsize[L] + nsize[R] > omega) return;
    if ((u64)nin[L] + nin[R] > delta) return;
    mate[L] = R;
    mate[R] = L;
}
__global__ void k_group_heads(u32 n, const u32 *__restrict__ mate, u32 *__restrict__ head) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) head[v] = (mate[v] == NONE || v < mate[v]) ? 1u : 0u;
}
__global__ void k_group_assign(u32 n, const u32 *__restrict__ mate, const u32 *__restrict__ gid,
                               u32 *__restrict__ groups) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    u32 m = mate[v];
    groups[v] = gid[(m == NONE || v < m) ? v : m];
}

// ---------------------------------------------------------------- greedy merge (-ipm)
__global__ void k_group_sums(u32 n, const u32 *__restrict__ groups, const u32 *__restrict__ nsize,
                             const u32 *__restrict__ nin, u32 *__restrict__ gs, unsigned long long *__restrict__ gi) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    atomicAdd(&gs[groups[v]], nsize[v]);
    atomicAdd(&gi[groups[v]], (unsigned long long)nin[v]);
}
__global__ void k_split64(const u64 *__restrict__ x, const u32 *__restrict__ ids, u32 m, u32 *__restrict__ hi,
                          u32 *__restrict__ lo) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    u64 v = x[ids ? ids[i] : i];
    hi[i] = (u32)(v >> 32);
    lo[i] = (u32)v;
}
__global__ void k_gather_sz64(const u32 *__restrict__ ord, u32 m, const u32 *__restrict__ gs, const u64 *__restrict__ gi,
                              u64 *__restrict__ ss, u64 *__restrict__ si) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    ss[i] = gs[ord[i]];
    si[i] = gi[ord[i]];
}
__global__ void k_pack_rep(const u32 *__restrict__ ord, const u32 *__restrict__ packid, u32 m, u32 *__restrict__ rep) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) atomicMin(&rep[packid[i]], ord[i]);
}
__global__ void k_pack_map(const u32 *__restrict__ ord, const u32 *__restrict__ packid, const u32 *__restrict__ rep,
                           u32 m, u32 *__restrict__ gmap) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) gmap[ord[i]] = rep[packid[i]];
}
__global__ void k_self_head(const u32 *__restrict__ gmap, u32 m, u32 *__restrict__ head) {
    u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < m) head[x] = gmap[x] == x ? 1u : 0u;
}
__global__ void k_remap_groups(u32 n, u32 *__restrict__ groups, const u32 *__restrict__ gmap, const u32 *__restrict__ nid) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) groups[v] = nid[gmap[groups[v]]];
}

}  // namespace

// out += sum of v[list[i]] over i < nl
__global__ void k_list_sum(const u32 *__restrict__ list, u32 nl, const u64 *__restrict__ v,
                           unsigned long long *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    const u64 s = warp_sum(i < nl ? v[list[i]] : (u64)0);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// out[0] += sum of v[0, n), out[1] = max(out[1], max of v[0, n))
__global__ void k_sum_max(const u64 *__restrict__ v, u32 n, unsigned long long *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    u64 x = i < n ? v[i] : 0;
    const u64 s = warp_sum(x), m = warp_max_u64(x);
    if ((threadIdx.x & 31) == 0) {
        if (s) atomicAdd(&out[0], (unsigned long long)s);
        if (m) atomicMax(&out[1], (unsigned long long)m);
    }
}

void setup_coarsen_kernels(Ctx &c) {
    AXC_CUDA(cudaFuncSetAttribute(k_rate_block<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * 16384 * 4));
    AXC_CUDA(cudaFuncSetAttribute(k_rate_block<(int)AXC_MAX_CANDIDATES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  3 * 16384 * 4));
}

// A rating kernel with per-thread top lists of 4 when cnc <= 4 (the reference scripts' -cnc 4),
// else of AXC_MAX_CANDIDATES: shorter lists hold fewer registers, so more blocks fit an SM.
#define RATE_LAUNCH(c, kname, cnc, grid, block, smem, ...)                                                   \
    do {                                                                                                     \
        if ((cnc) <= 4) LAUNCH_AS(c, #kname, kname<4>, grid, block, smem, __VA_ARGS__);                      \
        else LAUNCH_AS(c, #kname, kname<(int)AXC_MAX_CANDIDATES>, grid, block, smem, __VA_ARGS__);           \
    } while (0)

void rating(Ctx &c, const DLevel &L, const u32 *wfx, u32 omega, u32 delta, u32 cnc, u32 *pairs, u32 *scores,
            u64 *pin_visits) {
    const u32 n = L.n;
    if (n == 0) return;
    size_t m = c.arena.mark();
    u64 *work = c.arena.alloc<u64>(n);
    RateArgs A{n, cnc, omega, delta, L.off, L.pins, L.nsrc, wfx, L.toff, L.touch, L.nin, L.nsize, pairs, scores,
               c.d_status, work};
    u32 *flag = c.arena.alloc<u32>(n);
    u32 *lists[4];
    for (auto &l : lists) l = c.arena.alloc<u32>(n);
    // device counters, read back in one round trip: [0..3] tier sizes, [4] work sum, [5] work max
    u64 *dc = c.arena.alloc<u64>(6);
    AXC_CUDA(cudaMemsetAsync(dc, 0, 48, c.stream));
    fill_u32(c, pairs, NONE, (u64)n * cnc);
    LAUNCH(c, k_rate_work, cdiv((u64)n * 32, 256), 256, 0, n, L.toff, L.touch, L.off, work);
    LAUNCH(c, k_sum_max, cdiv(n, 256), 256, 0, work, n, (unsigned long long *)(dc + 4));
    const u64 lim[5] = {0, RT_WARP_W, RT_BLK1_W, RT_BLK2_W, ~0ull};
    for (int t = 0; t < 4; ++t) {
        LAUNCH(c, k_rate_tier, cdiv(n, 256), 256, 0, n, work, lim[t], lim[t + 1], flag);
        compact_indices_dn(c, flag, lists[t], n, (u32 *)(dc + t));
    }
    u64 h[6];
    fetch(c, h, dc, 48);
    if (pin_visits) *pin_visits = h[4];
    const u32 *list = lists[0], *list2 = lists[1], *list3 = lists[2], *list4 = lists[3];
    // Kernel timer: algorithmic bytes of the block tiers, 4 per pin visit (the pin id) and 8 per
    // candidate slot written (pair and score), per launch.
    u64 tier_visits[3] = {0, 0, 0};
    if (c.profiling("k_rate_block")) {
        u64 *dv = c.arena.alloc<u64>(3);
        AXC_CUDA(cudaMemsetAsync(dv, 0, 24, c.stream));
        for (int t = 0; t < 3; ++t)
            if (h[1 + t])
                LAUNCH(c, k_list_sum, cdiv(h[1 + t], 256), 256, 0, lists[1 + t], (u32)h[1 + t], work,
                       (unsigned long long *)(dv + t));
        fetch(c, tier_visits, dv, 24);
        for (int t = 0; t < 2; ++t)  // the heavy tier counts below, if it runs on k_rate_block
            if (h[1 + t]) c.prof_bytes += 4 * tier_visits[t] + 8ull * cnc * h[1 + t];
    }
    // tier: one warp per node, table in static smem
    u32 nl = (u32)h[0];
    RATE_LAUNCH(c, k_rate_warp, cnc, cdiv(nl, RT_WARPS), RT_WARPS * 32, 0, A, list, nl);
    // tier: one block per node, 4096-slot table in dynamic smem
    nl = (u32)h[1];
    // shared tables sized by the largest node table the tier can need (distinct neighbours never
    // exceed min(work, n)), so smaller tables fit more blocks per SM
    const u64 wcap = std::min<u64>(h[5], n);
    auto tier_cap = [&](u64 hi, u32 cap_hi) {
        u32 cap = 64;
        while (cap < 2 * std::min<u64>(wcap, hi) && cap < cap_hi) cap <<= 1;
        return cap;
    };
    const u32 cap1 = tier_cap(RT_BLK1_W, 4096u), cap2 = tier_cap(RT_BLK2_W, 16384u);
    // Nodes' work bounds count pins with multiplicity; their distinct neighbours are usually far
    // fewer. A first launch tries rt_try-slot tables (more blocks per SM); nodes that outgrow
    // theirs are redone by a second launch with the tier's full tables.
    // A node that outgrows an rt_try table retries at rt_mid slots (two blocks per SM) when the
    // tier's tables are larger still, and only past that at the tier's full size.
    u32 *retry = c.arena.alloc<u32>(n), *retry2 = c.arena.alloc<u32>(n);
    u32 *d_retry = (u32 *)(dc + 4), *d_retry2 = d_retry + 1;  // dc[4] was read already
    const u32 rt_try = c.tune.rate_try, rt_mid = std::max(c.tune.rate_mid, c.tune.rate_try);
    auto block_tier = [&](const u32 *lst, u32 cnt, u32 cap_full) {
        if (!cnt) return;
        if (cap_full <= rt_try) {
            RATE_LAUNCH(c, k_rate_block, cnc, cnt, RT_BLOCK, 3 * cap_full * 4, A, lst, cnt, cap_full, (u32 *)nullptr,
                   (const u32 *)nullptr, (u32 *)nullptr, (u32 *)nullptr, (u32 *)nullptr);
            return;
        }
        AXC_CUDA(cudaMemsetAsync(d_retry, 0, 8, c.stream));  // d_retry and d_retry2
        RATE_LAUNCH(c, k_rate_block, cnc, cnt, RT_BLOCK, 3 * rt_try * 4, A, lst, cnt, rt_try, (u32 *)nullptr,
               (const u32 *)nullptr, retry, d_retry, (u32 *)nullptr);
        const u32 *rl = retry, *dn = d_retry;
        if (cap_full > rt_mid) {
            RATE_LAUNCH(c, k_rate_block, cnc, std::min<u32>(cnt, (u32)c.sms * 2), RT_BLOCK, 3 * rt_mid * 4, A, rl, cnt, rt_mid,
                   (u32 *)nullptr, dn, retry2, d_retry2, (u32 *)nullptr);
            rl = retry2;
            dn = d_retry2;
        }
        const u32 grid = std::min<u32>(cnt, (u32)c.sms * 2);
        RATE_LAUNCH(c, k_rate_block, cnc, grid, RT_BLOCK, 3 * cap_full * 4, A, rl, cnt, cap_full, (u32 *)nullptr, dn,
               (u32 *)nullptr, (u32 *)nullptr, (u32 *)nullptr);
    };
    block_tier(list2, nl, cap1);
    // tier: one block per node, up to 16384-slot table in dynamic smem
    nl = (u32)h[2];
    block_tier(list3, nl, cap2);
    // tier: heavy nodes, tables in a global scratch slice per resident block
    nl = (u32)h[3];
    if (nl) {
        u64 wmax = h[5];
        if (wmax > n) wmax = n;  // distinct neighbours never exceed the node count
        u32 cap = 64;
        while (cap < 2 * wmax && cap < (1u << 30)) cap <<= 1;
        const u64 split_bytes = (u64)nl * 3 * cap * 4;
        if (nl < (u32)c.sms * 2 && split_bytes <= (512ull << 20)) {
            // few heavy nodes: several blocks per node on a per-node table, then selection
            const u32 splits = std::min<u32>(64, cdiv((u64)c.sms * 4, nl));
            u32 *gtab = c.arena.alloc<u32>((u64)nl * 3 * cap);
            AXC_CUDA(cudaMemsetAsync(gtab, 0xFF, (size_t)nl * cap * 4, c.stream));
            AXC_CUDA(cudaMemsetAsync(gtab + (u64)nl * cap, 0, (size_t)nl * cap * 8, c.stream));
            LAUNCH(c, k_rate_split_acc, nl * splits, RT_BLOCK, 0, A, list4, nl, cap, splits, gtab);
            RATE_LAUNCH(c, k_rate_split_select, cnc, nl, RT_BLOCK, 0, A, list4, nl, cap, gtab);
        } else {
            u32 grid = nl < (u32)c.sms * 2 ? nl : (u32)c.sms * 2;
            u32 *gtab = c.arena.alloc<u32>((u64)grid * 3 * cap), *gused = c.arena.alloc<u32>((u64)grid * cap);
            if (c.profiling("k_rate_block")) c.prof_bytes += 4 * tier_visits[2] + 8ull * cnc * nl;
            RATE_LAUNCH(c, k_rate_block, cnc, grid, RT_BLOCK, 0, A, list4, nl, cap, gtab, (const u32 *)nullptr, (u32 *)nullptr,
                   (u32 *)nullptr, gused);
        }
    }
    check_status(c);
    c.arena.release(m);
}

u32 matching(Ctx &c, u32 n, u32 cnc, const u32 *pairs, const u32 *scores, const u32 *nsize, const u32 *nin,
             u32 omega, u32 delta, u32 rounds, u32 *groups) {
    if (n == 0) return 0;
    size_t m = c.arena.mark();
    u32 *mate = c.arena.alloc<u32>(n), *ptr = c.arena.alloc<u32>(n), *prop = c.arena.alloc<u32>(n);
    unsigned long long *best = c.arena.alloc<unsigned long long>(n);
    u32 *changed = c.arena.alloc<u32>(rounds + 1);
    fill_u32(c, mate, NONE, n);
    AXC_CUDA(cudaMemsetAsync(ptr, 0, (size_t)n * 4, c.stream));
    AXC_CUDA(cudaMemsetAsync(changed, 0, (size_t)(rounds + 1) * 4, c.stream));
    MatchArgs A{n, cnc, pairs, scores, mate, ptr, prop, best, changed};
    bool done = false;
    if (c.coop_supported) {
        int per_sm = 0;
        AXC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_match_coop, 256, 0));
        u32 grid = (u32)per_sm * c.sms;
        u32 need = cdiv(n, 256);
        if (grid > need) grid = need;
        if (grid >= 1 && per_sm > 0) {
            void *args[] = {(void *)&A, (void *)&rounds};
            AXC_CUDA(cudaLaunchCooperativeKernel((void *)k_match_coop, grid, 256, args, 0, c.stream));
            c.launches++;
            done = true;
        }
    }
    if (!done) {
        u32 grid = cdiv(n, 256);
        for (u32 r = 0; r < rounds; ++r)
            for (int ph = 0; ph < 3; ++ph) LAUNCH(c, k_match_phase, grid, 256, 0, A, r, ph);
    }
    // two-hop pass
    {
        size_t m2 = c.arena.mark();
        u32 *flag = c.arena.alloc<u32>(n), *ids = c.arena.alloc<u32>(n), *key = c.arena.alloc<u32>(n);
        u32 *head = c.arena.alloc<u32>(n), *sid = c.arena.alloc<u32>(n), *start = c.arena.alloc<u32>(n);
        u32 *dm = c.arena.alloc<u32>(1);
        LAUNCH(c, k_hop_flags, cdiv(n, 256), 256, 0, n, cnc, pairs, mate, flag);
        compact_indices_dn(c, flag, ids, n, dm);
        LAUNCH(c, k_hop_keys, cdiv(n, 256), 256, 0, ids, dm, cnc, pairs, key);
        radix_sort_pairs_dn(c, key, ids, dm, n, bits_for(n - 1));
        LAUNCH(c, k_hop_heads, cdiv(n, 256), 256, 0, key, dm, n, head);
        scan_excl_u32(c, head, sid, n);
        LAUNCH(c, k_hop_start, cdiv(n, 256), 256, 0, head, sid, dm, start);
        LAUNCH(c, k_hop_pair, cdiv(n, 256), 256, 0, ids, key, head, sid, start, dm, nsize, nin, omega, delta, mate);
        c.arena.release(m2);
    }
    // orphans
    u32 *flag = c.arena.alloc<u32>(n), *orph = c.arena.alloc<u32>(n);
    LAUNCH(c, k_orphan_flags, cdiv(n, 256), 256, 0, n, cnc, pairs, flag);
    u32 mo = compact_indices(c, flag, orph, n);
    if (mo >= 2) {
        u32 *key = c.arena.alloc<u32>(mo);
        LAUNCH(c, k_gather_size, cdiv(mo, 256), 256, 0, orph, mo, nsize, key);
        u32 maxs = reduce_max_u32(c, key, mo);
        radix_sort_pairs(c, key, orph, mo, bits_for(maxs));
        LAUNCH(c, k_orphan_pair, cdiv(mo / 2, 256), 256, 0, orph, mo, nsize, nin, omega, delta, mate);
    }
    // relabel in order of the smallest member
    u32 *head = flag, *gid = orph;
    LAUNCH(c, k_group_heads, cdiv(n, 256), 256, 0, n, mate, head);
    scan_excl_u32(c, head, gid, n);
    u64 tail[2];
    {
        u32 *d = c.arena.alloc<u32>(2);
        AXC_CUDA(cudaMemcpyAsync(d, gid + n - 1, 4, cudaMemcpyDeviceToDevice, c.stream));
        AXC_CUDA(cudaMemcpyAsync(d + 1, head + n - 1, 4, cudaMemcpyDeviceToDevice, c.stream));
        fetch(c, tail, d, 8);
    }
    const u32 *t32 = (const u32 *)tail;
    u32 ng = t32[0] + t32[1];
    LAUNCH(c, k_group_assign, cdiv(n, 256), 256, 0, n, mate, gid, groups);
    c.arena.release(m);
    return ng;
}

u32 greedy_merge_groups(Ctx &c, u32 n, const u32 *nsize, const u32 *nin, u32 *groups, u32 ng, u32 omega,
                        u32 delta) {
    if (n == 0 || ng < 2) return ng;
    size_t mk = c.arena.mark();
    const u32 m = ng;
    u32 *gs = c.arena.alloc<u32>(m);
    u64 *gi = c.arena.alloc<u64>(m);
    AXC_CUDA(cudaMemsetAsync(gs, 0, (size_t)m * 4, c.stream));
    AXC_CUDA(cudaMemsetAsync(gi, 0, (size_t)m * 8, c.stream));
    LAUNCH(c, k_group_sums, cdiv(n, 256), 256, 0, n, groups, nsize, nin, gs, (unsigned long long *)gi);
    // order by (size, inbound, id): ids ascending, stable by inbound (64-bit), stable by size
    u32 *ord = c.arena.alloc<u32>(m), *hi = c.arena.alloc<u32>(m), *lo = c.arena.alloc<u32>(m);
    iota_u32(c, ord, m);
    LAUNCH(c, k_split64, cdiv(m, 256), 256, 0, gi, (const u32 *)nullptr, m, hi, lo);
    radix_sort_pairs64(c, hi, lo, ord, m, 32, 32);
    LAUNCH(c, k_gather_size, cdiv(m, 256), 256, 0, ord, m, gs, lo);
    radix_sort_pairs(c, lo, ord, m, 32);
    u64 *ss = c.arena.alloc<u64>(m), *si = c.arena.alloc<u64>(m);
    LAUNCH(c, k_gather_sz64, cdiv(m, 256), 256, 0, ord, m, gs, gi, ss, si);
    u32 *msc = c.arena.alloc<u32>(m), *packid = c.arena.alloc<u32>(m), *rep = c.arena.alloc<u32>(m);
    greedy_pack(c, ss, si, m, (u64)omega, (u64)delta, packid);
    fill_u32(c, rep, NONE, m);
    LAUNCH(c, k_pack_rep, cdiv(m, 256), 256, 0, ord, packid, m, rep);
    u32 *gmap = hi;
    LAUNCH(c, k_pack_map, cdiv(m, 256), 256, 0, ord, packid, rep, m, gmap);
    u32 *head = lo, *nid = msc;
    LAUNCH(c, k_self_head, cdiv(m, 256), 256, 0, gmap, m, head);
    scan_excl_u32(c, head, nid, m);
    u32 t[2];
    {
        u32 *d = c.arena.alloc<u32>(2);
        AXC_CUDA(cudaMemcpyAsync(d, nid + m - 1, 4, cudaMemcpyDeviceToDevice, c.stream));
        AXC_CUDA(cudaMemcpyAsync(d + 1, head + m - 1, 4, cudaMemcpyDeviceToDevice, c.stream));
        u64 tmp;
        fetch(c, &tmp, d, 8);
        memcpy(t, &tmp, 8);
    }
    const u32 newg = t[0] + t[1];
    LAUNCH(c, k_remap_groups, cdiv(n, 256), 256, 0, n, groups, gmap, nid);
    c.arena.release(mk);
    return newg;
}

}  // namespace axc
