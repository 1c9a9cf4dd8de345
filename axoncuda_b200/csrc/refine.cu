// Refinement (sources/refinement.cu:18-582 and kernels/refinement.cu:9-652 restated with exact
// integer arithmetic and a sparse per-hyperedge census instead of the dense E x K table).
//
// One round:
//  1. census: for every hyperedge the partitions among its pins with (pins, destination pins),
//     in first-occurrence order (hashed) or ascending order (partition-indexed, K <= 256);
//     partition sizes and distinct-inbound counts.
//  2. gains: every node's best feasible target among the partitions adjacent to it; only moves
//     with positive gain are proposed. With K <= 256 from per-hyperedge partition bitmasks
//     (O(K/32) per incidence and lane), else from hash tables (O(lambda) per incidence).
//  3. rank by (gain desc, id asc).
//  4. cascade: each move's gain recomputed assuming every better-ranked move is applied, by a
//     sweep over each hyperedge's movers in rank order (O(pins) instead of the reference's
//     per-move re-read of every incident hyperedge), 32 movers at a time per warp with exact
//     prefix counts.
//  5. prefix sums of cascaded gains; size-excess and inbound-validity of every prefix from sorted
//     event streams (sources/refinement.cu:239-491); best prefix by best_move_functor
//     (headers/data_types.cuh:113-136); apply when valid with non-negative prefix gain.
//
// Work lists that depend only on the level (hyperedge-length tiers, per-node gain-work bounds)
// are built once per level. Inside a round every count stays in device memory; the host reads a
// single word per round (whether moves were applied), which drives the round schedule.
#include <cstdlib>

#include "common.cuh"
#include "kernels.h"
#include "blocksort.cuh"

namespace axc {
namespace {

constexpr u32 CS_WARP_CAP = 256;
constexpr u32 CS_BLOCK_CAP = 4096;
constexpr u32 CS_WARPS = 4;

// Slots of a block's census or candidate hash table for `len` keys: a power of two, at most 2/3
// full. The hyperedge's entries and their order do not depend on it.
__host__ __device__ __forceinline__ u32 cs_cap(u64 len) {
    u32 cap = 32;
    while (cap < len + (len >> 1)) cap <<= 1;
    return cap;
}
// Bytes of dynamic shared memory this launch was given.
__device__ __forceinline__ u32 dyn_smem_bytes() {
    u32 b;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(b));
    return b;
}

// What a node saves by leaving partition p of a hyperedge (weight w) where p holds c of its pins:
// INCC (encourage) floor(w / c^2), k-way w when the node is the last pin in p.
__device__ __forceinline__ i64 leave_gain(int encourage, u32 w, u32 c) {
    if (encourage) return c >= 1 ? (i64)((u64)w / ((u64)c * c)) : 0;
    return c == 1 ? (i64)w : 0;
}

// ------------------------------------------------------------------ census
struct CensusArgs {
    const u64 *off;
    const u32 *pins, *nsrc, *part;
    u32 *cpart, *ccnt, *cdcnt, *lam;
    u32 *status;
    // when set: every pin adds leave_gain(w, count of its partition) to its node's saving
    unsigned long long *save;
    const u32 *wfx;
    int encourage;
    // partition-indexed census only, when set: the hyperedge's masks of partitions present and
    // with destination pins, mw words each
    u32 *mask, *dmask;
    u32 mw;
    // when set (kernel timer on k_census_direct_warp): each hyperedge's algorithmic bytes are added
    unsigned long long *pbytes;
};

// insert phase: keys = partition, mn = first position, cnt/dcnt counters
__device__ __forceinline__ void cs_insert(const CensusArgs &A, u64 a, u64 b, u64 s, u32 *keys, u32 *mn, u32 *cnt,
                                          u32 *dcnt, u32 mask, u32 t, u32 nt) {
    for (u64 k = a + t; k < b; k += nt) {
        u32 p = A.part[A.pins[k]];
        u32 slot = hash_find_or_insert(keys, mask, p);
        if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); continue; }
        atomicMin(&mn[slot], (u32)(k - a));
        atomicAdd(&cnt[slot], 1u);
        if (k >= s) atomicAdd(&dcnt[slot], 1u);
    }
}

__global__ void k_census_warp(u32 e, CensusArgs A) {
    __shared__ u32 tk[CS_WARPS][2 * CS_WARP_CAP], tm[CS_WARPS][2 * CS_WARP_CAP], tc[CS_WARPS][2 * CS_WARP_CAP],
        td[CS_WARPS][2 * CS_WARP_CAP];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 h = blockIdx.x * CS_WARPS + w;
    if (h >= e) return;
    const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
    const u32 len = (u32)(b - a);
    if (len > CS_WARP_CAP) return;
    u32 cap = 32;
    while (cap < 2 * len) cap <<= 1;
    u32 *keys = tk[w], *mn = tm[w], *cnt = tc[w], *dcnt = td[w];
    for (u32 i = lane; i < cap; i += 32) { keys[i] = NONE; mn[i] = NONE; cnt[i] = 0; dcnt[i] = 0; }
    __syncwarp();
    cs_insert(A, a, b, s, keys, mn, cnt, dcnt, cap - 1, lane, 32);
    __syncwarp();
    u32 o = 0;
    for (u64 base = a; base < b; base += 32) {
        u64 k = base + lane;
        u32 slot = NONE, p = 0;
        if (k < b) {
            p = A.part[A.pins[k]];
            slot = hash_find(keys, cap - 1, p);
        }
        if (A.save && slot != NONE)
            atomicAdd(&A.save[A.pins[k]], (unsigned long long)leave_gain(A.encourage, A.wfx[h], cnt[slot]));
        bool first = slot != NONE && mn[slot] == (u32)(k - a);
        u32 bal = __ballot_sync(0xFFFFFFFFu, first);
        if (first) {
            u64 dst = a + o + __popc(bal & ((1u << lane) - 1u));
            A.cpart[dst] = p;
            A.ccnt[dst] = cnt[slot];
            A.cdcnt[dst] = dcnt[slot];
        }
        o += __popc(bal);
    }
    if (lane == 0) A.lam[h] = o;
}

__global__ void k_census_block(const u32 *__restrict__ list, u32 nlist, CensusArgs A, u32 *gtab,
                               const u64 *__restrict__ gtab_off) {
    extern __shared__ u32 dyn[];
    __shared__ u32 wsum[33];
    if (blockIdx.x >= nlist) return;
    const u32 h = list[blockIdx.x];
    const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
    const u32 len = (u32)(b - a);
    const u32 cap = cs_cap(len);
    if (!gtab && 16ull * cap > dyn_smem_bytes()) {  // launched with too small a table: refuse
        if (threadIdx.x == 0) atomicExch(A.status, DEV_HASH_FULL);
        return;
    }
    u32 *keys = gtab ? gtab + 4 * gtab_off[blockIdx.x] : dyn;
    u32 *mn = keys + cap, *cnt = mn + cap, *dcnt = cnt + cap;
    for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = NONE; mn[i] = NONE; cnt[i] = 0; dcnt[i] = 0; }
    __syncthreads();
    cs_insert(A, a, b, s, keys, mn, cnt, dcnt, cap - 1, threadIdx.x, blockDim.x);
    __syncthreads();
    u32 o = 0;  // running count, identical in every thread
    const u32 lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (u64 base = a; base < b; base += blockDim.x) {
        u64 k = base + threadIdx.x;
        u32 slot = NONE, p = 0;
        if (k < b) {
            p = A.part[A.pins[k]];
            slot = hash_find(keys, cap - 1, p);
        }
        if (A.save && slot != NONE)
            atomicAdd(&A.save[A.pins[k]], (unsigned long long)leave_gain(A.encourage, A.wfx[h], cnt[slot]));
        bool first = slot != NONE && mn[slot] == (u32)(k - a);
        u32 bal = __ballot_sync(0xFFFFFFFFu, first);
        if (lane == 0) wsum[w] = __popc(bal);
        __syncthreads();
        u32 before = 0, tot = 0;
        for (u32 i = 0; i < nw; ++i) {
            if (i < w) before += wsum[i];
            tot += wsum[i];
        }
        if (first) {
            u64 dst = a + o + before + __popc(bal & ((1u << lane) - 1u));
            A.cpart[dst] = p;
            A.ccnt[dst] = cnt[slot];
            A.cdcnt[dst] = dcnt[slot];
        }
        o += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) A.lam[h] = o;
}

// Partition-indexed census for K <= CD_K: the counters are K-slot arrays indexed by partition id,
// so a hyperedge of any length fits in shared memory and needs no hashing. Entries are emitted in
// ascending partition order (the hashed census emits them in order of first occurrence; every
// consumer reads them as a set). With A.save set, every pin then adds its saving from the count
// of its own partition.
constexpr u32 CD_K = 256;
constexpr u32 CD_WARP_LEN = 1024;  // longer hyperedges take a block

// Counts of hyperedge h's pins over [t0, len) step nt into cnt / dcnt (shared, zeroed).
__device__ __forceinline__ void cd_count(const CensusArgs &A, u64 a, u64 b, u64 s, u32 *cnt, u32 *dcnt, u32 t0,
                                         u32 nt) {
    for (u64 k = a + t0; k < b; k += nt) {
        const u32 q = A.part[A.pins[k]];
        atomicAdd(&cnt[q], 1u);
        if (k >= s) atomicAdd(&dcnt[q], 1u);
    }
}
// Returns how many savings this thread added.
__device__ __forceinline__ u32 cd_save(const CensusArgs &A, u32 h, u64 a, u64 b, const u32 *cnt, u32 t0, u32 nt) {
    if (!A.save) return 0;
    const u32 w = A.wfx[h];
    u32 added = 0;
    for (u64 k = a + t0; k < b; k += nt) {
        const u32 v = A.pins[k];
        const i64 g = leave_gain(A.encourage, w, cnt[A.part[v]]);
        if (g) {
            atomicAdd(&A.save[v], (unsigned long long)g);
            ++added;
        }
    }
    return added;
}
// One warp: the nonzero counters in ascending partition order, then lam. The ballots of the
// counters are the hyperedge's masks, written when A.mask is set.
// Returns the entries written (lam).
__device__ __forceinline__ u32 cd_emit(const CensusArgs &A, u32 h, u64 a, const u32 *cnt, const u32 *dcnt, u32 K) {
    const u32 lane = threadIdx.x & 31;
    u32 o = 0;
    const u32 qend = A.mask ? 32 * A.mw : K;
    for (u32 qb = 0; qb < qend; qb += 32) {
        const u32 q = qb + lane;
        const u32 c = q < K ? cnt[q] : 0;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, c > 0);
        if (A.mask) {
            const u32 dbal = __ballot_sync(0xFFFFFFFFu, c > 0 && dcnt[q] > 0);
            if (lane == 0) {
                A.mask[(u64)h * A.mw + qb / 32] = bal;
                A.dmask[(u64)h * A.mw + qb / 32] = dbal;
            }
        }
        if (c > 0) {
            const u64 dst = a + o + __popc(bal & ((1u << lane) - 1u));
            A.cpart[dst] = q;
            A.ccnt[dst] = c;
            A.cdcnt[dst] = dcnt[q];
        }
        o += __popc(bal);
    }
    if (lane == 0) A.lam[h] = o;
    return o;
}

__global__ void k_census_direct_warp(u32 e, CensusArgs A, u32 K) {
    __shared__ u32 tc[CS_WARPS][CD_K], td[CS_WARPS][CD_K];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 h = blockIdx.x * CS_WARPS + w;
    if (h >= e) return;
    const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
    if (b - a > CD_WARP_LEN) return;
    u32 *cnt = tc[w], *dcnt = td[w];
    for (u32 i = lane; i < K; i += 32) { cnt[i] = 0; dcnt[i] = 0; }
    __syncwarp();
    cd_count(A, a, b, s, cnt, dcnt, lane, 32);
    __syncwarp();
    const u32 saved = __reduce_add_sync(0xFFFFFFFFu, cd_save(A, h, a, b, cnt, lane, 32));
    const u32 lm = cd_emit(A, h, a, cnt, dcnt, K);
    if (A.pbytes && lane == 0)  // algorithmic bytes (kernel timer): offsets and source count, each
        // pin's id and partition, the entries and their count, the masks, the weight and savings
        prof_add(A.pbytes, h, 20 + 8 * (b - a) + 12ull * lm + 4 + (A.mask ? 8ull * A.mw : 0) +
                                  (A.save ? 4 + 8ull * saved : 0));
}

__global__ void k_census_direct_block(const u32 *__restrict__ list, u32 nlist, CensusArgs A, u32 K) {
    __shared__ u32 cnt[CD_K], dcnt[CD_K];
    for (u32 idx = blockIdx.x; idx < nlist; idx += gridDim.x) {
        const u32 h = list[idx];
        const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
        for (u32 i = threadIdx.x; i < K; i += blockDim.x) { cnt[i] = 0; dcnt[i] = 0; }
        __syncthreads();
        cd_count(A, a, b, s, cnt, dcnt, threadIdx.x, blockDim.x);
        __syncthreads();
        cd_save(A, h, a, b, cnt, threadIdx.x, blockDim.x);
        if (threadIdx.x < 32) cd_emit(A, h, a, cnt, dcnt, K);
        __syncthreads();
    }
}

// ---- incremental partition-indexed census (levels that are not small, K <= CD_K) ---------------
// The level keeps one census across its rounds. Round r recomputes only the hyperedges holding a
// node that moved in round r - 1 (all of them in round 0): their entries, count and masks are
// rewritten, and each pin's saving changes by leave_gain(w, its partition's new count) minus
// leave_gain(w, its partition's count at the previous census). A node's partition at the
// previous census is its current one, unless it moved in round r - 1: then the apply kernel kept
// the old one in prev[] and stamped the move with the round counter. The results are those of a
// census rebuilt from scratch (integer sums, the same entries in the same order).
struct IncArgs {
    const u32 *list, *nlist;   // the hyperedges to recompute
    u32 *work;                 // the warps' work counter (zeroed before the launch)
    const u32 *dirty;          // their flags (the block kernel's filter)
    const u32 *prev, *stamp;   // [n]
    const u32 *ctr;            // rounds run at this level (0 in round 0)
};

// Old counts from the hyperedge's previous entries [a, a + lm) into ocnt (zeroed, K slots).
__device__ __forceinline__ void ci_old_counts(const CensusArgs &A, u64 a, u32 lm, u32 *ocnt, u32 t0, u32 nt) {
    for (u32 j = t0; j < lm; j += nt) ocnt[A.cpart[a + j]] = A.ccnt[a + j];
}
// The savings' change of pins t0, t0 + nt, ... (all of their saving in round 0); returns how many
// this thread added.
__device__ __forceinline__ u32 ci_save(const CensusArgs &A, const IncArgs &I, u32 h, u64 a, u64 b, const u32 *cnt,
                                       const u32 *ocnt, u32 r, u32 t0, u32 nt) {
    const u32 w = A.wfx[h];
    u32 added = 0;
    for (u64 k = a + t0; k < b; k += nt) {
        const u32 v = A.pins[k], p = A.part[v];
        i64 g = leave_gain(A.encourage, w, cnt[p]);
        if (r) {
            const u32 po = I.stamp[v] == r - 1 ? I.prev[v] : p;
            g -= leave_gain(A.encourage, w, ocnt[po]);
        }
        if (g) {
            atomicAdd(&A.save[v], (unsigned long long)g);
            ++added;
        }
    }
    return added;
}

// Listed hyperedges of at most CD_WARP_LEN pins, one warp each; warps take 32 list entries at a
// time from a shared counter.
__global__ void k_census_inc_warp(CensusArgs A, u32 K, IncArgs I) {
    __shared__ u32 tc[CS_WARPS][CD_K], td[CS_WARPS][CD_K], to[CS_WARPS][CD_K];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 nl = *I.nlist, r = *I.ctr;
    u32 *cnt = tc[w], *dcnt = td[w], *ocnt = to[w];
    u64 bytes = 0;  // algorithmic bytes of this warp's hyperedges (kernel timer)
    for (;;) {
        u32 base = 0;
        if (lane == 0) base = atomicAdd(I.work, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= nl) break;
        const u32 end = base + 32 < nl ? base + 32 : nl;
        for (u32 idx = base; idx < end; ++idx) {
            const u32 h = I.list[idx];
            const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
            if (b - a > CD_WARP_LEN) continue;  // the block kernel's
            const u32 lm_old = r ? A.lam[h] : 0;
            __syncwarp();  // the previous hyperedge's tables are no longer read
            for (u32 i = lane; i < K; i += 32) { cnt[i] = 0; dcnt[i] = 0; ocnt[i] = 0; }
            __syncwarp();
            if (r) ci_old_counts(A, a, lm_old, ocnt, lane, 32);
            cd_count(A, a, b, s, cnt, dcnt, lane, 32);
            __syncwarp();  // old entries read, counts complete, before the entries are rewritten
            const u32 saved = __reduce_add_sync(0xFFFFFFFFu, ci_save(A, I, h, a, b, cnt, ocnt, r, lane, 32));
            const u32 lm = cd_emit(A, h, a, cnt, dcnt, K);
            // the list entry, offsets and source count, each pin's id, partition (and move stamp),
            // the old entries, the new entries and their count, the masks, the weight and savings
            bytes += 24 + 12 * (b - a) + 8ull * lm_old + 12ull * lm + 4 + (A.mask ? 8ull * A.mw : 0) + 4 +
                     8ull * saved;
        }
    }
    if (A.pbytes && lane == 0 && bytes) prof_add(A.pbytes, blockIdx.x * CS_WARPS + w, bytes);
}

// Hyperedges of more than CD_WARP_LEN pins (the level's block list), one block each, when flagged.
__global__ void k_census_inc_block(const u32 *__restrict__ list, u32 nlist, CensusArgs A, u32 K, IncArgs I) {
    __shared__ u32 cnt[CD_K], dcnt[CD_K], ocnt[CD_K];
    const u32 r = *I.ctr;
    for (u32 idx = blockIdx.x; idx < nlist; idx += gridDim.x) {
        const u32 h = list[idx];
        if (!I.dirty[h]) continue;  // uniform over the block
        const u64 a = A.off[h], b = A.off[h + 1], s = a + A.nsrc[h];
        const u32 lm_old = r ? A.lam[h] : 0;
        for (u32 i = threadIdx.x; i < K; i += blockDim.x) { cnt[i] = 0; dcnt[i] = 0; ocnt[i] = 0; }
        __syncthreads();
        if (r) ci_old_counts(A, a, lm_old, ocnt, threadIdx.x, blockDim.x);
        cd_count(A, a, b, s, cnt, dcnt, threadIdx.x, blockDim.x);
        __syncthreads();
        ci_save(A, I, h, a, b, cnt, ocnt, r, threadIdx.x, blockDim.x);
        __syncthreads();  // every thread has read lam and the old entries
        if (threadIdx.x < 32) cd_emit(A, h, a, cnt, dcnt, K);
        __syncthreads();
    }
}

// After the apply: the hyperedges of the nodes this round moved (stamped with the round counter)
// are flagged for the next round's census. One warp per mover.
__global__ void k_mark_moved(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u32 *__restrict__ stamp,
                             const u32 *__restrict__ ctr, const u64 *__restrict__ toff, const u32 *__restrict__ touch,
                             u32 *__restrict__ dirty) {
    const u32 lane = threadIdx.x & 31u, nw = (gridDim.x * blockDim.x) >> 5;
    const u32 M = *dM, r = *ctr;
    for (u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < M; i += nw) {
        const u32 v = mv[i];
        if (stamp[v] != r) continue;  // not applied this round
        for (u64 j = toff[v] + lane; j < toff[v + 1]; j += 32) dirty[touch[j]] = 1u;
    }
}
__global__ void k_round_tick(u32 *ctr) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctr[0] += 1;
}

__global__ void k_flag_len(u32 e, const u64 *__restrict__ off, u64 lo, u64 hi, u32 *__restrict__ flag) {
    u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < e) {
        u64 l = off[h + 1] - off[h];
        flag[h] = (l > lo && l <= hi) ? 1u : 0u;
    }
}
__global__ void k_tab_sizes(const u32 *__restrict__ list, u32 nl, const u64 *__restrict__ off, u64 *__restrict__ sz) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == nl) sz[i] = 0;
    if (i >= nl) return;
    u32 h = list[i];
    u64 len = off[h + 1] - off[h], cap = 32;
    while (cap < 2 * len) cap <<= 1;
    sz[i] = cap;
}

__global__ void k_part_sizes(u32 n, const u32 *__restrict__ part, const u32 *__restrict__ nsize,
                             unsigned long long *__restrict__ ps) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) atomicAdd(&ps[part[v]], (unsigned long long)nsize[v]);
}
// Few partitions (K <= PS_SMEM_K): per-block sums in shared memory, one global add per partition
// and block, over a grid-stride range (every node's global atomic would hit the same K words).
constexpr u32 PS_SMEM_K = 1024;
__global__ void k_part_sizes_smem(u32 n, u32 K, const u32 *__restrict__ part, const u32 *__restrict__ nsize,
                                  unsigned long long *__restrict__ ps) {
    __shared__ unsigned long long sh[PS_SMEM_K];
    for (u32 i = threadIdx.x; i < K; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (u32 v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const u32 q = part[v];
        if (q < K) atomicAdd(&sh[q], (unsigned long long)nsize[v]);  // ids are below K by contract
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < K; i += blockDim.x)
        if (sh[i]) atomicAdd(&ps[i], sh[i]);
}
__global__ void k_part_inbound(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ lam,
                               const u32 *__restrict__ cpart, const u32 *__restrict__ cdcnt,
                               unsigned long long *__restrict__ pinb) {
    const u32 h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (h >= e) return;
    const u64 a = off[h];
    for (u32 j = lane; j < lam[h]; j += 32)
        if (cdcnt[a + j] > 0) atomicAdd(&pinb[cpart[a + j]], 1ull);
}

constexpr u32 PI_SMEM_K = 8192;
// k_part_inbound for K <= PI_SMEM_K: warps stride over the hyperedges and count into a shared
// histogram, which the block adds to pinb once; this avoids contended global atomics on few
// partitions.
__global__ void k_part_inbound_smem(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ lam,
                                    const u32 *__restrict__ cpart, const u32 *__restrict__ cdcnt, u32 K,
                                    unsigned long long *__restrict__ pinb) {
    extern __shared__ u32 hist[];
    for (u32 i = threadIdx.x; i < K; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const u32 lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (u32 h = blockIdx.x * nw + (threadIdx.x >> 5); h < e; h += gridDim.x * nw) {
        const u64 a = off[h];
        const u32 lm = lam[h];
        for (u32 j = lane; j < lm; j += 32)
            if (cdcnt[a + j] > 0) atomicAdd(&hist[cpart[a + j]], 1u);
    }
    __syncthreads();
    for (u32 i = threadIdx.x; i < K; i += blockDim.x)
        if (hist[i]) atomicAdd(&pinb[i], (unsigned long long)hist[i]);
}

// ------------------------------------------------------------------ gains
struct GainArgs {
    u32 n, omega, delta, discount, round;
    u32 seed;
    int encourage;
    const u64 *off;
    const u32 *lam, *cpart, *ccnt, *cdcnt, *wfx;
    const u32 *pins, *nsrc;  // the level's hyperedges (pin-centric passes)
    const u64 *toff;
    const u32 *touch, *nin, *nsize, *part;
    const u64 *psize, *pinb;
    u32 *target;
    i64 *gain;
    u32 *status;
    const u32 *dyn;  // when set: discount and round read from device memory (graph replays)
    const i64 *save; // partition-indexed gains: each node's saving from leaving its partition
    u32 K;           // partitions: with K <= GN_DIRECT_K the tables are indexed by partition id
};

constexpr u32 GN_DIRECT_K = 256;

// Slots of a node's table: K (rounded up) when indexed by partition id, else from its work bound.
// Rounds with K <= GN_DIRECT_K take the mask kernels (k_gain_mask_*); the partition-indexed
// branches of the table kernels below are kept so that those kernels stay correct for any K.
__device__ __forceinline__ bool gain_direct(const GainArgs &A) { return A.K <= GN_DIRECT_K; }
__device__ __forceinline__ u32 gain_cap(const GainArgs &A, u64 work, u32 cap_max) {
    u32 cap = 32;
    if (gain_direct(A)) {
        while (cap < A.K) cap <<= 1;
        return cap;
    }
    while (cap < 2 * work && cap < cap_max) cap <<= 1;
    return cap;
}

// The launch's arguments with the per-round scalars resolved.
__device__ __forceinline__ GainArgs gain_args_now(const GainArgs &A0) {
    GainArgs A = A0;
    if (A0.dyn) {
        A.discount = A0.dyn[0];
        A.round = A0.dyn[1];
    }
    return A;
}

// Per-level bounds of a node's gain work: the partitions adjacent to it in any round number at
// most min(sum over incident hyperedges of min(|e|, K), K), which sizes its accumulator table; the
// sum of incident weights bounds its gain.
__global__ void k_gain_bounds(u32 n, u32 K, const u64 *__restrict__ toff, const u32 *__restrict__ touch,
                              const u64 *__restrict__ off, const u32 *__restrict__ wfx, u64 *__restrict__ work,
                              unsigned long long *__restrict__ wmax) {
    const u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (u >= n) return;
    u64 s = 0, ws = 0;
    for (u64 j = toff[u] + lane; j < toff[u + 1]; j += 32) {
        u32 h = touch[j];
        u64 len = off[h + 1] - off[h];
        s += len < K ? len : K;
        ws += wfx[h];
    }
    s = warp_sum(s);
    ws = warp_sum(ws);
    if (lane == 0) {
        work[u] = s < K ? s : K;
        atomicMax(wmax, (unsigned long long)ws);
    }
}
__host__ __device__ __forceinline__ u32 table_cap(u64 work, u32 cap_max) {
    u32 cap = 32;
    while (cap < 2 * work && cap < cap_max) cap <<= 1;
    return cap;
}

// Accumulate node u's adjacency to other partitions into (keys, conn, dconn). Warp-cooperative:
// the calling warp takes the node's incidences in batches of 32 starting at `first`, every
// `stride` entries. A batch's hyperedge metadata loads in parallel; its census entries are then
// flattened across the lanes (each lane finds its entry's hyperedge by a 5-step search over the
// prefix of the batch's lambdas). saving and wtot are per-lane partial sums.
//
// With `trk` the block counts the distinct partitions it inserts. In a first try (limit below the
// table size) passing the limit, or a full table, sets *ovf and the warps stop at their next batch;
// the caller retries the node with a larger table. With trk->used the inserted slots are listed,
// so the caller can scan and clear only those.
struct GainTrack {
    u32 *ndist;
    u32 limit;
    volatile u32 *ovf;
    u32 *used;
};
__device__ __forceinline__ void gain_flat(const GainArgs &A, u32 u, u32 p, u32 *keys, unsigned long long *conn,
                                          u32 *dconn, u32 mask, u32 first, u32 stride, i64 &saving, i64 &wtot,
                                          const GainTrack *trk = nullptr) {
    const u32 lane = threadIdx.x & 31u;
    const u64 t0 = A.toff[u];
    const u32 deg = (u32)(A.toff[u + 1] - t0), nin_u = A.nin[u];
    for (u32 jb = first; jb < deg; jb += stride) {
        if (trk && __any_sync(0xFFFFFFFFu, *trk->ovf != 0)) return;
        const u32 j = jb + lane;
        const bool has = j < deg;
        const u32 h = has ? A.touch[t0 + j] : 0;
        const u32 lm = has ? A.lam[h] : 0;
        const u32 wh = has ? A.wfx[h] : 0;
        const u64 ah = has ? A.off[h] : 0;
        const u32 ib = (has && j < nin_u) ? 1u : 0u;
        wtot += wh;
        u32 x = lm;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if ((int)lane >= o) x += y;
        }
        const u32 total = __shfl_sync(0xFFFFFFFFu, x, 31), excl = x - lm;
        const u32 chunk = (deg - jb) < 32 ? (deg - jb) : 32;
        for (u32 fb = 0; fb < total; fb += 32) {
            const u32 f = fb + lane;
            u32 lo = 0, hi = chunk - 1;
            for (int it = 0; it < 5; ++it) {
                const u32 mid = (lo + hi + 1) >> 1;
                const u32 em = __shfl_sync(0xFFFFFFFFu, excl, mid & 31);
                if (lo < hi) { if (em <= f) lo = mid; else hi = mid - 1; }
            }
            const u32 eo = __shfl_sync(0xFFFFFFFFu, excl, lo);
            const u64 ao = __shfl_sync(0xFFFFFFFFu, ah, lo);
            const u32 wo = __shfl_sync(0xFFFFFFFFu, wh, lo);
            const u32 io = __shfl_sync(0xFFFFFFFFu, ib, lo);
            if (f >= total) continue;
            const u64 k = ao + (f - eo);
            const u32 q = A.cpart[k];
            if (q == p) {
                saving += leave_gain(A.encourage, wo, A.ccnt[k]);
                continue;
            }
            u32 slot;
            if (gain_direct(A)) {  // the slot is the partition id: no probing
                slot = q;
                keys[q] = q;
            } else if (trk) {
                bool fresh;
                slot = hash_insert_fresh(keys, mask, q, fresh);
                if (slot == NONE) {  // full: a first try overflows, a sized table is an error
                    if (trk->limit <= mask) *trk->ovf = 1u;
                    else atomicExch(A.status, DEV_HASH_FULL);
                    continue;
                }
                if (fresh) {
                    const u32 idx = atomicAdd(trk->ndist, 1u);
                    if (trk->used) trk->used[idx] = slot;
                    if (idx >= trk->limit) *trk->ovf = 1u;
                }
            } else {
                slot = hash_find_or_insert(keys, mask, q);
                if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); continue; }
            }
            atomicAdd(&conn[slot], (unsigned long long)wo);
            if (io && A.cdcnt[k] > 0) atomicAdd(&dconn[slot], 1u);
        }
    }
}

// candidate key: the larger wins. (gain, tie-hash, -id) packed into two u64 words.
struct Cand {
    i64 g;
    u64 tie;  // hash << 32 | ~q
};
__device__ __forceinline__ bool cand_better(const Cand &x, const Cand &y) {
    return x.g > y.g || (x.g == y.g && x.tie > y.tie);
}

__device__ __forceinline__ Cand gain_candidate(const GainArgs &A, u32 u, u32 q, u64 cw, u32 dc, i64 saving,
                                               i64 wtot) {
    Cand c{INT64_MIN, 0};
    const u64 s = A.nsize[u];
    if (A.psize[q] + s - s / A.discount > A.omega) return c;
    if (A.pinb[q] + (u64)(A.nin[u] - dc) > A.delta) return c;
    c.g = saving - (wtot - (i64)cw);
    c.tie = ((u64)mix32(q + A.round + A.seed) << 32) | (u64)(~q);
    return c;
}

__device__ __forceinline__ Cand warp_best(Cand c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Cand d;
        d.g = __shfl_xor_sync(0xFFFFFFFFu, c.g, o);
        d.tie = __shfl_xor_sync(0xFFFFFFFFu, c.tie, o);
        if (cand_better(d, c)) c = d;
    }
    return c;
}

constexpr u32 GN_WARP_W = 128;
constexpr u32 GN_WARPS = 4;
constexpr u32 GN_BLOCK = 256;
constexpr u32 GN_BLOCK_W = 4096;
constexpr u32 GN_WARP_DEG = 256;      // incidences one warp takes; more go to a block
constexpr u32 GN_SMALL_LEVEL = 1024;  // levels with at most this many nodes use blocks only
constexpr u32 GM_WARP_DEG = 4096;     // incidences one warp takes in the mask gains; more go to a block

// ------------------------------------------------------------------ partition-indexed gains
// For K <= GN_DIRECT_K a hyperedge's census is also kept as two K-bit masks of MW words: the
// partitions present, and those holding destination pins. A node's table is then MW registers
// per lane (lane l owns partitions l, l + 32, ...), so an incidence costs O(MW) per lane whatever
// its lambda, against lambda hash updates in the general path. The node's saving from leaving
// its own partition comes from the census pass (Census::save); candidates, connectivity and the
// inbound count per candidate are the same quantities the general path accumulates.
__global__ void k_census_masks(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ lam,
                               const u32 *__restrict__ cpart, const u32 *__restrict__ cdcnt, u32 MW,
                               u32 *__restrict__ mask, u32 *__restrict__ dmask) {
    const u32 h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (h >= e) return;
    const u64 a = off[h];
    const u32 lm = lam[h];
    u32 mw[8], dw[8];
#pragma unroll
    for (u32 k = 0; k < 8; ++k) mw[k] = dw[k] = 0;
    for (u32 j = lane; j < lm; j += 32) {
        const u32 q = cpart[a + j], bit = 1u << (q & 31), wd = q >> 5;
        const bool d = cdcnt[a + j] > 0;
#pragma unroll
        for (u32 k = 0; k < 8; ++k)
            if (k == wd) {
                mw[k] |= bit;
                if (d) dw[k] |= bit;
            }
    }
#pragma unroll
    for (u32 k = 0; k < 8; ++k) {
        if (k < MW) {
            const u32 m = __reduce_or_sync(0xFFFFFFFFu, mw[k]), d = __reduce_or_sync(0xFFFFFFFFu, dw[k]);
            if (lane == 0) {
                mask[(u64)h * MW + k] = m;
                dmask[(u64)h * MW + k] = d;
            }
        }
    }
}

template <u32 MW>
__device__ __forceinline__ void load_words(const u32 *p, u32 (&w)[MW]) {
    if constexpr (MW == 1) {
        w[0] = *p;
    } else if constexpr (MW == 2) {
        const uint2 v = *(const uint2 *)p;
        w[0] = v.x; w[1] = v.y;
    } else {
#pragma unroll
        for (u32 k = 0; k < MW; k += 4) {
            const uint4 v = *(const uint4 *)(p + k);
            w[k] = v.x; w[k + 1] = v.y; w[k + 2] = v.z; w[k + 3] = v.w;
        }
    }
}
template <u32 MW>
__device__ __forceinline__ void store_words(u32 *p, const u32 (&w)[MW]) {
    if constexpr (MW == 1) {
        *p = w[0];
    } else if constexpr (MW == 2) {
        *(uint2 *)p = make_uint2(w[0], w[1]);
    } else {
#pragma unroll
        for (u32 k = 0; k < MW; k += 4) *(uint4 *)(p + k) = make_uint4(w[k], w[k + 1], w[k + 2], w[k + 3]);
    }
}

template <u32 MW>
struct MaskAcc {
    unsigned long long conn[MW];  // this lane's partitions: summed weights of incidences holding them
    u32 dconn[MW];                // inbound incidences with destination pins in them
    u32 pres[MW];                 // OR of the mask words seen (bit `lane` of word k: partition lane + 32k)
};

// Accumulate node u's incidences first, first + stride, ... in batches of 32 (one warp). Each
// batch stages its masks in the warp's shared slots (sm, sd, sw: 32 entries), which every lane
// then reads as broadcasts.
template <u32 MW>
__device__ __forceinline__ void gain_mask_acc(const GainArgs &A, const u32 *__restrict__ mask,
                                              const u32 *__restrict__ dmask, u32 u, u32 first, u32 stride,
                                              u32 (*sm)[MW], u32 (*sd)[MW], u32 *sw, MaskAcc<MW> &acc, i64 &wtot) {
    const u32 lane = threadIdx.x & 31u;
    const u64 t0 = A.toff[u];
    const u32 deg = (u32)(A.toff[u + 1] - t0), nin_u = A.nin[u];
    for (u32 jb = first; jb < deg; jb += stride) {
        const u32 j = jb + lane;
        const bool has = j < deg;
        const u32 h = has ? A.touch[t0 + j] : 0;
        const u32 wh = has ? A.wfx[h] : 0;
        wtot += wh;
        u32 mw[MW], dw[MW];
#pragma unroll
        for (u32 k = 0; k < MW; ++k) mw[k] = dw[k] = 0;
        if (has) load_words<MW>(mask + (u64)h * MW, mw);
        if (has && j < nin_u) load_words<MW>(dmask + (u64)h * MW, dw);
        store_words<MW>(sm[lane], mw);
        store_words<MW>(sd[lane], dw);
        sw[lane] = wh;
        __syncwarp();
        const u32 chunk = (deg - jb) < 32 ? (deg - jb) : 32;
        for (u32 t = 0; t < chunk; ++t) {
            const u32 wt = sw[t];
            u32 mk[MW], dk[MW];
            load_words<MW>(sm[t], mk);
            load_words<MW>(sd[t], dk);
#pragma unroll
            for (u32 k = 0; k < MW; ++k) {
                if ((mk[k] >> lane) & 1u) acc.conn[k] += wt;
                acc.dconn[k] += (dk[k] >> lane) & 1u;
                acc.pres[k] |= mk[k];
            }
        }
        __syncwarp();
    }
}

template <u32 MW>
__device__ __forceinline__ Cand mask_best(const GainArgs &A, u32 u, u32 p, const MaskAcc<MW> &acc, i64 saving,
                                          i64 wtot) {
    const u32 lane = threadIdx.x & 31u;
    Cand best{INT64_MIN, 0};
#pragma unroll
    for (u32 k = 0; k < MW; ++k) {
        const u32 q = lane + 32 * k;
        if (q < A.K && q != p && ((acc.pres[k] >> lane) & 1u)) {
            const Cand c = gain_candidate(A, u, q, acc.conn[k], acc.dconn[k], saving, wtot);
            if (cand_better(c, best)) best = c;
        }
    }
    return warp_best(best);
}

__device__ __forceinline__ void write_move(const GainArgs &A, u32 u, const Cand &b) {
    if (b.g != INT64_MIN && b.g > 0) {
        A.target[u] = ~(u32)b.tie;
        A.gain[u] = b.g;
    } else {
        A.target[u] = NONE;
        A.gain[u] = 0;
    }
}

// One warp per node.
template <u32 MW>
__global__ void __launch_bounds__(GN_WARPS * 32) k_gain_mask_warp(GainArgs A0, const u32 *__restrict__ list, u32 nl,
                                                                 const u32 *__restrict__ mask,
                                                                 const u32 *__restrict__ dmask) {
    const GainArgs A = gain_args_now(A0);
    __shared__ __align__(16) u32 sm[GN_WARPS][32][MW], sd[GN_WARPS][32][MW];
    __shared__ u32 sw[GN_WARPS][32];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 idx = blockIdx.x * GN_WARPS + w;
    if (idx >= nl) return;
    const u32 u = list[idx], p = A.part[u];
    MaskAcc<MW> acc;
#pragma unroll
    for (u32 k = 0; k < MW; ++k) { acc.conn[k] = 0; acc.dconn[k] = 0; acc.pres[k] = 0; }
    i64 wtot = 0;
    gain_mask_acc<MW>(A, mask, dmask, u, 0, 32, sm[w], sd[w], sw[w], acc, wtot);
    wtot = warp_sum(wtot);
    const Cand best = mask_best<MW>(A, u, p, acc, A.save[u], wtot);
    if (lane == 0) write_move(A, u, best);
}

// One block per node (its warps split the incidences), for heavy nodes and small levels; the
// warps' tables are summed in shared memory.
template <u32 MW>
__global__ void __launch_bounds__(GN_BLOCK) k_gain_mask_block(GainArgs A0, const u32 *__restrict__ list, u32 nl,
                                                             const u32 *__restrict__ mask,
                                                             const u32 *__restrict__ dmask) {
    constexpr u32 NW = GN_BLOCK / 32;
    const GainArgs A = gain_args_now(A0);
    __shared__ __align__(16) u32 sm[NW][32][MW], sd[NW][32][MW];
    __shared__ u32 sw[NW][32];
    __shared__ unsigned long long rc[MW][32];
    __shared__ u32 rd[MW][32], rp[MW];
    __shared__ i64 rw[NW];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (u32 i = threadIdx.x; i < MW * 32; i += blockDim.x) { rc[i / 32][i % 32] = 0; rd[i / 32][i % 32] = 0; }
    if (threadIdx.x < MW) rp[threadIdx.x] = 0;
    __syncthreads();
    for (u32 idx = blockIdx.x; idx < nl; idx += gridDim.x) {
        const u32 u = list[idx], p = A.part[u];
        MaskAcc<MW> acc;
#pragma unroll
        for (u32 k = 0; k < MW; ++k) { acc.conn[k] = 0; acc.dconn[k] = 0; acc.pres[k] = 0; }
        i64 wtot = 0;
        gain_mask_acc<MW>(A, mask, dmask, u, 32 * w, GN_BLOCK, sm[w], sd[w], sw[w], acc, wtot);
        wtot = warp_sum(wtot);
#pragma unroll
        for (u32 k = 0; k < MW; ++k) {
            if (acc.conn[k]) atomicAdd(&rc[k][lane], acc.conn[k]);
            if (acc.dconn[k]) atomicAdd(&rd[k][lane], acc.dconn[k]);
            if (lane == 0 && acc.pres[k]) atomicOr(&rp[k], acc.pres[k]);
        }
        if (lane == 0) rw[w] = wtot;
        __syncthreads();
        if (w == 0) {
#pragma unroll
            for (u32 k = 0; k < MW; ++k) {
                acc.conn[k] = rc[k][lane];
                acc.dconn[k] = rd[k][lane];
                acc.pres[k] = rp[k];
            }
            wtot = 0;
            for (u32 i = 0; i < NW; ++i) wtot += rw[i];
            const Cand best = mask_best<MW>(A, u, p, acc, A.save[u], wtot);
            if (lane == 0) write_move(A, u, best);
        }
        __syncthreads();  // warp 0 has read the sums: clear them for the next node
        for (u32 i = threadIdx.x; i < MW * 32; i += blockDim.x) { rc[i / 32][i % 32] = 0; rd[i / 32][i % 32] = 0; }
        if (threadIdx.x < MW) rp[threadIdx.x] = 0;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(GN_WARPS * 32) k_gain_warp(GainArgs A0, const u32 *__restrict__ list, u32 nl,
                                                             const u64 *__restrict__ work) {
    const GainArgs A = gain_args_now(A0);
    __shared__ u32 tk[GN_WARPS][2 * GN_WARP_W], td[GN_WARPS][2 * GN_WARP_W];
    __shared__ unsigned long long tcw[GN_WARPS][2 * GN_WARP_W];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 idx = blockIdx.x * GN_WARPS + w;
    if (idx >= nl) return;
    const u32 u = list[idx], p = A.part[u];
    u32 *keys = tk[w], *dconn = td[w];
    unsigned long long *conn = tcw[w];
    const u32 cap = gain_cap(A, work[u], 2 * GN_WARP_W);
    for (u32 i = lane; i < cap; i += 32) { keys[i] = NONE; dconn[i] = 0; conn[i] = 0; }
    __syncwarp();
    i64 saving = 0, wtot = 0;
    gain_flat(A, u, p, keys, conn, dconn, cap - 1, 0, 32, saving, wtot);
    saving = warp_sum(saving);
    wtot = warp_sum(wtot);
    __syncwarp();
    Cand best{INT64_MIN, 0};
    for (u32 i = lane; i < cap; i += 32) {
        if (keys[i] == NONE) continue;
        Cand c = gain_candidate(A, u, keys[i], conn[i], dconn[i], saving, wtot);
        if (cand_better(c, best)) best = c;
    }
    best = warp_best(best);
    if (lane == 0) {
        if (best.g != INT64_MIN && best.g > 0) {
            A.target[u] = ~(u32)best.tie;
            A.gain[u] = best.g;
        } else {
            A.target[u] = NONE;
            A.gain[u] = 0;
        }
    }
}

// One block per node. Three table modes:
// - shared, sized (gtab null, try_limit 0): the node's table bound fits in shared memory;
// - shared, first try (try_limit > 0): a cap_max-slot shared table for nodes whose bound does not
//   fit; a node with more than try_limit distinct partitions is appended to retry / *nretry;
// - global (gtab set): this block's slice of gtab, sized by the bound. Inserted slots are listed
//   in this block's slice of gused, so candidates are read from and cleared in those slots only;
//   the slice is cleared once at the start.
// With dnl set, the node count is read from device memory.
__global__ void __launch_bounds__(GN_BLOCK) k_gain_block(GainArgs A0, const u32 *__restrict__ list, u32 nl,
                                                        const u32 *__restrict__ dnl, u32 cap_max, u32 *gtab,
                                                        u32 *gused, const u64 *__restrict__ work, u32 try_limit,
                                                        u32 *__restrict__ retry, u32 *__restrict__ nretry) {
    const GainArgs A = gain_args_now(A0);
    extern __shared__ unsigned long long dyn64[];
    __shared__ i64 red[2][32];
    __shared__ Cand cred[32];
    __shared__ u32 ndist, ovf;
    if (dnl) nl = *dnl;
    // this block's global slice: conn u64 [cap_max], keys and dconn u32 [cap_max]; a node uses
    // the first `cap` slots of each, and leaves every slot empty again when it is done
    u32 *gbase = gtab ? gtab + (u64)blockIdx.x * 4 * cap_max : nullptr;
    u32 *used = gtab ? gused + (u64)blockIdx.x * cap_max : nullptr;
    if (gtab && blockIdx.x < nl) {
        for (u32 i = threadIdx.x; i < 2 * cap_max; i += blockDim.x) gbase[i] = 0;
        for (u32 i = threadIdx.x; i < cap_max; i += blockDim.x) { gbase[2 * cap_max + i] = NONE; gbase[3 * cap_max + i] = 0; }
    }
    for (u32 idx = blockIdx.x; idx < nl; idx += gridDim.x) {
        const u32 u = list[idx], p = A.part[u];
        unsigned long long *conn;
        u32 *keys, *dconn;
        const u32 cap = try_limit ? cap_max : gain_cap(A, work[u], cap_max);
        if (gtab) {
            conn = (unsigned long long *)gbase;
            keys = gbase + 2 * cap_max;
            dconn = keys + cap_max;
        } else {
            conn = dyn64;
            keys = (u32 *)(dyn64 + cap);
            dconn = keys + cap;
            for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = NONE; dconn[i] = 0; conn[i] = 0; }
        }
        if (threadIdx.x == 0) { ndist = 0; ovf = 0; }
        __syncthreads();
        const bool track = (try_limit || gtab) && !gain_direct(A);
        const GainTrack trk{&ndist, try_limit ? try_limit : cap, &ovf, used};
        i64 saving = 0, wtot = 0;
        gain_flat(A, u, p, keys, conn, dconn, cap - 1, 32 * (threadIdx.x >> 5), blockDim.x, saving, wtot,
                  track ? &trk : nullptr);
        saving = warp_sum(saving);
        wtot = warp_sum(wtot);
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = saving; red[1][threadIdx.x >> 5] = wtot; }
        __syncthreads();
        if (ovf) {  // first try overflowed: the global tier takes the node
            if (threadIdx.x == 0) retry[atomicAdd(nretry, 1u)] = u;
            __syncthreads();
            continue;
        }
        saving = 0;
        wtot = 0;
        for (u32 i = 0; i < blockDim.x / 32; ++i) { saving += red[0][i]; wtot += red[1][i]; }
        Cand best{INT64_MIN, 0};
        const bool listed = track && used;
        const u32 nscan = listed ? ndist : cap;
        for (u32 t = threadIdx.x; t < nscan; t += blockDim.x) {
            const u32 i = listed ? used[t] : t;
            if (keys[i] == NONE) continue;
            Cand c = gain_candidate(A, u, keys[i], conn[i], dconn[i], saving, wtot);
            if (cand_better(c, best)) best = c;
        }
        if (gtab) {
            __syncthreads();  // every candidate is read before the slots are emptied
            for (u32 t = threadIdx.x; t < nscan; t += blockDim.x) {
                const u32 i = listed ? used[t] : t;
                keys[i] = NONE;
                conn[i] = 0;
                dconn[i] = 0;
            }
        }
        best = warp_best(best);
        if ((threadIdx.x & 31) == 0) cred[threadIdx.x >> 5] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            Cand b = cred[0];
            for (u32 i = 1; i < blockDim.x / 32; ++i)
                if (cand_better(cred[i], b)) b = cred[i];
            if (b.g != INT64_MIN && b.g > 0) {
                A.target[u] = ~(u32)b.tie;
                A.gain[u] = b.g;
            } else {
                A.target[u] = NONE;
                A.gain[u] = 0;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ sampled gains (K > AXC_SPARSE_GAIN_K)
// With more partitions than AXC_SPARSE_GAIN_K a heavy node's adjacent partitions number in the
// tens of thousands and no per-node table fits on chip. Its gains follow the sampled rule of
// include/axc.h in two kernels:
//  - k_gain_sample (one block per node, the sample table in shared memory) finds the sample
//    prefix, accumulates the sampled connectivity and, when the prefix is the whole node, settles
//    the node exactly as k_gain_block would; otherwise it writes the node's candidates;
//  - k_cands_warp / k_cands_block (one warp or block per hyperedge holding such a node) put the
//    hyperedge's census in a hash table and add, for each such pin, the hyperedge's weight to its
//    candidates' sums, and k_cands_best picks each node's best feasible candidate. A node's exact
//    pass so costs its incidences times GS_C + 1 lookups, not its whole census.
constexpr u32 GS_K = AXC_SPARSE_GAIN_K;
constexpr u32 GS_SAMPLE = AXC_SPARSE_GAIN_SAMPLE;
constexpr u32 GS_C = AXC_SPARSE_GAIN_CANDIDATES;
constexpr u32 GS_TAB = 2 * GS_SAMPLE;                // sample table slots: at most half full
constexpr u32 GS_BLOCK = 256;
constexpr u32 GS_PER_SM = 2;                         // resident sample blocks per SM
constexpr u32 GS_DC_BITS = 13;                       // a slot's inbound count (<= GS_SAMPLE) in its low bits
constexpr u64 GS_DC_MASK = (1ull << GS_DC_BITS) - 1;
constexpr u64 GS_RULED_OUT = 1ull << 63;             // slot mark: the size or inbound bound rules it out
static_assert(GS_SAMPLE <= GS_DC_MASK && GS_DC_BITS + 32 + 13 <= 64 && GS_SAMPLE <= 8192,
              "packed slot: inbound count below the connectivity (<= GS_SAMPLE u32 weights)");
static_assert(GS_TAB <= 65536, "used-slot list holds 16-bit slots");
constexpr size_t GS_SMEM = (size_t)GS_TAB * 12 + (size_t)GS_SAMPLE * 2;  // packed u64 and key u32 per
                                                     // slot; the used-slot list (u16)
// Nodes outside the sampled kernels (gain tiers 0 and 1) have at most GN_BLOCK_W census entries,
// so their sample would be the whole node and the exact kernels give the rule's result.
static_assert(GN_BLOCK_W <= GS_SAMPLE, "tier-1 nodes must fit the sample");

// The census entries [ao, ao + lo) of one hyperedge read by the whole calling warp, CF_UNROLL
// independent loads in flight per lane: f(k, cpart[k], w, inbound) for each entry k.
constexpr u32 CF_UNROLL = 8;
template <class F>
__device__ __forceinline__ void census_edge_warp(const GainArgs &A, u64 ao, u32 lo, u32 w, u32 io, F &&f) {
    const u32 lane = threadIdx.x & 31u;
    for (u32 i0 = 0; i0 < lo; i0 += 32 * CF_UNROLL) {
        u32 x[CF_UNROLL];
#pragma unroll
        for (u32 r = 0; r < CF_UNROLL; ++r) {
            const u32 i = i0 + 32 * r + lane;
            x[r] = i < lo ? A.cpart[ao + i] : NONE;
        }
#pragma unroll
        for (u32 r = 0; r < CF_UNROLL; ++r) {
            const u32 i = i0 + 32 * r + lane;
            if (i < lo) f(ao + i, x[r], w, io);
        }
    }
}

// Census entries of u's incidences j = first, first + stride, ... below jend, flattened across the
// calling warp's lanes in batches of 32 incidences (the scheme of gain_flat): f(k, cpart[k], w,
// inbound) is called for each entry k, and every incidence adds its weight to wtot once (per
// lane). A batch whose entries average CF_LONG or more per incidence is read one hyperedge at a
// time by the whole warp instead (coalesced, no search). The calls are the same set either way.
constexpr u32 CF_LONG = 16;
template <class F>
__device__ __forceinline__ void census_flat(const GainArgs &A, u32 u, u32 first, u32 stride, u32 jend, i64 &wtot,
                                            F &&f) {
    const u32 lane = threadIdx.x & 31u;
    const u64 t0 = A.toff[u];
    const u32 nin_u = A.nin[u];
    for (u32 jb = first; jb < jend; jb += stride) {
        const u32 j = jb + lane;
        const bool has = j < jend;
        const u32 h = has ? A.touch[t0 + j] : 0;
        const u32 lm = has ? A.lam[h] : 0;
        const u32 wh = has ? A.wfx[h] : 0;
        const u64 ah = has ? A.off[h] : 0;
        const u32 ib = (has && j < nin_u) ? 1u : 0u;
        wtot += wh;
        u32 x = lm;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if ((int)lane >= o) x += y;
        }
        const u32 total = __shfl_sync(0xFFFFFFFFu, x, 31), excl = x - lm;
        const u32 chunk = (jend - jb) < 32 ? (jend - jb) : 32;
        if (total >= 32 * CF_LONG) {  // long lists: the warp reads one hyperedge's entries at a time
            for (u32 t = 0; t < chunk; ++t) {
                const u64 ao = __shfl_sync(0xFFFFFFFFu, ah, t);
                const u32 lo = __shfl_sync(0xFFFFFFFFu, lm, t), wo = __shfl_sync(0xFFFFFFFFu, wh, t);
                const u32 io = __shfl_sync(0xFFFFFFFFu, ib, t);
                census_edge_warp(A, ao, lo, wo, io, f);
            }
            continue;
        }
        for (u32 fb = 0; fb < total; fb += 32) {
            const u32 fi = fb + lane;
            u32 lo = 0, hi = chunk - 1;
            for (int it = 0; it < 5; ++it) {
                const u32 mid = (lo + hi + 1) >> 1;
                const u32 em = __shfl_sync(0xFFFFFFFFu, excl, mid & 31);
                if (lo < hi) { if (em <= fi) lo = mid; else hi = mid - 1; }
            }
            const u32 eo = __shfl_sync(0xFFFFFFFFu, excl, lo);
            const u64 ao = __shfl_sync(0xFFFFFFFFu, ah, lo);
            const u32 wo = __shfl_sync(0xFFFFFFFFu, wh, lo);
            const u32 io = __shfl_sync(0xFFFFFFFFu, ib, lo);
            if (fi < total) f(ao + (fi - eo), A.cpart[ao + (fi - eo)], wo, io);
        }
    }
}

// Block-wide sum of a u64 over GS_BLOCK threads (every thread gets it). `sh` holds one word per warp.
__device__ __forceinline__ u64 block_sum_u64(u64 v, unsigned long long *sh) {
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    u64 t = 0;
    for (u32 i = 0; i < blockDim.x / 32; ++i) t += sh[i];
    return t;
}

// Sampled-connectivity order of the candidate selection: (sconn desc, hash desc, id asc) as one
// (hi, lo) pair compared as unsigned, the larger first.
struct SKey {
    u64 hi, lo;
};
__device__ __forceinline__ bool skey_better(const SKey &a, const SKey &b) {
    return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo);
}

// Candidates and accumulator rows of the sampled rule's exact pass (k_cands_*).
struct CandAcc {
    u32 *spos;                 // [n]
    u32 *cand;                 // [n * GS_C], NONE-padded
    unsigned long long *conn;  // [rows * GS_C]
    u32 *dcon;                 // [rows * GS_C]
    unsigned long long *sacc, *wacc;  // [rows]
};

// Inserts k into the descending list top[0, GS_C) (keys not above the last entry drop out).
__device__ __forceinline__ void skey_insert(SKey (&top)[GS_C], SKey k) {
#pragma unroll
    for (u32 i = 0; i < GS_C; ++i)
        if (skey_better(k, top[i])) {
            const SKey t = top[i];
            top[i] = k;
            k = t;
        }
}
// The warp's best of its lanes' lists, GS_C times: out[r] = the r-th best over the warp (empty
// keys are {0, 0}, below every real key, whose low word holds ~q with q < 2^32 - 2).
__device__ __forceinline__ void skey_warp_top(SKey (&top)[GS_C], SKey *out) {
    const u32 lane = threadIdx.x & 31u;
    for (u32 r = 0; r < GS_C; ++r) {
        SKey b = top[0];
        u32 bl = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const SKey c{__shfl_xor_sync(0xFFFFFFFFu, b.hi, o), __shfl_xor_sync(0xFFFFFFFFu, b.lo, o)};
            const u32 cl = __shfl_xor_sync(0xFFFFFFFFu, bl, o);
            if (skey_better(c, b) || (!skey_better(b, c) && cl < bl)) { b = c; bl = cl; }
        }
        if (lane == 0) out[r] = b;
        if (lane == bl) {  // the winner drops its head
#pragma unroll
            for (u32 i = 0; i + 1 < GS_C; ++i) top[i] = top[i + 1];
            top[GS_C - 1] = SKey{0, 0};
        }
    }
}

__global__ void __launch_bounds__(GS_BLOCK, GS_PER_SM) k_gain_sample(GainArgs A0, const u32 *__restrict__ list, u32 nl,
                                                             CandAcc C) {
    const GainArgs A = gain_args_now(A0);
    extern __shared__ unsigned long long gs_dyn[];
    unsigned long long *sacc = gs_dyn;       // [GS_TAB]: sampled connectivity << GS_DC_BITS | inbound count
    u32 *keys = (u32 *)(gs_dyn + GS_TAB);    // [GS_TAB]
    unsigned short *used = (unsigned short *)(keys + GS_TAB);  // [GS_SAMPLE]: the slots the node filled
    __shared__ unsigned long long wsh[GS_BLOCK / 32];
    __shared__ unsigned long long s_acc;
    __shared__ Cand cred[GS_BLOCK / 32];
    __shared__ SKey kred[(GS_BLOCK / 32) * GS_C];
    __shared__ u32 ndist;
    // the first GS_BLOCK incidences: exclusive census prefix (entry GS_BLOCK or m = the sample's
    // total), census offset and weight
    __shared__ u32 s_ex[GS_BLOCK + 1], s_w[GS_BLOCK];
    __shared__ u64 s_off[GS_BLOCK];
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (u32 i = threadIdx.x; i < GS_TAB; i += GS_BLOCK) { keys[i] = NONE; sacc[i] = 0; }
    for (u32 idx = blockIdx.x; idx < nl; idx += gridDim.x) {
        const u32 u = list[idx], p = A.part[u];
        const u64 t0 = A.toff[u];
        const u32 deg = (u32)(A.toff[u + 1] - t0), nin_u = A.nin[u];
        if (threadIdx.x == 0) ndist = 0;
        // 1. the sample: the longest incidence prefix with at most GS_SAMPLE census entries
        u32 m = 0;
        u64 acc = 0;
        for (u32 base = 0; base < deg; base += GS_BLOCK) {
            const u32 j = base + threadIdx.x;
            const u32 h = j < deg ? A.touch[t0 + j] : 0;
            const u32 lm = j < deg ? A.lam[h] : 0;
            if (base == 0 && j < deg) {
                s_off[j] = A.off[h];
                s_w[j] = A.wfx[h];
            }
            u64 x = lm;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u64 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if ((int)lane >= o) x += y;
            }
            if (lane == 31) wsh[warp] = x;
            __syncthreads();
            for (u32 i = 0; i < warp; ++i) x += wsh[i];
            if (base == 0) s_ex[threadIdx.x] = (u32)(x - lm < GS_SAMPLE ? x - lm : GS_SAMPLE);  // exact for j < m
            const bool take = j < deg && acc + x <= GS_SAMPLE;
            const u32 cnt = (u32)__syncthreads_count(take);
            if (cnt > 0 && threadIdx.x == cnt - 1) s_acc = acc + x;
            __syncthreads();
            m += cnt;
            if (cnt > 0) acc = s_acc;
            if (cnt < GS_BLOCK) break;
        }
        if (threadIdx.x == 0 && m <= GS_BLOCK) s_ex[m] = (u32)acc;
        __syncthreads();
        // 2. sampled connectivity; saving and wtot are exact when the sample is the whole node
        i64 saving = 0, wtot = 0;
        const auto put = [&](u64 k, u32 q, u32 w, bool dst) {
            if (q == p) { saving += leave_gain(A.encourage, w, A.ccnt[k]); return; }
            bool fresh = false;
            const u32 slot = hash_insert_fresh(keys, GS_TAB - 1, q, fresh);
            if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); return; }
            if (fresh) used[atomicAdd(&ndist, 1u)] = (unsigned short)slot;  // at most GS_SAMPLE distinct keys
            atomicAdd(&sacc[slot], ((unsigned long long)w << GS_DC_BITS) | (dst ? 1ull : 0ull));
        };
        if (m <= GS_BLOCK) {
            // the sample's acc entries split evenly over the block: thread t takes entries t,
            // t + GS_BLOCK, ..., finding each one's incidence with a cursor over s_ex
            constexpr u32 U = 4;
            u32 j = 0;
            for (u32 f0 = threadIdx.x; f0 < acc; f0 += U * GS_BLOCK) {
                u64 kk[U];
                u32 xx[U], jj[U], dd[U];
#pragma unroll
                for (u32 r = 0; r < U; ++r) {
                    const u32 f = f0 + r * GS_BLOCK;
                    jj[r] = NONE;
                    if (f < acc) {
                        while (s_ex[j + 1] <= f) ++j;  // s_ex[m] = acc > f ends it below m
                        jj[r] = j;
                        kk[r] = s_off[j] + (f - s_ex[j]);
                        xx[r] = A.cpart[kk[r]];
                        dd[r] = j < nin_u ? A.cdcnt[kk[r]] : 0;
                    }
                }
#pragma unroll
                for (u32 r = 0; r < U; ++r)
                    if (jj[r] != NONE) put(kk[r], xx[r], s_w[jj[r]], dd[r] > 0);
            }
            if (threadIdx.x < m) wtot = s_w[threadIdx.x];
        } else {
            census_flat(A, u, 32 * warp, GS_BLOCK, m, wtot,
                        [&](u64 k, u32 q, u32 w, u32 io) { put(k, q, w, io && q != p && A.cdcnt[k] > 0); });
        }
        __syncthreads();
        const u32 nd = ndist;
        const u64 s = A.nsize[u];
        if (m == deg) {  // 3a. the whole node: exact, as the table kernels
            saving = (i64)block_sum_u64((u64)saving, wsh);
            wtot = (i64)block_sum_u64((u64)wtot, wsh);
            Cand best{INT64_MIN, 0};
            for (u32 t = threadIdx.x; t < nd; t += GS_BLOCK) {
                const u32 i = used[t];
                const Cand c = gain_candidate(A, u, keys[i], sacc[i] >> GS_DC_BITS, (u32)(sacc[i] & GS_DC_MASK), saving,
                                              wtot);
                if (cand_better(c, best)) best = c;
            }
            best = warp_best(best);
            if (lane == 0) cred[warp] = best;
            __syncthreads();
            if (threadIdx.x == 0) {
                Cand b = cred[0];
                for (u32 i = 1; i < GS_BLOCK / 32; ++i)
                    if (cand_better(cred[i], b)) b = cred[i];
                write_move(A, u, b);  // spos[u] stays NONE
            }
        } else {
            // 3b. the GS_C best by (sampled connectivity, tie hash, -id) among the keys the size
            // limit and the inbound bound do not rule out. Pass 1 marks the ruled-out slots and
            // takes each warp's best key; the least of those GS_BLOCK / 32 >= GS_C keys is no
            // better than the GS_C-th best, so pass 2 lists only the keys at or above it
            // (per-thread lists, then per warp, then warp 0 over the warps' lists).
            const u64 in_sample = m < nin_u ? m : nin_u;
            SKey best1{0, 0};
            constexpr u32 U = 4;  // keys per thread whose partition loads are in flight together
            for (u32 t0 = threadIdx.x; t0 < nd; t0 += U * GS_BLOCK) {
                u32 qs[U], is[U];
                u64 ps[U], pb[U];
#pragma unroll
                for (u32 r = 0; r < U; ++r) {
                    const u32 t = t0 + r * GS_BLOCK;
                    is[r] = t < nd ? used[t] : 0;
                    qs[r] = t < nd ? keys[is[r]] : NONE;
                    ps[r] = qs[r] != NONE ? A.psize[qs[r]] : 0;
                    pb[r] = qs[r] != NONE ? A.pinb[qs[r]] : 0;
                }
#pragma unroll
                for (u32 r = 0; r < U; ++r) {
                    const u32 q = qs[r], i = is[r];
                    if (q == NONE) continue;
                    const u64 v = sacc[i];
                    if (ps[r] + s - s / A.discount > A.omega || pb[r] + in_sample - (v & GS_DC_MASK) > A.delta) {
                        sacc[i] = v | GS_RULED_OUT;
                        continue;
                    }
                    const SKey k{v >> GS_DC_BITS, ((u64)mix32(q + A.round + A.seed) << 32) | (u64)(~q)};
                    if (skey_better(k, best1)) best1 = k;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const SKey c{__shfl_xor_sync(0xFFFFFFFFu, best1.hi, o), __shfl_xor_sync(0xFFFFFFFFu, best1.lo, o)};
                if (skey_better(c, best1)) best1 = c;
            }
            if (lane == 0) kred[warp] = best1;
            __syncthreads();
            SKey thr = kred[0];
            for (u32 w2 = 1; w2 < GS_BLOCK / 32; ++w2)
                if (skey_better(thr, kred[w2])) thr = kred[w2];
            __syncthreads();  // kred is reused below
            SKey top[GS_C];
#pragma unroll
            for (u32 r = 0; r < GS_C; ++r) top[r] = SKey{0, 0};
            for (u32 t = threadIdx.x; t < nd; t += GS_BLOCK) {
                const u32 i = used[t];
                const u64 v = sacc[i];
                if (v & GS_RULED_OUT) continue;
                const u32 q = keys[i];
                const SKey k{v >> GS_DC_BITS, ((u64)mix32(q + A.round + A.seed) << 32) | (u64)(~q)};
                if (!skey_better(thr, k)) skey_insert(top, k);
            }
            skey_warp_top(top, kred + warp * GS_C);
            __syncthreads();
            if (warp == 0) {
#pragma unroll
                for (u32 r = 0; r < GS_C; ++r) top[r] = SKey{0, 0};
                for (u32 t = lane; t < (GS_BLOCK / 32) * GS_C; t += 32) skey_insert(top, kred[t]);
                __syncwarp();  // every lane has read kred before lane 0 overwrites its head
                skey_warp_top(top, kred);
                __syncwarp();
                if (lane < GS_C) {  // the candidates and a zeroed accumulator row (row = list index)
                    const SKey b = kred[lane];
                    C.cand[(u64)u * GS_C + lane] = (b.hi | b.lo) ? ~(u32)b.lo : NONE;
                    C.conn[(u64)idx * GS_C + lane] = 0;
                    C.dcon[(u64)idx * GS_C + lane] = 0;
                }
                if (lane == 0) {
                    C.sacc[idx] = 0;
                    C.wacc[idx] = 0;
                    C.spos[u] = idx;
                }
            }
        }
        __syncthreads();
        for (u32 t = threadIdx.x; t < nd; t += GS_BLOCK) {  // empty the node's slots for the next one
            const u32 i = used[t];
            keys[i] = NONE;
            sacc[i] = 0;
        }
        __syncthreads();
    }
}

// The exact pass of the sampled rule, pin-centric. Each listed node u whose sample was not the
// whole node has row r = spos[u] of the accumulators (k_gain_sample sets it and zeroes the row;
// spos is NONE for every other node): conn[r * GS_C + i], the weight of u's hyperedges holding its
// candidate i; dcon[r * GS_C + i], u's inbound hyperedges with a destination pin in candidate i;
// sacc[r], u's saving from leaving its partition; wacc[r], the weight of all u's hyperedges. One
// pass over the hyperedges fills them: a hyperedge's census goes into a hash table (partition ->
// count, plus a has-destination bit) and each listed pin looks up its own partition and its
// candidates. k_cands_best then takes the best feasible candidate from these integer sums, which
// are those a scan of each node's incidences would give.
static_assert(GS_C == 8, "k_cands_* read a node's candidates as two 16-byte words");
constexpr u32 CV_DBIT = 0x80000000u;  // census value: the partition holds a destination pin
constexpr u32 CV_WARPS = 4;
constexpr u32 CV_WARP_LEN = 256;      // longer hyperedges take a block (CS_WARP_CAP)
constexpr u32 CV_BLOCK_LEN = 4096;    // longer still: a table in device memory (CS_BLOCK_CAP)
constexpr u32 CV_BLOCK = 256;
constexpr size_t CV_BLOCK_SMEM = (size_t)8 * 8192;  // keys and values of cs_cap(CV_BLOCK_LEN) slots

// Census entries [a, a + lm) of one hyperedge into keys/vals (mask + 1 cleared slots), threads
// t, t + nt, ...: each partition appears once in a census, so each slot is written once.
__device__ __forceinline__ void cv_fill(const GainArgs &A, u64 a, u32 lm, u32 *keys, u32 *vals, u32 mask, u32 t,
                                        u32 nt) {
    for (u32 j = t; j < lm; j += nt) {
        const u32 slot = hash_find_or_insert(keys, mask, A.cpart[a + j]);
        if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); continue; }
        vals[slot] = A.ccnt[a + j] | (A.cdcnt[a + j] > 0 ? CV_DBIT : 0u);
    }
}
// Listed pin v (row r) of a hyperedge of weight w; io: v is one of its destinations.
__device__ __forceinline__ void cv_pin(const GainArgs &A, const CandAcc &C, u32 v, u32 r, bool io, u32 w,
                                       const u32 *keys, const u32 *vals, u32 mask) {
    const u32 sp = hash_find(keys, mask, A.part[v]);  // present: v's own partition
    if (sp != NONE) {
        const i64 g = leave_gain(A.encourage, w, vals[sp] & ~CV_DBIT);
        if (g) atomicAdd(&C.sacc[r], (unsigned long long)g);
    }
    if (w) atomicAdd(&C.wacc[r], (unsigned long long)w);
    const uint4 *cp = reinterpret_cast<const uint4 *>(C.cand + (u64)v * GS_C);
    const uint4 c0 = cp[0], c1 = cp[1];
    const u32 q[GS_C] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
    for (u32 i = 0; i < GS_C; ++i) {
        if (q[i] == NONE) break;
        const u32 s = hash_find(keys, mask, q[i]);
        if (s == NONE) continue;
        if (w) atomicAdd(&C.conn[(u64)r * GS_C + i], (unsigned long long)w);
        if (io && (vals[s] & CV_DBIT)) atomicAdd(&C.dcon[(u64)r * GS_C + i], 1u);
    }
}

// One warp per hyperedge of at most CV_WARP_LEN pins; skipped when it holds no listed pin.
__global__ void __launch_bounds__(CV_WARPS * 32) k_cands_warp(GainArgs A, CandAcc C, u32 e) {
    __shared__ u32 tk[CV_WARPS][2 * CV_WARP_LEN], tv[CV_WARPS][2 * CV_WARP_LEN];
    const u32 wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 h = blockIdx.x * CV_WARPS + wp;
    if (h >= e) return;
    const u64 a = A.off[h], b = A.off[h + 1];
    if (b - a > CV_WARP_LEN) return;
    constexpr u32 R = CV_WARP_LEN / 32;
    u32 pv[R], pr[R];
    bool any = false;
#pragma unroll
    for (u32 i = 0; i < R; ++i) {
        const u64 k = a + lane + 32 * i;
        pv[i] = k < b ? A.pins[k] : 0;
        pr[i] = k < b ? C.spos[pv[i]] : NONE;
        any |= pr[i] != NONE;
    }
    if (!__any_sync(0xFFFFFFFFu, any)) return;
    const u32 lm = A.lam[h];
    const u32 cap = cs_cap(lm);
    u32 *keys = tk[wp], *vals = tv[wp];
    for (u32 i = lane; i < cap; i += 32) keys[i] = NONE;
    __syncwarp();
    cv_fill(A, a, lm, keys, vals, cap - 1, lane, 32);
    __syncwarp();
    const u32 w = A.wfx[h];
    const u64 s = a + A.nsrc[h];
#pragma unroll
    for (u32 i = 0; i < R; ++i)
        if (pr[i] != NONE) cv_pin(A, C, pv[i], pr[i], a + lane + 32 * i >= s, w, keys, vals, cap - 1);
}

// One block per listed hyperedge: `list` holds those of CV_WARP_LEN < |e| <= CV_BLOCK_LEN pins
// (tables in shared memory) or, with gtab set, the longer ones (tables at gtab + 2 * gtab_off[i],
// 2 * |e| slots rounded up to a power of two, as k_tab_sizes sizes them).
__global__ void __launch_bounds__(CV_BLOCK) k_cands_block(GainArgs A, CandAcc C, const u32 *__restrict__ list,
                                                          u32 nlist, u32 *gtab, const u64 *__restrict__ gtab_off) {
    extern __shared__ u32 cv_dyn[];
    if (blockIdx.x >= nlist) return;
    const u32 h = list[blockIdx.x];
    const u64 a = A.off[h], b = A.off[h + 1];
    bool any = false;
    for (u64 k = a + threadIdx.x; k < b && !any; k += CV_BLOCK) any = C.spos[A.pins[k]] != NONE;
    if (!__syncthreads_or(any)) return;
    const u32 lm = A.lam[h];
    const u32 cap = cs_cap(lm);
    if (!gtab && 8ull * cap > dyn_smem_bytes()) {  // launched with too small a table: refuse
        if (threadIdx.x == 0) atomicExch(A.status, DEV_HASH_FULL);
        return;
    }
    u32 *keys = gtab ? gtab + 2 * gtab_off[blockIdx.x] : cv_dyn;
    u32 *vals = keys + cap;
    for (u32 i = threadIdx.x; i < cap; i += CV_BLOCK) keys[i] = NONE;
    __syncthreads();
    cv_fill(A, a, lm, keys, vals, cap - 1, threadIdx.x, CV_BLOCK);
    __syncthreads();
    const u32 w = A.wfx[h];
    const u64 s = a + A.nsrc[h];
    for (u64 k = a + threadIdx.x; k < b; k += CV_BLOCK) {
        const u32 v = A.pins[k], r = C.spos[v];
        if (r != NONE) cv_pin(A, C, v, r, k >= s, w, keys, vals, cap - 1);
    }
}

// Each listed node with a row: its best feasible candidate (the order of gain_candidate).
__global__ void k_cands_best(GainArgs A0, CandAcc C, const u32 *__restrict__ list, u32 nl) {
    const GainArgs A = gain_args_now(A0);
    const u32 idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nl) return;
    const u32 u = list[idx], r = C.spos[u];
    if (r == NONE) return;  // settled by k_gain_sample
    const i64 saving = (i64)C.sacc[r], wtot = (i64)C.wacc[r];
    Cand best{INT64_MIN, 0};
#pragma unroll
    for (u32 i = 0; i < GS_C; ++i) {
        const u32 q = C.cand[(u64)u * GS_C + i];
        if (q == NONE) break;
        const Cand c = gain_candidate(A, u, q, C.conn[(u64)r * GS_C + i], C.dcon[(u64)r * GS_C + i], saving, wtot);
        if (cand_better(c, best)) best = c;
    }
    write_move(A, u, best);
}

__global__ void k_list_degree(const u32 *__restrict__ list, u32 nl, const u64 *__restrict__ toff,
                              unsigned long long *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    u64 d = i < nl ? toff[list[i] + 1] - toff[list[i]] : 0;
    d = warp_sum(d);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(out, (unsigned long long)d);
}
__global__ void k_list_max(const u32 *__restrict__ list, u32 nl, const u64 *__restrict__ v,
                           unsigned long long *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    u64 m = i < nl ? v[list[i]] : 0;
    m = warp_max_u64(m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, (unsigned long long)m);
}
// Gain tiers: 0 = one warp (small table, at most GN_WARP_DEG incidences), 1 = one block with the
// table in shared memory, 2 = one block with the table in global scratch. Levels of at most
// GN_SMALL_LEVEL nodes use no warp tier: their few nodes carry long census chains, which a block
// splits over its warps while the rest of the GPU would idle anyway.
__device__ __forceinline__ u32 gain_tier(u32 n, u32 K, u64 wk, u64 deg) {
    if (K <= GN_DIRECT_K)  // partition-indexed gains: a warp or a block, by incidences
        return (n > GN_SMALL_LEVEL && deg <= GM_WARP_DEG) ? 0u : 1u;
    if (wk > GN_BLOCK_W) return 2u;
    return (n > GN_SMALL_LEVEL && wk <= GN_WARP_W && deg <= GN_WARP_DEG) ? 0u : 1u;
}
__global__ void k_tier(u32 n, u32 K, const u64 *__restrict__ work, const u64 *__restrict__ toff, u32 tier,
                       u32 *__restrict__ flag) {
    u32 u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    flag[u] = gain_tier(n, K, work[u], toff[u + 1] - toff[u]) == tier ? 1u : 0u;
}

// ------------------------------------------------------------------ ranking
// Mover flags, and every node's rank reset (k_set_rank then ranks the movers) and cascaded gain
// zeroed.
__global__ void k_move_flags(u32 n, const u32 *__restrict__ target, u32 *__restrict__ flag, u32 *__restrict__ rank,
                             unsigned long long *__restrict__ g2) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) {
        flag[v] = target[v] != NONE ? 1u : 0u;
        rank[v] = NONE;
        g2[v] = 0;
    }
}
__global__ void k_move_keys(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const i64 *__restrict__ gain,
                            u64 gbound, u32 *__restrict__ hi, u32 *__restrict__ lo) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *dM) return;
    u64 k = gbound - (u64)gain[mv[i]];  // ascending key = descending gain
    hi[i] = (u32)(k >> 32);
    lo[i] = (u32)k;
}
// rank[mv[i]] = i; also the size-event count 2M into *twice.
__global__ void k_set_rank(const u32 *__restrict__ mv, const u32 *__restrict__ dM, u32 *__restrict__ rank,
                           u32 *__restrict__ twice) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *twice = 2 * *dM;
    if (i < *dM) rank[mv[i]] = i;
}

// k-way pair ranking (include/axc.h AXC_PAIR_RANK_MAX_K): the moves, in (gain desc, id asc)
// order, get the key of their direction group: (min(p,q) * K + max(p,q)) * 2 + (p > q).
constexpr u32 PAIR_RANK_MAX_K = AXC_PAIR_RANK_MAX_K;
__global__ void k_pair_group(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u32 *__restrict__ part,
                             const u32 *__restrict__ target, u32 K, u32 *__restrict__ gk, u32 *__restrict__ pos) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *dM) return;
    const u32 u = mv[i], p = part[u], q = target[u];
    gk[i] = (((p < q ? p : q) * K + (p < q ? q : p)) << 1) | (p < q ? 0u : 1u);
    pos[i] = i;
}
__device__ __forceinline__ u32 lower_bound_u32(const u32 *a, u32 n, u32 x) {
    u32 lo = 0, hi = n;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// After the stable sort by group key: the move at position j is the i-th of its group; the i-th of
// the opposite direction is its partner. Pair gain into psn[node] (indexed by node, so later
// passes can rebuild the key after any permutation), (pair position << 1 | d) into k1.
__global__ void k_pair_keys(const u32 *__restrict__ gk, const u32 *__restrict__ pos, const u32 *__restrict__ dM,
                            const u32 *__restrict__ mv, const i64 *__restrict__ gain, i64 *__restrict__ psn,
                            u32 *__restrict__ k1, u32 *__restrict__ node) {
    const u32 M = *dM, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    const u32 g = gk[j], d = g & 1u;
    const u32 i = j - lower_bound_u32(gk, M, g);
    const u32 s2 = lower_bound_u32(gk, M, g ^ 1u), e2 = lower_bound_u32(gk, M, (g ^ 1u) + 1u);
    const u32 u = mv[pos[j]];
    i64 ps = gain[u];
    u32 pk = j;
    if (i < e2 - s2) {
        ps += gain[mv[pos[s2 + i]]];
        if (d) pk = s2 + i;
    }
    psn[u] = ps;
    k1[j] = (pk << 1) | d;
    node[j] = u;
}
// Descending pair-gain keys of the permuted movers (hi and lo words of pbound - ps).
__global__ void k_pair_gain_keys(const u32 *__restrict__ node, const u32 *__restrict__ dM, const i64 *__restrict__ psn,
                                 u64 pbound, u32 *__restrict__ hi, u32 *__restrict__ lo) {
    const u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= *dM) return;
    const u64 k = pbound - (u64)psn[node[j]];
    hi[j] = (u32)(k >> 32);
    lo[j] = (u32)k;
}

// ------------------------------------------------------------------ cascade
constexpr u32 CC_WARPS = 4;
constexpr u32 CC_MOV = 128;    // movers per hyperedge handled by the warp kernel
constexpr u32 CC_TAB = 512;    // partition table slots of the warp kernel

struct CascadeArgs {
    u32 e;
    int encourage;
    const u64 *off;
    const u32 *pins, *nsrc, *wfx, *lam, *cpart, *ccnt, *cdcnt, *rank, *part, *target;
    unsigned long long *g2;
    // inbound-set transitions (INCC): a (partition, hyperedge) destination count going 0 -> 1 or
    // 1 -> 0 at a move's rank; appended as (partition, rank, +-1)
    int track;
    u32 *tp, *tr;
    int32_t *tdv;
    u32 *dT;
    u64 tcap;
    // when set (small levels), transitions are summed per (partition, rank) instead: entry
    // p * dense_stride + r gets ((d << 32) + 1) per transition, its count below and its net above
    unsigned long long *tdense;
    u32 dense_stride;
    u32 *status;
    u32 K;  // partitions: with K <= CC_DIRECT_K the per-hyperedge tables are indexed by partition id
    // when set (kernel timer on k_cascade_warp): each hyperedge's algorithmic bytes are added here
    unsigned long long *pbytes;
};

constexpr u32 MV_DST = 0x80000000u;  // mover flag in the node field: the pin is a destination
constexpr u32 CC_DIRECT_K = 256;

__device__ __forceinline__ bool cascade_direct(const CascadeArgs &A) { return A.K <= CC_DIRECT_K; }

// The hyperedge's census into the table: partition -> (pins, destination pins). Block- or
// warp-wide over threads [t0, t0 + nt); direct tables hold K slots, hashed ones `cap`.
__device__ __forceinline__ void cascade_fill(const CascadeArgs &A, u64 a, u32 lm, u32 *tk, u32 *tc, u32 *td, u32 cap,
                                             u32 t0, u32 nt) {
    const bool direct = cascade_direct(A);
    for (u32 i = t0; i < lm; i += nt) {
        const u32 q = A.cpart[a + i];
        const u32 s = direct ? q : hash_find_or_insert(tk, cap - 1, q);
        if (s != NONE) { tc[s] = A.ccnt[a + i]; td[s] = A.cdcnt[a + i]; }
    }
}

__device__ __forceinline__ void emit_at(const CascadeArgs &A, u32 s, u32 p, u32 r, int32_t d) {
    if (A.tdense) {
        atomicAdd(&A.tdense[(u64)p * A.dense_stride + r], ((unsigned long long)(i64)d << 32) + 1ull);
        return;
    }
    if (s >= A.tcap) { atomicExch(A.status, DEV_BAD_INDEX); return; }
    A.tp[s] = p;
    A.tr[s] = r;
    A.tdv[s] = d;
}
__device__ __forceinline__ void emit_transition(const CascadeArgs &A, u32 p, u32 r, int32_t d) {
    emit_at(A, atomicAdd(A.dT, 1u), p, r, d);
}

// Table slots of every mover's source and target partition, sl[i] = slot(p) | slot(q) << 16,
// gathered in parallel so the sequential sweep reads no global memory. Hashed tables insert the
// partitions missing from the census (their counts stay zero); they need cap <= 65536.
__device__ __forceinline__ void cascade_slots(const CascadeArgs &A, const u64 *mv, u32 *sl, u32 m, u32 *tk, u32 cap,
                                              u32 t0, u32 nt) {
    const bool direct = cascade_direct(A);
    for (u32 i = t0; i < m; i += nt) {
        const u32 v = (u32)mv[i] & ~MV_DST;
        const u32 p = A.part[v], q = A.target[v];
        u32 sp = p, sq = q;  // direct tables: the slot is the partition id
        if (!direct) {
            sp = hash_find_or_insert(tk, cap - 1, p);
            sq = hash_find_or_insert(tk, cap - 1, q);
            if (sp == NONE || sq == NONE) { atomicExch(A.status, DEV_HASH_FULL); sp = sq = 0; }
        }
        sl[i] = sp | sq << 16;
    }
}

// Sweep the movers of one hyperedge sequentially in rank order. mv[i] = rank << 32 | dst flag |
// node; tc / td hold the hyperedge's pins / destination pins per partition (hash slots in tk,
// or the partition id itself for direct tables). With sl the slots come precomputed from
// cascade_slots; without it (hashed tables too large for 16-bit slots) they are looked up here.
// One thread; cascade_sweep_warp is the warp-wide form used wherever the slots fit 16 bits.
__device__ void cascade_sweep(const CascadeArgs &A, u32 h, const u64 *mv, const u32 *sl, u32 m, u32 *tk, u32 *tc,
                              u32 *td, u32 mask) {
    const u32 w = A.wfx[h];
    const bool direct = cascade_direct(A);
    for (u32 i = 0; i < m; ++i) {
        const u32 lowv = (u32)mv[i], r = (u32)(mv[i] >> 32);
        const u32 v = lowv & ~MV_DST;
        u32 sp, sq;
        if (sl) {
            sp = sl[i] & 0xFFFFu;
            sq = sl[i] >> 16;
        } else {
            sp = A.part[v];
            sq = A.target[v];
            if (!direct) {
                sp = hash_find_or_insert(tk, mask, sp);
                sq = hash_find_or_insert(tk, mask, sq);
                if (sp == NONE || sq == NONE) { atomicExch(A.status, DEV_HASH_FULL); return; }
            }
        }
        const u32 cp = tc[sp], cq = tc[sq];
        const i64 d = leave_gain(A.encourage, w, cp) - (cq == 0 ? (i64)w : 0);
        atomicAdd(&A.g2[v], (unsigned long long)d);
        tc[sp] = cp - 1;
        tc[sq] = tc[sq] + 1;
        if (A.track && (lowv & MV_DST)) {
            if (td[sp] == 1) emit_transition(A, direct ? sp : tk[sp], r, -1);
            if (td[sq] == 0) emit_transition(A, direct ? sq : tk[sq], r, +1);
            td[sp] -= 1;
            td[sq] += 1;
        }
    }
}

// Table size for a hyperedge with lm census partitions and m movers: its keys are the census
// partitions plus at most m targets, at load factor <= 1/2.
__host__ __device__ __forceinline__ u64 cascade_cap(u64 lm, u64 m) {
    u64 cap = 32;
    while (cap < 2 * (lm + m)) cap <<= 1;
    return cap;
}
__device__ __forceinline__ u32 cascade_cap32(u32 lm, u32 m) {
    const u64 cap = cascade_cap(lm, m);
    return cap > (1ull << 31) ? (1u << 31) : (u32)cap;
}

// Hyperedges with at most CC_MOV movers, one warp each (hashed tables also need at most CC_TAB
// slots); the others are appended to `big` for the block kernel.
// The same sweep with a whole warp, 32 movers at a time (slots from cascade_slots required). The
// counts a mover sees are the table's counts before its chunk plus what the chunk's earlier lanes
// did to its two partitions: leaves of the same source (match_any), joins of the same target
// (match_any), and the cross terms, lanes whose target is its source or whose source is its
// target (one shuffle pass over the chunk). The tables are then updated by the whole chunk at once.
// Equal to the sequential sweep: the counts are exact prefix sums, and transitions are a set.
__device__ void cascade_sweep_warp(const CascadeArgs &A, u32 h, const u64 *mv, const u32 *sl, u32 m, const u32 *tk,
                                   u32 *tc, u32 *td, u32 *lmask) {
    const u32 lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    const u32 w = A.wfx[h];
    const bool direct = cascade_direct(A);
    for (u32 base = 0; base < m; base += 32) {
        const u32 i = base + lane;
        const bool act = i < m;
        const u64 e = act ? mv[i] : 0;
        // inactive lanes get slots no table has (slots are below 65536), distinct per lane
        const u32 sp = act ? (sl[i] & 0xFFFFu) : 0x10000u + lane, sq = act ? (sl[i] >> 16) : 0x20000u + lane;
        const bool dst = act && ((u32)e & MV_DST);
        const u32 dmask = __ballot_sync(0xFFFFFFFFu, dst);
        u32 m_pp, m_qq, m_qp = 0, m_pq = 0;  // lanes with my source / my target as source / target
        if (lmask) {  // direct tables: lmask[x] / lmask[K + x] = lanes with source / target x
            u32 *pm = lmask, *qm = lmask + A.K;
            if (act) {
                atomicOr(&pm[sp], 1u << lane);
                atomicOr(&qm[sq], 1u << lane);
            }
            __syncwarp();
            m_pp = act ? pm[sp] : 0u;
            m_qq = act ? qm[sq] : 0u;
            m_qp = act ? qm[sp] : 0u;
            m_pq = act ? pm[sq] : 0u;
            __syncwarp();
            if (act) {
                pm[sp] = 0;
                qm[sq] = 0;
            }
        } else {
            m_pp = __match_any_sync(0xFFFFFFFFu, sp);
            m_qq = __match_any_sync(0xFFFFFFFFu, sq);
#pragma unroll 8
            for (u32 j = 0; j < 32; ++j) {
                const u32 spj = __shfl_sync(0xFFFFFFFFu, sp, j), sqj = __shfl_sync(0xFFFFFFFFu, sq, j);
                m_qp |= (u32)(sqj == sp) << j;
                m_pq |= (u32)(spj == sq) << j;
            }
        }
        const int before_p = __popc(m_qp & lt) - __popc(m_pp & lt);
        const int before_q = __popc(m_qq & lt) - __popc(m_pq & lt);
        if (act) {
            const u32 cp = (u32)((int)tc[sp] + before_p), cq = (u32)((int)tc[sq] + before_q);
            const i64 d = leave_gain(A.encourage, w, cp) - (cq == 0 ? (i64)w : 0);
            atomicAdd(&A.g2[(u32)e & ~MV_DST], (unsigned long long)d);
        }
        if (A.track) {  // warp-uniform
            bool ep = false, eq = false;
            if (dst) {
                const int dp = __popc(m_qp & lt & dmask) - __popc(m_pp & lt & dmask);
                const int dq = __popc(m_qq & lt & dmask) - __popc(m_pq & lt & dmask);
                ep = (int)td[sp] + dp == 1;
                eq = (int)td[sq] + dq == 0;
            }
            // one reservation per chunk: p-transitions first, then q-transitions
            const u32 bp = __ballot_sync(0xFFFFFFFFu, ep), bq = __ballot_sync(0xFFFFFFFFu, eq);
            const u32 tot = __popc(bp) + __popc(bq);
            u32 s0 = 0;
            if (lane == 0 && tot) s0 = atomicAdd(A.dT, tot);
            s0 = __shfl_sync(0xFFFFFFFFu, s0, 0);
            const u32 r = (u32)(e >> 32);
            if (ep) emit_at(A, s0 + __popc(bp & lt), direct ? sp : tk[sp], r, -1);
            if (eq) emit_at(A, s0 + __popc(bp) + __popc(bq & lt), direct ? sq : tk[sq], r, +1);
        }
        __syncwarp();
        if (act) {
            atomicSub(&tc[sp], 1u);
            atomicAdd(&tc[sq], 1u);
            if (dst) {
                atomicSub(&td[sp], 1u);
                atomicAdd(&td[sq], 1u);
            }
        }
        __syncwarp();
    }
}

// The hyperedges that hold a mover: every incidence of every mover flags its hyperedge (flag[]
// zeroed before), then the flags are compacted into the cascade's list. One warp per mover.
__global__ void k_mover_hedges(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u64 *__restrict__ toff,
                               const u32 *__restrict__ touch, u32 *__restrict__ flag) {
    const u32 lane = threadIdx.x & 31u, nw = (gridDim.x * blockDim.x) >> 5;
    const u32 M = *dM;
    for (u32 r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < M; r += nw) {
        const u32 u = mv[r];
        for (u64 j = toff[u] + lane; j < toff[u + 1]; j += 32) flag[touch[j]] = 1u;
    }
}

__global__ void k_cascade_warp(CascadeArgs A, const u32 *__restrict__ list, const u32 *__restrict__ nlist,
                               u32 *__restrict__ big, u32 *__restrict__ nbig) {
    __shared__ u64 mvs[CC_WARPS][CC_MOV];
    __shared__ u32 sl[CC_WARPS][CC_MOV];
    __shared__ u32 tk[CC_WARPS][CC_TAB], tc[CC_WARPS][CC_TAB], td[CC_WARPS][CC_TAB];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 nl = *nlist;
    u64 bytes = 0;  // algorithmic bytes of this warp's hyperedges (kernel timer)
    for (u32 idx = blockIdx.x * CC_WARPS + w; idx < nl; idx += gridDim.x * CC_WARPS) {
        __syncwarp();  // the previous hyperedge's shared state is no longer read
        const u32 h = list[idx];
        const u64 a = A.off[h], b = A.off[h + 1], d0 = a + A.nsrc[h];
        // collect movers (rank << 32 | dst flag | node)
        u32 m = 0;
        for (u64 base = a; base < b; base += 32) {
            u64 k = base + lane;
            u32 v = k < b ? A.pins[k] : 0, r = k < b ? A.rank[v] : NONE;
            bool mvr = r != NONE;
            u32 bal = __ballot_sync(0xFFFFFFFFu, mvr);
            if (mvr) {
                u32 pos = m + __popc(bal & ((1u << lane) - 1u));
                if (pos < CC_MOV) mvs[w][pos] = ((u64)r << 32) | (k >= d0 ? MV_DST : 0u) | v;
            }
            m += __popc(bal);
        }
        // algorithmic bytes (kernel timer): the list entry, offsets and source count, each pin's id
        // and rank, the census size, then the hand-off to the block kernel or the census entries,
        // each mover's partition, target and cascaded gain, and the weight (transitions not counted)
        const u64 bytes_read = 24 + 8 * (b - a);
        if (m == 0) {  // (a listed hyperedge always has a mover)
            bytes += bytes_read;
            continue;
        }
        const u32 lm = A.lam[h];
        const bool direct = cascade_direct(A);
        const u32 cap = direct ? A.K : cascade_cap32(lm, m);
        if (m > CC_MOV || cap > CC_TAB) {
            if (lane == 0) big[atomicAdd(nbig, 1u)] = h;  // handled by the block kernel
            bytes += bytes_read + 8;
            continue;
        }
        bytes += bytes_read + 8 + 12ull * lm + 16ull * m;
        __syncwarp();
        // sort movers by rank: each key's position is the number of smaller keys (keys are unique)
        u64 mine[CC_MOV / 32];
        u32 posv[CC_MOV / 32];
        for (u32 i = 0; i < CC_MOV / 32; ++i) mine[i] = (lane + 32 * i < m) ? mvs[w][lane + 32 * i] : ~0ull;
        for (u32 i = 0; i < CC_MOV / 32; ++i) {
            posv[i] = 0;
            if (lane + 32 * i >= m) continue;
            for (u32 j = 0; j < m; ++j) posv[i] += mvs[w][j] < mine[i];
        }
        __syncwarp();
        for (u32 i = 0; i < CC_MOV / 32; ++i)
            if (lane + 32 * i < m) mvs[w][posv[i]] = mine[i];
        // table of partition counts from the census, then the movers' slots; direct tables leave
        // tk to the sweep's lane masks (2K <= CC_TAB words, zeroed)
        for (u32 i = lane; i < cap; i += 32) { tc[w][i] = 0; td[w][i] = 0; }
        const u32 ntk = direct ? 2 * A.K : cap;
        for (u32 i = lane; i < ntk; i += 32) tk[w][i] = direct ? 0u : NONE;
        __syncwarp();
        cascade_fill(A, a, lm, tk[w], tc[w], td[w], cap, lane, 32);
        __syncwarp();
        cascade_slots(A, mvs[w], sl[w], m, tk[w], cap, lane, 32);
        __syncwarp();
        cascade_sweep_warp(A, h, mvs[w], sl[w], m, tk[w], tc[w], td[w], direct ? tk[w] : nullptr);
    }
    if (A.pbytes && lane == 0 && bytes) prof_add(A.pbytes, blockIdx.x * CC_WARPS + w, bytes);
}

// Block-wide bitonic sort of buf[0, P) ascending (P a power of two).
__device__ void block_bitonic_u64(u64 *buf, u32 P) {
    for (u32 k = 2; k <= P; k <<= 1) {
        for (u32 j = k >> 1; j > 0; j >>= 1) {
            for (u32 i = threadIdx.x; i < P; i += blockDim.x) {
                const u32 ixj = i ^ j;
                if (ixj > i) {
                    const u64 x = buf[i], y = buf[ixj];
                    if ((x > y) == ((i & k) == 0)) {
                        buf[i] = y;
                        buf[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

constexpr u32 CB_THREADS = 128;
constexpr u32 CB_MOV_MAX = 2048;  // movers of the block kernel, in shared memory
constexpr u32 CB_TAB_HASH = 8192; // hashed table slots of the block kernel, at most
constexpr size_t CB_DYN_MAX = (size_t)CB_MOV_MAX * 12 + (size_t)CB_TAB_HASH * 12;
// The block kernel's middle tier (hashed tables): hyperedges with at most CB_MID_MOV movers and
// CB_MID_TAB table slots take blocks small enough for several per SM; the rest go on to the
// launch sized by the level's largest hyperedge.
constexpr u32 CB_MID_MOV = 512;
constexpr u32 CB_MID_TAB = 2048;

// Gather the movers of hyperedge h (rank << 32 | dst flag | node) into mvs[0, min(m, lim)) with
// the whole block; returns m (all of them, counted past lim) and their largest rank in *rmax.
// Warps reserve their movers' slots with one atomic each. Ends with the block synchronised.
__device__ __forceinline__ u32 cascade_gather(const CascadeArgs &A, u32 h, u64 *mvs, u32 lim, u32 *cntm, u32 *smax,
                                              u32 &rmax) {
    const u64 a = A.off[h], b = A.off[h + 1], d0 = a + A.nsrc[h];
    const u32 lane = threadIdx.x & 31;
    if (threadIdx.x == 0) { *cntm = 0; *smax = 0; }
    __syncthreads();
    u32 mymax = 0;
    for (u64 base = a; base < b; base += blockDim.x) {  // same trip count in every thread
        const u64 k = base + threadIdx.x;
        const u32 v = k < b ? A.pins[k] : 0, r = k < b ? A.rank[v] : NONE;
        const bool mvr = r != NONE;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, mvr);
        u32 wbase = 0;
        if (lane == 0 && bal) wbase = atomicAdd(cntm, (u32)__popc(bal));
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (mvr) {
            const u32 pos = wbase + __popc(bal & ((1u << lane) - 1u));
            if (pos < lim) mvs[pos] = ((u64)r << 32) | (k >= d0 ? MV_DST : 0u) | v;
            mymax = r > mymax ? r : mymax;
        }
    }
    mymax = __reduce_max_sync(0xFFFFFFFFu, mymax);
    if (lane == 0 && mymax) atomicMax(smax, mymax);
    __syncthreads();
    const u32 m = *cntm;
    rmax = *smax;
    __syncthreads();  // read before the next hyperedge resets them
    return m;
}

constexpr u32 CB_SORT_R = 8;                          // keys per thread in the block radix sort
constexpr u32 CB_RADIX_MAX = CB_SORT_R * CB_THREADS;  // more movers sort bitonically

// Stable LSD radix sort of buf[0, m) (m <= CB_RADIX_MAX, CB_THREADS threads) by key bits
// [32, 32 + nbits), 2 bits per pass. Thread t holds positions [t*R, t*R + R) in registers; a
// pass counts its keys' digits in four 16-bit fields of one u64, scans those across the block
// (warp shuffles plus one shared word per warp) and writes each key to its digit's offset plus
// the count of equal digits before it. About 30 instructions per key and pass, against the
// bitonic sort's log^2 m / 2 compare-exchange stages.
__device__ __forceinline__ void block_radix_sort_hi(u64 *buf, u32 m, u32 nbits, u64 *wsum) {
    constexpr u32 NW = CB_THREADS / 32;
    const u32 R = (m + CB_THREADS - 1) / CB_THREADS;
    const u32 t = threadIdx.x, lane = t & 31, w = t >> 5;
    u64 key[CB_SORT_R];
#pragma unroll
    for (u32 r = 0; r < CB_SORT_R; ++r) {
        const u32 i = t * R + r;
        key[r] = (r < R && i < m) ? buf[i] : 0;
    }
    for (u32 sh = 0; sh < nbits; sh += 2) {
        u64 cnt = 0, pre[CB_SORT_R];
#pragma unroll
        for (u32 r = 0; r < CB_SORT_R; ++r) {
            pre[r] = cnt;
            if (r < R && t * R + r < m) cnt += 1ull << (16 * ((u32)(key[r] >> (32 + sh)) & 3u));
        }
        u64 x = cnt;
#pragma unroll
        for (u32 o = 1; o < 32; o <<= 1) {
            const u64 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        u64 wpre = 0, tot = 0;
#pragma unroll
        for (u32 i = 0; i < NW; ++i) {
            if (i < w) wpre += wsum[i];
            tot += wsum[i];
        }
        const u64 excl = wpre + x - cnt;
        const u32 c0 = (u32)(tot & 0xFFFFu), c1 = (u32)((tot >> 16) & 0xFFFFu), c2 = (u32)((tot >> 32) & 0xFFFFu);
#pragma unroll
        for (u32 r = 0; r < CB_SORT_R; ++r) {
            if (r < R && t * R + r < m) {
                const u32 d = (u32)(key[r] >> (32 + sh)) & 3u;
                const u32 off = d == 0 ? 0u : d == 1 ? c0 : d == 2 ? c0 + c1 : c0 + c1 + c2;
                buf[off + (u32)(((excl + pre[r]) >> (16 * d)) & 0xFFFFu)] = key[r];
            }
        }
        __syncthreads();
#pragma unroll
        for (u32 r = 0; r < CB_SORT_R; ++r) {
            const u32 i = t * R + r;
            if (r < R && i < m) key[r] = buf[i];
        }
    }
}

// Sort, tables, slots and sweep of one hyperedge whose m movers (largest rank rmax) are in mvs,
// block-wide. The shared-memory kernel sorts up to CB_RADIX_MAX of them with the block radix sort
// (wsum set); more, and the scratch kernel's, sort bitonically. Direct tables leave tk to the sweep's lane masks (2K words, zeroed).
__device__ __forceinline__ void cascade_block_one(const CascadeArgs &A, u32 h, u64 *mvs, u32 *sl, u32 m, u32 rmax,
                                                  u32 *tk, u32 *tc, u32 *td, u32 cap, u64 *wsum) {
    const bool direct = cascade_direct(A);
    u32 P = 1;
    while (P < m) P <<= 1;
    const bool radix = wsum && m <= CB_RADIX_MAX;
    if (!radix)
        for (u32 i = m + threadIdx.x; i < P; i += blockDim.x) mvs[i] = ~0ull;
    for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { tc[i] = 0; td[i] = 0; }
    const u32 ntk = direct ? 2 * A.K : cap;
    for (u32 i = threadIdx.x; i < ntk; i += blockDim.x) tk[i] = direct ? 0u : NONE;
    __syncthreads();
    if (radix) block_radix_sort_hi(mvs, m, 32 - __clz(rmax), wsum);
    else block_bitonic_u64(mvs, P);
    cascade_fill(A, A.off[h], A.lam[h], tk, tc, td, cap, threadIdx.x, blockDim.x);
    __syncthreads();
    if (sl) {
        cascade_slots(A, mvs, sl, m, tk, cap, threadIdx.x, blockDim.x);
        __syncthreads();
    }
    if (sl) {
        if (threadIdx.x < 32) cascade_sweep_warp(A, h, mvs, sl, m, tk, tc, td, direct ? tk : nullptr);
    } else if (threadIdx.x == 0) {
        cascade_sweep(A, h, mvs, sl, m, tk, tc, td, cap - 1);
    }
    __syncthreads();
}

// Hyperedges with more movers than a warp takes: one block per hyperedge, everything in shared
// memory (dynamic: smov movers and their slots, then three tables of stab slots). A hyperedge
// with more than smov movers, or a hashed table above stab slots, is appended to `huge`.
__global__ void __launch_bounds__(CB_THREADS) k_cascade_block(CascadeArgs A, const u32 *__restrict__ list,
                                                              const u32 *__restrict__ nl, u32 smov, u32 stab,
                                                              u32 *__restrict__ huge, u32 *__restrict__ nhuge) {
    extern __shared__ __align__(16) unsigned char cb_smem[];
    __shared__ u32 cntm, smax;
    __shared__ u64 wsum[CB_THREADS / 32];
    u64 *mvs = (u64 *)cb_smem;
    u32 *sl = (u32 *)(mvs + smov), *tk = sl + smov, *tc = tk + stab, *td = tc + stab;
    const bool direct = cascade_direct(A);
    for (u32 idx = blockIdx.x; idx < *nl; idx += gridDim.x) {
        const u32 h = list[idx];
        u32 rmax;
        const u32 m = cascade_gather(A, h, mvs, smov, &cntm, &smax, rmax);
        const u32 cap = direct ? A.K : cascade_cap32(A.lam[h], m);
        if (m > smov || cap > stab) {
            if (threadIdx.x == 0) huge[atomicAdd(nhuge, 1u)] = h;
            continue;
        }
        cascade_block_one(A, h, mvs, sl, m, rmax, tk, tc, td, cap, wsum);
    }
}

// The rest: one block per SM, each with its slice of scratch regions sized by the level's
// largest hyperedge (mv_cap movers and slots, three tables of tab_cap slots).
__global__ void __launch_bounds__(CB_THREADS) k_cascade_huge(CascadeArgs A, const u32 *__restrict__ list,
                                                             const u32 *__restrict__ nl, u64 *scratch_mv,
                                                             u32 *scratch_sl, u32 *scratch_tab, u64 mv_cap,
                                                             u64 tab_cap) {
    __shared__ u32 cntm, smax;
    u64 *mvs = scratch_mv + (u64)blockIdx.x * mv_cap;
    u32 *tk = scratch_tab + (u64)blockIdx.x * 3 * tab_cap, *tc = tk + tab_cap, *td = tc + tab_cap;
    const bool direct = cascade_direct(A);
    for (u32 idx = blockIdx.x; idx < *nl; idx += gridDim.x) {
        const u32 h = list[idx];
        u32 rmax;
        const u32 m = cascade_gather(A, h, mvs, (u32)mv_cap, &cntm, &smax, rmax);
        const u32 cap = direct ? A.K : cascade_cap32(A.lam[h], m);
        // 16-bit slots cover every direct table and hashed tables of up to 65536 slots
        u32 *sl = (direct || cap <= 65536) ? scratch_sl + (u64)blockIdx.x * mv_cap : nullptr;
        cascade_block_one(A, h, mvs, sl, m, rmax, tk, tc, td, cap, nullptr);
    }
}

// ------------------------------------------------------------------ prefix and validity
// G[i] = the cascaded gain of the i-th mover; the two following nmax-entry blocks (the size and
// inbound violations) start at zero.
__global__ void k_gather_g2(const u32 *__restrict__ mv, const u32 *__restrict__ dM, u32 nmax,
                            const unsigned long long *__restrict__ g2, i64 *__restrict__ G) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nmax) {
        G[i] = i < *dM ? (i64)g2[mv[i]] : 0;
        G[(u64)nmax + i] = 0;
        G[2 * (u64)nmax + i] = 0;
    }
}

// size events: 2r = leave p, 2r+1 = join q
__global__ void k_size_events(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u32 *__restrict__ part,
                              const u32 *__restrict__ target, u32 *__restrict__ key, u32 *__restrict__ val) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * *dM) return;
    u32 v = mv[i >> 1];
    key[i] = (i & 1) ? target[v] : part[v];
    val[i] = i;
}
__global__ void k_size_delta(const u32 *__restrict__ mv, const u32 *__restrict__ val, const u32 *__restrict__ dne,
                             u32 nmax, const u32 *__restrict__ nsize, i64 *__restrict__ d) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmax) return;
    if (i >= *dne) { d[i] = 0; return; }
    u32 ev = val[i];
    i64 s = nsize[mv[ev >> 1]];
    d[i] = (ev & 1) ? s : -s;
}
__global__ void k_size_flags(const u32 *__restrict__ key, const u32 *__restrict__ val, const i64 *__restrict__ d,
                             const i64 *__restrict__ E, const u32 *__restrict__ dne, const u64 *__restrict__ psize,
                             u64 omega, unsigned long long *__restrict__ Vs) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 ne = *dne;
    if (i >= ne) return;
    u32 p = key[i];
    u32 st = lower_bound_u32(key, ne, p);
    i64 before = (i64)psize[p] + (E[i] - E[st]);
    i64 after = before + d[i];
    i64 exb = before > (i64)omega ? before - (i64)omega : 0;
    i64 exa = after > (i64)omega ? after - (i64)omega : 0;
    if (exa != exb) atomicAdd(&Vs[val[i] >> 1], (unsigned long long)(exa - exb));
}

__global__ void k_gather_by_dn(const u32 *__restrict__ src, const u32 *__restrict__ idx, u32 *__restrict__ dst,
                               const u32 *__restrict__ dn) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < *dn) dst[i] = src[idx[i]];
}
// transition keys: (partition, rank) in one word when both fit, else the rank alone (the
// partition is then a second stable pass). The count is clamped to the capacity nmax first (an
// overflow has already set the status word); later kernels read the clamped count.
__global__ void k_trans_keys(u32 *__restrict__ dT, u64 nmax, const u32 *__restrict__ tp,
                             const u32 *__restrict__ tr, u32 rbits, int combined, u32 *__restrict__ key,
                             u32 *__restrict__ perm) {
    u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 cnt = *dT < nmax ? *dT : nmax;
    if (j == 0 && cnt < *dT) atomicMin(dT, (u32)cnt);
    if (j >= cnt) return;
    key[j] = combined ? ((tp[j] << rbits) | tr[j]) : tr[j];
    perm[j] = (u32)j;
}
// after ordering by (p, r): partition, rank and delta of position i
__global__ void k_trans_perm(const u32 *__restrict__ perm, const u32 *__restrict__ dT, u64 nmax,
                             const u32 *__restrict__ tp, const u32 *__restrict__ tr, const int32_t *__restrict__ td,
                             u32 *__restrict__ sp, u32 *__restrict__ sr, i64 *__restrict__ sd) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmax) return;
    if (i >= *dT) { sd[i] = 0; return; }
    const u32 j = perm[i];
    sp[i] = tp[j];
    sr[i] = tr[j];
    sd[i] = td[j];
}
// per partition, the running inbound-set size along the move sequence; an event that makes the
// partition exceed delta adds +1 at its rank, one that brings it back adds -1. The first event of a
// partition assumes it started valid (kernels/refinement.cu:632-651).
__global__ void k_trans_flags(const u32 *__restrict__ sp, const u32 *__restrict__ sr, const i64 *__restrict__ sd,
                              const i64 *__restrict__ E, const u32 *__restrict__ dT, const u64 *__restrict__ pinb,
                              u64 delta, unsigned long long *__restrict__ Vi) {
    u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 nt = *dT;
    if (j >= nt) return;
    const u32 p = sp[j];
    const u32 st = lower_bound_u32(sp, nt, p);  // the partition's first transition (sp is sorted)
    const i64 before = (i64)pinb[p] + (E[j] - E[st]);
    const i64 after = before + sd[j];
    const bool was_bad = (j != st) && before > (i64)delta;
    const bool is_bad = after > (i64)delta;
    if (was_bad != is_bad) atomicAdd(&Vi[sr[j]], (unsigned long long)(i64)(is_bad ? 1 : -1));
}

// ---- size and inbound validity of every prefix on small levels: one block per partition ----------
// The same quantities as the event pipelines above (k_size_events ... k_size_flags and
// k_trans_keys ... k_trans_flags), without sorting: a partition's size events are its movers in
// rank order, and its inbound transitions arrive summed per rank (CascadeArgs::tdense).
//  - sizes: Vs[r] += excess(after rank r) - excess(before), excess = max(size - omega, 0);
//  - inbound: Vi[r] += bad(after r) - bad(before r) at each rank with transitions, bad = the
//    running inbound count above delta, and "before" taken as good at the partition's first
//    such rank (kernels/refinement.cu:632-651). Both telescope over the events of one rank, so
//    the order of events within a rank does not matter.
constexpr u32 VS_THREADS = 1024;
constexpr u32 VS_MAX_K = 256;    // partitions (blocks)

__device__ __forceinline__ i64 block_incl_scan_i64(i64 v, i64 *sh, i64 &total) {
    const u32 lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const i64 y = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if ((int)lane >= o) v += y;
    }
    __syncthreads();
    if (lane == 31) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        i64 x = lane < (blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const i64 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if ((int)lane >= o) x += y;
        }
        sh[lane] = x;  // inclusive warp prefixes
    }
    __syncthreads();
    total = sh[(blockDim.x >> 5) - 1];
    return v + (w ? sh[w - 1] : 0);
}
__global__ void __launch_bounds__(VS_THREADS) k_validity_small(
    const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u32 *__restrict__ part,
    const u32 *__restrict__ target, const u32 *__restrict__ nsize, const u64 *__restrict__ psize, u64 omega,
    unsigned long long *__restrict__ Vs, int track, const unsigned long long *__restrict__ tdense, u32 stride,
    const u64 *__restrict__ pinb, u64 delta, unsigned long long *__restrict__ Vi) {
    __shared__ i64 sh[32];
    const u32 p = blockIdx.x, M = *dM;
    i64 run = (i64)psize[p];
    const i64 om = (i64)omega;
    for (u32 base = 0; base < M; base += VS_THREADS) {
        const u32 r = base + threadIdx.x;
        i64 d = 0;
        if (r < M) {
            const u32 v = mv[r];
            if (part[v] == p) d = -(i64)nsize[v];
            else if (target[v] == p) d = (i64)nsize[v];
        }
        i64 tot;
        const i64 incl = block_incl_scan_i64(d, sh, tot);
        if (d != 0) {
            const i64 after = run + incl, before = after - d;
            const i64 dx = (after > om ? after - om : 0) - (before > om ? before - om : 0);
            if (dx) atomicAdd(&Vs[r], (unsigned long long)dx);
        }
        run += tot;
    }
    if (!track) return;
    const i64 dl = (i64)delta;
    i64 run2 = (i64)pinb[p];
    bool seen = false;  // a rank with transitions of p came before this chunk
    for (u32 base = 0; base < M; base += VS_THREADS) {
        const u32 r = base + threadIdx.x;
        const unsigned long long x = r < M ? tdense[(u64)p * stride + r] : 0ull;
        const bool has = (u32)x != 0u;
        const i64 D = has ? (i64)(int32_t)(u32)(x >> 32) : 0;
        i64 tot, htot;
        const i64 incl = block_incl_scan_i64(D, sh, tot);
        const i64 hincl = block_incl_scan_i64(has ? 1 : 0, sh, htot);
        if (has) {
            const i64 after = run2 + incl, before = after - D;
            const bool first = !seen && hincl == 1;
            const bool bad_before = !first && before > dl, bad_after = after > dl;
            if (bad_before != bad_after) atomicAdd(&Vi[r], (unsigned long long)(i64)(bad_after ? 1 : -1));
        }
        run2 += tot;
        seen = seen || htot > 0;
    }
}

// best prefix (best_move_functor): inbound-valid first, then fewer size violations, then larger
// gain, then the earlier rank.
struct Best {
    u32 ok;
    i64 vs, g;
    u32 r;
};
__device__ __forceinline__ bool best_better(const Best &b, const Best &a) {  // is b better than a
    if (a.ok != b.ok) return b.ok > a.ok;
    if (!a.ok) return b.r < a.r;
    if (a.vs != b.vs) return b.vs < a.vs;
    if (a.g != b.g) return b.g > a.g;
    return b.r < a.r;
}
__device__ __forceinline__ Best best_pick(const Best &a, const Best &b) {  // the better one; r = ~0 is empty
    if (b.r == 0xFFFFFFFFu) return a;
    if (a.r == 0xFFFFFFFFu) return b;
    return best_better(b, a) ? b : a;
}
__device__ __forceinline__ Best warp_best_prefix(Best b) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Best c;
        c.ok = __shfl_xor_sync(0xFFFFFFFFu, b.ok, o);
        c.vs = __shfl_xor_sync(0xFFFFFFFFu, b.vs, o);
        c.g = __shfl_xor_sync(0xFFFFFFFFu, b.g, o);
        c.r = __shfl_xor_sync(0xFFFFFFFFu, b.r, o);
        b = best_pick(b, c);
    }
    return b;
}
// ---- small levels (n <= RSS_CAP): ranking, and prefix sums + best prefix + apply, one block each ----
// The movers in id order, ranked by (gain desc, id asc): compaction by block scans, the stable
// radix sort of the descending gain keys (a second pass over the high words when the gain bound
// needs more than 32 bits), then the ranks. Also resets every node's rank and cascaded gain and
// writes the mover count and the size-event count, as k_move_flags ... k_set_rank do.
__global__ void __launch_bounds__(RSS_WARPS * 32) k_rank_small(u32 n, const u32 *__restrict__ target,
                                                              const i64 *__restrict__ gain, u64 gbound, u32 kb,
                                                              u32 *__restrict__ mv, u32 *__restrict__ rank,
                                                              unsigned long long *__restrict__ g2, u32 *__restrict__ dM,
                                                              u32 *__restrict__ twice) {
    extern __shared__ u32 sm[];
    __shared__ i64 sh[32];
    u32 M = 0;
    for (u32 b = 0; b < n; b += blockDim.x) {
        const u32 v = b + threadIdx.x;
        const bool f = v < n && target[v] != NONE;
        if (v < n) { rank[v] = NONE; g2[v] = 0; }
        i64 tot;
        const i64 incl = block_incl_scan_i64(f ? 1 : 0, sh, tot);
        if (f) {
            const u32 pos = M + (u32)incl - 1;
            sm[pos] = (u32)(gbound - (u64)gain[v]);
            sm[RSS_CAP + pos] = v;
        }
        M += (u32)tot;
    }
    const u32 *ko, *vo;
    block_radix_sort(sm, M, kb < 32 ? kb : 32, ko, vo);
    if (kb > 32) {  // high words of the movers in their low-word order
        u32 hv[RSS_ITEMS], nv[RSS_ITEMS];
#pragma unroll
        for (int k = 0; k < RSS_ITEMS; ++k) {
            const u32 i = threadIdx.x + (u32)k * blockDim.x;
            nv[k] = i < M ? vo[i] : 0u;
            hv[k] = i < M ? (u32)((gbound - (u64)gain[nv[k]]) >> 32) : 0u;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < RSS_ITEMS; ++k) {
            const u32 i = threadIdx.x + (u32)k * blockDim.x;
            if (i < M) { sm[i] = hv[k]; sm[RSS_CAP + i] = nv[k]; }
        }
        block_radix_sort(sm, M, kb - 32, ko, vo);
    }
    for (u32 i = threadIdx.x; i < M; i += blockDim.x) {
        const u32 v = vo[i];
        mv[i] = v;
        rank[v] = i;
    }
    if (threadIdx.x == 0) {
        *dM = M;
        *twice = 2 * M;
    }
}

// The inclusive prefix sums by rank of the cascaded gains, size violations (Vs) and inbound
// violations (Vi), the best prefix by best_better, and its application when it is valid with a
// non-negative gain: k_gather_g2, the 3n scan, k_best, k_best_final and k_apply in one block.
__global__ void __launch_bounds__(1024) k_tail_small(const u32 *__restrict__ mv, const u32 *__restrict__ dM,
                                                     const unsigned long long *__restrict__ g2,
                                                     const i64 *__restrict__ Vs, const i64 *__restrict__ Vi, int has_vi,
                                                     const u32 *__restrict__ target, u32 *__restrict__ part,
                                                     u32 *__restrict__ apply) {
    __shared__ i64 sh[32];
    __shared__ Best bsh[32];
    __shared__ i64 vsh[32];
    __shared__ Best s_best;
    __shared__ i64 s_vi;
    const u32 M = *dM, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) { s_best = Best{0, 0, 0, 0xFFFFFFFFu}; s_vi = 0; }
    i64 rg = 0, rs = 0, ri = 0;
    for (u32 base = 0; base < M; base += blockDim.x) {
        const u32 r = base + threadIdx.x;
        const bool in = r < M;
        i64 tg, ts, ti;
        const i64 pg = rg + block_incl_scan_i64(in ? (i64)g2[mv[r]] : 0, sh, tg);
        const i64 ps = rs + block_incl_scan_i64(in ? Vs[r] : 0, sh, ts);
        const i64 pi = ri + block_incl_scan_i64(in ? Vi[r] : 0, sh, ti);
        Best b{has_vi ? (pi == 0 ? 1u : 0u) : 1u, ps, pg, in ? r : 0xFFFFFFFFu};
        i64 bvi = pi;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            Best c;
            c.ok = __shfl_xor_sync(0xFFFFFFFFu, b.ok, o);
            c.vs = __shfl_xor_sync(0xFFFFFFFFu, b.vs, o);
            c.g = __shfl_xor_sync(0xFFFFFFFFu, b.g, o);
            c.r = __shfl_xor_sync(0xFFFFFFFFu, b.r, o);
            const i64 cvi = __shfl_xor_sync(0xFFFFFFFFu, bvi, o);
            const Best x = best_pick(b, c);
            if (x.r != b.r) bvi = cvi;
            b = x;
        }
        if (lane == 0) { bsh[w] = b; vsh[w] = bvi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            Best x = s_best;
            i64 xv = s_vi;
            for (u32 k = 0; k < blockDim.x / 32; ++k) {
                const Best y = best_pick(x, bsh[k]);
                if (y.r != x.r) xv = vsh[k];
                x = y;
            }
            s_best = x;
            s_vi = xv;
        }
        rg += tg;
        rs += ts;
        ri += ti;
    }
    __syncthreads();
    const Best x = s_best;
    const i64 vi = has_vi ? s_vi : 0;
    const bool ok = x.r != 0xFFFFFFFFu && x.vs <= 0 && vi <= 0 && x.g >= 0;
    if (threadIdx.x == 0) *apply = ok ? 1u : 0u;
    if (!ok) return;
    for (u32 i = threadIdx.x; i <= x.r; i += blockDim.x) {
        const u32 v = mv[i];
        part[v] = target[v];
    }
}

// best_better is a strict total order (ties end on the rank), so the tree reduction picks the
// same prefix as a sequential scan would.
// pre = inclusive scan of [gain deltas | size-violation deltas | inbound-violation deltas] by rank,
// each n long: the prefix of segment s at rank r is pre[s*n + r] - pre[s*n - 1].
__device__ __forceinline__ i64 seg_prefix(const i64 *pre, u32 n, u32 s, u32 r) {
    const u64 base = (u64)s * n;
    return pre[base + r] - (s ? pre[base - 1] : 0);
}
__global__ void k_best(const i64 *__restrict__ pre, u32 n, int has_vi, const u32 *__restrict__ dM,
                       Best *__restrict__ out) {
    __shared__ Best sh[32];
    Best b{0, 0, 0, 0xFFFFFFFFu};
    const u32 M = *dM;
    for (u32 r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const u32 ok = has_vi ? (seg_prefix(pre, n, 2, r) == 0 ? 1u : 0u) : 1u;
        Best c{ok, seg_prefix(pre, n, 1, r), seg_prefix(pre, n, 0, r), r};
        b = best_pick(b, c);
    }
    b = warp_best_prefix(b);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        Best x = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : Best{0, 0, 0, 0xFFFFFFFFu};
        x = warp_best_prefix(x);
        if (threadIdx.x == 0) out[blockIdx.x] = x;
    }
}
__global__ void k_best_final(const Best *__restrict__ in, u32 nb, const i64 *__restrict__ pre, u32 n, int has_vi,
                             Best *__restrict__ out, u32 *__restrict__ apply) {
    Best x = in[0];
    for (u32 i = 1; i < nb; ++i)
        if (in[i].r != 0xFFFFFFFFu && (x.r == 0xFFFFFFFFu || best_better(in[i], x))) x = in[i];
    *out = x;
    const i64 vi = (has_vi && x.r != 0xFFFFFFFFu) ? seg_prefix(pre, n, 2, x.r) : 0;
    *apply = (x.r != 0xFFFFFFFFu && x.vs <= 0 && vi <= 0 && x.g >= 0) ? 1u : 0u;
}
// With prev set (incremental census), a moved node's old partition and the round counter are kept.
__global__ void k_apply(const u32 *__restrict__ mv, const u32 *__restrict__ target, const Best *__restrict__ best,
                        const u32 *__restrict__ apply, u32 *__restrict__ part, u32 *__restrict__ prev,
                        u32 *__restrict__ stamp, const u32 *__restrict__ ctr) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (!*apply || i > best->r) return;
    u32 v = mv[i];
    if (prev) {
        prev[v] = part[v];
        stamp[v] = *ctr;
    }
    part[v] = target[v];
}

// Copies (the k-way multi-start): moves are sorted by copy last, so every copy owns one rank
// segment; ck[r] is the copy of rank r. One block per copy finds its segment's best prefix with
// the prefix values taken relative to the segment start, and decides its own application.
__global__ void k_copy_keys(const u32 *__restrict__ mv, const u32 *__restrict__ dM, u32 copy_n, u32 *__restrict__ ck) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < *dM) ck[i] = mv[i] / copy_n;
}
__global__ void k_best_seg(const i64 *__restrict__ pre, u32 n, int has_vi, const u32 *__restrict__ dM,
                           const u32 *__restrict__ ck, Best *__restrict__ best, u32 *__restrict__ capply,
                           u32 *__restrict__ apply) {
    __shared__ Best sh[32];
    const u32 M = *dM, t = blockIdx.x;
    const u32 s = lower_bound_u32(ck, M, t), e = lower_bound_u32(ck, M, t + 1);
    const i64 g0 = s ? seg_prefix(pre, n, 0, s - 1) : 0, v0 = s ? seg_prefix(pre, n, 1, s - 1) : 0;
    const i64 i0 = (s && has_vi) ? seg_prefix(pre, n, 2, s - 1) : 0;
    Best b{0, 0, 0, 0xFFFFFFFFu};
    for (u32 r = s + threadIdx.x; r < e; r += blockDim.x) {
        const u32 ok = has_vi ? (seg_prefix(pre, n, 2, r) - i0 == 0 ? 1u : 0u) : 1u;
        Best c{ok, seg_prefix(pre, n, 1, r) - v0, seg_prefix(pre, n, 0, r) - g0, r};
        b = best_pick(b, c);
    }
    b = warp_best_prefix(b);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x < 32) {
        Best x = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : Best{0, 0, 0, 0xFFFFFFFFu};
        x = warp_best_prefix(x);
        if (threadIdx.x == 0) {
            best[t] = x;
            const i64 vi = (has_vi && x.r != 0xFFFFFFFFu) ? seg_prefix(pre, n, 2, x.r) - i0 : 0;
            const u32 ap = (x.r != 0xFFFFFFFFu && x.vs <= 0 && vi <= 0 && x.g >= 0) ? 1u : 0u;
            capply[t] = ap;
            if (ap) atomicOr(apply, 1u);
        }
    }
}
__global__ void k_apply_seg(const u32 *__restrict__ mv, const u32 *__restrict__ dM, const u32 *__restrict__ ck,
                            const u32 *__restrict__ target, const Best *__restrict__ best,
                            const u32 *__restrict__ capply, u32 *__restrict__ part, u32 *__restrict__ prev,
                            u32 *__restrict__ stamp, const u32 *__restrict__ ctr) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *dM) return;
    const u32 t = ck[i];
    if (!capply[t] || i > best[t].r) return;
    const u32 v = mv[i];
    if (prev) {
        prev[v] = part[v];
        stamp[v] = *ctr;
    }
    part[v] = target[v];
}

GainArgs make_gain_args(const DLevel &L, const u32 *wfx, const RefineParams &rp, const Census &cs, const u32 *part,
                        const u64 *psize, const u64 *pinb, u32 discount, u32 round, u32 *target, i64 *gain,
                        u32 *status) {
    GainArgs A;
    A.n = L.n; A.omega = rp.omega; A.delta = rp.delta; A.discount = discount; A.round = round; A.K = rp.K;
    A.seed = (u32)rp.seed; A.encourage = rp.encourage ? 1 : 0;
    A.off = L.off; A.pins = L.pins; A.nsrc = L.nsrc; A.lam = cs.lam; A.cpart = cs.part; A.ccnt = cs.cnt; A.cdcnt = cs.dcnt; A.wfx = wfx;
    A.toff = L.toff; A.touch = L.touch; A.nin = L.nin; A.nsize = L.nsize; A.part = part;
    A.psize = psize; A.pinb = pinb; A.target = target; A.gain = gain; A.status = status;
    A.dyn = nullptr;
    A.save = cs.save;
    return A;
}

}  // namespace

// Work lists of one level for the census (hyperedge length tiers) and the gains (node gain-work
// bound tiers), plus the bounds that size per-round buffers. Built once per level.
struct LevelPrep {
    u32 *hblock = nullptr, n_hblock = 0;       // 256 < |e| <= 4096
    u32 *hhuge = nullptr, n_hhuge = 0;         // |e| > 4096
    u64 *huge_tab = nullptr, huge_tot = 0;     // table offsets of the huge hyperedges
    u32 *ntier[3] = {nullptr, nullptr, nullptr};
    u32 ncount[3] = {0, 0, 0};
    u64 *work = nullptr;     // per-node table bound of the gains
    u64 heavy_work_max = 0;  // largest gain-work bound of the heavy tier
    u64 block_work_max = 0;  // largest gain-work bound of the block tier (sizes its shared table)
    u64 gain_bound = 0;     // no gain exceeds this (sum of incident weights)
    u64 max_len = 0;         // largest hyperedge
    u64 dst_pins = 0;        // destination pins (bounds the inbound events: 2 per pin)
    u64 tier_deg[3] = {0, 0, 0};  // incidence entries of each gain tier (kernel timer only)
    u32 census_K = 0;        // nonzero: partition-indexed census over this many partitions, and
                             // hblock holds the hyperedges above CD_WARP_LEN pins
};

// Movers the cascade's block kernel keeps in shared memory: CB_MOV_MAX, or less when the context's
// tuning (c.tune.cascade_movers) or the environment variable AXC_CASCADE_BLOCK_MOVERS asks for it
// (a power of two >= 128), which sends hyperedges with more movers to the scratch kernel; the tests
// use it to reach that kernel on small inputs. Read at each level's launch.
static u32 cascade_block_movers(const Ctx &c) {
    unsigned long v = c.tune.cascade_movers;
    if (!v) {
        const char *s = std::getenv("AXC_CASCADE_BLOCK_MOVERS");
        if (!s || !*s) return CB_MOV_MAX;
        v = std::strtoul(s, nullptr, 10);
    }
    u32 lim = 128;
    while ((unsigned long)lim * 2 <= v && lim < CB_MOV_MAX) lim <<= 1;
    return lim;
}

// The incremental census is on unless the environment variable AXC_INC_CENSUS is "0" (then every
// round rebuilds the census; the same results).
static bool inc_census_enabled() {
    const char *s = std::getenv("AXC_INC_CENSUS");
    return !(s && s[0] == '0');
}

static bool round_loop_enabled() {
    const char *s = std::getenv("AXC_ROUND_LOOP");
    return !(s && s[0] == '0');
}

void setup_refine_kernels(Ctx &c) {
    AXC_CUDA(cudaFuncSetAttribute(k_census_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * 2 * CS_BLOCK_CAP * 4));
    AXC_CUDA(cudaFuncSetAttribute(k_gain_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * GN_BLOCK_W * 16));
    AXC_CUDA(cudaFuncSetAttribute(k_cascade_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CB_DYN_MAX));
    AXC_CUDA(cudaFuncSetAttribute(k_gain_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GS_SMEM));
    AXC_CUDA(cudaFuncSetAttribute(k_gain_sample, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    AXC_CUDA(cudaFuncSetAttribute(k_cands_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CV_BLOCK_SMEM));
    AXC_CUDA(cudaFuncSetAttribute(k_rank_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RSS_SMEM));
}

__global__ void k_level_bounds(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ nsrc,
                               unsigned long long *__restrict__ out);

// Largest gain-work bound over all nodes (out[0]) and over the block tier (out[1]).
__global__ void k_tier_max(u32 n, u32 K, const u64 *__restrict__ work, const u64 *__restrict__ toff,
                           unsigned long long *__restrict__ out) {
    u32 u = blockIdx.x * blockDim.x + threadIdx.x;
    u64 all = 0, blk = 0;
    if (u < n) {
        const u64 wk = work[u], deg = toff[u + 1] - toff[u];
        all = wk;
        if (gain_tier(n, K, wk, deg) == 1u) blk = wk;
    }
    all = warp_max_u64(all);
    blk = warp_max_u64(blk);
    if ((threadIdx.x & 31) == 0) {
        if (all) atomicMax(&out[0], (unsigned long long)all);
        if (blk) atomicMax(&out[1], (unsigned long long)blk);
    }
}

// Everything the level's rounds need sized on the host comes back in one round trip (a second
// one only when some hyperedge is longer than CS_BLOCK_CAP).
static LevelPrep prepare_level(Ctx &c, const DLevel &L, const u32 *wfx, u32 K) {
    LevelPrep lp;
    const u32 e = L.e, n = L.n;
    // [0] census block list, [1] census huge list, [2..4] node tiers, [5] gain bound,
    // [6] largest work, [7] largest block-tier work, [8] largest hyperedge, [9] destination pins
    u64 *dc = c.arena.alloc<u64>(10);
    AXC_CUDA(cudaMemsetAsync(dc, 0, 80, c.stream));
    lp.census_K = K <= CD_K ? K : 0;
    if (e) {
        u32 *flag = c.arena.alloc<u32>(e);
        lp.hblock = c.arena.alloc<u32>(e);
        if (lp.census_K) {  // partition-indexed census: a warp, or a block above CD_WARP_LEN pins
            LAUNCH(c, k_flag_len, cdiv(e, 256), 256, 0, e, L.off, (u64)CD_WARP_LEN, ~0ull, flag);
            compact_indices_dn(c, flag, lp.hblock, e, (u32 *)(dc + 0));
        } else {
            lp.hhuge = c.arena.alloc<u32>(e);
            LAUNCH(c, k_flag_len, cdiv(e, 256), 256, 0, e, L.off, (u64)CS_WARP_CAP, (u64)CS_BLOCK_CAP, flag);
            compact_indices_dn(c, flag, lp.hblock, e, (u32 *)(dc + 0));
            LAUNCH(c, k_flag_len, cdiv(e, 256), 256, 0, e, L.off, (u64)CS_BLOCK_CAP, ~0ull, flag);
            compact_indices_dn(c, flag, lp.hhuge, e, (u32 *)(dc + 1));
        }
        LAUNCH(c, k_level_bounds, cdiv(e, 256), 256, 0, e, L.off, L.nsrc, (unsigned long long *)(dc + 8));
    }
    if (n) {
        u64 *work = c.arena.alloc<u64>(n);
        lp.work = work;
        LAUNCH(c, k_gain_bounds, cdiv((u64)n * 32, 256), 256, 0, n, K, L.toff, L.touch, L.off, wfx, work,
               (unsigned long long *)(dc + 5));
        u32 *flag = c.arena.alloc<u32>(n);
        for (u32 t = 0; t < 3; ++t) {
            lp.ntier[t] = c.arena.alloc<u32>(n);
            LAUNCH(c, k_tier, cdiv(n, 256), 256, 0, n, K, work, L.toff, t, flag);
            compact_indices_dn(c, flag, lp.ntier[t], n, (u32 *)(dc + 2 + t));
        }
        LAUNCH(c, k_tier_max, cdiv(n, 256), 256, 0, n, K, work, L.toff, (unsigned long long *)(dc + 6));
    }
    u64 h[10];
    fetch(c, h, dc, 80);
    lp.n_hblock = (u32)h[0];
    lp.n_hhuge = (u32)h[1];
    for (int t = 0; t < 3; ++t) lp.ncount[t] = (u32)h[2 + t];
    lp.gain_bound = h[5];
    lp.heavy_work_max = lp.ncount[2] ? h[6] : 0;
    lp.block_work_max = h[7];
    lp.max_len = h[8];
    lp.dst_pins = h[9];
    if (lp.n_hhuge) {
        lp.huge_tab = c.arena.alloc<u64>(lp.n_hhuge + 1);
        LAUNCH(c, k_tab_sizes, cdiv(lp.n_hhuge + 1, 256), 256, 0, lp.hhuge, lp.n_hhuge, L.off, lp.huge_tab);
        scan_excl_u64(c, lp.huge_tab, lp.huge_tab, lp.n_hhuge + 1);
        lp.huge_tot = fetch1(c, lp.huge_tab + lp.n_hhuge);
    }
    if (n) {
        if (c.profiling("k_gain_warp") || c.profiling("k_gain_block")) {
            unsigned long long *dg = c.arena.alloc<unsigned long long>(3);
            AXC_CUDA(cudaMemsetAsync(dg, 0, 24, c.stream));
            for (int t = 0; t < 3; ++t)
                LAUNCH(c, k_list_degree, cdiv(lp.ncount[t], 256), 256, 0, lp.ntier[t], lp.ncount[t], L.toff, dg + t);
            fetch(c, lp.tier_deg, dg, 24);
        }
    }
    return lp;
}

// Longest hyperedge a block-tier table must hold: the level's longest, capped by the tier's bound
// (the bound itself when the level's is not known).
static u64 block_tier_len(const LevelPrep &lp, u64 bound) { return lp.max_len && lp.max_len < bound ? lp.max_len : bound; }

static void run_census(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *part, Census &cs) {
    cs.beg = L.off;
    if (L.e == 0) return;
    CensusArgs A{L.off, L.pins, L.nsrc, part, cs.part, cs.cnt, cs.dcnt, cs.lam, c.d_status,
                 (unsigned long long *)cs.save, cs.wfx, cs.encourage, nullptr, nullptr, 0, nullptr};
    if (c.profiling("k_census_direct_warp")) A.pbytes = c.d_prof_bytes();
    if (lp.census_K) {
        A.mask = cs.mask;  // masks come with the partition-indexed census
        A.dmask = cs.dmask;
        A.mw = cs.mw;
        LAUNCH(c, k_census_direct_warp, cdiv(L.e, CS_WARPS), CS_WARPS * 32, 0, L.e, A, lp.census_K);
        if (lp.n_hblock)
            LAUNCH(c, k_census_direct_block, lp.n_hblock, 256, 0, lp.hblock, lp.n_hblock, A, lp.census_K);
        return;
    }
    LAUNCH(c, k_census_warp, cdiv(L.e, CS_WARPS), CS_WARPS * 32, 0, L.e, A);
    if (lp.n_hblock)
        LAUNCH(c, k_census_block, lp.n_hblock, 256, 16 * (size_t)cs_cap(block_tier_len(lp, CS_BLOCK_CAP)),
               lp.hblock, lp.n_hblock, A,
               (u32 *)nullptr, (const u64 *)nullptr);
    if (lp.n_hhuge) {
        size_t m = c.arena.mark();
        u32 *gtab = c.arena.alloc<u32>(4 * lp.huge_tot);
        LAUNCH(c, k_census_block, lp.n_hhuge, 512, 0, lp.hhuge, lp.n_hhuge, A, gtab, (const u64 *)lp.huge_tab);
        c.arena.release(m);
    }
}

static Census alloc_census(Ctx &c, const DLevel &L) {
    Census cs;
    cs.beg = L.off;
    cs.part = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.cnt = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.dcnt = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.lam = c.arena.alloc<u32>(L.e ? L.e : 1);
    return cs;
}

// Algorithmic bytes of one gains launch over a node list: 8 per incidence entry (the touching id
// and the census reads of the node's own and the candidate partitions) and 16 per node (its
// move, gain and rank).
static u64 gain_bytes(const LevelPrep &lp, int t) { return 8 * lp.tier_deg[t] + 16 * (u64)lp.ncount[t]; }

// Distinct partitions a node may reach in the first try of the heavy gain tier: 3/4 of the
// table, or fewer when the environment variable AXC_GAIN_TRY_LIMIT asks for it (at least 1),
// which sends more nodes to the global retry; the tests use it to reach that path on small inputs.
static u32 gain_try_limit(u32 cap) {
    const u32 lim = cap / 4 * 3;
    const char *s = std::getenv("AXC_GAIN_TRY_LIMIT");
    if (!s || !*s) return lim;
    const unsigned long v = std::strtoul(s, nullptr, 10);
    return v < 1 ? 1u : (v < lim ? (u32)v : lim);
}

template <u32 MW>
static void run_gains_masked(Ctx &c, const LevelPrep &lp, const GainArgs &A, const Census &cs) {
    if (lp.ncount[0])
        LAUNCH(c, k_gain_mask_warp<MW>, cdiv(lp.ncount[0], GN_WARPS), GN_WARPS * 32, 0, A, lp.ntier[0], lp.ncount[0],
               cs.mask, cs.dmask);
    if (lp.ncount[1])
        LAUNCH(c, k_gain_mask_block<MW>, lp.ncount[1], GN_BLOCK, 0, A, lp.ntier[1], lp.ncount[1], cs.mask, cs.dmask);
}

static void run_gains(Ctx &c, const DLevel &L, const LevelPrep &lp, const GainArgs &A, const Census &cs) {
    if (cs.mask) {  // partition-indexed gains (K <= GN_DIRECT_K); their two tiers write every node
        if (c.profiling("k_gain_mask_warp")) c.prof_bytes += gain_bytes(lp, 0);
        if (c.profiling("k_gain_mask_block")) c.prof_bytes += gain_bytes(lp, 1);
        switch (cs.mw) {
            case 1: run_gains_masked<1>(c, lp, A, cs); break;
            case 2: run_gains_masked<2>(c, lp, A, cs); break;
            case 4: run_gains_masked<4>(c, lp, A, cs); break;
            default: run_gains_masked<8>(c, lp, A, cs); break;
        }
        return;
    }
    fill_u32(c, A.target, NONE, L.n);
    if (c.profiling("k_gain_warp") && lp.ncount[0]) c.prof_bytes += gain_bytes(lp, 0);
    if (c.profiling("k_gain_block")) c.prof_bytes += gain_bytes(lp, 1) + gain_bytes(lp, 2);
    LAUNCH(c, k_gain_warp, cdiv(lp.ncount[0], GN_WARPS), GN_WARPS * 32, 0, A, lp.ntier[0], lp.ncount[0], lp.work);
    if (lp.ncount[1]) {
        // shared table sized by the tier's largest bound (16 B per slot)
        u32 cap1 = table_cap(lp.block_work_max, 2 * GN_BLOCK_W);
        if (A.K <= GN_DIRECT_K)  // indexed by partition id: K slots (rounded up) per node
            while (cap1 < A.K) cap1 <<= 1;
        LAUNCH(c, k_gain_block, lp.ncount[1], GN_BLOCK, cap1 * 16, A, lp.ntier[1], lp.ncount[1], (const u32 *)nullptr,
               cap1, (u32 *)nullptr, (u32 *)nullptr, lp.work, 0u, (u32 *)nullptr, (u32 *)nullptr);
    }
    if (lp.ncount[2] && A.K > GS_K) {  // the sampled rule (include/axc.h AXC_SPARSE_GAIN_*)
        size_t m = c.arena.mark();
        const u32 rows = lp.ncount[2];
        CandAcc C;
        C.cand = c.arena.alloc<u32>((u64)L.n * GS_C);
        C.spos = c.arena.alloc<u32>(L.n);
        C.conn = c.arena.alloc<unsigned long long>((u64)rows * GS_C);
        C.dcon = c.arena.alloc<u32>((u64)rows * GS_C);
        C.sacc = c.arena.alloc<unsigned long long>(rows);
        C.wacc = c.arena.alloc<unsigned long long>(rows);
        fill_u32(c, C.spos, NONE, L.n);
        LAUNCH(c, k_gain_sample, std::min<u32>(rows, (u32)c.sms * GS_PER_SM), GS_BLOCK, GS_SMEM, A, lp.ntier[2], rows, C);
        LAUNCH(c, k_cands_warp, cdiv(L.e, CV_WARPS), CV_WARPS * 32, 0, A, C, L.e);
        if (lp.n_hblock)
            LAUNCH(c, k_cands_block, lp.n_hblock, CV_BLOCK, 8 * (size_t)cs_cap(block_tier_len(lp, CV_BLOCK_LEN)), A,
                   C, lp.hblock, lp.n_hblock, (u32 *)nullptr,
                   (const u64 *)nullptr);
        if (lp.n_hhuge) {
            u32 *gtab = c.arena.alloc<u32>(2 * lp.huge_tot);
            LAUNCH(c, k_cands_block, lp.n_hhuge, CV_BLOCK, 0, A, C, lp.hhuge, lp.n_hhuge, gtab, (const u64 *)lp.huge_tab);
        }
        LAUNCH(c, k_cands_best, cdiv(rows, 256), 256, 0, A, C, lp.ntier[2], rows);
        c.arena.release(m);
    } else if (lp.ncount[2]) {
        size_t m = c.arena.mark();
        const u32 *heavy = lp.ntier[2];
        const u32 *dn = nullptr;
        if (A.K > GN_DIRECT_K) {
            // Bounds overestimate: partitions recur across a node's hyperedges. First try with the
            // largest shared table; a node with more than 3/4 of its slots distinct is retried.
            const u32 cap_try = 2 * GN_BLOCK_W;
            u32 *retry = c.arena.alloc<u32>(lp.ncount[2]), *nretry = c.arena.alloc<u32>(1);
            AXC_CUDA(cudaMemsetAsync(nretry, 0, 4, c.stream));
            LAUNCH(c, k_gain_block, lp.ncount[2], GN_BLOCK, cap_try * 16, A, lp.ntier[2], lp.ncount[2],
                   (const u32 *)nullptr, cap_try, (u32 *)nullptr, (u32 *)nullptr, lp.work, gain_try_limit(cap_try), retry,
                   nretry);
            heavy = retry;
            dn = nretry;
        }
        u32 cap = 64;
        while (cap < 2 * lp.heavy_work_max && cap < (1u << 28)) cap <<= 1;
        u32 grid = lp.ncount[2] < (u32)c.sms * 2 ? lp.ncount[2] : (u32)c.sms * 2;
        u32 *gtab = c.arena.alloc<u32>((u64)grid * 4 * cap), *gused = c.arena.alloc<u32>((u64)grid * cap);
        LAUNCH(c, k_gain_block, grid, GN_BLOCK, 0, A, heavy, lp.ncount[2], dn, cap, gtab, gused, lp.work, 0u,
               (u32 *)nullptr, (u32 *)nullptr);
        c.arena.release(m);
    }
}

Census build_census(Ctx &c, const DLevel &L, const u32 *part) {
    Census cs = alloc_census(c, L);
    size_t m = c.arena.mark();
    LevelPrep lp;
    if (L.e) {
        u32 *flag = c.arena.alloc<u32>(L.e);
        lp.hblock = c.arena.alloc<u32>(L.e);
        LAUNCH(c, k_flag_len, cdiv(L.e, 256), 256, 0, L.e, L.off, (u64)CS_WARP_CAP, (u64)CS_BLOCK_CAP, flag);
        lp.n_hblock = compact_indices(c, flag, lp.hblock, L.e);
        lp.hhuge = c.arena.alloc<u32>(L.e);
        LAUNCH(c, k_flag_len, cdiv(L.e, 256), 256, 0, L.e, L.off, (u64)CS_BLOCK_CAP, ~0ull, flag);
        lp.n_hhuge = compact_indices(c, flag, lp.hhuge, L.e);
        if (lp.n_hhuge) {
            lp.huge_tab = c.arena.alloc<u64>(lp.n_hhuge + 1);
            LAUNCH(c, k_tab_sizes, cdiv(lp.n_hhuge + 1, 256), 256, 0, lp.hhuge, lp.n_hhuge, L.off, lp.huge_tab);
            scan_excl_u64(c, lp.huge_tab, lp.huge_tab, lp.n_hhuge + 1);
            lp.huge_tot = fetch1(c, lp.huge_tab + lp.n_hhuge);
        }
    }
    run_census(c, L, lp, part, cs);
    c.arena.release(m);
    return cs;
}

void part_sizes(Ctx &c, u32 n, const u32 *part, const u32 *nsize, u64 *psize, u32 K) {
    AXC_CUDA(cudaMemsetAsync(psize, 0, (size_t)K * 8, c.stream));
    if (n && K <= PS_SMEM_K)
        LAUNCH(c, k_part_sizes_smem, std::min<u32>(cdiv(n, 256), (u32)c.sms * 4), 256, 0, n, K, part, nsize,
               (unsigned long long *)psize);
    else if (n)
        LAUNCH(c, k_part_sizes, cdiv(n, 256), 256, 0, n, part, nsize, (unsigned long long *)psize);
}
void part_inbound(Ctx &c, const DLevel &L, const Census &cs, u64 *pinb, u32 K) {
    AXC_CUDA(cudaMemsetAsync(pinb, 0, (size_t)K * 8, c.stream));
    if (L.e && K <= PI_SMEM_K) {  // per-block counts in shared memory, one global add per partition
        const u32 grid = std::min<u32>(cdiv(L.e, 256 / 32), 2 * (u32)c.sms);
        LAUNCH(c, k_part_inbound_smem, grid, 256, (size_t)K * 4, L.e, L.off, cs.lam, cs.part, cs.dcnt, K,
               (unsigned long long *)pinb);
    } else if (L.e)
        LAUNCH(c, k_part_inbound, cdiv((u64)L.e * 32, 256), 256, 0, L.e, L.off, cs.lam, cs.part, cs.dcnt,
               (unsigned long long *)pinb);
}

// Whether a round needs the partitions' inbound counts. With no inbound limit (delta 2^31 - 1,
// k-way) the inbound check pinb[q] + nin[u] - dc > delta never holds while the level has fewer
// than 2^30 hyperedges (both terms are at most e), so zero counts decide it the same way.
static bool inbound_binds(const DLevel &L, const RefineParams &rp) {
    return rp.delta < 0x7FFFFFFFu || (u64)L.e >= (1ull << 30);
}

// Mask words per hyperedge for K partitions: 1, 2, 4 or 8.
static u32 mask_words(u32 K) {
    u32 mw = 1;
    while (32 * mw < K) mw <<= 1;
    return mw;
}

// The round's census, with the extras of the partition-indexed gains when K <= GN_DIRECT_K:
// each node's saving (pushed by the census pass) and the per-hyperedge masks.
static Census census_for_gains(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *wfx, const RefineParams &rp,
                               const u32 *part) {
    Census cs = alloc_census(c, L);
    const bool direct = rp.K <= GN_DIRECT_K;
    if (direct) {
        cs.save = c.arena.alloc<i64>(L.n ? L.n : 1);
        AXC_CUDA(cudaMemsetAsync(cs.save, 0, (size_t)L.n * 8, c.stream));
        cs.wfx = wfx;
        cs.encourage = rp.encourage ? 1 : 0;
    }
    if (direct) {
        cs.mw = mask_words(rp.K);
        cs.mask = c.arena.alloc<u32>((u64)(L.e ? L.e : 1) * cs.mw);
        cs.dmask = c.arena.alloc<u32>((u64)(L.e ? L.e : 1) * cs.mw);
    }
    run_census(c, L, lp, part, cs);
    if (direct && L.e && !lp.census_K)  // a hashed census: masks from its entries
        LAUNCH(c, k_census_masks, cdiv((u64)L.e * 32, 256), 256, 0, L.e, L.off, cs.lam, cs.part, cs.dcnt, cs.mw,
               cs.mask, cs.dmask);
    return cs;
}

void refine_gains_only(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, const u32 *part,
                       u32 discount, u32 round, u32 *target, i64 *gain) {
    size_t m = c.arena.mark();
    LevelPrep lp = prepare_level(c, L, wfx, rp.K);
    Census cs = census_for_gains(c, L, lp, wfx, rp, part);
    u64 *psize = c.arena.alloc<u64>(rp.K), *pinb = c.arena.alloc<u64>(rp.K);
    part_sizes(c, L.n, part, L.nsize, psize, rp.K);
    part_inbound(c, L, cs, pinb, rp.K);
    GainArgs A = make_gain_args(L, wfx, rp, cs, part, psize, pinb, discount, round, target, gain, c.d_status);
    run_gains(c, L, lp, A, cs);
    check_status(c);
    c.arena.release(m);
}

// The level-persistent census of the incremental rounds (k_census_inc_*), for levels with a
// partition-indexed census (K <= CD_K) that are not small.
struct IncCensus {
    Census cs;              // entries, counts, masks and node savings, kept across the rounds
    u32 *dirty = nullptr;   // [e] hyperedges to recompute at the next census (all before round 0)
    u32 *dlist = nullptr;   // [e] their compacted list
    u32 *prev = nullptr;    // [n] a moved node's partition before its last move
    u32 *stamp = nullptr;   // [n] the round counter at the node's last move (NONE: none)
    u32 *ctr = nullptr;     // [0] rounds run at this level, [1] the list count, [2] the warps' work
};

static bool inc_census_eligible(const DLevel &L, const LevelPrep &lp, const RefineParams &rp) {
    const bool small = rp.K <= VS_MAX_K && L.n <= (u32)RSS_CAP && rp.copies == 1;
    return lp.census_K && rp.K <= GN_DIRECT_K && !small && L.e;
}

static void inc_census_init(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, IncCensus &ic) {
    ic.cs = alloc_census(c, L);
    ic.cs.save = c.arena.alloc<i64>(L.n ? L.n : 1);
    AXC_CUDA(cudaMemsetAsync(ic.cs.save, 0, (size_t)L.n * 8, c.stream));
    ic.cs.wfx = wfx;
    ic.cs.encourage = rp.encourage ? 1 : 0;
    ic.cs.mw = mask_words(rp.K);
    ic.cs.mask = c.arena.alloc<u32>((u64)L.e * ic.cs.mw);
    ic.cs.dmask = c.arena.alloc<u32>((u64)L.e * ic.cs.mw);
    ic.dirty = c.arena.alloc<u32>(L.e);
    ic.dlist = c.arena.alloc<u32>(L.e);
    ic.prev = c.arena.alloc<u32>(L.n ? L.n : 1);
    ic.stamp = c.arena.alloc<u32>(L.n ? L.n : 1);
    ic.ctr = c.arena.alloc<u32>(4);
    fill_u32(c, ic.dirty, 1u, L.e);
    fill_u32(c, ic.stamp, NONE, L.n);
    AXC_CUDA(cudaMemsetAsync(ic.ctr, 0, 16, c.stream));
}

// The round's census in incremental form: the flagged hyperedges are listed, recomputed and
// unflagged.
static void inc_census_round(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *part, IncCensus &ic) {
    const Census &cs = ic.cs;
    CensusArgs A{L.off, L.pins, L.nsrc, part, cs.part, cs.cnt, cs.dcnt, cs.lam, c.d_status,
                 (unsigned long long *)cs.save, cs.wfx, cs.encourage, cs.mask, cs.dmask, cs.mw, nullptr};
    if (c.profiling("k_census_inc_warp")) A.pbytes = c.d_prof_bytes();
    compact_indices_dn(c, ic.dirty, ic.dlist, L.e, ic.ctr + 1);
    AXC_CUDA(cudaMemsetAsync(ic.ctr + 2, 0, 4, c.stream));
    const IncArgs I{ic.dlist, ic.ctr + 1, ic.ctr + 2, ic.dirty, ic.prev, ic.stamp, ic.ctr};
    int per_sm = 1;
    AXC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_census_inc_warp, CS_WARPS * 32, 0));
    LAUNCH(c, k_census_inc_warp, std::min<u32>(cdiv(L.e, CS_WARPS), (u32)c.sms * (u32)std::max(per_sm, 1)),
           CS_WARPS * 32, 0, A, lp.census_K, I);
    if (lp.n_hblock) LAUNCH(c, k_census_inc_block, lp.n_hblock, 256, 0, lp.hblock, lp.n_hblock, A, lp.census_K, I);
    AXC_CUDA(cudaMemsetAsync(ic.dirty, 0, (size_t)L.e * 4, c.stream));
}

// The launches of one round, with no host synchronization: safe to capture in a CUDA graph.
// dyn (device, optional) holds the round's discount and round number for graph replays. Returns
// the device word that says whether the moves were applied; its arena slot lies below `keep`,
// the mark the caller releases to after reading it.
static u32 *round_body(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *wfx, const RefineParams &rp,
                       u32 *part, u32 discount, u32 round, const u32 *dyn, size_t &keep, IncCensus *ic) {
    const u32 n = L.n;
    u32 *apply = c.arena.alloc<u32>(1);
    keep = c.arena.mark();
    Census cs;
    if (ic) {
        inc_census_round(c, L, lp, part, *ic);
        cs = ic->cs;
    } else {
        cs = census_for_gains(c, L, lp, wfx, rp, part);
    }
    u64 *psize = c.arena.alloc<u64>(rp.K), *pinb = c.arena.alloc<u64>(rp.K);
    part_sizes(c, n, part, L.nsize, psize, rp.K);
    if (inbound_binds(L, rp)) {
        part_inbound(c, L, cs, pinb, rp.K);
    } else {
        AXC_CUDA(cudaMemsetAsync(pinb, 0, (size_t)rp.K * 8, c.stream));
    }
    u32 *target = c.arena.alloc<u32>(n);
    i64 *gain = c.arena.alloc<i64>(n);
    GainArgs A = make_gain_args(L, wfx, rp, cs, part, psize, pinb, discount, round, target, gain, c.d_status);
    A.dyn = dyn;
    run_gains(c, L, lp, A, cs);
    // counters on the device: [0] M movers, [1] 2M size events, [2] inbound transitions,
    // [3] cascade hyperedges for the block kernel, [4] for the scratch kernel, [5] for the block
    // kernel's full-size launch after its middle tier, [6] hyperedges holding a mover
    u32 *cnt = c.arena.alloc<u32>(8);
    AXC_CUDA(cudaMemsetAsync(cnt, 0, 32, c.stream));
    u32 *dM = cnt, *dSE = cnt + 1, *dT = cnt + 2, *dBig = cnt + 3, *dHuge = cnt + 4, *dBig2 = cnt + 5;
    u32 *dHl = cnt + 6;  // hyperedges holding a mover
    // small levels: ranking, validity and the best prefix in one block each (SMALL_*)
    const bool small = rp.K <= VS_MAX_K && n <= (u32)RSS_CAP && rp.copies == 1;
    // movers in id order, then ranked by (gain desc, id asc)
    u32 *flag = c.arena.alloc<u32>(n), *mv = c.arena.alloc<u32>(n), *rank = c.arena.alloc<u32>(n);
    unsigned long long *g2 = c.arena.alloc<unsigned long long>(n);  // cascaded gains, zeroed here
    const u32 kb = bits_for(lp.gain_bound);
    u32 *khi = c.arena.alloc<u32>(n), *klo = c.arena.alloc<u32>(n);
    if (small) {
        LAUNCH(c, k_rank_small, 1, RSS_WARPS * 32, RSS_SMEM, n, target, gain, lp.gain_bound, kb, mv, rank, g2, dM, dSE);
    } else {
    LAUNCH(c, k_move_flags, cdiv(n, 256), 256, 0, n, target, flag, rank, g2);
    compact_indices_dn(c, flag, mv, n, dM);
    LAUNCH(c, k_move_keys, cdiv(n, 256), 256, 0, mv, dM, gain, lp.gain_bound, khi, klo);
    if (kb > 32) {
        // stable by the low word, then by the high word (a 64-bit LSD sort); the high words are
        // recomputed for the permuted movers between the two passes
        u32 *tmp = c.arena.alloc<u32>(n);
        radix_sort_pairs_dn(c, klo, mv, dM, n, 32);
        LAUNCH(c, k_move_keys, cdiv(n, 256), 256, 0, mv, dM, gain, lp.gain_bound, khi, tmp);
        radix_sort_pairs_dn(c, khi, mv, dM, n, kb - 32);
    } else {
        radix_sort_pairs_dn(c, klo, mv, dM, n, kb);
    }
    }
    const bool pairs = !rp.encourage && rp.K <= PAIR_RANK_MAX_K;
    if (pairs) {  // k-way: moves in p <-> q pairs
        u32 *gk = khi, *pos = klo;  // the gain keys are spent
        LAUNCH(c, k_pair_group, cdiv(n, 256), 256, 0, mv, dM, part, target, rp.K, gk, pos);
        radix_sort_pairs_dn(c, gk, pos, dM, n, bits_for(2 * (u64)rp.K * rp.K));
        i64 *psn = c.arena.alloc<i64>(n);
        u32 *k1 = c.arena.alloc<u32>(n), *node = c.arena.alloc<u32>(n);
        LAUNCH(c, k_pair_keys, cdiv(n, 256), 256, 0, gk, pos, dM, mv, gain, psn, k1, node);
        radix_sort_pairs_dn(c, k1, node, dM, n, bits_for(2 * (u64)n));
        const u64 pbound = 2 * lp.gain_bound;
        const u32 pb = bits_for(pbound);
        LAUNCH(c, k_pair_gain_keys, cdiv(n, 256), 256, 0, node, dM, psn, pbound, khi, klo);
        radix_sort_pairs_dn(c, klo, node, dM, n, pb < 32 ? pb : 32);
        if (pb > 32) {
            LAUNCH(c, k_pair_gain_keys, cdiv(n, 256), 256, 0, node, dM, psn, pbound, khi, klo);
            radix_sort_pairs_dn(c, khi, node, dM, n, pb - 32);
        }
        AXC_CUDA(cudaMemcpyAsync(mv, node, (size_t)n * 4, cudaMemcpyDeviceToDevice, c.stream));
    }
    u32 *ck = nullptr;  // copies: the copy of every rank, ascending
    if (rp.copies > 1) {
        ck = c.arena.alloc<u32>(n);
        LAUNCH(c, k_copy_keys, cdiv(n, 256), 256, 0, mv, dM, rp.copy_n, ck);
        radix_sort_pairs_dn(c, ck, mv, dM, n, bits_for(rp.copies - 1));
    }
    if (!small || pairs || rp.copies > 1) LAUNCH(c, k_set_rank, cdiv(n, 256), 256, 0, mv, dM, rank, dSE);
    // cascade

    // inbound-set transitions (INCC): each destination pin of a mover gives at most two
    const bool track = rp.delta < 0x7FFFFFFFu && lp.dst_pins;
    // small levels check every prefix with one block per partition (k_validity_small), the
    // transitions summed per (partition, rank) in a dense K x n table
    const u64 tcap = track && !small ? 2 * lp.dst_pins : 0;
    u32 *tp = nullptr, *tr = nullptr;
    int32_t *tdv = nullptr;
    unsigned long long *tdense = nullptr;
    if (track && small) {
        tdense = c.arena.alloc<unsigned long long>((u64)rp.K * n);
        AXC_CUDA(cudaMemsetAsync(tdense, 0, (size_t)rp.K * n * 8, c.stream));
    } else if (track) {
        tp = c.arena.alloc<u32>(tcap);
        tr = c.arena.alloc<u32>(tcap);
        tdv = (int32_t *)c.arena.alloc<u32>(tcap);
    }
    {
        CascadeArgs C;
        C.e = L.e; C.encourage = rp.encourage ? 1 : 0; C.off = L.off; C.pins = L.pins; C.nsrc = L.nsrc;
        C.wfx = wfx; C.lam = cs.lam; C.cpart = cs.part; C.ccnt = cs.cnt; C.cdcnt = cs.dcnt; C.rank = rank;
        C.part = part; C.target = target; C.g2 = g2;
        C.track = track ? 1 : 0; C.tp = tp; C.tr = tr; C.tdv = tdv; C.dT = dT; C.tcap = tcap;
        C.tdense = tdense; C.dense_stride = n;
        C.status = c.d_status;
        C.K = rp.K;
        C.pbytes = c.profiling("k_cascade_warp") ? c.d_prof_bytes() : nullptr;
        const bool direct = rp.K <= CC_DIRECT_K;
        size_t m1 = c.arena.mark();
        u32 *big = c.arena.alloc<u32>(L.e ? L.e : 1), *huge = c.arena.alloc<u32>(L.e ? L.e : 1);
        u32 *big2 = c.arena.alloc<u32>(L.e ? L.e : 1);
        if (L.e) {
            // only the hyperedges that hold a mover: flagged from the movers' incidences
            u32 *hflag = c.arena.alloc<u32>(L.e), *hlist = c.arena.alloc<u32>(L.e);
            AXC_CUDA(cudaMemsetAsync(hflag, 0, (size_t)L.e * 4, c.stream));
            LAUNCH(c, k_mover_hedges, (u32)c.sms * 8, 256, 0, mv, dM, L.toff, L.touch, hflag);
            compact_indices_dn(c, hflag, hlist, L.e, dHl);
            int per_w = 1;
            AXC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_w, k_cascade_warp, CC_WARPS * 32, 0));
            const u32 gw = std::min<u32>(cdiv(L.e, CC_WARPS), (u32)c.sms * (u32)std::max(per_w, 1));
            LAUNCH(c, k_cascade_warp, gw, CC_WARPS * 32, 0, C, hlist, dHl, big, dBig);
            // block kernel: shared memory sized by the level's largest hyperedge, all resident blocks
            u32 smov = 128;
            while (smov < lp.max_len && smov < cascade_block_movers(c)) smov <<= 1;
            // hashed tables: sized for the level's largest hyperedge within the block's limit
            const u32 stab = direct ? std::max(2 * rp.K, 32u)  // tk: the sweep's 2K lane masks
                                    : (u32)std::min<u64>(cascade_cap(std::min<u64>(lp.max_len, rp.K),
                                                                     std::min<u64>(lp.max_len, smov)),
                                                         CB_TAB_HASH);
            const u32 *blist = big, *bcount = dBig;
            if (!direct && (smov > CB_MID_MOV || stab > CB_MID_TAB)) {  // middle tier first
                const u32 smid = std::min(smov, CB_MID_MOV), tmid = std::min(stab, CB_MID_TAB);
                const size_t dmid = (size_t)smid * 12 + (size_t)tmid * 12;
                int per_mid = 1;
                AXC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_mid, k_cascade_block, CB_THREADS, dmid));
                LAUNCH(c, k_cascade_block, (u32)c.sms * (u32)std::max(per_mid, 1), CB_THREADS, dmid, C, big, dBig, smid,
                       tmid, big2, dBig2);
                blist = big2;
                bcount = dBig2;
            }
            const size_t dyn = (size_t)smov * 12 + (size_t)stab * 12;
            int per_sm = 1;
            AXC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cascade_block, CB_THREADS, dyn));
            const u32 grid = (u32)c.sms * (u32)std::max(per_sm, 1);
            LAUNCH(c, k_cascade_block, grid, CB_THREADS, dyn, C, blist, bcount, smov, stab, huge, dHuge);
            // scratch kernel, only when some hyperedge can outgrow the block kernel: one slice of
            // movers, slots and tables per block, at most 1 GiB in all
            u64 mv_cap = 1;
            while (mv_cap < lp.max_len) mv_cap <<= 1;
            const u64 tab_cap = direct ? stab : cascade_cap(std::min<u64>(lp.max_len, rp.K), lp.max_len);
            if (mv_cap > smov || tab_cap > stab) {
                const u64 per_block = mv_cap * 12 + tab_cap * 12;
                const u32 gh = (u32)std::max<u64>(1, std::min<u64>((u64)c.sms, (1ull << 30) / per_block));
                u64 *smv = c.arena.alloc<u64>((u64)gh * mv_cap);
                u32 *ssl = c.arena.alloc<u32>((u64)gh * mv_cap);
                u32 *stb = c.arena.alloc<u32>((u64)gh * 3 * tab_cap);
                LAUNCH(c, k_cascade_huge, gh, CB_THREADS, 0, C, huge, dHuge, smv, ssl, stb, mv_cap, tab_cap);
            }
        }
        c.arena.release(m1);
    }
    // prefix gains in rank order
    // per-rank deltas of the cascaded gain, the size violations and the inbound violations, in
    // one buffer [G | Vs | Vi] so one inclusive scan makes all three prefix sums
    i64 *raw = c.arena.alloc<i64>(3 * (u64)n), *pre = c.arena.alloc<i64>(3 * (u64)n);
    i64 *Gx = raw, *Vs = raw + n, *Vi = raw + 2 * (u64)n;
    if (small) {
        AXC_CUDA(cudaMemsetAsync(Vs, 0, 2 * (size_t)n * 8, c.stream));  // Vs and Vi
        LAUNCH(c, k_validity_small, rp.K, VS_THREADS, 0, mv, dM, part, target, L.nsize, psize, (u64)rp.omega,
               (unsigned long long *)Vs, track ? 1 : 0, tdense, n, pinb, (u64)rp.delta, (unsigned long long *)Vi);
        LAUNCH(c, k_tail_small, 1, 1024, 0, mv, dM, (const unsigned long long *)g2, Vs, Vi, track ? 1 : 0, target,
               part, apply);
        c.arena.release(keep);
        return apply;
    }
    LAUNCH(c, k_gather_g2, cdiv(n, 256), 256, 0, mv, dM, n, g2, Gx);  // also zeroes Vs and Vi
    // size validity
    if (!small) {
        size_t m1 = c.arena.mark();
        const u32 nemax = 2 * n;
        u32 *key = c.arena.alloc<u32>(nemax), *val = c.arena.alloc<u32>(nemax);
        LAUNCH(c, k_size_events, cdiv(nemax, 256), 256, 0, mv, dM, part, target, key, val);
        radix_sort_pairs_dn(c, key, val, dSE, nemax, bits_for(rp.K ? rp.K - 1 : 0));
        i64 *d = c.arena.alloc<i64>(nemax), *E = c.arena.alloc<i64>(nemax);
        LAUNCH(c, k_size_delta, cdiv(nemax, 256), 256, 0, mv, val, dSE, nemax, L.nsize, d);
        scan_excl_i64(c, d, E, nemax);
        LAUNCH(c, k_size_flags, cdiv(nemax, 256), 256, 0, key, val, d, E, dSE, psize, (u64)rp.omega,
               (unsigned long long *)Vs);
        c.arena.release(m1);
    }
    // inbound validity (INCC only): the transitions ordered by (partition, rank), the running
    // inbound-set size of each partition along them
    if (track && !small) {
        size_t m1 = c.arena.mark();
        const u64 nt = tcap;
        const u32 rb = bits_for(n ? n - 1 : 0), pb = bits_for(rp.K ? rp.K - 1 : 0);
        const bool combined = rb + pb <= 32;
        u32 *key = c.arena.alloc<u32>(nt), *perm = c.arena.alloc<u32>(nt);
        LAUNCH(c, k_trans_keys, cdiv(nt, 256), 256, 0, dT, nt, tp, tr, rb, combined ? 1 : 0, key, perm);
        if (combined) {
            radix_sort_pairs_dn(c, key, perm, dT, nt, rb + pb);
        } else {
            radix_sort_pairs_dn(c, key, perm, dT, nt, rb);
            LAUNCH(c, k_gather_by_dn, cdiv(nt, 256), 256, 0, tp, perm, key, dT);
            radix_sort_pairs_dn(c, key, perm, dT, nt, pb);
        }
        u32 *sp = c.arena.alloc<u32>(nt), *sr = key;
        i64 *sd = c.arena.alloc<i64>(nt), *E2 = c.arena.alloc<i64>(nt);
        LAUNCH(c, k_trans_perm, cdiv(nt, 256), 256, 0, perm, dT, nt, tp, tr, tdv, sp, sr, sd);
        scan_excl_i64(c, sd, E2, nt);
        LAUNCH(c, k_trans_flags, cdiv(nt, 256), 256, 0, sp, sr, sd, E2, dT, pinb, (u64)rp.delta,
               (unsigned long long *)Vi);
        c.arena.release(m1);
    }
    scan_incl_i64(c, raw, pre, 3 * (u64)n);
    // best prefix and apply
    if (rp.copies > 1) {  // every copy its own
        Best *bs = (Best *)c.arena.alloc<u64>(4 * (u64)rp.copies);
        u32 *capply = c.arena.alloc<u32>(rp.copies);
        AXC_CUDA(cudaMemsetAsync(apply, 0, 4, c.stream));
        LAUNCH(c, k_best_seg, rp.copies, 256, 0, pre, n, track ? 1 : 0, dM, ck, bs, capply, apply);
        LAUNCH(c, k_apply_seg, cdiv(n, 256), 256, 0, mv, dM, ck, target, bs, capply, part, ic ? ic->prev : nullptr,
               ic ? ic->stamp : nullptr, ic ? (const u32 *)ic->ctr : nullptr);
    } else {
        const u32 nbk = cdiv(n, 256) < 64u ? cdiv(n, 256) : 64u;
        Best *bb = (Best *)c.arena.alloc<u64>(4 * (nbk + 1));
        LAUNCH(c, k_best, nbk, 256, 0, pre, n, track ? 1 : 0, dM, bb + 1);
        LAUNCH(c, k_best_final, 1, 1, 0, bb + 1, nbk, pre, n, track ? 1 : 0, bb, apply);
        LAUNCH(c, k_apply, cdiv(n, 256), 256, 0, mv, target, bb, apply, part, ic ? ic->prev : nullptr,
               ic ? ic->stamp : nullptr, ic ? (const u32 *)ic->ctr : nullptr);
    }
    if (ic) {  // flag the moved nodes' hyperedges for the next census, then count the round
        LAUNCH(c, k_mark_moved, (u32)c.sms * 8, 256, 0, mv, dM, ic->stamp, ic->ctr, L.toff, L.touch, ic->dirty);
        LAUNCH(c, k_round_tick, 1, 32, 0, ic->ctr);
    }
    c.arena.release(keep);
    return apply;
}

// The round's one host round trip: the apply flag and the status word.
static bool round_result(Ctx &c, const u32 *apply) {
    AXC_CUDA(cudaMemcpyAsync(c.h_pinned, apply, 4, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaMemcpyAsync((char *)c.h_pinned + 4, c.d_status, 4, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    u32 hv[2];
    memcpy(hv, c.h_pinned, 8);
    if (hv[1] != DEV_OK) {
        AXC_CUDA(cudaMemsetAsync(c.d_status, 0, 4, c.stream));
        throw Error(AXC_EINTERNAL, "device status word = " + std::to_string(hv[1]));
    }
    return hv[0] != 0;
}

// One round, launched eagerly; returns true when moves were applied.
static bool refine_round(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *wfx, const RefineParams &rp,
                         u32 *part, u32 discount, u32 round, IncCensus *ic) {
    const size_t m0 = c.arena.mark();
    size_t keep;
    const u32 *apply = round_body(c, L, lp, wfx, rp, part, discount, round, nullptr, keep, ic);
    const bool r = round_result(c, apply);
    c.arena.release(m0);
    return r;
}

// The rounds of one level replayed from one CUDA graph of the round body.
struct RoundGraph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~RoundGraph() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

// Kernel nodes of a captured graph (memset and copy nodes are not kernel launches).
static u32 rg_kernels(cudaGraph_t g) {
    size_t k = 0;
    if (cudaGraphGetNodes(g, nullptr, &k) != cudaSuccess || k == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(k);
    if (cudaGraphGetNodes(g, nodes.data(), &k) != cudaSuccess) return 0;
    u32 kernels = 0;
    for (size_t i = 0; i < k; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
    }
    return kernels;
}

// The round schedule on the device, for the level's rounds run as the body of one conditional
// WHILE graph node. rs = {r, R, rounds done}; after each round: the next r by the skip rule after
// a round without moves (sources/refinement.cu:539-542; the host loop of refine_level is the same
// rule), its discount (1, 2, none by thirds) and round number into dyn, and the loop goes on while
// r < R and the status word is clear.
__global__ void k_round_next(cudaGraphConditionalHandle h, u32 *__restrict__ rs, u32 *__restrict__ dyn,
                             const u32 *__restrict__ apply, const u32 *__restrict__ status) {
    u32 r = rs[0];
    const u32 R = rs[1];
    rs[2] += 1;
    if (!*apply) {
        if (r < R / 3) r = R / 2;
        else if (r < 2 * R / 3) r = 2 * R / 3;
        else r = R;
    }
    r += 1;
    rs[0] = r;
    const bool go = r < R && *(volatile const u32 *)status == 0;
    if (go) {
        dyn[0] = r < R / 3 ? 1u : (r < 2 * R / 3 ? 2u : 0xFFFFFFFFu);
        dyn[1] = r;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// level bounds that need the offsets: the largest hyperedge and the destination pin count
__global__ void k_level_bounds(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ nsrc,
                               unsigned long long *__restrict__ out) {
    u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    u64 len = 0, dst = 0;
    if (h < e) {
        len = off[h + 1] - off[h];
        dst = len - nsrc[h];
    }
    len = warp_max_u64(len);
    dst = warp_sum(dst);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], (unsigned long long)len);
        atomicAdd(&out[1], (unsigned long long)dst);
    }
}

// All rounds of a level in one graph launch: a conditional WHILE node whose body is one round
// (round_body) followed by k_round_next, which applies the round schedule on the device. Returns
// the rounds run.
static u32 refine_level_loop(Ctx &c, const DLevel &L, const LevelPrep &lp, const u32 *wfx, const RefineParams &rp,
                             u32 *part, IncCensus *ic) {
    const u32 R = rp.rounds;
    u32 *dyn = c.arena.alloc<u32>(2), *rs = c.arena.alloc<u32>(4);
    {
        u32 *hp = (u32 *)((char *)c.h_pinned + 64);
        hp[0] = 0 < R / 3 ? 1u : (0 < 2 * R / 3 ? 2u : 0xFFFFFFFFu);  // discount of round 0 (2 when R = 2)
        hp[1] = 0u;
        hp[2] = 0u;  // rs: r, R, rounds done
        hp[3] = R;
        hp[4] = 0u;
        hp[5] = 0u;
        AXC_CUDA(cudaMemcpyAsync(dyn, hp, 8, cudaMemcpyHostToDevice, c.stream));
        AXC_CUDA(cudaMemcpyAsync(rs, hp + 2, 16, cudaMemcpyHostToDevice, c.stream));
    }
    RoundGraph rg;
    AXC_CUDA(cudaGraphCreate(&rg.g, 0));
    cudaGraphConditionalHandle h;
    AXC_CUDA(cudaGraphConditionalHandleCreate(&h, rg.g, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    AXC_CUDA(cudaGraphAddNode(&wn, rg.g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const size_t m1 = c.arena.mark();
    const u32 launches0 = c.launches;
    size_t keep;
    u32 *apply = nullptr;
    AXC_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    c.capturing = true;
    try {
        apply = round_body(c, L, lp, wfx, rp, part, 1, 0, dyn, keep, ic);
        LAUNCH(c, k_round_next, 1, 1, 0, h, rs, dyn, apply, c.d_status);
    } catch (...) {
        c.capturing = false;
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c.stream, &junk);
        throw;
    }
    c.capturing = false;
    AXC_CUDA(cudaStreamEndCapture(c.stream, &body));
    c.launches = launches0;
    const u32 body_kernels = rg_kernels(body);
    AXC_CUDA(cudaGraphInstantiate(&rg.x, rg.g, 0));
    // the round's scratch above m1 stays unallocated, and nothing else allocates, while the graph runs
    c.arena.release(m1);
    AXC_CUDA(cudaGraphLaunch(rg.x, c.stream));
    u32 *hp = (u32 *)((char *)c.h_pinned + 64);
    AXC_CUDA(cudaMemcpyAsync(hp, rs, 16, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaMemcpyAsync(hp + 4, c.d_status, 4, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    const u32 done = hp[2];
    c.launches += done * body_kernels;
    if (hp[4] != DEV_OK) {
        AXC_CUDA(cudaMemsetAsync(c.d_status, 0, 4, c.stream));
        throw Error(AXC_EINTERNAL, "device status word = " + std::to_string(hp[4]));
    }
    return done;
}

u32 refine_level(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, u32 *part) {
    const u32 R = rp.rounds;
    if (R == 0 || L.n == 0) return 0;
    size_t m = c.arena.mark();
    LevelPrep lp = prepare_level(c, L, wfx, rp.K);
    // one census kept across the rounds where the level allows it (k_census_inc_*)
    IncCensus icv, *ic = nullptr;
    if (inc_census_eligible(L, lp, rp) && inc_census_enabled()) {
        inc_census_init(c, L, wfx, rp, icv);
        ic = &icv;
    }
    // Graph replays need the round's scalars in device memory. Kernel-timer pairs captured in the
    // graph are read back after every replay; the bytes of the captured launches count per replay.
    const bool graph = R > 1;
    // Without the kernel timer the rounds run as one conditional WHILE graph: the schedule lives
    // on the device and the host waits once per level. With the timer on, each round is one replay
    // of the round graph, so that its event pairs are read after every round. The environment
    // variable AXC_ROUND_LOOP=0 also selects the replays (the same kernels and results; profilers
    // that do not follow kernels into conditional graph nodes see them then).
    if (graph && !c.prof_on && round_loop_enabled()) {
        const u32 done = refine_level_loop(c, L, lp, wfx, rp, part, ic);
        c.arena.release(m);
        return done;
    }
    size_t ev0 = 0, ev1 = 0;
    u64 bytes_per_round = 0;
    RoundGraph rg;
    u32 *dyn = nullptr, *apply = nullptr, graph_kernels = 0;
    if (graph) {
        dyn = c.arena.alloc<u32>(2);
        const size_t m1 = c.arena.mark();
        size_t keep;
        const u32 launches0 = c.launches;  // captured launches run only when replayed
        const u64 bytes0 = c.prof_bytes;
        ev0 = c.prof_used;
        AXC_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        c.capturing = true;
        try {
            apply = round_body(c, L, lp, wfx, rp, part, 1, 0, dyn, keep, ic);
        } catch (...) {
            c.capturing = false;
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(c.stream, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        c.capturing = false;
        ev1 = c.prof_used;
        bytes_per_round = c.prof_bytes - bytes0;
        c.prof_bytes = bytes0;
        AXC_CUDA(cudaStreamEndCapture(c.stream, &rg.g));
        AXC_CUDA(cudaGraphInstantiate(&rg.x, rg.g, 0));
        c.launches = launches0;
        graph_kernels = rg_kernels(rg.g);
        c.arena.release(m1);
        c.arena.alloc<u32>(1);  // keep the apply word below the round's scratch, as captured
    }
    u32 done = 0;
    for (u32 r = 0; r < R; ++r) {
        const u32 discount = r < R / 3 ? 1u : (r < 2 * R / 3 ? 2u : 0xFFFFFFFFu);
        ++done;
        bool applied;
        if (graph) {
            u32 *hp = (u32 *)((char *)c.h_pinned + 64);
            hp[0] = discount;
            hp[1] = r;
            AXC_CUDA(cudaMemcpyAsync(dyn, hp, 8, cudaMemcpyHostToDevice, c.stream));
            AXC_CUDA(cudaGraphLaunch(rg.x, c.stream));
            c.launches += graph_kernels;
            applied = round_result(c, apply);
            c.prof_collect(ev0, ev1);
            c.prof_bytes += bytes_per_round;
        } else {
            applied = refine_round(c, L, lp, wfx, rp, part, discount, r, ic);
        }
        if (!applied) {
            if (r < R / 3) r = R / 2;
            else if (r < 2 * R / 3) r = 2 * R / 3;
            else r = R;
        }
    }
    if (graph) c.prof_used = ev0;  // the captured pairs go back to the pool with the graph
    c.arena.release(m);
    return done;
}

}  // namespace axc
