// Refinement (sources/refinement.cu:18-582 and kernels/refinement.cu:9-652 restated with exact
// integer arithmetic and a sparse per-hyperedge census instead of the dense E x K table).
//
// One round:
//  1. census: for every hyperedge the partitions among its pins with (pins, destination pins),
//     in first-occurrence order; partition sizes and distinct-inbound counts.
//  2. gains: every node's best feasible target among the partitions adjacent to it; only moves
//     with positive gain are proposed.
//  3. rank by (gain desc, id asc).
//  4. cascade: each move's gain recomputed assuming every better-ranked move is applied, by a
//     sweep over each hyperedge's movers in rank order (O(pins) instead of the reference's
//     per-move re-read of every incident hyperedge).
//  5. prefix sums of cascaded gains; size-excess and inbound-validity of every prefix from sorted
//     event streams (sources/refinement.cu:239-491); best prefix by best_move_functor
//     (headers/data_types.cuh:113-136); apply when valid with non-negative prefix gain.
#include "common.cuh"
#include "kernels.h"

namespace axc {
namespace {

constexpr u32 CS_WARP_CAP = 256;
constexpr u32 CS_BLOCK_CAP = 4096;
constexpr u32 CS_WARPS = 4;

// ------------------------------------------------------------------ census
struct CensusArgs {
    const u64 *off;
    const u32 *pins, *nsrc, *part;
    u32 *cpart, *ccnt, *cdcnt, *lam;
    u32 *status;
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
    u32 cap = 32;
    while (cap < 2 * len) cap <<= 1;
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
__global__ void k_part_inbound(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ lam,
                               const u32 *__restrict__ cpart, const u32 *__restrict__ cdcnt,
                               unsigned long long *__restrict__ pinb) {
    const u32 h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (h >= e) return;
    const u64 a = off[h];
    for (u32 j = lane; j < lam[h]; j += 32)
        if (cdcnt[a + j] > 0) atomicAdd(&pinb[cpart[a + j]], 1ull);
}

// ------------------------------------------------------------------ gains
struct GainArgs {
    u32 n, omega, delta, discount, round;
    u32 seed;
    int encourage;
    const u64 *off;
    const u32 *lam, *cpart, *ccnt, *cdcnt, *wfx;
    const u64 *toff;
    const u32 *touch, *nin, *nsize, *part;
    const u64 *psize, *pinb;
    u32 *target;
    i64 *gain;
    u32 *status;
};

__device__ __forceinline__ i64 leave_gain(int encourage, u32 w, u32 c) {
    if (encourage) return c >= 1 ? (i64)((u64)w / ((u64)c * c)) : 0;
    return c == 1 ? (i64)w : 0;
}

__global__ void k_gain_work(u32 n, const u64 *__restrict__ toff, const u32 *__restrict__ touch,
                            const u32 *__restrict__ lam, u64 *__restrict__ work) {
    const u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (u >= n) return;
    u64 s = 0;
    for (u64 j = toff[u] + lane; j < toff[u + 1]; j += 32) s += lam[touch[j]];
    s = warp_sum(s);
    if (lane == 0) work[u] = s;
}

// Accumulate node u's adjacency to other partitions into (keys, conn, dconn); returns the saving
// and the total incident weight through the reference arguments (valid in thread t == 0 after
// the caller's reduction). Threads [0, nt) of the group cooperate hyperedge by hyperedge.
__device__ __forceinline__ void gain_accumulate(const GainArgs &A, u32 u, u32 p, u32 *keys,
                                                unsigned long long *conn, u32 *dconn, u32 mask, u32 t, u32 nt,
                                                i64 &saving, i64 &wtot) {
    const u64 t0 = A.toff[u], t1 = A.toff[u + 1];
    const u32 nin_u = A.nin[u];
    for (u64 j = t0; j < t1; ++j) {
        const u32 h = A.touch[j];
        const bool inb = (j - t0) < nin_u;
        const u32 w = A.wfx[h];
        const u64 a = A.off[h];
        const u32 lm = A.lam[h];
        if (t == 0) wtot += w;
        for (u32 i = t; i < lm; i += nt) {
            const u32 q = A.cpart[a + i];
            if (q == p) {
                saving += leave_gain(A.encourage, w, A.ccnt[a + i]);
                continue;
            }
            const u32 slot = hash_find_or_insert(keys, mask, q);
            if (slot == NONE) { atomicExch(A.status, DEV_HASH_FULL); continue; }
            atomicAdd(&conn[slot], (unsigned long long)w);
            if (inb && A.cdcnt[a + i] > 0) atomicAdd(&dconn[slot], 1u);
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

__global__ void __launch_bounds__(GN_WARPS * 32) k_gain_warp(GainArgs A, const u32 *__restrict__ list, u32 nl) {
    __shared__ u32 tk[GN_WARPS][2 * GN_WARP_W], td[GN_WARPS][2 * GN_WARP_W];
    __shared__ unsigned long long tcw[GN_WARPS][2 * GN_WARP_W];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 idx = blockIdx.x * GN_WARPS + w;
    if (idx >= nl) return;
    const u32 u = list[idx], p = A.part[u];
    u32 *keys = tk[w], *dconn = td[w];
    unsigned long long *conn = tcw[w];
    const u32 cap = 2 * GN_WARP_W;
    for (u32 i = lane; i < cap; i += 32) { keys[i] = NONE; dconn[i] = 0; conn[i] = 0; }
    __syncwarp();
    i64 saving = 0, wtot = 0;
    gain_accumulate(A, u, p, keys, conn, dconn, cap - 1, lane, 32, saving, wtot);
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

__global__ void __launch_bounds__(GN_BLOCK) k_gain_block(GainArgs A, const u32 *__restrict__ list, u32 nl, u32 cap_max,
                                                        u32 *gtab) {
    extern __shared__ unsigned long long dyn64[];
    __shared__ i64 red[2][32];
    __shared__ Cand cred[32];
    for (u32 idx = blockIdx.x; idx < nl; idx += gridDim.x) {
        const u32 u = list[idx], p = A.part[u];
        unsigned long long *conn;
        u32 *keys, *dconn;
        const u32 cap = cap_max;
        if (gtab) {
            u32 *base = gtab + (u64)blockIdx.x * 4 * cap;
            conn = (unsigned long long *)base;
            keys = base + 2 * cap;
            dconn = keys + cap;
        } else {
            conn = dyn64;
            keys = (u32 *)(dyn64 + cap);
            dconn = keys + cap;
        }
        for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = NONE; dconn[i] = 0; conn[i] = 0; }
        __syncthreads();
        i64 saving = 0, wtot = 0;
        gain_accumulate(A, u, p, keys, conn, dconn, cap - 1, threadIdx.x, blockDim.x, saving, wtot);
        saving = warp_sum(saving);
        wtot = warp_sum(wtot);
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = saving; red[1][threadIdx.x >> 5] = wtot; }
        __syncthreads();
        saving = 0;
        wtot = 0;
        for (u32 i = 0; i < blockDim.x / 32; ++i) { saving += red[0][i]; wtot += red[1][i]; }
        Cand best{INT64_MIN, 0};
        for (u32 i = threadIdx.x; i < cap; i += blockDim.x) {
            if (keys[i] == NONE) continue;
            Cand c = gain_candidate(A, u, keys[i], conn[i], dconn[i], saving, wtot);
            if (cand_better(c, best)) best = c;
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

// ------------------------------------------------------------------ ranking
__global__ void k_move_flags(u32 n, const u32 *__restrict__ target, u32 *__restrict__ flag) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) flag[v] = target[v] != NONE ? 1u : 0u;
}
__global__ void k_move_keys(const u32 *__restrict__ mv, u32 M, const i64 *__restrict__ gain, u64 gmax,
                            u32 *__restrict__ hi, u32 *__restrict__ lo) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    u64 k = gmax - (u64)gain[mv[i]];  // ascending key = descending gain
    hi[i] = (u32)(k >> 32);
    lo[i] = (u32)k;
}
__global__ void k_gain_max(const u32 *__restrict__ mv, u32 M, const i64 *__restrict__ gain,
                           unsigned long long *__restrict__ out) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    u64 g = i < M ? (u64)gain[mv[i]] : 0;
    g = warp_max_u64(g);
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)g);
}
__global__ void k_set_rank(const u32 *__restrict__ mv, u32 M, u32 *__restrict__ rank) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) rank[mv[i]] = i;
}

// ------------------------------------------------------------------ cascade
constexpr u32 CC_WARPS = 4;
constexpr u32 CC_MOV = 128;    // movers per hyperedge handled by the warp kernel
constexpr u32 CC_TAB = 512;    // partition table slots of the warp kernel

struct CascadeArgs {
    u32 e;
    int encourage;
    const u64 *off;
    const u32 *pins, *wfx, *lam, *cpart, *ccnt, *rank, *part, *target;
    unsigned long long *g2;
    u32 *status;
};

// Sweep the movers (sorted by rank) of one hyperedge sequentially.
__device__ void cascade_sweep(const CascadeArgs &A, u32 h, const u64 *mv, u32 m, u32 *tk, u32 *tc, u32 mask) {
    const u32 w = A.wfx[h];
    for (u32 i = 0; i < m; ++i) {
        const u32 v = (u32)mv[i];
        const u32 p = A.part[v], q = A.target[v];
        const u32 sp = hash_find_or_insert(tk, mask, p), sq = hash_find_or_insert(tk, mask, q);
        if (sp == NONE || sq == NONE) { atomicExch(A.status, DEV_HASH_FULL); return; }
        const u32 cp = tc[sp], cq = tc[sq];
        const i64 d = leave_gain(A.encourage, w, cp) - (cq == 0 ? (i64)w : 0);
        atomicAdd(&A.g2[v], (unsigned long long)d);
        tc[sp] = cp - 1;
        tc[sq] = tc[sq] + 1;
    }
}

__global__ void k_cascade_warp(CascadeArgs A, u32 *__restrict__ big) {
    __shared__ u64 mvs[CC_WARPS][CC_MOV];
    __shared__ u32 tk[CC_WARPS][CC_TAB], tc[CC_WARPS][CC_TAB];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 h = blockIdx.x * CC_WARPS + w;
    if (h >= A.e) return;
    const u64 a = A.off[h], b = A.off[h + 1];
    // collect movers (rank << 32 | node)
    u32 m = 0;
    for (u64 base = a; base < b; base += 32) {
        u64 k = base + lane;
        u32 v = k < b ? A.pins[k] : 0, r = k < b ? A.rank[v] : NONE;
        bool mvr = r != NONE;
        u32 bal = __ballot_sync(0xFFFFFFFFu, mvr);
        if (mvr) {
            u32 pos = m + __popc(bal & ((1u << lane) - 1u));
            if (pos < CC_MOV) mvs[w][pos] = ((u64)r << 32) | v;
        }
        m += __popc(bal);
    }
    if (m == 0) return;
    const u32 lm = A.lam[h];
    if (m > CC_MOV || 2 * (lm + 2 * m) > CC_TAB) {
        if (lane == 0) big[h] = 1;
        return;
    }
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
    // table of partition counts from the census
    u32 cap = 32;
    while (cap < 2 * (lm + 2 * m)) cap <<= 1;
    for (u32 i = lane; i < cap; i += 32) { tk[w][i] = NONE; tc[w][i] = 0; }
    __syncwarp();
    for (u32 i = lane; i < lm; i += 32) {
        u32 s = hash_find_or_insert(tk[w], cap - 1, A.cpart[a + i]);
        if (s != NONE) tc[w][s] = A.ccnt[a + i];
    }
    __syncwarp();
    if (lane == 0) cascade_sweep(A, h, mvs[w], m, tk[w], tc[w], cap - 1);
}

// Large hyperedges: one block each, movers and tables in global scratch.
__global__ void k_cascade_big(CascadeArgs A, const u32 *__restrict__ list, u32 nl, u64 *scratch_mv, u32 *scratch_tab,
                              const u64 *__restrict__ mv_off, const u64 *__restrict__ tab_off) {
    if (blockIdx.x >= nl) return;
    const u32 h = list[blockIdx.x];
    const u64 a = A.off[h], b = A.off[h + 1];
    u64 *mvs = scratch_mv + mv_off[blockIdx.x];
    const u32 lm = A.lam[h];
    __shared__ u32 cntm;
    if (threadIdx.x == 0) cntm = 0;
    __syncthreads();
    for (u64 k = a + threadIdx.x; k < b; k += blockDim.x) {
        u32 v = A.pins[k], r = A.rank[v];
        if (r != NONE) mvs[atomicAdd(&cntm, 1u)] = ((u64)r << 32) | v;
    }
    __syncthreads();
    const u32 m = cntm;
    // sort by rank: odd-even transposition over the block (m is bounded by the hyperedge size)
    for (u32 phase = 0; phase < m; ++phase) {
        for (u32 i = 2 * threadIdx.x + (phase & 1); i + 1 < m; i += 2 * blockDim.x) {
            u64 x = mvs[i], y = mvs[i + 1];
            if (x > y) { mvs[i] = y; mvs[i + 1] = x; }
        }
        __syncthreads();
    }
    u32 cap = 32;
    while (cap < 2 * (lm + 2 * m)) cap <<= 1;
    u32 *tk = scratch_tab + tab_off[blockIdx.x], *tc = tk + cap;
    for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { tk[i] = NONE; tc[i] = 0; }
    __syncthreads();
    for (u32 i = threadIdx.x; i < lm; i += blockDim.x) {
        u32 s = hash_find_or_insert(tk, cap - 1, A.cpart[a + i]);
        if (s != NONE) tc[s] = A.ccnt[a + i];
    }
    __syncthreads();
    if (threadIdx.x == 0) cascade_sweep(A, h, mvs, m, tk, tc, cap - 1);
}
__global__ void k_big_sizes(const u32 *__restrict__ list, u32 nl, const u64 *__restrict__ off, const u32 *__restrict__ lam,
                            u64 *__restrict__ mvsz, u64 *__restrict__ tabsz) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == nl) { mvsz[i] = 0; tabsz[i] = 0; }
    if (i >= nl) return;
    u32 h = list[i];
    u64 len = off[h + 1] - off[h];
    u64 cap = 32;
    while (cap < 2 * (lam[h] + 2 * len)) cap <<= 1;
    mvsz[i] = len;
    tabsz[i] = 2 * cap;
}

// ------------------------------------------------------------------ prefix and validity
__global__ void k_gather_g2(const u32 *__restrict__ mv, u32 M, const unsigned long long *__restrict__ g2,
                            i64 *__restrict__ G) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) G[i] = (i64)g2[mv[i]];
}
__global__ void k_incl_fix(const i64 *__restrict__ x, i64 *__restrict__ ex, u32 M) {  // ex := ex + x
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) ex[i] += x[i];
}

// size events: 2r = leave p, 2r+1 = join q
__global__ void k_size_events(const u32 *__restrict__ mv, u32 M, const u32 *__restrict__ part,
                              const u32 *__restrict__ target, u32 *__restrict__ key, u32 *__restrict__ val) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * M) return;
    u32 v = mv[i >> 1];
    key[i] = (i & 1) ? target[v] : part[v];
    val[i] = i;
}
__global__ void k_size_delta(const u32 *__restrict__ mv, const u32 *__restrict__ val, u32 ne,
                             const u32 *__restrict__ nsize, i64 *__restrict__ d) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    u32 ev = val[i];
    i64 s = nsize[mv[ev >> 1]];
    d[i] = (ev & 1) ? s : -s;
}
__device__ __forceinline__ u32 lower_bound_u32(const u32 *a, u32 len, u32 x) {
    u32 lo = 0, hi = len;
    while (lo < hi) {
        u32 mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__global__ void k_size_flags(const u32 *__restrict__ key, const u32 *__restrict__ val, const i64 *__restrict__ d,
                             const i64 *__restrict__ E, u32 ne, const u64 *__restrict__ psize, u64 omega,
                             unsigned long long *__restrict__ Vs) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    u32 p = key[i];
    u32 st = lower_bound_u32(key, ne, p);
    i64 before = (i64)psize[p] + (E[i] - E[st]);
    i64 after = before + d[i];
    i64 exb = before > (i64)omega ? before - (i64)omega : 0;
    i64 exa = after > (i64)omega ? after - (i64)omega : 0;
    if (exa != exb) atomicAdd(&Vs[val[i] >> 1], (unsigned long long)(exa - exb));
}

// inbound events: mover r, its i-th inbound hyperedge: 2i = leave p (-1), 2i+1 = join q (+1)
__global__ void k_inb_counts(const u32 *__restrict__ mv, u32 M, const u32 *__restrict__ nin, u32 *__restrict__ c) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) c[i] = 2 * nin[mv[i]];
}
__global__ void k_inb_events(const u32 *__restrict__ mv, u32 M, const u64 *__restrict__ base,
                             const u64 *__restrict__ toff, const u32 *__restrict__ touch, const u32 *__restrict__ nin,
                             const u32 *__restrict__ part, const u32 *__restrict__ target, u32 *__restrict__ keyH,
                             u32 *__restrict__ keyP, u32 *__restrict__ val) {
    const u32 r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= M) return;
    const u32 v = mv[r];
    const u64 b0 = base[r], t0 = toff[v];
    const u32 ni = nin[v], p = part[v], q = target[v];
    for (u32 i = lane; i < ni; i += 32) {
        u32 h = touch[t0 + i];
        u64 e0 = b0 + 2 * i;
        keyH[e0] = h; keyP[e0] = p; val[e0] = (u32)e0;
        keyH[e0 + 1] = h; keyP[e0 + 1] = q; val[e0 + 1] = (u32)(e0 + 1);
    }
}
__global__ void k_gather_by(const u32 *__restrict__ src, const u32 *__restrict__ idx, u32 *__restrict__ dst, u64 n) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
__device__ __forceinline__ u32 upper_bound_u64d(const u64 *a, u32 len, u64 x) {
    u32 lo = 0, hi = len;
    while (lo < hi) {
        u32 mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// per sorted event: hyperedge, partition, sign, rank; heads of (p,h) segments
__global__ void k_inb_decode(const u32 *__restrict__ val, const u32 *__restrict__ keyP, u64 ne, const u64 *__restrict__ base,
                             u32 M, const u32 *__restrict__ mv, const u64 *__restrict__ toff,
                             const u32 *__restrict__ touch, u32 *__restrict__ ev_h, u32 *__restrict__ ev_r,
                             i64 *__restrict__ ev_d, u32 *__restrict__ head) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    u32 ev = val[i];
    u32 r = upper_bound_u64d(base, M + 1, ev) - 1;
    u32 k = (u32)((ev - base[r]) >> 1);
    ev_h[i] = touch[toff[mv[r]] + k];
    ev_r[i] = r;
    ev_d[i] = (ev & 1) ? 1 : -1;
    (void)keyP;
}
__global__ void k_seg_heads(const u32 *__restrict__ a, const u32 *__restrict__ b, u64 ne, u32 *__restrict__ head) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    head[i] = (i == 0 || a[i] != a[i - 1] || (b && b[i] != b[i - 1])) ? 1u : 0u;
}
__global__ void k_seg_start(const u32 *__restrict__ head, const u32 *__restrict__ sid, u64 ne, u32 *__restrict__ start) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ne && head[i]) start[sid[i]] = (u32)i;
}
__device__ __forceinline__ u32 census_dcnt(const u64 *off, const u32 *lam, const u32 *cpart, const u32 *cdcnt, u32 h,
                                           u32 p) {
    const u64 a = off[h];
    for (u32 j = 0; j < lam[h]; ++j)
        if (cpart[a + j] == p) return cdcnt[a + j];
    return 0;
}
// transitions of a (partition, hyperedge) destination count through 0
__global__ void k_inb_trans(const u32 *__restrict__ keyP, const u32 *__restrict__ ev_h, const u32 *__restrict__ ev_r,
                            const i64 *__restrict__ ev_d, const i64 *__restrict__ E, const u32 *__restrict__ head,
                            const u32 *__restrict__ sid, const u32 *__restrict__ start, u64 ne,
                            const u64 *__restrict__ off, const u32 *__restrict__ lam, const u32 *__restrict__ cpart,
                            const u32 *__restrict__ cdcnt, u32 *__restrict__ tflag, int32_t *__restrict__ tdelta) {
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    const u32 st = start[sid[i]];
    const i64 base = census_dcnt(off, lam, cpart, cdcnt, ev_h[i], keyP[i]);
    const i64 before = base + (E[i] - E[st]);
    const i64 after = before + ev_d[i];
    int32_t t = 0;
    if (before == 0 && after > 0) t = 1;
    if (before > 0 && after == 0) t = -1;
    tflag[i] = t != 0;
    tdelta[i] = t;
    (void)head;
}
// transition j (in (p, h, r) order): partition, rank, +-1
__global__ void k_trans_gather(const u32 *__restrict__ idx, u32 T, const u32 *__restrict__ keyP,
                               const u32 *__restrict__ ev_r, const int32_t *__restrict__ tdelta, u32 *__restrict__ tp,
                               u32 *__restrict__ tr, int32_t *__restrict__ td) {
    u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T) return;
    tp[j] = keyP[idx[j]];
    tr[j] = ev_r[idx[j]];
    td[j] = tdelta[idx[j]];
}
// after ordering by (p, r): sorted rank and delta of position i
__global__ void k_trans_perm(const u32 *__restrict__ perm, u32 T, const u32 *__restrict__ tr,
                             const int32_t *__restrict__ td, u32 *__restrict__ sr, i64 *__restrict__ sd) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T) return;
    sr[i] = tr[perm[i]];
    sd[i] = td[perm[i]];
}
// per partition, the running inbound-set size along the move sequence; an event that makes the
// partition exceed delta adds +1 at its rank, one that brings it back adds -1. The first event of a
// partition assumes it started valid (kernels/refinement.cu:632-651).
__global__ void k_trans_flags(const u32 *__restrict__ sp, const u32 *__restrict__ sr, const i64 *__restrict__ sd,
                              const i64 *__restrict__ E, const u32 *__restrict__ sid, const u32 *__restrict__ start,
                              u32 T, const u64 *__restrict__ pinb, u64 delta, unsigned long long *__restrict__ Vi) {
    u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T) return;
    const u32 p = sp[j];
    const u32 st = start[sid[j]];
    const i64 before = (i64)pinb[p] + (E[j] - E[st]);
    const i64 after = before + sd[j];
    const bool was_bad = (j != st) && before > (i64)delta;
    const bool is_bad = after > (i64)delta;
    if (was_bad != is_bad) atomicAdd(&Vi[sr[j]], (unsigned long long)(i64)(is_bad ? 1 : -1));
}
__global__ void k_iota(u32 *p, u32 n) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
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
__global__ void k_best(const i64 *__restrict__ G, const i64 *__restrict__ Vs, const i64 *__restrict__ Vi, u32 M,
                       Best *__restrict__ out) {
    __shared__ Best sh[256];
    Best b{0, 0, 0, 0xFFFFFFFFu};
    for (u32 r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        Best c{Vi ? (Vi[r] == 0 ? 1u : 0u) : 1u, Vs[r], G[r], r};
        if (b.r == 0xFFFFFFFFu || best_better(c, b)) b = c;
    }
    sh[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        Best x = sh[0];
        for (u32 i = 1; i < blockDim.x; ++i)
            if (sh[i].r != 0xFFFFFFFFu && (x.r == 0xFFFFFFFFu || best_better(sh[i], x))) x = sh[i];
        out[blockIdx.x] = x;
    }
}
__global__ void k_best_final(const Best *__restrict__ in, u32 nb, const i64 *__restrict__ Vi, Best *__restrict__ out,
                             u32 *__restrict__ apply) {
    Best x = in[0];
    for (u32 i = 1; i < nb; ++i)
        if (in[i].r != 0xFFFFFFFFu && (x.r == 0xFFFFFFFFu || best_better(in[i], x))) x = in[i];
    *out = x;
    const i64 vi = Vi ? Vi[x.r] : 0;
    *apply = (x.r != 0xFFFFFFFFu && x.vs <= 0 && vi <= 0 && x.g >= 0) ? 1u : 0u;
}
__global__ void k_apply(const u32 *__restrict__ mv, const u32 *__restrict__ target, const Best *__restrict__ best,
                        const u32 *__restrict__ apply, u32 *__restrict__ part) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (!*apply || i > best->r) return;
    u32 v = mv[i];
    part[v] = target[v];
}

__global__ void k_rate_tier_g(u32 n, const u64 *__restrict__ work, u64 lo, u64 hi, u32 *__restrict__ flag) {
    u32 u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) flag[u] = (work[u] > lo && work[u] <= hi) ? 1u : 0u;
}

GainArgs make_gain_args(const DLevel &L, const u32 *wfx, const RefineParams &rp, const Census &cs, const u32 *part,
                        const u64 *psize, const u64 *pinb, u32 discount, u32 round, u32 *target, i64 *gain,
                        u32 *status) {
    GainArgs A;
    A.n = L.n; A.omega = rp.omega; A.delta = rp.delta; A.discount = discount; A.round = round;
    A.seed = (u32)rp.seed; A.encourage = rp.encourage ? 1 : 0;
    A.off = L.off; A.lam = cs.lam; A.cpart = cs.part; A.ccnt = cs.cnt; A.cdcnt = cs.dcnt; A.wfx = wfx;
    A.toff = L.toff; A.touch = L.touch; A.nin = L.nin; A.nsize = L.nsize; A.part = part;
    A.psize = psize; A.pinb = pinb; A.target = target; A.gain = gain; A.status = status;
    return A;
}

void run_gains(Ctx &c, const DLevel &L, const GainArgs &A) {
    const u32 n = L.n;
    size_t m = c.arena.mark();
    u64 *work = c.arena.alloc<u64>(n);
    u32 *flag = c.arena.alloc<u32>(n), *list = c.arena.alloc<u32>(n);
    LAUNCH(c, k_gain_work, cdiv((u64)n * 32, 256), 256, 0, n, L.toff, L.touch, A.lam, work);
    // warp tier: adjacency work <= 128 -> 256-slot table
    LAUNCH(c, k_rate_tier_g, cdiv(n, 256), 256, 0, n, work, 0ull, (u64)GN_WARP_W, flag);
    u32 nl = compact_indices(c, flag, list, n);
    LAUNCH(c, k_gain_warp, cdiv(nl, GN_WARPS), GN_WARPS * 32, 0, A, list, nl);
    // block tier: <= 4096 -> 8192-slot table in dynamic smem (16 B per slot)
    LAUNCH(c, k_rate_tier_g, cdiv(n, 256), 256, 0, n, work, (u64)GN_WARP_W, 4096ull, flag);
    nl = compact_indices(c, flag, list, n);
    LAUNCH(c, k_gain_block, nl, GN_BLOCK, 8192 * 16, A, list, nl, 8192u, (u32 *)nullptr);
    // heavy tier: global tables
    LAUNCH(c, k_rate_tier_g, cdiv(n, 256), 256, 0, n, work, 4096ull, ~0ull, flag);
    nl = compact_indices(c, flag, list, n);
    if (nl) {
        u64 wmax = reduce_max_u64(c, work, n);
        u32 cap = 64;
        while (cap < 2 * wmax && cap < (1u << 28)) cap <<= 1;
        u32 grid = nl < (u32)c.sms * 2 ? nl : (u32)c.sms * 2;
        u32 *gtab = c.arena.alloc<u32>((u64)grid * 4 * cap);
        LAUNCH(c, k_gain_block, grid, GN_BLOCK, 0, A, list, nl, cap, gtab);
    }
    c.arena.release(m);
}

}  // namespace


void setup_refine_kernels(Ctx &c) {
    AXC_CUDA(cudaFuncSetAttribute(k_census_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * 2 * CS_BLOCK_CAP * 4));
    AXC_CUDA(cudaFuncSetAttribute(k_gain_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 16));
}

Census build_census(Ctx &c, const DLevel &L, const u32 *part) {
    Census cs;
    const u32 e = L.e;
    cs.beg = L.off;
    cs.part = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.cnt = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.dcnt = c.arena.alloc<u32>(L.P ? L.P : 1);
    cs.lam = c.arena.alloc<u32>(e ? e : 1);
    if (e == 0) return cs;
    CensusArgs A{L.off, L.pins, L.nsrc, part, cs.part, cs.cnt, cs.dcnt, cs.lam, c.d_status};
    LAUNCH(c, k_census_warp, cdiv(e, CS_WARPS), CS_WARPS * 32, 0, e, A);
    size_t m = c.arena.mark();
    u32 *flag = c.arena.alloc<u32>(e), *list = c.arena.alloc<u32>(e);
    LAUNCH(c, k_flag_len, cdiv(e, 256), 256, 0, e, L.off, (u64)CS_WARP_CAP, (u64)CS_BLOCK_CAP, flag);
    u32 nb = compact_indices(c, flag, list, e);
    if (nb)
        LAUNCH(c, k_census_block, nb, 256, 4 * 2 * CS_BLOCK_CAP * 4, list, nb, A, (u32 *)nullptr,
               (const u64 *)nullptr);
    LAUNCH(c, k_flag_len, cdiv(e, 256), 256, 0, e, L.off, (u64)CS_BLOCK_CAP, ~0ull, flag);
    u32 nh = compact_indices(c, flag, list, e);
    if (nh) {
        u64 *tsz = c.arena.alloc<u64>(nh + 1);
        LAUNCH(c, k_tab_sizes, cdiv(nh + 1, 256), 256, 0, list, nh, L.off, tsz);
        scan_excl_u64(c, tsz, tsz, nh + 1);
        u64 tot = fetch1(c, tsz + nh);
        u32 *gtab = c.arena.alloc<u32>(4 * tot);
        LAUNCH(c, k_census_block, nh, 512, 0, list, nh, A, gtab, (const u64 *)tsz);
    }
    c.arena.release(m);
    return cs;
}

void part_sizes(Ctx &c, u32 n, const u32 *part, const u32 *nsize, u64 *psize, u32 K) {
    AXC_CUDA(cudaMemsetAsync(psize, 0, (size_t)K * 8, c.stream));
    if (n) LAUNCH(c, k_part_sizes, cdiv(n, 256), 256, 0, n, part, nsize, (unsigned long long *)psize);
}
void part_inbound(Ctx &c, const DLevel &L, const Census &cs, u64 *pinb, u32 K) {
    AXC_CUDA(cudaMemsetAsync(pinb, 0, (size_t)K * 8, c.stream));
    if (L.e)
        LAUNCH(c, k_part_inbound, cdiv((u64)L.e * 32, 256), 256, 0, L.e, L.off, cs.lam, cs.part, cs.dcnt,
               (unsigned long long *)pinb);
}

void refine_gains_only(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, const u32 *part,
                       u32 discount, u32 round, u32 *target, i64 *gain) {
    size_t m = c.arena.mark();
    Census cs = build_census(c, L, part);
    u64 *psize = c.arena.alloc<u64>(rp.K), *pinb = c.arena.alloc<u64>(rp.K);
    part_sizes(c, L.n, part, L.nsize, psize, rp.K);
    part_inbound(c, L, cs, pinb, rp.K);
    GainArgs A = make_gain_args(L, wfx, rp, cs, part, psize, pinb, discount, round, target, gain, c.d_status);
    run_gains(c, L, A);
    check_status(c);
    c.arena.release(m);
}

// One round; returns true when moves were applied.
static bool refine_round(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, u32 *part, u32 discount,
                         u32 round) {
    const u32 n = L.n;
    size_t m0 = c.arena.mark();
    Census cs = build_census(c, L, part);
    u64 *psize = c.arena.alloc<u64>(rp.K), *pinb = c.arena.alloc<u64>(rp.K);
    part_sizes(c, n, part, L.nsize, psize, rp.K);
    part_inbound(c, L, cs, pinb, rp.K);
    u32 *target = c.arena.alloc<u32>(n);
    i64 *gain = c.arena.alloc<i64>(n);
    GainArgs A = make_gain_args(L, wfx, rp, cs, part, psize, pinb, discount, round, target, gain, c.d_status);
    run_gains(c, L, A);
    // movers in id order, then ranked by (gain desc, id asc)
    u32 *flag = c.arena.alloc<u32>(n), *mv = c.arena.alloc<u32>(n);
    LAUNCH(c, k_move_flags, cdiv(n, 256), 256, 0, n, target, flag);
    const u32 M = compact_indices(c, flag, mv, n);
    if (M == 0) {
        check_status(c);
        c.arena.release(m0);
        return false;
    }
    unsigned long long *gm = c.arena.alloc<unsigned long long>(1);
    AXC_CUDA(cudaMemsetAsync(gm, 0, 8, c.stream));
    LAUNCH(c, k_gain_max, cdiv(M, 256), 256, 0, mv, M, gain, gm);
    const u64 gmax = fetch1(c, (const u64 *)gm);
    const u32 kb = bits_for(gmax);
    u32 *khi = c.arena.alloc<u32>(M), *klo = c.arena.alloc<u32>(M);
    LAUNCH(c, k_move_keys, cdiv(M, 256), 256, 0, mv, M, gain, gmax, khi, klo);
    if (kb > 32) radix_sort_pairs64(c, khi, klo, mv, M, kb - 32, 32);
    else radix_sort_pairs(c, klo, mv, M, kb);
    u32 *rank = flag;
    fill_u32(c, rank, NONE, n);
    LAUNCH(c, k_set_rank, cdiv(M, 256), 256, 0, mv, M, rank);
    // cascade
    unsigned long long *g2 = c.arena.alloc<unsigned long long>(n);
    AXC_CUDA(cudaMemsetAsync(g2, 0, (size_t)n * 8, c.stream));
    {
        CascadeArgs C{L.e, rp.encourage ? 1 : 0, L.off, L.pins, wfx, cs.lam, cs.part, cs.cnt, rank, part, target, g2,
                      c.d_status};
        size_t m1 = c.arena.mark();
        u32 *big = c.arena.alloc<u32>(L.e), *blist = c.arena.alloc<u32>(L.e);
        AXC_CUDA(cudaMemsetAsync(big, 0, (size_t)L.e * 4, c.stream));
        LAUNCH(c, k_cascade_warp, cdiv(L.e, CC_WARPS), CC_WARPS * 32, 0, C, big);
        u32 nb = compact_indices(c, big, blist, L.e);
        if (nb) {
            u64 *mvsz = c.arena.alloc<u64>(nb + 1), *tabsz = c.arena.alloc<u64>(nb + 1);
            LAUNCH(c, k_big_sizes, cdiv(nb + 1, 256), 256, 0, blist, nb, L.off, cs.lam, mvsz, tabsz);
            scan_excl_u64(c, mvsz, mvsz, nb + 1);
            scan_excl_u64(c, tabsz, tabsz, nb + 1);
            u64 t2[2];
            t2[0] = fetch1(c, mvsz + nb);
            t2[1] = fetch1(c, tabsz + nb);
            u64 *smv = c.arena.alloc<u64>(t2[0] + 1);
            u32 *stab = c.arena.alloc<u32>(t2[1] + 1);
            LAUNCH(c, k_cascade_big, nb, 256, 0, C, blist, nb, smv, stab, mvsz, tabsz);
        }
        c.arena.release(m1);
    }
    // prefix gains in rank order
    i64 *G = c.arena.alloc<i64>(M), *Gx = c.arena.alloc<i64>(M);
    LAUNCH(c, k_gather_g2, cdiv(M, 256), 256, 0, mv, M, g2, Gx);
    scan_excl_i64(c, Gx, G, M);
    LAUNCH(c, k_incl_fix, cdiv(M, 256), 256, 0, Gx, G, M);
    // size validity
    i64 *Vs = c.arena.alloc<i64>(M);
    AXC_CUDA(cudaMemsetAsync(Vs, 0, (size_t)M * 8, c.stream));
    {
        size_t m1 = c.arena.mark();
        const u32 ne = 2 * M;
        u32 *key = c.arena.alloc<u32>(ne), *val = c.arena.alloc<u32>(ne);
        LAUNCH(c, k_size_events, cdiv(ne, 256), 256, 0, mv, M, part, target, key, val);
        radix_sort_pairs(c, key, val, ne, bits_for(rp.K ? rp.K - 1 : 0));
        i64 *d = c.arena.alloc<i64>(ne), *E = c.arena.alloc<i64>(ne);
        LAUNCH(c, k_size_delta, cdiv(ne, 256), 256, 0, mv, val, ne, L.nsize, d);
        scan_excl_i64(c, d, E, ne);
        LAUNCH(c, k_size_flags, cdiv(ne, 256), 256, 0, key, val, d, E, ne, psize, (u64)rp.omega,
               (unsigned long long *)Vs);
        c.arena.release(m1);
    }
    i64 *Vsx = c.arena.alloc<i64>(M);
    scan_excl_i64(c, Vs, Vsx, M);
    LAUNCH(c, k_incl_fix, cdiv(M, 256), 256, 0, Vs, Vsx, M);
    Vs = Vsx;
    // inbound validity (INCC only)
    i64 *Vi = nullptr;
    if (rp.delta < 0x7FFFFFFFu) {
        Vi = c.arena.alloc<i64>(M);
        AXC_CUDA(cudaMemsetAsync(Vi, 0, (size_t)M * 8, c.stream));
        size_t m1 = c.arena.mark();
        u32 *cnt = c.arena.alloc<u32>(M);
        u64 *base = c.arena.alloc<u64>(M + 1);
        LAUNCH(c, k_inb_counts, cdiv(M, 256), 256, 0, mv, M, L.nin, cnt);
        offsets_from_counts(c, cnt, base, M);
        const u64 ne = fetch1(c, base + M);
        if (ne) {
            u32 *keyH = c.arena.alloc<u32>(ne), *keyP = c.arena.alloc<u32>(ne), *val = c.arena.alloc<u32>(ne);
            LAUNCH(c, k_inb_events, cdiv((u64)M * 32, 256), 256, 0, mv, M, base, L.toff, L.touch, L.nin, part, target,
                   keyH, keyP, val);
            radix_sort_pairs(c, keyH, val, ne, bits_for(L.e ? L.e - 1 : 0));
            u32 *kp2 = c.arena.alloc<u32>(ne);
            LAUNCH(c, k_gather_by, cdiv(ne, 256), 256, 0, keyP, val, kp2, ne);
            radix_sort_pairs(c, kp2, val, ne, bits_for(rp.K ? rp.K - 1 : 0));
            u32 *ev_h = keyH, *ev_r = keyP;  // reuse
            i64 *ev_d = c.arena.alloc<i64>(ne);
            u32 *head = c.arena.alloc<u32>(ne), *sid = c.arena.alloc<u32>(ne), *start = c.arena.alloc<u32>(ne);
            LAUNCH(c, k_inb_decode, cdiv(ne, 256), 256, 0, val, kp2, ne, base, M, mv, L.toff, L.touch, ev_h, ev_r,
                   ev_d, head);
            LAUNCH(c, k_seg_heads, cdiv(ne, 256), 256, 0, kp2, ev_h, ne, head);
            scan_excl_u32(c, head, sid, ne);
            LAUNCH(c, k_seg_start, cdiv(ne, 256), 256, 0, head, sid, ne, start);
            i64 *E = c.arena.alloc<i64>(ne);
            scan_excl_i64(c, ev_d, E, ne);
            u32 *tflag = c.arena.alloc<u32>(ne);
            int32_t *tdelta = (int32_t *)c.arena.alloc<u32>(ne);
            LAUNCH(c, k_inb_trans, cdiv(ne, 256), 256, 0, kp2, ev_h, ev_r, ev_d, E, head, sid, start, ne, L.off,
                   cs.lam, cs.part, cs.dcnt, tflag, tdelta);
            u32 *tidx = c.arena.alloc<u32>(ne);
            const u32 T = compact_indices(c, tflag, tidx, ne);
            if (T) {
                u32 *tp = c.arena.alloc<u32>(T), *tr = c.arena.alloc<u32>(T), *perm = c.arena.alloc<u32>(T);
                int32_t *td = (int32_t *)c.arena.alloc<u32>(T);
                LAUNCH(c, k_trans_gather, cdiv(T, 256), 256, 0, tidx, T, kp2, ev_r, tdelta, tp, tr, td);
                // order (p, r): stable by r, then stable by p
                u32 *kr = c.arena.alloc<u32>(T), *kpp = c.arena.alloc<u32>(T);
                AXC_CUDA(cudaMemcpyAsync(kr, tr, (size_t)T * 4, cudaMemcpyDeviceToDevice, c.stream));
                LAUNCH(c, k_iota, cdiv(T, 256), 256, 0, perm, T);
                radix_sort_pairs(c, kr, perm, T, bits_for(M - 1));
                LAUNCH(c, k_gather_by, cdiv(T, 256), 256, 0, tp, perm, kpp, T);
                radix_sort_pairs(c, kpp, perm, T, bits_for(rp.K ? rp.K - 1 : 0));
                u32 *sr = kr;
                i64 *sd = c.arena.alloc<i64>(T), *E2 = c.arena.alloc<i64>(T);
                LAUNCH(c, k_trans_perm, cdiv(T, 256), 256, 0, perm, T, tr, td, sr, sd);
                scan_excl_i64(c, sd, E2, T);
                u32 *h2 = c.arena.alloc<u32>(T), *sid2 = c.arena.alloc<u32>(T), *st2 = c.arena.alloc<u32>(T);
                LAUNCH(c, k_seg_heads, cdiv(T, 256), 256, 0, kpp, (const u32 *)nullptr, T, h2);
                scan_excl_u32(c, h2, sid2, T);
                LAUNCH(c, k_seg_start, cdiv(T, 256), 256, 0, h2, sid2, T, st2);
                LAUNCH(c, k_trans_flags, cdiv(T, 256), 256, 0, kpp, sr, sd, E2, sid2, st2, T, pinb, (u64)rp.delta,
                       (unsigned long long *)Vi);
            }
        }
        c.arena.release(m1);
        i64 *Vix = c.arena.alloc<i64>(M);
        scan_excl_i64(c, Vi, Vix, M);
        LAUNCH(c, k_incl_fix, cdiv(M, 256), 256, 0, Vi, Vix, M);
        Vi = Vix;
    }
    // best prefix and apply
    const u32 nbk = cdiv(M, 256) < 64u ? cdiv(M, 256) : 64u;
    Best *bb = (Best *)c.arena.alloc<u64>(4 * (nbk + 1));
    u32 *apply = c.arena.alloc<u32>(1);
    LAUNCH(c, k_best, nbk, 256, 0, G, Vs, Vi, M, bb + 1);
    LAUNCH(c, k_best_final, 1, 1, 0, bb + 1, nbk, Vi, bb, apply);
    LAUNCH(c, k_apply, cdiv(M, 256), 256, 0, mv, target, bb, apply, part);
    const u32 applied = fetch1(c, apply);
    check_status(c);
    c.arena.release(m0);
    return applied != 0;
}

u32 refine_level(Ctx &c, const DLevel &L, const u32 *wfx, const RefineParams &rp, u32 *part) {
    const u32 R = rp.rounds;
    u32 done = 0;
    for (u32 r = 0; r < R; ++r) {
        const u32 discount = r < R / 3 ? 1u : (r < 2 * R / 3 ? 2u : 0xFFFFFFFFu);
        ++done;
        if (!refine_round(c, L, wfx, rp, part, discount, r)) {
            if (r < R / 3) r = R / 2;
            else if (r < 2 * R / 3) r = 2 * R / 3;
            else r = R;
        }
    }
    return done;
}

}  // namespace axc
