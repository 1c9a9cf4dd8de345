// Construction kernels: fixed-point weights, per-hyperedge uniqueness (level-0 rule-2 dedupe and
// level-to-level contraction share one kernel family), compaction into a new pin CSR, and the
// incidence ("touching") CSR built as a stable transpose.
//
// Uniqueness rule. Every pin occurrence k of hyperedge h gets a key (the pin, or its group at
// contraction) and a priority (cls << 31 | position). For each key the occurrence of minimum
// priority survives. Level 0 (includes/hgraph.hpp:518-581, rule 2): cls = 0 everywhere, so the
// first occurrence in flat order survives and sources (stored first) win over destinations.
// Contraction (kernels/construction.cu:304-489): cls = 1 for sources, 0 for destinations, so a
// group that is both keeps its destination occurrence. Survivors are compacted in position order,
// so the output keeps sources first and is deterministic.
#include "common.cuh"
#include "kernels.h"

namespace axc {
namespace {

__global__ void k_wfx(const float *__restrict__ w, u32 *__restrict__ wfx, u32 e) {
    u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= e) return;
    float x = w ? w[h] : 1.0f;
    double y = x > 0.0f ? floor((double)x * 262144.0) : 0.0;
    wfx[h] = y >= 4294967295.0 ? 0xFFFFFFFFu : (u32)y;
}

constexpr u32 UQ_WARP_CAP = 256;      // hyperedges up to this size: one warp, table in smem
constexpr u32 UQ_BLOCK_CAP = 8192;    // up to this size: one block, table in dynamic smem
constexpr u32 UQ_WARPS = 8;

__device__ __forceinline__ u32 uq_key(const u32 *pins, const u32 *groups, u64 k) {
    u32 v = pins[k];
    return groups ? groups[v] : v;
}

// Insert all occurrences of hyperedge [a,b) into the table (keys/vals, size mask+1), then mark
// survivors. Threads [t0, t0+nt) of the caller cooperate; caller syncs between phases.
__device__ __forceinline__ void uq_insert(const u32 *pins, const u32 *groups, u64 a, u64 b, u64 s,
                                          bool dst_wins, u32 *keys, u32 *vals, u32 mask, u32 t,
                                          u32 nt, u32 *status) {
    for (u64 k = a + t; k < b; k += nt) {
        u32 key = uq_key(pins, groups, k);
        u32 pri = ((dst_wins && k < s) ? 0x80000000u : 0u) | (u32)(k - a);
        u32 slot = hash_find_or_insert(keys, mask, key);
        if (slot == NONE) { atomicExch(status, DEV_HASH_FULL); continue; }
        atomicMin(&vals[slot], pri);
    }
}
__device__ __forceinline__ void uq_mark(const u32 *pins, const u32 *groups, u64 a, u64 b, u64 s,
                                        bool dst_wins, const u32 *keys, const u32 *vals, u32 mask,
                                        u32 t, u32 nt, uint8_t *keep, u32 &kept, u32 &kept_src) {
    for (u64 k = a + t; k < b; k += nt) {
        u32 key = uq_key(pins, groups, k);
        u32 pri = ((dst_wins && k < s) ? 0x80000000u : 0u) | (u32)(k - a);
        u32 slot = hash_find(keys, mask, key);
        bool kp = slot != NONE && vals[slot] == pri;
        keep[k] = kp;
        if (kp) { ++kept; if (k < s) ++kept_src; }
    }
}

__global__ void k_uniq_warp(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                            const u32 *__restrict__ nsrc, const u32 *__restrict__ groups, int dst_wins,
                            uint8_t *__restrict__ keep, u32 *__restrict__ cnt, u32 *__restrict__ cnt_src,
                            u32 *status) {
    __shared__ u32 tk[UQ_WARPS][2 * UQ_WARP_CAP], tv[UQ_WARPS][2 * UQ_WARP_CAP];
    const u32 w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 h = blockIdx.x * UQ_WARPS + w;
    if (h >= e) return;
    const u64 a = off[h], b = off[h + 1], s = a + nsrc[h];
    const u32 len = (u32)(b - a);
    if (len > UQ_WARP_CAP) return;  // handled by the block kernel
    u32 cap = 64;
    while (cap < 2 * len) cap <<= 1;
    u32 *keys = tk[w], *vals = tv[w];
    for (u32 i = lane; i < cap; i += 32) { keys[i] = NONE; vals[i] = NONE; }
    __syncwarp();
    uq_insert(pins, groups, a, b, s, dst_wins, keys, vals, cap - 1, lane, 32, status);
    __syncwarp();
    u32 kept = 0, ks = 0;
    uq_mark(pins, groups, a, b, s, dst_wins, keys, vals, cap - 1, lane, 32, keep, kept, ks);
    kept = warp_sum(kept);
    ks = warp_sum(ks);
    if (lane == 0) { cnt[h] = kept; cnt_src[h] = ks; }
}

__global__ void k_uniq_block(const u32 *__restrict__ list, u32 nlist, const u64 *__restrict__ off,
                             const u32 *__restrict__ pins, const u32 *__restrict__ nsrc,
                             const u32 *__restrict__ groups, int dst_wins, uint8_t *__restrict__ keep,
                             u32 *__restrict__ cnt, u32 *__restrict__ cnt_src, u32 *gtab,
                             const u64 *__restrict__ gtab_off, u32 *status) {
    extern __shared__ u32 dyn[];
    __shared__ u32 red[2][32];
    if (blockIdx.x >= nlist) return;
    const u32 h = list[blockIdx.x];
    const u64 a = off[h], b = off[h + 1], s = a + nsrc[h];
    const u32 len = (u32)(b - a);
    u32 cap = 64;
    while (cap < 2 * len) cap <<= 1;
    u32 *keys, *vals;
    if (gtab) {
        keys = gtab + 2 * gtab_off[blockIdx.x];
        vals = keys + cap;
    } else {
        keys = dyn;
        vals = dyn + cap;
    }
    for (u32 i = threadIdx.x; i < cap; i += blockDim.x) { keys[i] = NONE; vals[i] = NONE; }
    __syncthreads();
    uq_insert(pins, groups, a, b, s, dst_wins, keys, vals, cap - 1, threadIdx.x, blockDim.x, status);
    __syncthreads();
    u32 kept = 0, ks = 0;
    uq_mark(pins, groups, a, b, s, dst_wins, keys, vals, cap - 1, threadIdx.x, blockDim.x, keep, kept, ks);
    kept = warp_sum(kept);
    ks = warp_sum(ks);
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = kept; red[1][threadIdx.x >> 5] = ks; }
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 t0 = 0, t1 = 0;
        for (u32 i = 0; i < blockDim.x / 32; ++i) { t0 += red[0][i]; t1 += red[1][i]; }
        cnt[h] = t0;
        cnt_src[h] = t1;
    }
}

// Stable compaction of survivors, one warp per hyperedge.
__global__ void k_uniq_compact(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                               const u32 *__restrict__ groups, const uint8_t *__restrict__ keep,
                               const u64 *__restrict__ new_off, u32 *__restrict__ new_pins) {
    const u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= e) return;
    const u64 a = off[w], b = off[w + 1];
    u64 o = new_off[w];
    for (u64 base = a; base < b; base += 32) {
        u64 k = base + lane;
        bool kp = k < b && keep[k];
        u32 bal = __ballot_sync(0xFFFFFFFFu, kp);
        if (kp) new_pins[o + __popc(bal & ((1u << lane) - 1u))] = uq_key(pins, groups, k);
        o += __popc(bal);
    }
}

__global__ void k_flag_big(u32 e, const u64 *__restrict__ off, u32 lo, u32 hi, u32 *__restrict__ flag) {
    u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= e) return;
    u64 len = off[h + 1] - off[h];
    flag[h] = (len > lo && len <= hi) ? 1u : 0u;
}
__global__ void k_table_sizes(const u32 *__restrict__ list, u32 nlist, const u64 *__restrict__ off,
                              u64 *__restrict__ sz) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == nlist) sz[i] = 0;
    if (i >= nlist) return;
    u32 h = list[i];
    u64 len = off[h + 1] - off[h], cap = 64;
    while (cap < 2 * len) cap <<= 1;
    sz[i] = cap;
}

// ---------------------------------------------------------------- transpose
// key = 2*pin + is_source, value = hyperedge: a stable sort by key lists, per node, its inbound
// hyperedges ascending and then its outbound ones ascending (sources/construction.cu:17-62).
__global__ void k_touch_keys(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                             const u32 *__restrict__ nsrc, u32 *__restrict__ keys, u32 *__restrict__ vals,
                             u32 *__restrict__ deg, u32 *__restrict__ nin) {
    const u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= e) return;
    const u64 a = off[w], b = off[w + 1], s = a + nsrc[w];
    for (u64 k = a + lane; k < b; k += 32) {
        u32 v = pins[k];
        bool src = k < s;
        keys[k] = 2 * v + (src ? 1u : 0u);
        vals[k] = w;
        atomicAdd(&deg[v], 1u);
        if (!src) atomicAdd(&nin[v], 1u);
    }
}

// Input validation before any id is used as an index: offsets non-decreasing, source counts within
// their hyperedge, pin ids below n. Failures set the status word (no trap).
__global__ void k_check_input(u32 n, u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                              const u32 *__restrict__ nsrc, u32 *status) {
    const u32 w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= e) return;
    const u64 a = off[w], b = off[w + 1];
    if (b < a || nsrc[w] > b - a) {
        if (lane == 0) atomicExch(status, DEV_BAD_INDEX);
        return;
    }
    for (u64 k = a + lane; k < b; k += 32)
        if (pins[k] >= n) atomicExch(status, DEV_BAD_INDEX);
}

__global__ void k_group_sizes(u32 n, const u32 *__restrict__ groups, const u32 *__restrict__ nsize,
                              u32 *__restrict__ gsize) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) atomicAdd(&gsize[groups[v]], nsize[v]);
}

}  // namespace

void compute_wfx(Ctx &c, const float *d_w, u32 *d_wfx, u32 e) {
    if (e) LAUNCH(c, k_wfx, cdiv(e, 256), 256, 0, d_w, d_wfx, e);
}

u64 hedge_unique(Ctx &c, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc, const u32 *groups,
                 bool dst_wins, u64 *new_off, u32 *new_pins, u32 *new_nsrc, u64 pins_in) {
    if (e == 0) {
        AXC_CUDA(cudaMemsetAsync(new_off, 0, 8, c.stream));
        return 0;
    }
    size_t m = c.arena.mark();
    uint8_t *keep = c.arena.alloc<uint8_t>(pins_in ? pins_in : 1);
    u32 *cnt = c.arena.alloc<u32>(e);
    LAUNCH(c, k_uniq_warp, cdiv(e, UQ_WARPS), UQ_WARPS * 32, 0, e, off, pins, nsrc, groups,
           (int)dst_wins, keep, cnt, new_nsrc, c.d_status);
    // hyperedges larger than a warp's table
    u32 *flag = c.arena.alloc<u32>(e), *list = c.arena.alloc<u32>(e);
    LAUNCH(c, k_flag_big, cdiv(e, 256), 256, 0, e, off, UQ_WARP_CAP, UQ_BLOCK_CAP, flag);
    u32 nb = compact_indices(c, flag, list, e);
    if (nb) {
        size_t smem = 2 * 16384 * sizeof(u32);
        LAUNCH(c, k_uniq_block, nb, 512, smem, list, nb, off, pins, nsrc, groups, (int)dst_wins, keep,
               cnt, new_nsrc, (u32 *)nullptr, (const u64 *)nullptr, c.d_status);
    }
    LAUNCH(c, k_flag_big, cdiv(e, 256), 256, 0, e, off, UQ_BLOCK_CAP, 0xFFFFFFFFu, flag);
    u32 nh = compact_indices(c, flag, list, e);
    if (nh) {
        u64 *tsz = c.arena.alloc<u64>(nh + 1);
        LAUNCH(c, k_table_sizes, cdiv(nh + 1, 256), 256, 0, list, nh, off, tsz);
        scan_excl_u64(c, tsz, tsz, nh + 1);
        u64 tot = fetch1(c, tsz + nh);  // sum of table capacities
        u32 *gtab = c.arena.alloc<u32>(2 * tot);
        LAUNCH(c, k_uniq_block, nh, 512, 0, list, nh, off, pins, nsrc, groups, (int)dst_wins, keep, cnt,
               new_nsrc, gtab, (const u64 *)tsz, c.d_status);
    }
    offsets_from_counts(c, cnt, new_off, e);
    LAUNCH(c, k_uniq_compact, cdiv((u64)e * 32, 256), 256, 0, e, off, pins, groups, keep, new_off, new_pins);
    u64 total = fetch1(c, new_off + e);
    check_status(c);
    c.arena.release(m);
    return total;
}

void build_touching(Ctx &c, u32 n, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc, u64 P,
                    u64 *toff, u32 *touch, u32 *nin) {
    size_t m = c.arena.mark();
    u32 *keys = c.arena.alloc<u32>(P ? P : 1);
    u32 *deg = c.arena.alloc<u32>(n ? n : 1);
    AXC_CUDA(cudaMemsetAsync(deg, 0, (size_t)n * 4, c.stream));
    AXC_CUDA(cudaMemsetAsync(nin, 0, (size_t)n * 4, c.stream));
    if (e) LAUNCH(c, k_touch_keys, cdiv((u64)e * 32, 256), 256, 0, e, off, pins, nsrc, keys, touch, deg, nin);
    radix_sort_pairs(c, keys, touch, P, bits_for(n ? 2ull * n - 1 : 0));
    offsets_from_counts(c, deg, toff, n);
    c.arena.release(m);
}

void check_input(Ctx &c, u32 n, u32 e, const u64 *off, const u32 *pins, const u32 *nsrc) {
    if (e) LAUNCH(c, k_check_input, cdiv((u64)e * 32, 256), 256, 0, n, e, off, pins, nsrc, c.d_status);
    u32 s = fetch1(c, c.d_status);
    if (s != DEV_OK) {
        AXC_CUDA(cudaMemsetAsync(c.d_status, 0, 4, c.stream));
        throw Error(AXC_EINVAL, "hypergraph rejected: an offset, source count or pin id is out of range");
    }
}

void group_sizes(Ctx &c, u32 n, const u32 *groups, const u32 *nsize, u32 *gsize, u32 ng) {
    AXC_CUDA(cudaMemsetAsync(gsize, 0, (size_t)ng * 4, c.stream));
    if (n) LAUNCH(c, k_group_sizes, cdiv(n, 256), 256, 0, n, groups, nsize, gsize);
}

void setup_construct_kernels() {
    cudaFuncSetAttribute(k_uniq_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 16384 * 4);
}

}  // namespace axc
