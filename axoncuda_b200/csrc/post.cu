// Uncoarsening, the greedy packing shared by the -ipm group merge and the INCC small-partition
// merge, zero-basing, and metrics/validity on the device.
#include "common.cuh"
#include "kernels.h"

namespace axc {
namespace {

__global__ void k_uncoarsen(u32 n, const u32 *__restrict__ groups, const u32 *__restrict__ cp, u32 *__restrict__ part) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) part[v] = cp[groups[v]];
}

__device__ __forceinline__ u32 ub_u64(const u64 *a, u32 len, u64 x) {
    u32 lo = 0, hi = len;
    while (lo < hi) {
        u32 mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// next segment start of the greedy packing from pos (sources/postprocess.cu:118-137)
__global__ void k_pack_next(const u64 *__restrict__ ps, const u64 *__restrict__ pi, u32 m, u64 omega, u64 delta,
                            u32 *__restrict__ nxt) {
    u32 pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos > m) return;
    if (pos == m) { nxt[m] = m; return; }
    u32 js = ub_u64(ps, m + 1, ps[pos] + omega);
    u32 ji = ub_u64(pi, m + 1, pi[pos] + delta);
    u32 j = (js < ji ? js : ji) - 1;
    nxt[pos] = j > pos + 1 ? j : pos + 1;
}
__global__ void k_jump_double(const u32 *__restrict__ j, u32 *__restrict__ j2, u32 m) {
    u32 pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos <= m) j2[pos] = j[j[pos]];
}
__global__ void k_mark_orbit(const u32 *__restrict__ j, u32 *mark, u32 m) {
    u32 pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos <= m && ((volatile u32 *)mark)[pos]) mark[j[pos]] = 1u;
}
__global__ void k_set_one(u32 *p) { *p = 1u; }
__global__ void k_packid(const u32 *__restrict__ mark_scan, const u32 *__restrict__ mark, u32 m, u32 *__restrict__ packid) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) packid[i] = mark_scan[i] + mark[i] - 1;
}

__global__ void k_small_flags(u32 K, const u64 *__restrict__ psize, u32 *__restrict__ flag) {
    u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < K) flag[p] = psize[p] < 16 ? 1u : 0u;  // SMALL_PART_MERGE_SIZE_THRESHOLD (headers/defines.cuh:33)
}
__global__ void k_gather_key(const u32 *__restrict__ ids, u32 m, const u64 *__restrict__ x, u32 *__restrict__ key) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) key[i] = (u32)x[ids[i]];
}
__global__ void k_gather_u64(const u32 *__restrict__ ids, u32 m, const u64 *__restrict__ x, u64 *__restrict__ y) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) y[i] = x[ids[i]];
}
__global__ void k_rep_min(const u32 *__restrict__ ids, const u32 *__restrict__ packid, u32 m, u32 *__restrict__ rep) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) atomicMin(&rep[packid[i]], ids[i]);
}
__global__ void k_pmap_set(const u32 *__restrict__ ids, const u32 *__restrict__ packid, const u32 *__restrict__ rep,
                           u32 m, u32 *__restrict__ pmap) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) pmap[ids[i]] = rep[packid[i]];
}
__global__ void k_apply_map(u32 n, u32 *__restrict__ part, const u32 *__restrict__ pmap) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) part[v] = pmap[part[v]];
}
__global__ void k_used(u32 n, const u32 *__restrict__ part, u32 *__restrict__ used) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) used[part[v]] = 1u;
}

// metrics: per hyperedge lambda from the census
__global__ void k_metrics(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ lam, const u32 *__restrict__ wfx,
                          unsigned long long *__restrict__ acc) {
    u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    i64 conn = 0, cut = 0, soed = 0;
    if (h < e) {
        const i64 w = wfx[h];
        const i64 l = lam[h];
        const i64 len = (i64)(off[h + 1] - off[h]);
        const i64 l1 = l > 0 ? l - 1 : 0;  // an empty hyperedge connects nothing
        conn = w * l1;
        cut = l > 1 ? w : 0;
        soed = w * l1 * len;
    }
    conn = warp_sum(conn);
    cut = warp_sum(cut);
    soed = warp_sum(soed);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], (unsigned long long)conn);
        atomicAdd(&acc[1], (unsigned long long)cut);
        atomicAdd(&acc[2], (unsigned long long)soed);
    }
}
__global__ void k_part_stats(u32 K, const u64 *__restrict__ psize, const u64 *__restrict__ pinb,
                             unsigned long long *__restrict__ acc) {
    u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    u64 used = 0, ms = 0, mi = 0;
    if (p < K) {
        used = psize[p] > 0;
        ms = psize[p];
        mi = pinb[p];
    }
    used = warp_sum(used);
    ms = warp_max_u64(ms);
    mi = warp_max_u64(mi);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[3], (unsigned long long)used);
        atomicMax(&acc[4], (unsigned long long)ms);
        atomicMax(&acc[5], (unsigned long long)mi);
    }
}
__global__ void k_count_nodes(u32 n, const u32 *__restrict__ part, unsigned long long *__restrict__ cnt) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) atomicAdd(&cnt[part[v]], 1ull);
}

}  // namespace

void uncoarsen(Ctx &c, u32 n, const u32 *groups, const u32 *coarse_part, u32 *part) {
    if (n) LAUNCH(c, k_uncoarsen, cdiv(n, 256), 256, 0, n, groups, coarse_part, part);
}

// Greedy contiguous packing of m items with sizes ss and inbound bounds si (in their given
// order): a pack starting at pos ends before the first prefix slot that would exceed omega or
// delta (at least one item). The chain of pack starts from 0 is found by pointer doubling.
// packid[m] receives each item's pack index; returns the pack count.
u32 greedy_pack(Ctx &c, const u64 *ss, const u64 *si, u32 m, u64 omega, u64 delta, u32 *packid) {
    if (m == 0) return 0;
    size_t mk = c.arena.mark();
    u64 *s1 = c.arena.alloc<u64>(m + 1), *s2 = c.arena.alloc<u64>(m + 1);
    u64 *ps = c.arena.alloc<u64>(m + 1), *pi = c.arena.alloc<u64>(m + 1);
    AXC_CUDA(cudaMemcpyAsync(s1, ss, (size_t)m * 8, cudaMemcpyDeviceToDevice, c.stream));
    AXC_CUDA(cudaMemcpyAsync(s2, si, (size_t)m * 8, cudaMemcpyDeviceToDevice, c.stream));
    AXC_CUDA(cudaMemsetAsync(s1 + m, 0, 8, c.stream));
    AXC_CUDA(cudaMemsetAsync(s2 + m, 0, 8, c.stream));
    scan_excl_u64(c, s1, ps, m + 1);
    scan_excl_u64(c, s2, pi, m + 1);
    u32 levels = 1;
    while ((1ull << levels) < (u64)m + 1) ++levels;
    u32 *jt = c.arena.alloc<u32>((u64)(levels + 1) * (m + 1));
    LAUNCH(c, k_pack_next, cdiv(m + 1, 256), 256, 0, ps, pi, m, omega, delta, jt);
    for (u32 k = 1; k <= levels; ++k)
        LAUNCH(c, k_jump_double, cdiv(m + 1, 256), 256, 0, jt + (u64)(k - 1) * (m + 1), jt + (u64)k * (m + 1), m);
    u32 *mark = c.arena.alloc<u32>(m + 1);
    AXC_CUDA(cudaMemsetAsync(mark, 0, (size_t)(m + 1) * 4, c.stream));
    LAUNCH(c, k_set_one, 1, 1, 0, mark);
    for (u32 k = 0; k <= levels; ++k)
        LAUNCH(c, k_mark_orbit, cdiv(m + 1, 256), 256, 0, jt + (u64)k * (m + 1), mark, m);
    u32 *msc = c.arena.alloc<u32>(m);
    scan_excl_u32(c, mark, msc, m);
    LAUNCH(c, k_packid, cdiv(m, 256), 256, 0, msc, mark, m, packid);
    const u32 last = fetch1(c, packid + m - 1);
    c.arena.release(mk);
    return last + 1;
}

void merge_small_partitions(Ctx &c, const DLevel &L, u32 *part, u32 K, u32 omega, u32 delta) {
    if (K == 0) return;
    size_t mk = c.arena.mark();
    Census cs = build_census(c, L, part);
    u64 *psize = c.arena.alloc<u64>(K), *pinb = c.arena.alloc<u64>(K);
    part_sizes(c, L.n, part, L.nsize, psize, K);
    part_inbound(c, L, cs, pinb, K);
    u32 *flag = c.arena.alloc<u32>(K), *ids = c.arena.alloc<u32>(K);
    LAUNCH(c, k_small_flags, cdiv(K, 256), 256, 0, K, psize, flag);
    const u32 m = compact_indices(c, flag, ids, K);
    if (m > 0) {
        // order by (size, inbound, id): ids ascending, stable by inbound, stable by size
        u32 *key = c.arena.alloc<u32>(m);
        LAUNCH(c, k_gather_key, cdiv(m, 256), 256, 0, ids, m, pinb, key);
        radix_sort_pairs(c, key, ids, m, 32);
        LAUNCH(c, k_gather_key, cdiv(m, 256), 256, 0, ids, m, psize, key);
        radix_sort_pairs(c, key, ids, m, 4);
        u64 *ss = c.arena.alloc<u64>(m), *si = c.arena.alloc<u64>(m);
        LAUNCH(c, k_gather_u64, cdiv(m, 256), 256, 0, ids, m, psize, ss);
        LAUNCH(c, k_gather_u64, cdiv(m, 256), 256, 0, ids, m, pinb, si);
        u32 *packid = c.arena.alloc<u32>(m), *rep = c.arena.alloc<u32>(m);
        greedy_pack(c, ss, si, m, omega, delta, packid);
        fill_u32(c, rep, NONE, m);
        LAUNCH(c, k_rep_min, cdiv(m, 256), 256, 0, ids, packid, m, rep);
        u32 *pmap = c.arena.alloc<u32>(K);
        iota_u32(c, pmap, K);
        LAUNCH(c, k_pmap_set, cdiv(m, 256), 256, 0, ids, packid, rep, m, pmap);
        LAUNCH(c, k_apply_map, cdiv(L.n, 256), 256, 0, L.n, part, pmap);
    }
    c.arena.release(mk);
}

u32 zero_base(Ctx &c, u32 n, u32 *part, u32 K) {
    if (n == 0 || K == 0) return 0;
    size_t mk = c.arena.mark();
    u32 *used = c.arena.alloc<u32>(K + 1), *nid = c.arena.alloc<u32>(K + 1);
    AXC_CUDA(cudaMemsetAsync(used, 0, (size_t)(K + 1) * 4, c.stream));
    LAUNCH(c, k_used, cdiv(n, 256), 256, 0, n, part, used);
    scan_excl_u32(c, used, nid, K + 1);
    const u32 total = fetch1(c, nid + K);
    LAUNCH(c, k_apply_map, cdiv(n, 256), 256, 0, n, part, nid);
    c.arena.release(mk);
    return total;
}

void evaluate(Ctx &c, const DLevel &L, const u32 *wfx, const u32 *part, u32 omega, u32 delta, u32 max_parts,
              axc_stats *st) {
    size_t mk = c.arena.mark();
    const u32 K = L.n ? reduce_max_u32(c, part, L.n) + 1 : 0;
    Census cs = build_census(c, L, part);
    u64 *psize = c.arena.alloc<u64>(K ? K : 1), *pinb = c.arena.alloc<u64>(K ? K : 1);
    // validity counts nodes (not node weights), like sources/constr.cpp:95-115
    AXC_CUDA(cudaMemsetAsync(psize, 0, (size_t)K * 8, c.stream));
    if (L.n) LAUNCH(c, k_count_nodes, cdiv(L.n, 256), 256, 0, L.n, part, (unsigned long long *)psize);
    part_inbound(c, L, cs, pinb, K);
    unsigned long long *acc = c.arena.alloc<unsigned long long>(6);
    AXC_CUDA(cudaMemsetAsync(acc, 0, 48, c.stream));
    if (L.e) LAUNCH(c, k_metrics, cdiv(L.e, 256), 256, 0, L.e, L.off, cs.lam, wfx, acc);
    if (K) LAUNCH(c, k_part_stats, cdiv(K, 256), 256, 0, K, psize, pinb, acc);
    u64 h[6];
    fetch(c, h, acc, 48);
    st->connectivity_fx = (i64)h[0];
    st->cutnet_fx = (i64)h[1];
    st->soed_fx = (i64)h[2];
    st->connectivity = (double)(i64)h[0] / 262144.0;
    st->cutnet = (double)(i64)h[1] / 262144.0;
    st->soed = (double)(i64)h[2] / 262144.0;
    st->num_parts = (u32)h[3];
    st->max_part_size = (u32)h[4];
    st->max_part_inbound = (u32)h[5];
    const bool dense = h[3] == K;
    st->valid = dense && h[3] <= max_parts && h[4] <= omega && h[5] <= delta;
    c.arena.release(mk);
}

}  // namespace axc
