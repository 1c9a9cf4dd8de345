// K-way initial partition on the coarsest level (replaces the Mt-KaHyPar bridge of
// sources/init_part.cu:733-953). Level-synchronous BFS over hyperedges from node 0, re-rooted at
// the farthest node (largest distance, then largest id); nodes are ordered by (distance, id) with
// unreached nodes last, and cut into k consecutive chunks of equal node weight:
// node i goes to floor((2*W_before + s_i) * k / (2*W)). With coarse node weights capped at the
// balance slack (the driver caps cluster sizes in k-way mode) every chunk fits omega.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <vector>

namespace axc {
namespace {

__global__ void k_bfs_init(u32 n, u32 *__restrict__ dist, u32 root, u32 *__restrict__ front) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) dist[v] = v == root ? 0u : NONE;
    if (v == 0) front[0] = root;
}
__global__ void k_bfs_expand(const u32 *__restrict__ front, u32 nf, u32 level, const u64 *__restrict__ toff,
                             const u32 *__restrict__ touch, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                             u32 *__restrict__ hdone, u32 *__restrict__ dist, u32 *__restrict__ next, u32 *__restrict__ nn) {
    const u32 i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= nf) return;
    const u32 u = front[i];
    const u64 jend = toff[u + 1];
    // 32 incidences claimed at once (one per lane), then each claimed hyperedge expanded by the
    // whole warp; the distances do not depend on the order
    for (u64 jb = toff[u]; jb < jend; jb += 32) {
        const u64 j = jb + lane;
        const u32 h = j < jend ? touch[j] : 0;
        const bool mine = j < jend && atomicExch(&hdone[h], 1u) == 0;
        u32 bal = __ballot_sync(0xFFFFFFFFu, mine);
        while (bal) {
            const u32 t = __ffs(bal) - 1;
            bal &= bal - 1;
            const u32 hh = __shfl_sync(0xFFFFFFFFu, h, t);
            for (u64 k = off[hh] + lane; k < off[hh + 1]; k += 32) {
                const u32 v = pins[k];
                if (atomicCAS(&dist[v], NONE, level + 1) == NONE) next[atomicAdd(nn, 1u)] = v;
            }
        }
    }
}
__global__ void k_far_key(u32 n, const u32 *__restrict__ dist, u64 *__restrict__ key) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) key[v] = dist[v] == NONE ? 0ull : (((u64)dist[v] << 32) | v);
}
__global__ void k_order_keys(u32 n, const u32 *__restrict__ dist, u32 unreached, u32 *__restrict__ key) {
    u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) key[v] = dist[v] == NONE ? unreached : dist[v];
}
__global__ void k_gather_w(const u32 *__restrict__ ord, u32 n, const u32 *__restrict__ nsize, u64 *__restrict__ w) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = nsize[ord[i]];
}
__global__ void k_chunk(const u32 *__restrict__ ord, u32 n, const u64 *__restrict__ before, const u64 *__restrict__ w,
                        u64 W, u32 k, u32 base, u32 *__restrict__ part) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned __int128 x = (unsigned __int128)(2 * before[i] + w[i]) * k;
    u64 q = (u64)(x / (unsigned __int128)(2 * W));
    part[ord[i]] = base + (u32)(q < k - 1 ? q : k - 1);
}

// ---- the k-way multi-start (include/axc.h AXC_KWAY_TRIES) ----------------------------------------
__global__ void k_len2_flag(u32 e, const u64 *__restrict__ off, u32 *__restrict__ flag) {
    const u32 h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < e) flag[h] = off[h + 1] - off[h] >= 2 ? 1u : 0u;
}
__global__ void k_kept_len(const u32 *__restrict__ keep, u32 e2, const u64 *__restrict__ off, u64 *__restrict__ len) {
    const u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < e2) len[j] = off[keep[j] + 1] - off[keep[j]];
}
// hyperedge t * e2 + j of the copies is kept hyperedge j of copy t
__global__ void k_super_hedges(const u32 *__restrict__ keep, u32 e2, u32 nc, const u32 *__restrict__ nsrc,
                               const u32 *__restrict__ wfx, const u64 *__restrict__ offp, u64 P2,
                               u64 *__restrict__ offS, u32 *__restrict__ nsrcS, u32 *__restrict__ wfxS) {
    const u64 idx = (u64)blockIdx.x * blockDim.x + threadIdx.x, tot = (u64)nc * e2;
    if (idx == 0) offS[tot] = (u64)nc * P2;
    if (idx >= tot) return;
    const u32 t = (u32)(idx / e2), j = (u32)(idx % e2);
    offS[idx] = (u64)t * P2 + offp[j];
    nsrcS[idx] = nsrc[keep[j]];
    wfxS[idx] = wfx[keep[j]];
}
// one warp per (copy, kept hyperedge): its pins, shifted by t * n
__global__ void k_super_pins(const u32 *__restrict__ keep, u32 e2, u32 nc, const u64 *__restrict__ off,
                             const u32 *__restrict__ pins, const u64 *__restrict__ offp, u64 P2, u32 n,
                             u32 *__restrict__ pinsS) {
    const u64 wid = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5, tot = (u64)nc * e2;
    const u32 lane = threadIdx.x & 31;
    if (wid >= tot) return;
    const u32 t = (u32)(wid / e2), j = (u32)(wid % e2), h = keep[j];
    const u64 a = off[h], len = off[h + 1] - a, dst = (u64)t * P2 + offp[j];
    for (u64 i = lane; i < len; i += 32) pinsS[dst + i] = pins[a + i] + t * n;
}
// node t * n + v of the copies: its size; copy 0 starts from part
__global__ void k_super_nodes(u32 n, u32 nc, const u32 *__restrict__ nsize, const u32 *__restrict__ part,
                              u32 *__restrict__ nsizeS, u32 *__restrict__ partS) {
    const u64 idx = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (u64)nc * n) return;
    const u32 v = (u32)(idx % n);
    nsizeS[idx] = nsize[v];
    if (idx < n) partS[idx] = part[v];
}
__global__ void k_try_keys(u32 n, u32 salt, u32 *__restrict__ key, u32 *__restrict__ ord) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) { key[v] = mix32(v ^ salt); ord[v] = v; }
}
__global__ void k_copy_conn(u64 eS, u32 e2, const u32 *__restrict__ lam, const u32 *__restrict__ wfxS,
                            unsigned long long *__restrict__ conn) {
    const u64 h = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= eS) return;
    const u32 l = lam[h];
    if (l > 1) atomicAdd(&conn[h / e2], (unsigned long long)wfxS[h] * (l - 1));
}
__global__ void k_pick_copy(u32 n, const u32 *__restrict__ partS, u32 best, u32 k, u32 *__restrict__ part) {
    const u32 v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n) part[v] = partS[(u64)best * n + v] - best * k;
}

// BFS distances from root into dist[n]; returns the number of levels.
u32 bfs(Ctx &c, const DLevel &L, u32 root, u32 *dist) {
    size_t m = c.arena.mark();
    const u32 n = L.n;
    u32 *fa = c.arena.alloc<u32>(n), *fb = c.arena.alloc<u32>(n), *hd = c.arena.alloc<u32>(L.e ? L.e : 1);
    u32 *nn = c.arena.alloc<u32>(1);
    AXC_CUDA(cudaMemsetAsync(hd, 0, (size_t)L.e * 4, c.stream));
    LAUNCH(c, k_bfs_init, cdiv(n, 256), 256, 0, n, dist, root, fa);
    u32 nf = 1, lvl = 0;
    while (nf) {
        AXC_CUDA(cudaMemsetAsync(nn, 0, 4, c.stream));
        LAUNCH(c, k_bfs_expand, cdiv((u64)nf * 32, 256), 256, 0, fa, nf, lvl, L.toff, L.touch, L.off, L.pins, hd, dist,
               fb, nn);
        nf = fetch1(c, nn);
        std::swap(fa, fb);
        ++lvl;
    }
    c.arena.release(m);
    return lvl;
}

}  // namespace

void kway_initial(Ctx &c, const DLevel &L, u32 k, u32 *part) {
    const u32 n = L.n;
    if (n == 0) return;
    size_t m = c.arena.mark();
    u32 *dist = c.arena.alloc<u32>(n);
    bfs(c, L, 0, dist);
    u64 *key = c.arena.alloc<u64>(n);
    LAUNCH(c, k_far_key, cdiv(n, 256), 256, 0, n, dist, key);
    const u32 far = (u32)(reduce_max_u64(c, key, n) & 0xFFFFFFFFull);
    const u32 levels = bfs(c, L, far, dist);
    u32 *okey = c.arena.alloc<u32>(n), *ord = c.arena.alloc<u32>(n);
    LAUNCH(c, k_order_keys, cdiv(n, 256), 256, 0, n, dist, levels + 1, okey);
    iota_u32(c, ord, n);
    radix_sort_pairs(c, okey, ord, n, bits_for(levels + 1));
    u64 *w = c.arena.alloc<u64>(n + 1), *before = c.arena.alloc<u64>(n + 1);
    LAUNCH(c, k_gather_w, cdiv(n, 256), 256, 0, ord, n, L.nsize, w);
    AXC_CUDA(cudaMemsetAsync(w + n, 0, 8, c.stream));
    scan_excl_u64(c, w, before, n + 1);
    const u64 W = fetch1(c, before + n);
    LAUNCH(c, k_chunk, cdiv(n, 256), 256, 0, ord, n, before, w, W ? W : 1, k, 0u, part);
    c.arena.release(m);
}

// The multi-start of include/axc.h AXC_KWAY_TRIES: copies of the level without its hyperedges of
// fewer than 2 pins (they never change a k-way gain), copy 0 from `part` (the BFS chunks), copy t
// from the random order (mix32(v ^ mix32(t * 0x9E3779B9 + seed)), v) cut into weight chunks; all
// refined together, each copy taking its own best prefix, the least connected copy kept.
bool kway_multistart(Ctx &c, const DLevel &L, const u32 *wfx, u32 k, u32 omega, u64 seed, u32 *part) {
    const u32 n = L.n, e = L.e;
    if (n == 0 || e == 0) return false;
    const size_t m = c.arena.mark();
    u32 *flag = c.arena.alloc<u32>(e), *keep = c.arena.alloc<u32>(e);
    LAUNCH(c, k_len2_flag, cdiv(e, 256), 256, 0, e, L.off, flag);
    const u32 e2 = compact_indices(c, flag, keep, e);
    u64 *offp = c.arena.alloc<u64>((u64)e2 + 1);
    AXC_CUDA(cudaMemsetAsync(offp + e2, 0, 8, c.stream));
    if (e2) LAUNCH(c, k_kept_len, cdiv(e2, 256), 256, 0, keep, e2, L.off, offp);
    scan_excl_u64(c, offp, offp, (u64)e2 + 1);
    const u64 P2 = fetch1(c, offp + e2);
    const u64 nc64 = P2 ? std::min<u64>(AXC_KWAY_TRIES, AXC_KWAY_TRY_PINS / P2) : 0;
    if (nc64 < 2) {
        c.arena.release(m);
        return false;
    }
    const u32 nc = (u32)nc64;
    DLevel S;
    S.n = nc * n;
    S.e = nc * e2;
    S.P = nc64 * P2;
    S.off = c.arena.alloc<u64>((u64)S.e + 1);
    S.nsrc = c.arena.alloc<u32>(S.e);
    u32 *wfxS = c.arena.alloc<u32>(S.e);
    S.pins = c.arena.alloc<u32>(S.P);
    S.nsize = c.arena.alloc<u32>(S.n);
    u32 *partS = c.arena.alloc<u32>(S.n);
    LAUNCH(c, k_super_hedges, cdiv((u64)S.e, 256), 256, 0, keep, e2, nc, L.nsrc, wfx, offp, P2, S.off, S.nsrc, wfxS);
    LAUNCH(c, k_super_pins, cdiv((u64)S.e * 32, 256), 256, 0, keep, e2, nc, L.off, L.pins, offp, P2, n, S.pins);
    LAUNCH(c, k_super_nodes, cdiv((u64)S.n, 256), 256, 0, n, nc, L.nsize, part, S.nsize, partS);
    S.toff = c.arena.alloc<u64>((u64)S.n + 1);
    S.touch = c.arena.alloc<u32>(S.P);
    S.nin = c.arena.alloc<u32>(S.n);
    build_touching(c, S.n, S.e, S.off, S.pins, S.nsrc, S.P, S.toff, S.touch, S.nin);
    {  // the random starts: weight chunks of a hashed node order, partition ids shifted by t * k
        const size_t m1 = c.arena.mark();
        u32 *key = c.arena.alloc<u32>(n), *ord = c.arena.alloc<u32>(n);
        u64 *w = c.arena.alloc<u64>((u64)n + 1), *before = c.arena.alloc<u64>((u64)n + 1);
        for (u32 t = 1; t < nc; ++t) {
            LAUNCH(c, k_try_keys, cdiv(n, 256), 256, 0, n, mix32(t * 0x9E3779B9u + (u32)seed), key, ord);
            radix_sort_pairs(c, key, ord, n, 32);
            LAUNCH(c, k_gather_w, cdiv(n, 256), 256, 0, ord, n, L.nsize, w);
            AXC_CUDA(cudaMemsetAsync(w + n, 0, 8, c.stream));
            scan_excl_u64(c, w, before, (u64)n + 1);
            const u64 W = fetch1(c, before + n);
            LAUNCH(c, k_chunk, cdiv(n, 256), 256, 0, ord, n, before, w, W ? W : 1, k, t * k, partS + (u64)t * n);
        }
        c.arena.release(m1);
    }
    RefineParams rp{nc * k, omega, 0x7FFFFFFFu, false, AXC_KWAY_TRY_ROUNDS, seed};
    rp.copies = nc;
    rp.copy_n = n;
    refine_level(c, S, wfxS, rp, partS);
    Census cs = build_census(c, S, partS);
    unsigned long long *conn = c.arena.alloc<unsigned long long>(nc);
    AXC_CUDA(cudaMemsetAsync(conn, 0, (size_t)nc * 8, c.stream));
    LAUNCH(c, k_copy_conn, cdiv((u64)S.e, 256), 256, 0, (u64)S.e, e2, cs.lam, wfxS, conn);
    std::vector<u64> h(nc);
    fetch(c, h.data(), (const u64 *)conn, (size_t)nc * 8);
    u32 best = 0;
    for (u32 t = 1; t < nc; ++t)
        if (h[t] < h[best]) best = t;
    LAUNCH(c, k_pick_copy, cdiv(n, 256), 256, 0, n, partS, best, k, part);
    c.arena.release(m);
    return true;
}

}  // namespace axc
