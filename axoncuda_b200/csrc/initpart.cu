// K-way initial partition on the coarsest level (replaces the Mt-KaHyPar bridge of
// sources/init_part.cu:733-953). Level-synchronous BFS over hyperedges from node 0, re-rooted at
// the farthest node (largest distance, then largest id); nodes are ordered by (distance, id) with
// unreached nodes last, and cut into k consecutive chunks of equal node weight:
// node i goes to floor((2*W_before + s_i) * k / (2*W)). With coarse node weights capped at the
// balance slack (the driver caps cluster sizes in k-way mode) every chunk fits omega.
#include "common.cuh"
#include "kernels.h"

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
    for (u64 j = toff[u]; j < toff[u + 1]; ++j) {
        const u32 h = touch[j];
        u32 claim = 0;
        if (lane == 0) claim = atomicExch(&hdone[h], 1u);
        claim = __shfl_sync(0xFFFFFFFFu, claim, 0);
        if (claim) continue;
        for (u64 k = off[h] + lane; k < off[h + 1]; k += 32) {
            const u32 v = pins[k];
            if (atomicCAS(&dist[v], NONE, level + 1) == NONE) next[atomicAdd(nn, 1u)] = v;
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
                        u64 W, u32 k, u32 *__restrict__ part) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned __int128 x = (unsigned __int128)(2 * before[i] + w[i]) * k;
    u64 q = (u64)(x / (unsigned __int128)(2 * W));
    part[ord[i]] = (u32)(q < k - 1 ? q : k - 1);
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
    LAUNCH(c, k_chunk, cdiv(n, 256), 256, 0, ord, n, before, w, W ? W : 1, k, part);
    c.arena.release(m);
}

}  // namespace axc
