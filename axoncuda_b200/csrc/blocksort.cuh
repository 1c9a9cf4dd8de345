// One-block stable LSD radix sort in shared memory, shared by the sort primitive (prim.cu) and
// the small-level refinement kernels (refine.cu). A block of RSS_WARPS * 32 threads sorts at most
// RSS_CAP (key, value) pairs, 8 bits per pass. Warp w owns elements [w*256, (w+1)*256) in 8 rounds
// of 32, so the ranks (digit offset + earlier warps' counts + match_any rank in the warp) keep the
// sort stable.
#pragma once
#include "common.cuh"

namespace axc {

constexpr int RSS_WARPS = 32;
constexpr int RSS_ITEMS = 8;
constexpr int RSS_CAP = RSS_WARPS * 32 * RSS_ITEMS;  // 8192
constexpr size_t RSS_SMEM = (size_t)4 * RSS_CAP * 4 + (size_t)RSS_WARPS * 256 * 4 + 257 * 4;

#ifdef __CUDACC__
// sm (RSS_SMEM bytes of dynamic shared memory) holds the keys at [0, n) and the values at
// [RSS_CAP, RSS_CAP + n) on entry. On return ko / vo point at the sorted keys and values (in sm),
// and the block is synchronised.
__device__ __forceinline__ void block_radix_sort(u32 *sm, u32 n, u32 bits, const u32 *&ko, const u32 *&vo) {
    u32 *ka = sm, *va = ka + RSS_CAP, *kb = va + RSS_CAP, *vb = kb + RSS_CAP;
    u32 *wcnt = vb + RSS_CAP;             // [RSS_WARPS][256]
    u32 *dbase = wcnt + RSS_WARPS * 256;  // [257]
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const u32 lt = (1u << lane) - 1u;
    for (u32 shift = 0; shift < bits; shift += 8) {
        for (int i = threadIdx.x; i < RSS_WARPS * 256; i += blockDim.x) wcnt[i] = 0;
        __syncthreads();
        u32 dig[RSS_ITEMS], loc[RSS_ITEMS];
#pragma unroll
        for (int r = 0; r < RSS_ITEMS; ++r) {
            const u32 i = (u32)w * 32 * RSS_ITEMS + (u32)r * 32 + lane;
            const bool ok = i < n;
            const u32 d = ok ? ((ka[i] >> shift) & 255u) : 256u;
            dig[r] = d;
            const u32 peers = __match_any_sync(0xFFFFFFFFu, d);
            const u32 before = ok ? wcnt[w * 256 + d] : 0u;
            loc[r] = before + __popc(peers & lt);
            __syncwarp();
            if (ok && (peers & lt) == 0) wcnt[w * 256 + d] = before + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // per digit: counts over warps -> running offsets; then digit bases by a scan over 256
        if (threadIdx.x < 256) {
            const u32 d = threadIdx.x;
            u32 run = 0;
            for (int ww = 0; ww < RSS_WARPS; ++ww) {
                const u32 t = wcnt[ww * 256 + d];
                wcnt[ww * 256 + d] = run;
                run += t;
            }
            dbase[d] = run;
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // exclusive scan of the 256 digit totals, 8 per lane
            u32 v[8], s = 0;
            for (int k = 0; k < 8; ++k) { v[k] = dbase[lane * 8 + k]; s += v[k]; }
            u32 x = s;
            for (int o = 1; o < 32; o <<= 1) {
                const u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x += y;
            }
            u32 pre = x - s;
            for (int k = 0; k < 8; ++k) { dbase[lane * 8 + k] = pre; pre += v[k]; }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RSS_ITEMS; ++r) {
            const u32 d = dig[r];
            if (d < 256u) {
                const u32 i = (u32)w * 32 * RSS_ITEMS + (u32)r * 32 + lane;
                const u32 pos = dbase[d] + wcnt[w * 256 + d] + loc[r];
                kb[pos] = ka[i];
                vb[pos] = va[i];
            }
        }
        __syncthreads();
        u32 *t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    ko = ka;
    vo = va;
}
#endif

}  // namespace axc
