// Connectivity (lambda - 1), cut-net and SOED of a partition of a device-resident hypergraph,
// computed without allocating: the per-hyperedge distinct-partition census of evaluate() fused
// with its metric sums, with every scratch byte in one file-scope device array.
//
// Scratch (16 MiB + 256 B, one array per device, reused by every call):
//   header   [0] connectivity, [1] cut-net, [2] SOED (2^-18 weight units, as u64 sums of i64),
//            [3] status bits; cleared at the start of every call
//   slices   NA_BLOCKS hash tables of NA_SLICE keys, one per block of the large-hyperedge kernel,
//            used for hyperedges longer than NA_SMEM_LEN; cleared by the block before each use
// Hyperedges longer than NA_MAX_LEN are refused (AXC_EOVERFLOW).
#include <algorithm>

#include "common.cuh"

namespace axc {
namespace {

constexpr u32 NA_BLOCKS = 128;                 // blocks of the large-hyperedge kernel
constexpr u32 NA_SLICE = 32768;                // hash slots per block in global scratch
constexpr u32 NA_MAX_LEN = NA_SLICE / 2;       // longest hyperedge accepted (16384 pins)
constexpr u32 NA_SMEM_SLOTS = 4096;            // hash slots in shared memory
constexpr u32 NA_SMEM_LEN = NA_SMEM_SLOTS / 2;  // hyperedges up to this length use shared memory
constexpr u32 NA_HEADER_WORDS = 64;            // 256 B: accumulators and status
constexpr u32 NA_WORDS = NA_HEADER_WORDS + NA_BLOCKS * NA_SLICE;
constexpr u32 NA_TOO_LONG = 1u, NA_BAD_PART = 2u;

__device__ __align__(256) u32 g_noalloc_scratch[NA_WORDS];

// The hyperedge weight in fixed point: floor(w * 2^18) clamped to u32, unit when w is absent;
// the conversion every other entry point applies to the input weights.
__device__ __forceinline__ i64 na_weight(const float *w, u64 h) {
    const float x = w ? w[h] : 1.0f;
    const double y = x > 0.0f ? floor((double)x * 262144.0) : 0.0;
    return y >= 4294967295.0 ? (i64)0xFFFFFFFFu : (i64)y;
}

// Inserts key; true when this call put it in the table. The table is at most half full.
__device__ __forceinline__ bool na_insert(u32 *tab, u32 mask, u32 key) {
    u32 s = hslot(key, mask);
    for (u32 probes = 0; probes <= mask; ++probes) {
        const u32 k = tab[s];
        if (k == key) return false;
        if (k == NONE) {
            const u32 prev = atomicCAS(&tab[s], NONE, key);
            if (prev == NONE) return true;
            if (prev == key) return false;
        }
        s = (s + 1) & mask;
    }
    return false;
}

__device__ __forceinline__ void na_add(u32 *scratch, i64 conn, i64 cut, i64 soed) {
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(scratch);
    atomicAdd(&acc[0], (unsigned long long)conn);
    atomicAdd(&acc[1], (unsigned long long)cut);
    atomicAdd(&acc[2], (unsigned long long)soed);
}

// Hyperedges of at most 32 pins: one warp each, distinct partitions by lane matching.
__global__ void __launch_bounds__(256) k_na_small(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                                                  const float *__restrict__ w, const u32 *__restrict__ part,
                                                  u32 *scratch) {
    const u32 lane = threadIdx.x & 31u;
    const u32 nw = gridDim.x * (blockDim.x >> 5);
    i64 conn = 0, cut = 0, soed = 0;
    u32 bad = 0;
    for (u64 h = (u64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); h < e; h += nw) {
        const u64 a = off[h];
        const u64 len = off[h + 1] - a;
        if (len > 32) continue;
        const bool has = lane < len;
        const u32 p = has ? part[pins[a + lane]] : NONE;
        if (has && p == NONE) bad = 1;
        const u32 same = __match_any_sync(0xFFFFFFFFu, p);
        const bool first = p != NONE && (u32)(__ffs(same) - 1) == lane;
        const i64 l = __popc(__ballot_sync(0xFFFFFFFFu, first));
        if (lane == 0) {
            const i64 wf = na_weight(w, h);
            conn += wf * (l > 0 ? l - 1 : 0);  // an empty hyperedge connects nothing
            cut += l > 1 ? wf : 0;
            soed += wf * (l > 0 ? l - 1 : 0) * (i64)len;
        }
    }
    conn = warp_sum(conn);
    cut = warp_sum(cut);
    soed = warp_sum(soed);
    bad = __any_sync(0xFFFFFFFFu, bad);
    if (lane == 0) {
        if (conn || cut || soed) na_add(scratch, conn, cut, soed);
        if (bad) atomicOr(&scratch[6], NA_BAD_PART);
    }
}

// Longer hyperedges: one block each (grid-stride), partition ids hashed into shared memory up to
// NA_SMEM_LEN pins and into the block's slice of the scratch array up to NA_MAX_LEN.
__global__ void __launch_bounds__(256) k_na_large(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                                                  const float *__restrict__ w, const u32 *__restrict__ part,
                                                  u32 *scratch) {
    __shared__ u32 stab[NA_SMEM_SLOTS];
    __shared__ u32 distinct, bad;
    u32 *slice = scratch + NA_HEADER_WORDS + (u64)blockIdx.x * NA_SLICE;
    i64 conn = 0, cut = 0, soed = 0;
    if (threadIdx.x == 0) bad = 0;
    for (u64 h = blockIdx.x; h < e; h += gridDim.x) {
        const u64 a = off[h];
        const u64 len = off[h + 1] - a;
        if (len <= 32) continue;
        if (len > NA_MAX_LEN) {
            if (threadIdx.x == 0) atomicOr(&scratch[6], NA_TOO_LONG);
            continue;
        }
        u32 cap = 64;
        while (cap < 2 * len) cap <<= 1;
        u32 *tab = cap <= NA_SMEM_SLOTS ? stab : slice;
        for (u32 i = threadIdx.x; i < cap; i += blockDim.x) tab[i] = NONE;
        if (threadIdx.x == 0) distinct = 0;
        __syncthreads();
        for (u64 k = threadIdx.x; k < len; k += blockDim.x) {
            const u32 p = part[pins[a + k]];
            if (p == NONE) {
                bad = 1;
                continue;
            }
            if (na_insert(tab, cap - 1, p)) atomicAdd(&distinct, 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const i64 wf = na_weight(w, h), l = distinct;
            conn += wf * (l > 0 ? l - 1 : 0);  // an empty hyperedge connects nothing
            cut += l > 1 ? wf : 0;
            soed += wf * (l > 0 ? l - 1 : 0) * (i64)len;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (conn || cut || soed) na_add(scratch, conn, cut, soed);
        if (bad) atomicOr(&scratch[6], NA_BAD_PART);
    }
}

// Device address of the scratch array in the current context. A symbol's address belongs to a
// context, not to a device ordinal: after cudaDeviceReset, or under a driver-API context that the
// caller made current, an address cached by device would be stale. The lookup allocates nothing,
// so it is made on every call.
cudaError_t na_scratch(u32 **out) { return cudaGetSymbolAddress((void **)out, g_noalloc_scratch); }

}  // namespace
}  // namespace axc

using namespace axc;

extern "C" int axc_connectivity_noalloc(uint32_t e, const uint64_t *d_hedge_off, const uint32_t *d_pins,
                                        const float *d_hedge_w, const uint32_t *d_part, void *stream,
                                        int64_t *out_fx) {
    if (!out_fx || (e && (!d_hedge_off || !d_pins || !d_part))) return AXC_EINVAL;
    u32 *scratch = nullptr;
    if (na_scratch(&scratch) != cudaSuccess) return AXC_ECUDA;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(scratch, 0, NA_HEADER_WORDS * 4, s) != cudaSuccess) return AXC_ECUDA;
    if (e) {
        k_na_small<<<(u32)std::min<u64>(cdiv(e, 8), 148 * 16), 256, 0, s>>>(e, d_hedge_off, d_pins, d_hedge_w, d_part,
                                                                          scratch);
        k_na_large<<<NA_BLOCKS, 256, 0, s>>>(e, d_hedge_off, d_pins, d_hedge_w, d_part, scratch);
        if (cudaGetLastError() != cudaSuccess) return AXC_ECUDA;
    }
    uint64_t h[4];
    if (cudaMemcpyAsync(h, scratch, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return AXC_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return AXC_ECUDA;
    const u32 status = (u32)h[3];
    if (status & NA_TOO_LONG) return AXC_EOVERFLOW;
    if (status & NA_BAD_PART) return AXC_EINVAL;
    out_fx[0] = (int64_t)h[0];
    out_fx[1] = (int64_t)h[1];
    out_fx[2] = (int64_t)h[2];
    return AXC_OK;
}
