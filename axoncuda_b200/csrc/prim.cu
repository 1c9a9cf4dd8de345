// Device primitives owned by the library (no Thrust/CUB): single-pass scans and compaction
// (decoupled look-back over 2048-element tiles, Merrill & Garland 2016), a stable LSD radix sort
// with warp-level match_any ranking, fills and reductions. Every launch goes through the
// context's stream.
#include "common.cuh"
#include "blocksort.cuh"

namespace axc {

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T *warp_tot, T &block_total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        T t = lane < (blockDim.x >> 5) ? warp_tot[lane] : T(0);
        T s = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < (blockDim.x >> 5)) warp_tot[lane] = s - t;
        if (lane == (int)(blockDim.x >> 5) - 1) warp_tot[32] = s;
    }
    __syncthreads();
    T r = x - v + warp_tot[w];
    block_total = warp_tot[32];
    __syncthreads();
    return r;
}

template <class TI, class TO>
__global__ void k_tile_reduce(const TI *__restrict__ in, TO *__restrict__ part, u64 n) {
    __shared__ TO wt[33];
    const u64 base = (u64)blockIdx.x * SCAN_TILE;
    TO s = 0;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        u64 i = base + (u64)j * SCAN_THREADS + threadIdx.x;
        if (i < n) s += (TO)in[i];
    }
    TO tot;
    block_excl_scan<TO>(s, wt, tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

template <class TI, class TO>
__global__ void k_tile_scan(const TI *__restrict__ in, TO *__restrict__ out, const TO *__restrict__ part,
                            u64 n) {
    __shared__ TO wt[33];
    __shared__ TO stage[SCAN_TILE + SCAN_TILE / 32];
    const u64 base = (u64)blockIdx.x * SCAN_TILE;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = j * SCAN_THREADS + threadIdx.x;
        u64 i = base + li;
        stage[li + li / 32] = i < n ? (TO)in[i] : TO(0);
    }
    __syncthreads();
    TO loc[SCAN_ITEMS];
    TO s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = threadIdx.x * SCAN_ITEMS + j;
        loc[j] = stage[li + li / 32];
        s += loc[j];
    }
    TO tot;
    TO pre = block_excl_scan<TO>(s, wt, tot) + (part ? part[blockIdx.x] : TO(0));
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = threadIdx.x * SCAN_ITEMS + j;
        stage[li + li / 32] = pre;
        pre += loc[j];
    }
    __syncthreads();
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = j * SCAN_THREADS + threadIdx.x;
        u64 i = base + li;
        if (i < n) out[i] = stage[li + li / 32];
    }
}

// ------------------------------------------------------------------ single-pass look-back
constexpr u32 LB_SPIN_LIMIT = 1u << 24;  // polls of one predecessor flag before giving up

__device__ __forceinline__ u32 ld_flag(const u32 *p) { return *(const volatile u32 *)p; }

// Tile ticket and epoch of this block (every thread gets both).
__device__ __forceinline__ u32 lb_enter(const ScanState &S, u32 &s_tile, u32 &s_epoch, u32 &epoch) {
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&S.ctrl[0], 1u);
        s_epoch = *(volatile u32 *)&S.ctrl[2];
    }
    __syncthreads();
    epoch = s_epoch;
    return s_tile;
}
// The last block of the launch to finish resets the ticket and finish counters and advances the
// epoch for the next launch (every block has taken its ticket by then).
__device__ __forceinline__ void lb_leave(const ScanState &S, u32 epoch) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&S.ctrl[1], 1u) == gridDim.x - 1) {
            S.ctrl[0] = 0;
            S.ctrl[1] = 0;
            __threadfence();
            atomicExch(&S.ctrl[2], epoch + 1 < (1u << 30) ? epoch + 1 : 1u);
        }
    }
}

// Tiles take tickets in launch order, so a tile only ever waits on tiles already running. Each
// tile publishes its aggregate, then (after looking back over its predecessors with warp 0) its
// inclusive prefix. Returns the exclusive prefix of the tile to every thread.
template <class TO>
__device__ TO lookback_prefix(const ScanState &S, u32 epoch, u32 t, TO tile_total, u32 *status, TO *s_prefix,
                              u32 spin_limit = LB_SPIN_LIMIT) {
    const u32 lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) {
        if (t == 0) {
            S.incl[0] = (u64)tile_total;
            __threadfence();
            atomicExch(&S.flag[0], (epoch << 2) | 2u);
        } else {
            S.agg[t] = (u64)tile_total;
            __threadfence();
            atomicExch(&S.flag[t], (epoch << 2) | 1u);
        }
    }
    if (t > 0 && threadIdx.x < 32) {
        TO excl = 0;
        long long j = (long long)t - 1;
        bool gave_up = false;
        while (j >= 0) {
            const long long idx = j - (long long)lane;
            u32 st = 0;
            u64 v = 0;
            if (idx >= 0) {
                u32 f = 0;
                for (u32 it = 0;; ++it) {
                    f = ld_flag(&S.flag[idx]);
                    if ((f >> 2) == epoch && (f & 3u)) break;
                    if (it >= spin_limit) {
                        gave_up = true;
                        f = (epoch << 2) | 2u;
                        break;
                    }
                    if (it > 64) __nanosleep(64);
                }
                __threadfence();
                st = f & 3u;
                v = gave_up ? 0 : (st == 2u ? *(volatile u64 *)&S.incl[idx] : *(volatile u64 *)&S.agg[idx]);
            }
            const u32 inc = __ballot_sync(0xFFFFFFFFu, idx >= 0 && st == 2u);
            if (inc) {
                const u32 k = __ffs(inc) - 1;
                excl += warp_sum<TO>(lane <= k ? (TO)v : TO(0));
                break;
            }
            excl += warp_sum<TO>((TO)v);
            j -= 32;
        }
        if (__any_sync(0xFFFFFFFFu, gave_up) && lane == 0) atomicExch(status, (u32)DEV_SPIN_LIMIT);
        if (lane == 0) {
            S.incl[t] = (u64)(excl + tile_total);
            __threadfence();
            atomicExch(&S.flag[t], (epoch << 2) | 2u);
            *s_prefix = excl;
        }
    }
    __syncthreads();
    return t > 0 ? *s_prefix : TO(0);
}

// Scan: out[i] = sum of in[0..i) (exclusive) or in[0..i] (inclusive), in one pass.
// With skip_n set, a launch whose *skip_n is at most skip_le does nothing: every block returns
// before it takes a tile ticket, so the tile state is left as the previous launch left it.
template <class TI, class TO, bool INCL>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_lb(const TI *__restrict__ in, TO *__restrict__ out, u64 n,
                                                        ScanState S, u32 *status, const u32 *__restrict__ skip_n,
                                                        u32 skip_le) {
    __shared__ TO wt[33];
    __shared__ TO stage[SCAN_TILE + SCAN_TILE / 32];
    __shared__ u32 s_tile, s_epoch;
    __shared__ TO s_prefix;
    if (skip_n && *skip_n <= skip_le) return;
    u32 epoch;
    const u32 t = lb_enter(S, s_tile, s_epoch, epoch);
    const u64 base = (u64)t * SCAN_TILE;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = j * SCAN_THREADS + threadIdx.x;
        u64 i = base + li;
        stage[li + li / 32] = i < n ? (TO)in[i] : TO(0);
    }
    __syncthreads();
    TO loc[SCAN_ITEMS];
    TO s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = threadIdx.x * SCAN_ITEMS + j;
        loc[j] = stage[li + li / 32];
        s += loc[j];
    }
    TO tot;
    TO pre = block_excl_scan<TO>(s, wt, tot);
    pre += lookback_prefix<TO>(S, epoch, t, tot, status, &s_prefix);
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = threadIdx.x * SCAN_ITEMS + j;
        stage[li + li / 32] = INCL ? pre + loc[j] : pre;
        pre += loc[j];
    }
    __syncthreads();
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int li = j * SCAN_THREADS + threadIdx.x;
        u64 i = base + li;
        if (i < n) out[i] = stage[li + li / 32];
    }
    lb_leave(S, epoch);
}

// Stable compaction: out[k] = the k-th index i < n with flags[i] != 0; *total = their count.
__global__ void __launch_bounds__(SCAN_THREADS) k_compact_lb(const u32 *__restrict__ flags, u32 *__restrict__ out,
                                                           u64 n, u32 *__restrict__ total, ScanState S,
                                                           u32 *status) {
    __shared__ u32 wt[33];
    __shared__ u32 s_tile, s_epoch;
    __shared__ u32 s_prefix;
    u32 epoch;
    const u32 t = lb_enter(S, s_tile, s_epoch, epoch);
    // thread-contiguous items: thread k owns elements [base + k*ITEMS, base + (k+1)*ITEMS)
    const u64 base = (u64)t * SCAN_TILE + (u64)threadIdx.x * SCAN_ITEMS;
    u32 f[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        u64 i = base + j;
        f[j] = (i < n && flags[i]) ? 1u : 0u;
        s += f[j];
    }
    u32 tot;
    u32 pre = block_excl_scan<u32>(s, wt, tot);
    pre += lookback_prefix<u32>(S, epoch, t, tot, status, &s_prefix);
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        if (f[j]) out[pre] = (u32)(base + j);
        pre += f[j];
    }
    if (base < n && base + SCAN_ITEMS >= n) *total = pre;  // the thread holding element n-1
    lb_leave(S, epoch);
}

template <class TI, class TO, bool INCL = false>
void scan_impl(Ctx &c, const TI *in, TO *out, u64 n, const u32 *skip_n = nullptr, u32 skip_le = 0) {
    if (n == 0) return;
    const u32 tiles = cdiv(n, SCAN_TILE);
    if (tiles <= c.scan.cap_tiles) {
        LAUNCH(c, (k_scan_lb<TI, TO, INCL>), tiles, SCAN_THREADS, 0, in, out, n, c.scan, c.d_status, skip_n, skip_le);
        return;
    }
    if (INCL) throw Error(AXC_EOVERFLOW, "inclusive scan longer than the look-back tile state");
    if (tiles == 1) {
        LAUNCH(c, (k_tile_scan<TI, TO>), 1, SCAN_THREADS, 0, in, out, (const TO *)nullptr, n);
        return;
    }
    size_t m = c.arena.mark();
    TO *part = c.arena.alloc<TO>(tiles);
    LAUNCH(c, (k_tile_reduce<TI, TO>), tiles, SCAN_THREADS, 0, in, part, n);
    scan_impl<TO, TO>(c, part, part, tiles);
    LAUNCH(c, (k_tile_scan<TI, TO>), tiles, SCAN_THREADS, 0, in, out, (const TO *)part, n);
    c.arena.release(m);
}

// The bounded wait of the look-back, made to run out: the block plays tile 1 of epoch 1 in a
// private tile state whose tile 0 never publishes, so its warp polls that flag `spin_limit` times,
// gives up, sets the status word and returns.
__global__ void k_lookback_selftest(ScanState S, u32 *status, u32 spin_limit, u64 *out) {
    __shared__ u64 s_prefix;
    const u64 p = lookback_prefix<u64>(S, 1u, 1u, 5ull, status, &s_prefix, spin_limit);
    if (threadIdx.x == 0) *out = p;
}

__global__ void k_offsets_tail(const u32 *counts, u64 *out, u64 n) {
    out[n] = (n ? out[n - 1] + counts[n - 1] : 0);
}

// ------------------------------------------------------------------ radix sort
constexpr int RS_WARPS = 8;
constexpr int RS_ITEMS = 8;  // rounds of 32 per warp
constexpr int RS_TILE = RS_WARPS * 32 * RS_ITEMS;

// k_rs_hist / k_rs_scatter: with d_n set, a count of at most skip_le means the one-block sort
// has already sorted the data, and the launch does nothing.
__global__ void k_rs_hist(const u32 *__restrict__ keys, u64 n, u32 shift, u32 *__restrict__ hist,
                          u32 tiles, const u32 *__restrict__ d_n, u32 skip_le) {
    if (d_n && *d_n <= skip_le) return;
    __shared__ u32 cnt[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    if (d_n) n = *d_n;  // element count resident on the device (tiles past it count nothing)
    const u64 base = (u64)blockIdx.x * RS_TILE;
    for (int j = threadIdx.x; j < RS_TILE; j += blockDim.x) {
        u64 i = base + j;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(u64)d * tiles + blockIdx.x] = cnt[d];
}

__global__ void k_rs_scatter(const u32 *__restrict__ kin, const u32 *__restrict__ vin, u32 *__restrict__ kout,
                             u32 *__restrict__ vout, u64 n, u32 shift, const u32 *__restrict__ offs,
                             u32 tiles, const u32 *__restrict__ d_n, u32 skip_le) {
    if (d_n && *d_n <= skip_le) return;
    __shared__ u32 wcnt[RS_WARPS][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (d_n) n = *d_n;
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += blockDim.x) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const u64 base = (u64)blockIdx.x * RS_TILE + (u64)w * 32 * RS_ITEMS;
    u32 dig[RS_ITEMS], loc[RS_ITEMS], key[RS_ITEMS], val[RS_ITEMS];
    const u32 lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        u64 i = base + (u64)r * 32 + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : 0u;
        val[r] = ok ? vin[i] : 0u;
        u32 d = ok ? ((key[r] >> shift) & 255u) : 256u;
        dig[r] = d;
        u32 peers = __match_any_sync(0xFFFFFFFFu, d);
        u32 before = ok ? wcnt[w][d] : 0u;
        loc[r] = before + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) wcnt[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        u32 run = offs[(u64)d * tiles + blockIdx.x];
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            u32 t = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        if (dig[r] < 256u) {
            u32 pos = wcnt[w][dig[r]] + loc[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

__global__ void k_fill_u32(u32 *p, u32 v, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void k_iota_u32(u32 *p, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = (u32)i;
}
__global__ void k_gather_u32(const u32 *src, const u32 *idx, u32 *dst, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}
__global__ void k_reduce_sum(const u32 *p, u64 n, unsigned long long *out) {
    u64 s = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) s += p[i];
    s = warp_sum<u64>(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)s);
}
__global__ void k_reduce_max(const u32 *p, u64 n, u32 *out) {
    u32 m = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        m = max(m, p[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}
__global__ void k_reduce_sum64(const u64 *p, u64 n, unsigned long long *out) {
    u64 s = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) s += p[i];
    s = warp_sum<u64>(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)s);
}
__global__ void k_reduce_max64(const u64 *p, u64 n, unsigned long long *out) {
    u64 m = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        m = p[i] > m ? p[i] : m;
    m = warp_max_u64(m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)m);
}
__global__ void k_flag_to_u32(const u32 *flags, u32 *f01, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        f01[i] = flags[i] ? 1u : 0u;
}
__global__ void k_compact_write(const u32 *flags, const u32 *pos, u32 *out, u64 n, u32 *total) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        if (flags[i]) out[pos[i]] = (u32)i;
        if (i == n - 1) *total = pos[i] + (flags[i] ? 1u : 0u);
    }
}

// ------------------------------------------------------------------ small radix sort
// Arrays of at most RSS_CAP elements sort in one block (blocksort.cuh): every 8-bit pass in
// shared memory, one launch for the whole sort.
__global__ void __launch_bounds__(RSS_WARPS * 32) k_rs_small(u32 *__restrict__ keys, u32 *__restrict__ vals, u32 n_cap,
                                                             const u32 *__restrict__ d_n, u32 bits) {
    extern __shared__ u32 sm[];
    if (d_n && *d_n > n_cap) return;  // more than one block holds: the multi-pass sort takes it
    const u32 n = d_n ? *d_n : n_cap;
    for (u32 i = threadIdx.x; i < n; i += blockDim.x) { sm[i] = keys[i]; sm[RSS_CAP + i] = vals[i]; }
    const u32 *ko, *vo;
    block_radix_sort(sm, n, bits, ko, vo);
    for (u32 i = threadIdx.x; i < n; i += blockDim.x) { keys[i] = ko[i]; vals[i] = vo[i]; }
}

inline u32 grid_for(Ctx &c, u64 n, u32 threads = 256) {
    u64 b = (n + threads - 1) / threads;
    u64 cap = (u64)c.sms * 8;
    return (u32)(b < cap ? (b ? b : 1) : cap);
}

}  // namespace

void scan_excl_u32(Ctx &c, const u32 *in, u32 *out, u64 n) { scan_impl<u32, u32>(c, in, out, n); }
void scan_excl_u64(Ctx &c, const u64 *in, u64 *out, u64 n) { scan_impl<u64, u64>(c, in, out, n); }
void scan_excl_i64(Ctx &c, const i64 *in, i64 *out, u64 n) { scan_impl<i64, i64>(c, in, out, n); }
void scan_incl_i64(Ctx &c, const i64 *in, i64 *out, u64 n) { scan_impl<i64, i64, true>(c, in, out, n); }

void lookback_selftest(Ctx &c, u32 spin_limit) {
    const size_t m = c.arena.mark();
    ScanState S;
    S.flag = c.arena.alloc<u32>(2);
    S.agg = c.arena.alloc<u64>(2);
    S.incl = c.arena.alloc<u64>(2);
    S.ctrl = c.arena.alloc<u32>(4);
    S.cap_tiles = 2;
    u64 *out = c.arena.alloc<u64>(1);
    AXC_CUDA(cudaMemsetAsync(S.flag, 0, 8, c.stream));
    AXC_CUDA(cudaMemsetAsync(S.ctrl, 0, 16, c.stream));
    LAUNCH(c, k_lookback_selftest, 1, 32, 0, S, c.d_status, spin_limit, out);
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    c.arena.release(m);
    check_status(c);  // throws AXC_EINTERNAL with the status word (DEV_SPIN_LIMIT) when the wait gave up
}

void setup_prim_kernels() {
    AXC_CUDA(cudaFuncSetAttribute(k_rs_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RSS_SMEM));
}

void scan_state_create(Ctx &c, u32 cap_tiles) {
    ScanState &S = c.scan;
    AXC_CUDA(cudaMalloc(&S.flag, (size_t)cap_tiles * 4));
    AXC_CUDA(cudaMalloc(&S.agg, (size_t)cap_tiles * 8));
    AXC_CUDA(cudaMalloc(&S.incl, (size_t)cap_tiles * 8));
    AXC_CUDA(cudaMalloc(&S.ctrl, 16));
    AXC_CUDA(cudaMemset(S.flag, 0, (size_t)cap_tiles * 4));
    const u32 ctrl0[4] = {0, 0, 1, 0};  // epoch 1: no flag carries it yet
    AXC_CUDA(cudaMemcpy(S.ctrl, ctrl0, 16, cudaMemcpyHostToDevice));
    S.cap_tiles = cap_tiles;
}
void scan_state_destroy(Ctx &c) {
    ScanState &S = c.scan;
    if (S.flag) cudaFree(S.flag);
    if (S.agg) cudaFree(S.agg);
    if (S.incl) cudaFree(S.incl);
    if (S.ctrl) cudaFree(S.ctrl);
    S = ScanState();
}

void offsets_from_counts(Ctx &c, const u32 *counts, u64 *out, u64 n) {
    if (n) scan_impl<u32, u64>(c, counts, out, n);
    LAUNCH(c, k_offsets_tail, 1, 1, 0, counts, out, n);
}

void fill_u32(Ctx &c, u32 *p, u32 v, u64 n) {
    if (n) LAUNCH(c, k_fill_u32, grid_for(c, n), 256, 0, p, v, n);
}
void iota_u32(Ctx &c, u32 *p, u64 n) {
    if (n) LAUNCH(c, k_iota_u32, grid_for(c, n), 256, 0, p, n);
}

u64 reduce_sum_u32(Ctx &c, const u32 *p, u64 n) {
    size_t m = c.arena.mark();
    unsigned long long *d = c.arena.alloc<unsigned long long>(1);
    AXC_CUDA(cudaMemsetAsync(d, 0, 8, c.stream));
    if (n) LAUNCH(c, k_reduce_sum, grid_for(c, n), 256, 0, p, n, d);
    u64 r = fetch1(c, (const u64 *)d);
    c.arena.release(m);
    return r;
}
u32 reduce_max_u32(Ctx &c, const u32 *p, u64 n) {
    size_t m = c.arena.mark();
    u32 *d = c.arena.alloc<u32>(1);
    AXC_CUDA(cudaMemsetAsync(d, 0, 4, c.stream));
    if (n) LAUNCH(c, k_reduce_max, grid_for(c, n), 256, 0, p, n, d);
    u32 r = fetch1(c, d);
    c.arena.release(m);
    return r;
}

u64 reduce_sum_u64(Ctx &c, const u64 *p, u64 n) {
    size_t m = c.arena.mark();
    unsigned long long *d = c.arena.alloc<unsigned long long>(1);
    AXC_CUDA(cudaMemsetAsync(d, 0, 8, c.stream));
    if (n) LAUNCH(c, k_reduce_sum64, grid_for(c, n), 256, 0, p, n, d);
    u64 r = fetch1(c, (const u64 *)d);
    c.arena.release(m);
    return r;
}
u64 reduce_max_u64(Ctx &c, const u64 *p, u64 n) {
    size_t m = c.arena.mark();
    unsigned long long *d = c.arena.alloc<unsigned long long>(1);
    AXC_CUDA(cudaMemsetAsync(d, 0, 8, c.stream));
    if (n) LAUNCH(c, k_reduce_max64, grid_for(c, n), 256, 0, p, n, d);
    u64 r = fetch1(c, (const u64 *)d);
    c.arena.release(m);
    return r;
}

void compact_indices_dn(Ctx &c, const u32 *flags, u32 *out, u64 n, u32 *d_count) {
    if (n == 0) {
        AXC_CUDA(cudaMemsetAsync(d_count, 0, 4, c.stream));
        return;
    }
    const u32 tiles = cdiv(n, SCAN_TILE);
    if (tiles <= c.scan.cap_tiles) {
        LAUNCH(c, k_compact_lb, tiles, SCAN_THREADS, 0, flags, out, n, d_count, c.scan, c.d_status);
        return;
    }
    size_t m = c.arena.mark();
    u32 *f01 = c.arena.alloc<u32>(n);
    u32 *pos = c.arena.alloc<u32>(n);
    LAUNCH(c, k_flag_to_u32, grid_for(c, n), 256, 0, flags, f01, n);
    scan_excl_u32(c, f01, pos, n);
    LAUNCH(c, k_compact_write, grid_for(c, n), 256, 0, flags, pos, out, n, d_count);
    c.arena.release(m);
}

u32 compact_indices(Ctx &c, const u32 *flags, u32 *out, u64 n) {
    if (n == 0) return 0;
    size_t m = c.arena.mark();
    u32 *tot = c.arena.alloc<u32>(1);
    compact_indices_dn(c, flags, out, n, tot);
    u32 r = fetch1(c, tot);
    c.arena.release(m);
    return r;
}

void radix_sort_pairs(Ctx &c, u32 *keys, u32 *vals, u64 n, u32 bits) {
    radix_sort_pairs_dn(c, keys, vals, nullptr, n, bits);
}

// Same, with the element count read from device memory (d_n, at most n); no host round trip.
void radix_sort_pairs_dn(Ctx &c, u32 *keys, u32 *vals, const u32 *d_n, u64 n, u32 bits) {
    if ((!d_n && n <= 1) || n == 0 || bits == 0) return;
    if (n <= (u64)RSS_CAP) {  // one block, every pass in shared memory
        LAUNCH(c, k_rs_small, 1, RSS_WARPS * 32, RSS_SMEM, keys, vals, (u32)n, d_n, bits);
        return;
    }
    // Capacity above one block. With the count on the device both forms are launched: the
    // one-block sort acts when the count fits it, the passes below when it does not (each kernel
    // reads the count and returns at once otherwise), and an even number of passes leaves the
    // data in place either way.
    u32 skip_le = 0;
    u32 passes = (bits + 7) / 8;
    if (d_n) {
        LAUNCH(c, k_rs_small, 1, RSS_WARPS * 32, RSS_SMEM, keys, vals, (u32)RSS_CAP, d_n, bits);
        skip_le = RSS_CAP;
        passes += passes & 1u;
    }
    size_t m = c.arena.mark();
    const u32 tiles = cdiv(n, RS_TILE);
    u32 *k2 = c.arena.alloc<u32>(n), *v2 = c.arena.alloc<u32>(n);
    u32 *hist = c.arena.alloc<u32>((u64)tiles * 256);
    u32 *ka = keys, *va = vals, *kb = k2, *vb = v2;
    for (u32 pass = 0, shift = 0; pass < passes; ++pass, shift += 8) {
        LAUNCH(c, k_rs_hist, tiles, 256, 0, ka, n, shift, hist, tiles, d_n, skip_le);
        scan_impl<u32, u32>(c, hist, hist, (u64)tiles * 256, d_n, skip_le);
        LAUNCH(c, k_rs_scatter, tiles, RS_WARPS * 32, 0, ka, va, kb, vb, n, shift, hist, tiles, d_n, skip_le);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        AXC_CUDA(cudaMemcpyAsync(keys, ka, n * 4, cudaMemcpyDeviceToDevice, c.stream));
        AXC_CUDA(cudaMemcpyAsync(vals, va, n * 4, cudaMemcpyDeviceToDevice, c.stream));
    }
    c.arena.release(m);
}

void radix_sort_pairs64(Ctx &c, u32 *key_hi, u32 *key_lo, u32 *vals, u64 n, u32 bits_hi, u32 bits_lo) {
    if (n <= 1) return;
    size_t m = c.arena.mark();
    u32 *idx = c.arena.alloc<u32>(n), *tmp = c.arena.alloc<u32>(n);
    iota_u32(c, idx, n);
    radix_sort_pairs(c, key_lo, idx, n, bits_lo);           // idx: order by lo
    LAUNCH(c, k_gather_u32, grid_for(c, n), 256, 0, key_hi, idx, tmp, n);  // hi in that order
    radix_sort_pairs(c, tmp, idx, n, bits_hi);              // stable by hi
    LAUNCH(c, k_gather_u32, grid_for(c, n), 256, 0, vals, idx, key_lo, n);  // reuse key_lo as scratch
    AXC_CUDA(cudaMemcpyAsync(vals, key_lo, n * 4, cudaMemcpyDeviceToDevice, c.stream));
    AXC_CUDA(cudaMemcpyAsync(key_hi, tmp, n * 4, cudaMemcpyDeviceToDevice, c.stream));
    c.arena.release(m);
}

}  // namespace axc
