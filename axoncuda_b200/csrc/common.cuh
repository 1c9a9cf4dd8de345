// Shared internals of the B200 partitioner: context, device arena, launch bookkeeping and the
// warp/hash helpers every kernel file uses.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/axc.h"

namespace axc {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
constexpr u32 NONE = 0xFFFFFFFFu;
constexpr u32 WARP = 32;

// Device-side failure codes written to the context's status word (never trap).
enum DevStatus : u32 {
    DEV_OK = 0,
    DEV_HASH_FULL = 1,      // a bounded hash table could not take a key
    DEV_BAD_INDEX = 2,      // an index check failed
    DEV_SPIN_LIMIT = 3,     // a bounded wait gave up (a predecessor tile never published)
};

// Tile states of the single-pass scans: per tile a flag (epoch << 2 | 1 aggregate, 2 inclusive)
// and two values, kept for the context's lifetime so no scan has to clear them. ctrl[0] hands
// out tiles in launch order, ctrl[1] counts finished tiles and ctrl[2] is the launch's epoch: the
// last tile to finish resets the first two and advances the epoch, all on the device.
struct ScanState {
    u32 *flag = nullptr;
    u64 *agg = nullptr, *incl = nullptr;
    u32 *ctrl = nullptr;
    u32 cap_tiles = 0;
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define AXC_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            throw ::axc::Error(AXC_ECUDA, std::string(#call " failed: ") + cudaGetErrorString(_e) + \
                                              " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

// Bump allocator over one device allocation made when the context is created. Levels of the
// multilevel hierarchy are strictly nested, so allocation is LIFO: `mark()` / `release()`.
// Device byte counters of the kernel timer: PROF_SLOTS words, one per 128-byte line (PROF_STRIDE
// words apart) from byte STATUS_PROF_OFF of the status allocation, so that warps adding their
// bytes spread over as many L2 lines.
constexpr unsigned PROF_SLOTS = 32, PROF_STRIDE = 16, STATUS_PROF_OFF = 256;
constexpr size_t STATUS_BYTES = STATUS_PROF_OFF + (size_t)PROF_SLOTS * PROF_STRIDE * 8;
__device__ __forceinline__ void prof_add(unsigned long long *base, unsigned slot, unsigned long long v) {
    atomicAdd(&base[(slot & (PROF_SLOTS - 1)) * PROF_STRIDE], v);
}

struct Arena {
    char *base = nullptr;
    size_t cap = 0, top = 0, peak = 0;
    template <class T>
    T *alloc(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
        if (bytes == 0) bytes = 256;
        if (top + bytes > cap)
            throw Error(AXC_ENOMEM, "device arena exhausted: need " + std::to_string(top + bytes) +
                                        " of " + std::to_string(cap) + " bytes");
        T *p = reinterpret_cast<T *>(base + top);
        top += bytes;
        if (top > peak) peak = top;
        return p;
    }
    size_t mark() const { return top; }
    void release(size_t m) { top = m; }
};

// Tile and table sizes that change speed but never results (axc_tune_set): the block rating's
// first-try and second-try tables (slots, powers of two) and the movers the cascade's
// shared-memory block kernel keeps (0: its default, or AXC_CASCADE_BLOCK_MOVERS).
struct Tune {
    u32 rate_try = 2048;
    u32 rate_mid = 8192;
    u32 cascade_movers = 0;
};

struct Ctx {
    int device = 0;
    Tune tune;
    int sms = 148;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    Arena arena;
    u32 *d_status = nullptr;       // device status word
    u64 *h_pinned = nullptr;       // small pinned staging buffer for scalars (4 KiB)
    u32 launches = 0;
    std::string last_error;
    int coop_supported = 0;
    ScanState scan;
    // Kernel timer: while on, every launch of the kernel named `prof_name` is bracketed by a pair
    // of events on the context stream; launch sites with a byte model add the launch's
    // algorithmic bytes to prof_bytes.
    // Pairs recorded inside a CUDA graph capture become event-record nodes; the code that
    // replays the graph adds their durations to prof_ms / prof_launches after each replay.
    bool prof_on = false;
    std::string prof_name;
    std::vector<cudaEvent_t> prof_ev;
    size_t prof_used = 0;
    u64 prof_bytes = 0;
    double prof_ms = 0;
    u32 prof_launches = 0;
    bool capturing = false;
    bool profiling(const char *name) const { return prof_on && prof_name == name; }
    // Device-side byte counters of the kernels whose algorithmic bytes depend on device data (they
    // add them while profiled, through prof_add): summed and cleared by profile reads.
    unsigned long long *d_prof_bytes() const { return (unsigned long long *)((char *)d_status + STATUS_PROF_OFF); }
    cudaEvent_t prof_event() {
        if (prof_used == prof_ev.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            prof_ev.push_back(e);
        }
        return prof_ev[prof_used++];
    }
    void prof_record(cudaEvent_t e) {
        if (capturing) cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal);
        else cudaEventRecord(e, stream);
    }
    // Adds the durations of the recorded pairs [from, to) (their work must have completed).
    void prof_collect(size_t from, size_t to) {
        for (size_t i = from; i + 1 < to; i += 2) {
            float t = 0;
            if (cudaEventElapsedTime(&t, prof_ev[i], prof_ev[i + 1]) == cudaSuccess) {
                prof_ms += t;
                prof_launches++;
            }
        }
    }
};

// Launch bookkeeping: every kernel launch goes through here so stats can report the count and
// the kernel timer can bracket the launches it follows.
#define LAUNCH(ctx, kern, grid, block, smem, ...)                                              \
    do {                                                                                       \
        if ((grid) > 0) {                                                                      \
            const bool _prof = (ctx).profiling(#kern);                                         \
            cudaEvent_t _e0 = _prof ? (ctx).prof_event() : nullptr;                           \
            if (_e0) (ctx).prof_record(_e0);                                                   \
            kern<<<(grid), (block), (smem), (ctx).stream>>>(__VA_ARGS__);                      \
            (ctx).launches++;                                                                  \
            AXC_CUDA(cudaGetLastError());                                                      \
            if (_e0) {                                                                         \
                cudaEvent_t _e1 = (ctx).prof_event();                                          \
                if (_e1) (ctx).prof_record(_e1);                                               \
                else (ctx).prof_used--;                                                        \
            }                                                                                  \
        }                                                                                      \
    } while (0)

// The same with the kernel timer's name given: for template instances of one kernel, which the
// timer knows by the template's name.
#define LAUNCH_AS(ctx, name, kern, grid, block, smem, ...)                                     \
    do {                                                                                       \
        if ((grid) > 0) {                                                                      \
            const bool _prof = (ctx).profiling(name);                                          \
            cudaEvent_t _e0 = _prof ? (ctx).prof_event() : nullptr;                           \
            if (_e0) (ctx).prof_record(_e0);                                                   \
            kern<<<(grid), (block), (smem), (ctx).stream>>>(__VA_ARGS__);                      \
            (ctx).launches++;                                                                  \
            AXC_CUDA(cudaGetLastError());                                                      \
            if (_e0) {                                                                         \
                cudaEvent_t _e1 = (ctx).prof_event();                                          \
                if (_e1) (ctx).prof_record(_e1);                                               \
                else (ctx).prof_used--;                                                        \
            }                                                                                  \
        }                                                                                      \
    } while (0)

inline u32 cdiv(u64 a, u64 b) { return (u32)((a + b - 1) / b); }

// Read `count` u64 scalars back from device memory (one small synchronous round trip).
inline void fetch(Ctx &c, u64 *dst, const void *dsrc, size_t bytes) {
    AXC_CUDA(cudaMemcpyAsync(c.h_pinned, dsrc, bytes, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    memcpy(dst, c.h_pinned, bytes);
}
template <class T>
inline T fetch1(Ctx &c, const T *dsrc) {
    T v;
    AXC_CUDA(cudaMemcpyAsync(c.h_pinned, dsrc, sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    memcpy(&v, c.h_pinned, sizeof(T));
    return v;
}
inline void check_status(Ctx &c) {
    u32 s = fetch1(c, c.d_status);
    if (s != DEV_OK) {
        AXC_CUDA(cudaMemsetAsync(c.d_status, 0, 4, c.stream));
        throw Error(AXC_EINTERNAL, "device status word = " + std::to_string(s));
    }
}

// ---------------------------------------------------------------- device helpers
#ifdef __CUDACC__
__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}
__device__ __forceinline__ u64 warp_max_u64(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Symmetric noise in [0, 63] of an unordered id pair: the same integer mixing sequence as the
// reference's deterministic_noise (headers/utils.cuh:159-171), so ratings agree with it.
__host__ __device__ __forceinline__ u32 pair_noise(u32 a, u32 b) {
    u32 lo = a < b ? a : b, hi = a < b ? b : a;
    u32 x = lo * 0x9E3779B1u;
    x ^= hi + 0x85EBCA6Bu + (x << 6) + (x >> 2);
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 13;
    x *= 0x9E3779B1u;
    x ^= x >> 16;
    return x & 63u;
}

// 32-bit mixer for tie-breaks between refinement targets (headers/utils.cuh:252-261).
__host__ __device__ __forceinline__ u32 mix32(u32 x) {
    x ^= x >> 17;
    x *= 0xED5AD4BBu;
    x ^= x >> 11;
    x *= 0xAC4C1B51u;
    x ^= x >> 15;
    x *= 0x31848BABu;
    x ^= x >> 14;
    return x;
}

__device__ __forceinline__ u32 hslot(u32 key, u32 mask) { return (key * 0x9E3779B1u) & mask; }

// Open-addressing insert-or-find of `key` in keys[0..mask]; returns the slot or NONE when the
// table is full after a full probe cycle. Empty slots hold NONE.
__device__ __forceinline__ u32 hash_find_or_insert(u32 *keys, u32 mask, u32 key) {
    u32 h = hslot(key, mask);
    for (u32 probes = 0; probes <= mask; ++probes) {
        u32 k = keys[h];
        if (k == key) return h;
        if (k == NONE) {
            u32 prev = atomicCAS(&keys[h], NONE, key);
            if (prev == NONE || prev == key) return h;
        }
        h = (h + 1) & mask;
    }
    return NONE;
}
// hash_find_or_insert that also reports whether this call inserted the key (`fresh`).
__device__ __forceinline__ u32 hash_insert_fresh(u32 *keys, u32 mask, u32 key, bool &fresh) {
    fresh = false;
    u32 h = hslot(key, mask);
    for (u32 probes = 0; probes <= mask; ++probes) {
        const u32 k = keys[h];
        if (k == key) return h;
        if (k == NONE) {
            const u32 prev = atomicCAS(&keys[h], NONE, key);
            if (prev == NONE) { fresh = true; return h; }
            if (prev == key) return h;
        }
        h = (h + 1) & mask;
    }
    return NONE;
}
__device__ __forceinline__ u32 hash_find(const u32 *keys, u32 mask, u32 key) {
    u32 h = hslot(key, mask);
    for (u32 probes = 0; probes <= mask; ++probes) {
        u32 k = keys[h];
        if (k == key) return h;
        if (k == NONE) return NONE;
        h = (h + 1) & mask;
    }
    return NONE;
}
#endif

// ---------------------------------------------------------------- primitives (prim.cu)
// Exclusive scan; out may alias in. Returns nothing; total = out[n-1] + in[n-1] when needed.
void scan_excl_u32(Ctx &c, const u32 *in, u32 *out, u64 n);
void scan_excl_u64(Ctx &c, const u64 *in, u64 *out, u64 n);
void scan_excl_i64(Ctx &c, const i64 *in, i64 *out, u64 n);
void scan_incl_i64(Ctx &c, const i64 *in, i64 *out, u64 n);
// one look-back wait on a tile flag that nothing publishes, polled spin_limit times (the
// failure path of the scans' bounded waits); throws AXC_EINTERNAL when it gave up
void lookback_selftest(Ctx &c, u32 spin_limit);
// Tile state of the single-pass scans (made by axc_create, freed by axc_destroy).
void scan_state_create(Ctx &c, u32 cap_tiles);
void scan_state_destroy(Ctx &c);
// Kernel attributes of the primitives (shared memory opt-in); once per device.
void setup_prim_kernels();
// u32 counts -> u64 exclusive offsets with out[n] = total (out has n+1 entries)
void offsets_from_counts(Ctx &c, const u32 *counts, u64 *out, u64 n);
// Stable LSD radix sort of (key, value) pairs by the low `bits` bits of key. In place: on
// return keys/vals hold the sorted data. tmp buffers are taken from the arena.
void radix_sort_pairs(Ctx &c, u32 *keys, u32 *vals, u64 n, u32 bits);
// Same with the element count in device memory (*d_n <= n); buffers hold n entries.
void radix_sort_pairs_dn(Ctx &c, u32 *keys, u32 *vals, const u32 *d_n, u64 n, u32 bits);
// Stable compaction with the count left in device memory (no host round trip).
void compact_indices_dn(Ctx &c, const u32 *flags, u32 *out, u64 n, u32 *d_count);
// Stable sort by a 64-bit key given as (hi, lo) arrays: sorts by lo then by hi.
void radix_sort_pairs64(Ctx &c, u32 *key_hi, u32 *key_lo, u32 *vals, u64 n, u32 bits_hi, u32 bits_lo);
// Fill helpers
void fill_u32(Ctx &c, u32 *p, u32 v, u64 n);
void iota_u32(Ctx &c, u32 *p, u64 n);
// reductions
u64 reduce_sum_u32(Ctx &c, const u32 *p, u64 n);   // synchronous
u32 reduce_max_u32(Ctx &c, const u32 *p, u64 n);   // synchronous
u64 reduce_sum_u64(Ctx &c, const u64 *p, u64 n);   // synchronous
u64 reduce_max_u64(Ctx &c, const u64 *p, u64 n);   // synchronous
// Stable compaction of the indices i in [0,n) with flag[i] != 0 into out; returns the count.
u32 compact_indices(Ctx &c, const u32 *flags, u32 *out, u64 n);

inline u32 bits_for(u64 maxval) {
    u32 b = 0;
    while (b < 64 && (maxval >> b) != 0) ++b;
    return b;
}

}  // namespace axc
