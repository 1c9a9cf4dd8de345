// The quotient hypergraph of a partition (getPartitionsHypergraph(part, 2, squish=true),
// includes/hgraph.hpp:286-376), device part: for every hyperedge its distinct source partitions
// and its distinct destination partitions that are not also source partitions, each ascending.
//
// Every pin becomes a key (hyperedge, side, partition), side 0 for sources and 1 for
// destinations; one stable 64-bit radix sort orders them, so each hyperedge keeps its own pin
// range with its sources' partitions first. A warp per hyperedge then keeps the first entry of
// each run, drops destination partitions found among the sources (binary search in the sorted
// source run) and drops the hyperedge when it keeps at most one source partition and no
// destination one. The kept entries and per-hyperedge counts go back to the host, which merges
// identical (sources, destinations) pairs (quotient_merge in host_io.cpp).
#include "common.cuh"
#include "kernels.h"

namespace axc {
namespace {

__global__ void k_q_keys(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ pins,
                         const u32 *__restrict__ nsrc, const u32 *__restrict__ part, u32 pb, u32 *__restrict__ hi,
                         u32 *__restrict__ lo) {
    const u32 h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (h >= e) return;
    const u64 a = off[h], b = off[h + 1], s = a + nsrc[h];
    for (u64 k = a + lane; k < b; k += 32) {
        hi[k] = h;
        lo[k] = (k >= s ? 1u << pb : 0u) | part[pins[k]];
    }
}

// keep[k] for the sorted entries of hyperedge h; qcnt[h] (kept entries, 0 when the hyperedge
// vanishes) and qsrc[h] (kept source partitions).
__global__ void k_q_flags(u32 e, const u64 *__restrict__ off, const u32 *__restrict__ nsrc,
                          const u32 *__restrict__ lo, u32 pmask, u32 *__restrict__ keep, u32 *__restrict__ qcnt,
                          u32 *__restrict__ qsrc) {
    const u32 h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (h >= e) return;
    const u64 a = off[h], b = off[h + 1], s = a + nsrc[h];
    u32 ns = 0, nd = 0;
    for (u64 base = a; base < b; base += 32) {
        const u64 k = base + lane;
        bool kp = false, src = false;
        if (k < b) {
            const u32 x = lo[k];
            src = k < s;
            kp = k == a || lo[k - 1] != x;
            if (kp && !src) {  // a destination partition that is also a source one is not kept
                const u32 p = x & pmask;
                u64 l = a, r = s;  // sources hold (0, partition), ascending
                while (l < r) {
                    const u64 mid = (l + r) >> 1;
                    if (lo[mid] < p) l = mid + 1; else r = mid;
                }
                if (l < s && lo[l] == p) kp = false;
            }
            keep[k] = kp ? 1u : 0u;
        }
        ns += __popc(__ballot_sync(0xFFFFFFFFu, kp && src));
        nd += __popc(__ballot_sync(0xFFFFFFFFu, kp && !src));
    }
    const bool kept = ns > 1 || nd > 0;
    if (!kept)
        for (u64 k = a + lane; k < b; k += 32) keep[k] = 0;
    if (lane == 0) {
        qcnt[h] = kept ? ns + nd : 0;
        qsrc[h] = ns;
    }
}

__global__ void k_q_gather(const u32 *__restrict__ idx, u64 m, const u32 *__restrict__ lo, u32 pmask,
                           u32 *__restrict__ out) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = lo[idx[i]] & pmask;
}

}  // namespace

// g: the hypergraph already on the device (off, pins, nsrc; P pins); part: device, partition ids
// below K <= 2^31. Fills qcnt / qsrc (host, e entries) and qpins (host: the kept entries in
// hyperedge order, sources then destinations, each ascending).
void quotient_extract(Ctx &c, u32 e, u64 P, const u64 *off, const u32 *pins, const u32 *nsrc, const u32 *part, u32 K,
                      std::vector<u32> &qcnt, std::vector<u32> &qsrc, std::vector<u32> &qpins) {
    qcnt.assign(e, 0);
    qsrc.assign(e, 0);
    qpins.clear();
    if (e == 0 || P == 0) return;
    if (P > 0xFFFFFFFFull) throw Error(AXC_EOVERFLOW, "quotient: more than 2^32 pins");
    if (K > 0x80000000u) throw Error(AXC_EOVERFLOW, "quotient: partition ids above 2^31");
    const size_t m = c.arena.mark();
    const u32 pb = bits_for(K ? K - 1 : 0), pmask = (u32)((1ull << pb) - 1);  // side bit above the id
    u32 *hi = c.arena.alloc<u32>(P), *lo = c.arena.alloc<u32>(P), *key = c.arena.alloc<u32>(P);
    LAUNCH(c, k_q_keys, cdiv((u64)e * 32, 256), 256, 0, e, off, pins, nsrc, part, pb, hi, lo);
    // the sort carries a copy of the (side, partition) keys as its values: on return `key` holds
    // them in (hyperedge, side, partition) order, and hi / lo are free
    AXC_CUDA(cudaMemcpyAsync(key, lo, (size_t)P * 4, cudaMemcpyDeviceToDevice, c.stream));
    radix_sort_pairs64(c, hi, lo, key, P, bits_for(e - 1), pb + 1);
    u32 *keep = hi, *idx = lo;
    u32 *dcnt = c.arena.alloc<u32>(e), *dsrc = c.arena.alloc<u32>(e);
    LAUNCH(c, k_q_flags, cdiv((u64)e * 32, 256), 256, 0, e, off, nsrc, key, pmask, keep, dcnt, dsrc);
    const u32 nq = compact_indices(c, keep, idx, P);
    u32 *qp = c.arena.alloc<u32>(nq ? nq : 1);
    if (nq) LAUNCH(c, k_q_gather, cdiv(nq, 256), 256, 0, idx, (u64)nq, key, pmask, qp);
    qpins.resize(nq);
    AXC_CUDA(cudaMemcpyAsync(qcnt.data(), dcnt, (size_t)e * 4, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaMemcpyAsync(qsrc.data(), dsrc, (size_t)e * 4, cudaMemcpyDeviceToHost, c.stream));
    if (nq) AXC_CUDA(cudaMemcpyAsync(qpins.data(), qp, (size_t)nq * 4, cudaMemcpyDeviceToHost, c.stream));
    AXC_CUDA(cudaStreamSynchronize(c.stream));
    check_status(c);
    c.arena.release(m);
}

}  // namespace axc
