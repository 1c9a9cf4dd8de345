"""axc_connectivity_noalloc (connectivity, cut-net and SOED with its scratch in a fixed device
array, no allocation) against axc_evaluate on the same inputs, on two calls in a row so that the
second call sees the scratch the first one left behind. Named to run after every other test file;
it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

AXC_EINVAL, AXC_EOVERFLOW = 1, 11


def device(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def noalloc(torch, g, part, stream=None):
    """One call through the C ABI with the hypergraph and partition in device memory."""
    off = device(g.off.view(np.int64), torch)
    pins = device(g.pins.view(np.int32), torch)
    w = device(g.w, torch)
    dp = device(part.astype(np.uint32).view(np.int32), torch)
    out = (C.c_int64 * 3)()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    rc = ax.lib().axc_connectivity_noalloc(g.e, off.data_ptr(), pins.data_ptr(), w.data_ptr(), dp.data_ptr(),
                                           C.c_void_p(s), out)
    return rc, tuple(out)


def expected(ctx, g, part):
    k = int(part.max()) + 1 if len(part) else 1
    st = ctx.evaluate(g, ax.params_incc(g.n, 0x7FFFFFFF, max(k, 1)), part)
    return (st.connectivity_fx, st.cutnet_fx, st.soed_fx)


def long_edges(lengths, n, seed):
    """Hyperedges of the given lengths over n nodes (distinct pins, one source each), weights in
    (0, 4]."""
    rng = np.random.default_rng(seed)
    pins = [rng.choice(n, size=L, replace=False).astype(np.uint32) for L in lengths]
    off = np.zeros(len(lengths) + 1, np.uint64)
    off[1:] = np.cumsum(lengths)
    w = rng.uniform(0.01, 4.0, len(lengths)).astype(np.float32)
    return ax.Hypergraph(n, off, np.concatenate(pins), np.ones(len(lengths), np.uint32), w)


def cases():
    yield "circ_2k", ax.read(f"{GOLDEN}/circ_2k.hgr"), 7
    yield "snn_lognormal", ax.gen_snn(6, 3000, 200, 0.8, 2048, 0.7, 11), 40
    # shared-memory tier (33..2048 pins), global-scratch tier (2049..16384) and the longest accepted
    yield "long", long_edges([1, 2, 31, 32, 33, 500, 2048, 2049, 5000, 16384, 3, 16383], 40000, 3), 300


@pytest.mark.parametrize("name,g,k", list(cases()), ids=lambda x: x if isinstance(x, str) else "")
def test_noalloc_matches_evaluate_twice(ctx, name, g, k):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(17)
    part = rng.integers(0, k, g.n).astype(np.uint32)
    want = expected(ctx, g, part)
    first = noalloc(torch, g, part)
    second = noalloc(torch, g, part)
    assert first == (0, want)
    assert second == (0, want)


def with_empty_hyperedges():
    """Hyperedges of 0, 1 and 2+ pins mixed, weights not all 1: an empty hyperedge holds no
    partition and adds nothing to any of the three sums."""
    lens = [3, 0, 1, 4, 0, 2, 5]
    rng = np.random.default_rng(9)
    pins = np.concatenate([rng.choice(12, size=L, replace=False).astype(np.uint32) for L in lens])
    off = np.zeros(len(lens) + 1, np.uint64)
    off[1:] = np.cumsum(lens)
    w = np.array([1.0, 2.0, 0.5, 3.25, 1.0, 0.75, 1.5], np.float32)
    return ax.Hypergraph(12, off, pins, np.array([1, 0, 1, 2, 0, 1, 0], np.uint32), w)


SMALL = [("tiny_w", lambda: ax.read(f"{GOLDEN}/tiny_w.hgr"), 3), ("tiny_vw", lambda: ax.read(f"{GOLDEN}/tiny_vw.hgr"), 2),
         ("tiny_dups", lambda: ax.read(f"{GOLDEN}/tiny_dups.hgr"), 3), ("empty_hyperedges", with_empty_hyperedges, 4)]


@pytest.mark.parametrize("name,make,k", SMALL, ids=[c[0] for c in SMALL])
def test_noalloc_small_and_weighted_cases(ctx, name, make, k):
    """Weighted nets, duplicate pins and empty hyperedges: equal to axc_evaluate and to the
    oracle's evaluation, on two calls in a row."""
    from oracle import oracle as O
    torch = pytest.importorskip("torch")
    g = make()
    part = (np.arange(g.n) % k).astype(np.uint32)
    want = expected(ctx, g, part)
    ev = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, part, g.n, 0x7FFFFFFF, k)
    assert want == (ev["connectivity_fx"], ev["cutnet_fx"], ev["soed_fx"])
    assert noalloc(torch, g, part) == (0, want)
    assert noalloc(torch, g, part) == (0, want)


def test_noalloc_refuses_long_hyperedge_then_recovers(ctx):
    torch = pytest.importorskip("torch")
    g = long_edges([40, 16385, 7], 20000, 5)
    part = np.random.default_rng(1).integers(0, 5, g.n).astype(np.uint32)
    rc, _ = noalloc(torch, g, part)
    assert rc == AXC_EOVERFLOW
    ok = long_edges([40, 16384, 7], 20000, 5)
    assert noalloc(torch, ok, part) == (0, expected(ctx, ok, part))


def test_noalloc_rejects_reserved_partition_id(ctx):
    torch = pytest.importorskip("torch")
    g = ax.read(f"{GOLDEN}/circ_2k.hgr")
    part = np.zeros(g.n, np.uint32)
    part[3] = 0xFFFFFFFF
    rc, _ = noalloc(torch, g, part)
    assert rc == AXC_EINVAL
    part[3] = 1
    assert noalloc(torch, g, part) == (0, expected(ctx, g, part))


def test_noalloc_leaves_device_memory_alone(ctx):
    torch = pytest.importorskip("torch")
    g = ax.gen_snn(6, 3000, 200, 0.8, 2048, 0.7, 12)
    part = np.random.default_rng(2).integers(0, 50, g.n).astype(np.uint32)
    off = device(g.off.view(np.int64), torch)
    pins = device(g.pins.view(np.int32), torch)
    w = device(g.w, torch)
    dp = device(part.view(np.int32), torch)
    out = (C.c_int64 * 3)()

    def call():
        return ax.lib().axc_connectivity_noalloc(g.e, off.data_ptr(), pins.data_ptr(), w.data_ptr(),
                                                 dp.data_ptr(), None, out)

    torch.cuda.synchronize()
    assert call() == 0  # the first call in this context loads the kernels
    free0, _ = torch.cuda.mem_get_info()
    assert call() == 0
    assert call() == 0
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert tuple(out) == expected(ctx, g, part)
