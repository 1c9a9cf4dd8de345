"""GPU parity: every stage of the device pipeline, called through the C ABI, against the oracle.

Integer and index work must be bit-exact; the whole partitioner must return exactly the oracle's
partition (same algorithm, same integer arithmetic, same tie-breaks) and pass the constraint check.
"""
import os

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN, GOLDEN_INPUTS
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NONE = 0xFFFFFFFF


def golden(name):
    return ax.read(os.path.join(GOLDEN, name))


def dedup(g):
    off, pins, ns = O.dedupe(g.off, g.pins, g.nsrc)
    return ax.Hypergraph(g.n, off, pins, ns, g.w.copy())


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_construct_matches_oracle(ctx, name):
    g = golden(name)
    off, pins, ns, toff, touch, nin = ctx.stage_construct(g)
    o_off, o_pins, o_ns = O.dedupe(g.off, g.pins, g.nsrc)
    np.testing.assert_array_equal(off, o_off)
    np.testing.assert_array_equal(pins, o_pins)
    np.testing.assert_array_equal(ns, o_ns)
    t_off, t_touch, t_nin = O.touching(g.n, o_off, o_pins, o_ns)
    np.testing.assert_array_equal(toff, t_off)
    np.testing.assert_array_equal(touch, t_touch)
    np.testing.assert_array_equal(nin, t_nin)


@pytest.mark.parametrize("wl", ["snn-8x512", "circuit-200k-k2"])
def test_construct_full_size(ctx, wl):
    g, _ = ax.workload(wl)
    off, pins, ns, toff, touch, nin = ctx.stage_construct(g)
    o_off, o_pins, o_ns = O.dedupe(g.off, g.pins, g.nsrc)
    np.testing.assert_array_equal(pins, o_pins)
    t_off, t_touch, t_nin = O.touching(g.n, o_off, o_pins, o_ns)
    np.testing.assert_array_equal(toff, t_off)
    np.testing.assert_array_equal(touch, t_touch)
    np.testing.assert_array_equal(nin, t_nin)


def test_construct_with_duplicates_and_big_hyperedges(ctx):
    # hyperedges of 300 and 9000 pins exercise the block and global-table paths
    rng = np.random.default_rng(3)
    sizes = [5, 300, 40, 9000, 2]
    pins, off, ns = [], [0], []
    for s in sizes:
        v = rng.integers(0, 4000, s).astype(np.uint32)
        v[s // 2:] = v[: s - s // 2]  # many duplicates
        pins.append(v); off.append(off[-1] + s); ns.append(min(3, s - 1))
    g = ax.Hypergraph(4000, np.array(off, np.uint64), np.concatenate(pins), np.array(ns, np.uint32),
                      np.ones(len(sizes), np.float32))
    off2, pins2, ns2, *_ = ctx.stage_construct(g)
    o_off, o_pins, o_ns = O.dedupe(g.off, g.pins, g.nsrc)
    np.testing.assert_array_equal(off2, o_off)
    np.testing.assert_array_equal(pins2, o_pins)
    np.testing.assert_array_equal(ns2, o_ns)


RATING_CASES = [("snn_4x64.snn", 1, 1 << 20, 1 << 20, 4), ("snn_4x64.snn", 2, 3, 20, 8),
                ("circ_2k.hgr", 1, 1 << 20, 1 << 20, 16), ("snn_5x40_ln.snn", 3, 7, 9, 4),
                ("tiny_multi.axh", 1, 4, 4, 3), ("tiny_w.hgr", 1, 10, 10, 2)]


@pytest.mark.parametrize("name,size,omega,delta,cnc", RATING_CASES)
def test_rating_matches_oracle(ctx, name, size, omega, delta, cnc):
    g = dedup(golden(name))
    rng = np.random.default_rng(size)
    ns = rng.integers(1, size + 1, g.n).astype(np.uint32)
    pairs, scores = ctx.stage_rating(g, ns, omega, delta, cnc)
    o_pairs, o_scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, omega, delta, cnc)
    np.testing.assert_array_equal(pairs, o_pairs)
    np.testing.assert_array_equal(scores, o_scores)


def random_hyperedges(n, e, size, seed):
    """e hyperedges of `size` distinct uniform pins (the first one the source): neighbourhoods
    with almost no repeats, so nodes' distinct neighbours come close to their work bounds."""
    rng = np.random.default_rng(seed)
    pins = np.concatenate([rng.choice(n, size, replace=False) for _ in range(e)]).astype(np.uint32)
    off = np.arange(e + 1, dtype=np.uint64) * size
    return ax.Hypergraph(n, off, pins, np.ones(e, np.uint32), np.ones(e, np.float32))


# Rating tables: nodes whose distinct neighbours outgrow the first try (2048 slots) retry at
# 8192 slots, then at the tier's full size (about 40 hyperedges of 100 pins per node); nodes above
# 8192 pin visits use global tables whose filled slots are listed (about 100 per node).
@pytest.mark.parametrize("e", [8000, 20000])
def test_rating_retries_and_global_tables_match_oracle(ctx, e):
    g = random_hyperedges(20000, e, 100, e)
    ns = np.ones(g.n, np.uint32)
    pairs, scores = ctx.stage_rating(g, ns, 1 << 20, 1 << 20, 4)
    o_pairs, o_scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, 1 << 20, 1 << 20, 4)
    np.testing.assert_array_equal(pairs, o_pairs)
    np.testing.assert_array_equal(scores, o_scores)


@pytest.mark.parametrize("wl", ["snn-8x512", "circuit-200k-k2"])
def test_rating_full_size(ctx, wl):
    g, p = ax.workload(wl)
    g = dedup(g)
    ns = np.ones(g.n, np.uint32)
    omega = p.omega if p.mode == 0 else 1 << 20
    delta = p.delta if p.mode == 0 else 0x7FFFFFFF
    pairs, scores = ctx.stage_rating(g, ns, omega, delta, 4)
    o_pairs, o_scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, omega, delta, 4)
    np.testing.assert_array_equal(pairs, o_pairs)
    np.testing.assert_array_equal(scores, o_scores)


def long_and_short_snn():
    """Lognormal fan-out SNN: hyperedges on both sides of the rating's length limit (128 pins)."""
    return ax.gen_snn(5, 600, 100, 0.9, 400, 0.7, 21)


def test_rating_length_limit_matches_oracle(ctx):
    g = dedup(long_and_short_snn())
    lens = np.diff(g.off)
    assert (lens > ax.RATE_MAX_LEN).any() and (lens <= ax.RATE_MAX_LEN).any()
    ns = np.ones(g.n, np.uint32)
    pairs, scores = ctx.stage_rating(g, ns, 64, 4096, 4)
    o_pairs, o_scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, 64, 4096, 4)
    np.testing.assert_array_equal(pairs, o_pairs)
    np.testing.assert_array_equal(scores, o_scores)


def test_partition_with_long_hyperedges_matches_oracle(ctx):
    g = long_and_short_snn()
    p = ax.params_incc(64, 4096, 1048576, cnc=4, rfr=8)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1


# The refinement cascade sweeps each hyperedge's movers in rank order with one of three kernels:
# a warp (up to 128 movers), a block with shared-memory tables, or a block on scratch memory. Its
# tables are indexed by partition id up to 256 partitions and hashed above. The k-way case keeps
# K = 4 (direct tables); the INCC case with omega 8 ends with more than 256 partitions (hashed).
# AXC_CASCADE_BLOCK_MOVERS=128 sends every hyperedge with more than 128 movers to the scratch
# kernel, which the default routing reaches only for hyperedges above 2048 pins.
CASCADE_CASES = [ax.params_kway(4, 0.03, cnc=4, rfr=8), ax.params_incc(8, 2048, 1048576, cnc=4, rfr=8)]


@pytest.mark.parametrize("block_movers", [None, "128"])
@pytest.mark.parametrize("i", range(len(CASCADE_CASES)))
def test_cascade_kernels_match_oracle(ctx, monkeypatch, i, block_movers):
    g, p = long_and_short_snn(), CASCADE_CASES[i]
    if block_movers is None:
        monkeypatch.delenv("AXC_CASCADE_BLOCK_MOVERS", raising=False)
    else:
        monkeypatch.setenv("AXC_CASCADE_BLOCK_MOVERS", block_movers)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1
    if p.mode == ax.MODE_INCC:
        assert st.num_parts > 256


# Whole refinement levels (axc_stage_refine against the oracle's refine_level): every round count
# from 1 (one eager round) to 6 (rounds replayed on the device), INCC and k-way. R = 2 starts in
# the schedule's second third (discount 2) and R = 3 in the first.
REFINE_CASES = [("snn_5x40_ln.snn", True, 24, 12, 60), ("circ_2k.hgr", False, 8, 600, 1 << 20)]


@pytest.mark.parametrize("rounds", [1, 2, 3, 6])
@pytest.mark.parametrize("name,encourage,K,omega,delta", REFINE_CASES)
def test_refine_rounds_match_oracle(ctx, name, encourage, K, omega, delta, rounds):
    g = dedup(golden(name))
    rng = np.random.default_rng(rounds)
    part = rng.integers(0, K, g.n).astype(np.uint32)
    ns = rng.integers(1, 3, g.n).astype(np.uint32)
    out, ran = ctx.stage_refine(g, part, K, ns, omega, delta, encourage, rounds, 3)
    o = O.refine(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, part, K, omega, delta, encourage, rounds, 3)
    np.testing.assert_array_equal(out, o)
    assert 1 <= ran <= rounds and (out != part).any()


# The same on a level above the small-level bound (20,000 nodes, K <= 256): the rounds keep one
# census and recompute only the hyperedges of the previous round's moved nodes.
@pytest.mark.parametrize("rounds", [1, 2, 3, 6])
@pytest.mark.parametrize("encourage,K,omega,delta", [(False, 8, 4000, 1 << 20), (True, 200, 300, 1500)])
def test_refine_rounds_large_level_match_oracle(ctx, encourage, K, omega, delta, rounds):
    g = dedup(ax.gen_circuit(20000, 22000, 2, 64, 2.5, 0.9, 0.02, 5))
    rng = np.random.default_rng(rounds + 10)
    part = rng.integers(0, K, g.n).astype(np.uint32)
    ns = rng.integers(1, 3, g.n).astype(np.uint32)
    out, ran = ctx.stage_refine(g, part, K, ns, omega, delta, encourage, rounds, 3)
    o = O.refine(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, part, K, omega, delta, encourage, rounds, 3)
    np.testing.assert_array_equal(out, o)
    assert 1 <= ran <= rounds and (out != part).sum() > 1000


def test_refine_two_rounds_discount_matches_oracle(ctx):
    """Two rounds from a refined partition in which every node has a move: round 0 runs at
    discount 2, and the oracle applies one move in each round."""
    g0 = ax.gen_snn(3, 900, 650, 0.25, 1100, 1.0, 41)
    g = dedup(g0)
    start, K, _, _ = oracle_partition(g0, ax.params_incc(8, 2048, 1048576, cnc=4, rfr=1))
    ns = np.ones(g.n, np.uint32)
    out, ran = ctx.stage_refine(g, start, K, ns, 8, 2048, 1, 2)
    o = O.refine(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, start, K, 8, 2048, 1, 2)
    np.testing.assert_array_equal(out, o)
    assert ran == 2 and (o != start).sum() == 2


# Hashed cascade tables with hyperedges of up to 1101 pins: the block kernel's middle tier (at most
# 512 movers and 2048 table slots) takes the mid-size hyperedges and hands the larger ones to the
# launch sized by the level's longest hyperedge.
def test_cascade_middle_tier_matches_oracle(ctx):
    g = ax.gen_snn(3, 900, 650, 0.25, 1100, 1.0, 41)
    assert np.diff(g.off.astype(np.int64)).max() > 1024
    p = ax.params_incc(8, 2048, 1048576, cnc=4, rfr=2)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1 and st.num_parts > 256


# Nodes whose gain-table bound passes 4096 slots (here about 2000 partitions of two neurons and
# about 80 inbound hyperedges of about 80 pins) first try a shared-memory table and fall back to a
# global one when they reach too many distinct partitions. With at most 4096 partitions the first
# try always fits; AXC_GAIN_TRY_LIMIT=16 makes nearly every such node fall back.
@pytest.mark.parametrize("try_limit", [None, "16"])
def test_heavy_gain_tier_matches_oracle(ctx, monkeypatch, try_limit):
    g = ax.gen_snn(4, 1000, 80, 0.7, 300, 0.7, 31)
    p = ax.params_incc(2, 4096, 1048576, cnc=4, rfr=4)
    if try_limit is None:
        monkeypatch.delenv("AXC_GAIN_TRY_LIMIT", raising=False)
    else:
        monkeypatch.setenv("AXC_GAIN_TRY_LIMIT", try_limit)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1 and 256 < st.num_parts <= 4096


def census_entries_per_node(g, part):
    """Sum over each node's incident hyperedges of their distinct partitions (the sample measure of
    the sampled gain rule)."""
    off = g.off.astype(np.int64)
    lens = off[1:] - off[:-1]
    hid = np.repeat(np.arange(g.e), lens)
    pairs = np.unique(np.stack([hid, part[g.pins].astype(np.int64)], 1), axis=0)
    lam = np.bincount(pairs[:, 0], minlength=g.e)
    return np.bincount(g.pins.astype(np.int64), weights=lam[hid], minlength=g.n)


# More than AXC_SPARSE_GAIN_K = 4096 partitions: nodes whose incidences hold more than 4096 census
# entries take the sampled rule (candidates from an incidence prefix, exact evaluation of the best
# 8); the others the exact gains. Both against the oracle's restatement of the rule.
SAMPLED_CASES = [(6000, 1 << 20, 1 << 20, 1, 1), (6000, 40, 150, 1, 2), (9000, 3, 0x7FFFFFFF, 0, 1),
                 (5000, 1 << 20, 120, 1, 0xFFFFFFFF)]


@pytest.mark.parametrize("K,omega,delta,enc,disc", SAMPLED_CASES)
def test_sampled_gains_match_oracle(ctx, K, omega, delta, enc, disc):
    g = dedup(ax.gen_snn(4, 3000, 90, 0.5, 400, 0.7, 41))
    rng = np.random.default_rng(K + disc)
    part = rng.integers(0, K, g.n).astype(np.uint32)
    ns = rng.integers(1, 3, g.n).astype(np.uint32)
    ent = census_entries_per_node(g, part)
    assert (ent > 4096).sum() > 100 and (ent <= 4096).sum() > 100  # both paths are exercised
    tgt, gain = ctx.stage_gains(g, part, K, ns, omega, delta, enc, disc)
    o_tgt, o_gain = O.gains(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, part, K, omega, delta, enc, disc)
    np.testing.assert_array_equal(tgt, o_tgt)
    np.testing.assert_array_equal(gain, o_gain)
    assert (tgt[ent > 4096] != NONE).any()


def test_partition_with_sampled_gains_matches_oracle(ctx):
    """An INCC run whose inbound limit stops coarsening early, so every level refines with more
    than 4096 partitions and heavy nodes take the sampled rule; equal to the oracle's partition."""
    g = ax.gen_snn(10, 1000, 80, 0.0, 0, 1.0, 43)  # in-degrees up to 113: every node fits alone
    p = ax.params_incc(1024, 130, 1048576, cnc=4, rfr=6)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1 and st.num_parts > 4096


@pytest.mark.parametrize("name,cnc", [("snn_4x64.snn", 4), ("circ_2k.hgr", 8), ("snn_5x40_ln.snn", 2)])
def test_matching_matches_oracle(ctx, name, cnc):
    g = dedup(golden(name))
    ns = np.ones(g.n, np.uint32)
    toff, touch, nin = O.touching(g.n, g.off, g.pins, g.nsrc)
    pairs, scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, 1 << 20, 1 << 20, cnc)
    groups, ng = ctx.stage_matching(g.n, cnc, pairs, scores, ns, nin, 1 << 20, 1 << 20)
    o_groups, o_ng = O.matching(g.n, cnc, pairs, scores, ns, nin, 1 << 20, 1 << 20)
    assert ng == o_ng
    np.testing.assert_array_equal(groups, o_groups)


@pytest.mark.parametrize("wl", ["snn-8x512", "circuit-200k-k2"])
def test_matching_full_size(ctx, wl):
    g, _ = ax.workload(wl)
    g = dedup(g)
    ns = np.ones(g.n, np.uint32)
    toff, touch, nin = O.touching(g.n, g.off, g.pins, g.nsrc)
    pairs, scores = O.rating(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, 1 << 20, 0x7FFFFFFF, 4)
    groups, ng = ctx.stage_matching(g.n, 4, pairs, scores, ns, nin, 1 << 20, 0x7FFFFFFF)
    o_groups, o_ng = O.matching(g.n, 4, pairs, scores, ns, nin, 1 << 20, 0x7FFFFFFF)
    assert ng == o_ng
    np.testing.assert_array_equal(groups, o_groups)


def test_matching_orphans(ctx):
    # no candidates at all: everything is an orphan; pairing by (size, id) under omega and delta
    n, cnc = 11, 2
    pairs = np.full(n * cnc, NONE, np.uint32)
    scores = np.zeros(n * cnc, np.uint32)
    ns = np.array([3, 1, 4, 1, 5, 9, 2, 6, 5, 3, 5], np.uint32)
    nin = np.array([1, 0, 2, 7, 1, 0, 3, 1, 2, 0, 1], np.uint32)
    groups, ng = ctx.stage_matching(n, cnc, pairs, scores, ns, nin, 10, 5)
    o_groups, o_ng = O.matching(n, cnc, pairs, scores, ns, nin, 10, 5)
    assert ng == o_ng
    np.testing.assert_array_equal(groups, o_groups)


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_contract_matches_oracle(ctx, name):
    g = dedup(golden(name))
    rng = np.random.default_rng(1)
    ng = max(1, g.n // 2)
    groups = rng.integers(0, ng, g.n).astype(np.uint32)
    _, groups = np.unique(groups, return_inverse=True)
    groups = groups.astype(np.uint32)
    off, pins, ns = ctx.stage_contract(g, groups)
    o_off, o_pins, o_ns = O.contract(g.off, g.pins, g.nsrc, groups)
    np.testing.assert_array_equal(off, o_off)
    np.testing.assert_array_equal(pins, o_pins)
    np.testing.assert_array_equal(ns, o_ns)


GAIN_CASES = [("snn_4x64.snn", 8, 1 << 20, 1 << 20, 1, 1), ("snn_4x64.snn", 8, 40, 60, 1, 2),
              ("circ_2k.hgr", 4, 600, 0x7FFFFFFF, 0, 1), ("circ_2k.hgr", 17, 150, 0x7FFFFFFF, 0, 0xFFFFFFFF),
              ("snn_5x40_ln.snn", 6, 50, 30, 1, 0xFFFFFFFF)]


@pytest.mark.parametrize("name,K,omega,delta,enc,disc", GAIN_CASES)
def test_gains_match_oracle(ctx, name, K, omega, delta, enc, disc):
    g = dedup(golden(name))
    rng = np.random.default_rng(K)
    part = rng.integers(0, K, g.n).astype(np.uint32)
    ns = rng.integers(1, 3, g.n).astype(np.uint32)
    tgt, gain = ctx.stage_gains(g, part, K, ns, omega, delta, enc, disc)
    o_tgt, o_gain = O.gains(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, part, K, omega, delta, enc, disc)
    np.testing.assert_array_equal(tgt, o_tgt)
    np.testing.assert_array_equal(gain, o_gain)


def oracle_partition(g, p):
    if p.mode == ax.MODE_INCC:
        return O.partition(g.n, g.off, g.pins, g.nsrc, g.w, 0, omega=p.omega, delta=p.delta,
                           max_parts=p.max_parts, cnc=p.cnc, rfr=p.rfr, ipm=p.ipm, seed=p.seed)
    return O.partition(g.n, g.off, g.pins, g.nsrc, g.w, 1, k=p.k, eps=p.eps, cnc=p.cnc, rfr=p.rfr, seed=p.seed)


E2E_SMALL = [("snn_4x64.snn", ax.params_incc(16, 64, 1 << 20, cnc=4, rfr=8)),
             ("snn_4x64.snn", ax.params_kway(4, 0.05, cnc=4, rfr=8)),
             ("circ_2k.hgr", ax.params_incc(50, 400, 1 << 20, cnc=8, rfr=16)),
             ("circ_2k.hgr", ax.params_kway(8, 0.03, cnc=4, rfr=16)),
             ("snn_5x40_ln.snn", ax.params_incc(12, 30, 1 << 20, cnc=2, rfr=6, ipm=0)),
             ("tiny_multi.axh", ax.params_incc(3, 3, 1 << 20, cnc=2, rfr=4)),
             ("tiny_dups.hgr", ax.params_kway(2, 0.5, cnc=2, rfr=4))]


@pytest.mark.parametrize("i", range(len(E2E_SMALL)))
def test_partition_matches_oracle(ctx, i):
    name, p = E2E_SMALL[i]
    g = golden(name)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.num_parts == o_K
    assert st.valid == 1


@pytest.mark.parametrize("wl", ["snn-8x512", "circuit-200k-k2", "circuit-200k-k64"])
def test_partition_full_size_matches_oracle(ctx, wl):
    g, p = ax.workload(wl)
    part, st = ctx.partition(g, p)
    o_part, o_K, _, _ = oracle_partition(g, p)
    np.testing.assert_array_equal(part, o_part)
    assert st.valid == 1
    om = p.omega if p.mode == 0 else ax.kway_omega(g.n, p.k, p.eps)
    de = p.delta if p.mode == 0 else 0x7FFFFFFF
    kmax = p.max_parts if p.mode == 0 else p.k
    ev = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, part, om, de, kmax)
    assert ev["valid"] == 1
    assert ev["connectivity_fx"] == st.connectivity_fx


def host_quotient(g, part):
    import ctypes as C
    q = ax.HGraph()
    assert ax.lib().axc_quotient_hgraph(C.byref(g.c()), part.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(q)) == 0
    try:
        return ax.Hypergraph.from_c(q)
    finally:
        ax.lib().axc_free_hgraph(C.byref(q))


# The `-s` quotient hypergraph on the device must equal the host construction exactly: nodes,
# hyperedge order, source / destination lists and merged weights. Cases: SNN hyperedges with
# sources, hMETIS nets without, duplicate pins, one partition, many partitions, weights.
@pytest.mark.parametrize("name,K", [("snn_4x64.snn", 7), ("circ_2k.hgr", 40), ("tiny_dups.hgr", 3),
                                    ("snn_5x40_ln.snn", 1), ("tiny_w.hgr", 2), ("snn_4x64.snn", 256)])
def test_device_quotient_matches_host(ctx, name, K):
    g = golden(name)
    rng = np.random.default_rng(K)
    part = rng.integers(0, K, g.n).astype(np.uint32)
    q = ctx.quotient(g, part)
    h = host_quotient(g, part)
    assert q.n == h.n
    np.testing.assert_array_equal(q.off, h.off)
    np.testing.assert_array_equal(q.pins, h.pins)
    np.testing.assert_array_equal(q.nsrc, h.nsrc)
    np.testing.assert_array_equal(q.w, h.w)


def test_device_quotient_of_a_partition(ctx):
    g, p = ax.workload("snn-8x512")
    part, st = ctx.partition(g, p)
    q, h = ctx.quotient(g, part), host_quotient(g, part)
    assert q.n == st.num_parts and q.e == h.e
    np.testing.assert_array_equal(q.pins, h.pins)
    np.testing.assert_array_equal(q.w, h.w)


def test_evaluate_matches_oracle(ctx):
    g = golden("circ_2k.hgr")
    rng = np.random.default_rng(5)
    part = rng.integers(0, 9, g.n).astype(np.uint32)
    _, part = np.unique(part, return_inverse=True)
    part = part.astype(np.uint32)
    p = ax.params_incc(300, 2000, 9)
    st = ctx.evaluate(g, p, part)
    ev = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, part, 300, 2000, 9)
    assert (st.connectivity_fx, st.cutnet_fx, st.soed_fx) == (ev["connectivity_fx"], ev["cutnet_fx"], ev["soed_fx"])
    assert st.valid == ev["valid"] and st.num_parts == ev["num_parts"]
    assert st.max_part_inbound == ev["max_inbound"]


def test_same_seed_same_partition(ctx):
    g, p = ax.workload("circuit-200k-k64")
    a, _ = ctx.partition(g, p)
    b, _ = ctx.partition(g, p)
    np.testing.assert_array_equal(a, b)


def test_batch_queue_matches_solo(ctx):
    jobs = [(ax.gen_circuit(3000 + 500 * i, 3300 + 500 * i, 2, 32, 2.5, 0.9, 0.02, 100 + i),
             ax.params_kway([2, 8, 32][i % 3], 0.03, cnc=4, rfr=8)) for i in range(6)]
    solo = [ctx.partition(g, p)[0] for g, p in jobs]
    ids = [ctx.submit(g, p) for g, p in jobs]
    for (g, _), jid, s in zip(jobs, ids, solo):
        part, st = ctx.poll(jid, g.n)
        np.testing.assert_array_equal(part, s)
        assert st.valid == 1
