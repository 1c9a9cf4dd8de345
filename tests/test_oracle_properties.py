"""Size-independent properties of the oracle's refinement rule (CPU only; the GPU path is
bit-exact against this rule in tests/test_gpu_parity.py):
- k-way: a round applies a prefix of moves only when its cascaded gain, the exact change in
  λ−1 · w summed over the prefix, is non-negative, so λ−1 never rises; a balanced start stays
  within the size limit.
- INCC: a valid start stays valid under the size and inbound limits (the prefix is applied only
  with no size or inbound violation); partition ids are relabelled consecutively first, as the
  pipeline does after refinement."""
import os

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN
from oracle import oracle as O

DELTA_NONE = 0x7FFFFFFF


def dedup(name):
    g = ax.read(os.path.join(GOLDEN, name))
    off, pins, ns = O.dedupe(g.off, g.pins, g.nsrc)
    return ax.Hypergraph(g.n, off, pins, ns, g.w.copy())


@pytest.mark.parametrize("K", [2, 8, 32])
def test_kway_refinement_never_raises_connectivity(K):
    g = dedup("circ_2k.hgr")
    omega = ax.kway_omega(g.n, K, 0.03)
    start = (np.arange(g.n) % K).astype(np.uint32)
    ns = np.ones(g.n, np.uint32)
    before = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, start, omega, DELTA_NONE, K)
    assert before["valid"] == 1
    last = before["connectivity_fx"]
    for rounds in (1, 2, 6, 16):
        out = O.refine(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, start, K, omega, DELTA_NONE, False, rounds)
        after = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, out, omega, DELTA_NONE, K)
        assert after["valid"] == 1 and after["max_size"] <= omega
        assert after["connectivity_fx"] <= before["connectivity_fx"]
        last = min(last, after["connectivity_fx"])
    assert last < before["connectivity_fx"]  # the rounds did move something


@pytest.mark.parametrize("delta", [30, 60])
def test_incc_refinement_keeps_a_valid_start_valid(delta):
    g = dedup("snn_5x40_ln.snn")
    start = np.arange(g.n, dtype=np.uint32)  # every node alone: valid when delta covers a node
    ns = np.ones(g.n, np.uint32)
    assert O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, start, 12, delta, 1 << 20)["valid"] == 1
    for rounds in (1, 2, 6):
        out = O.refine(g.n, g.off, g.pins, g.nsrc, O.wfx(g.w), ns, start, g.n, 12, delta, True, rounds)
        relabelled = np.unique(out, return_inverse=True)[1].astype(np.uint32)
        after = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, relabelled, 12, delta, 1 << 20)
        assert after["valid"] == 1 and after["max_size"] <= 12 and after["max_inbound"] <= delta
        assert after["num_parts"] < g.n  # nodes did merge
