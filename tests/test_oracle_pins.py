"""Pins the oracle against the reference's own code.

The golden fixtures (tests/golden/*.ref.npz, *.grade.json) were produced by the reference's
HyperGraph loaders, deduplicateHyperedges(2) and incidence sets (includes/hgraph.hpp), and by its
grader (grading/grade.cpp), compiled here from the reference sources; tests/golden/make_golden.py
regenerates them. These tests need no GPU.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_INPUTS
from oracle import oracle as O


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".ref.npz"))


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_reader_matches_reference(name):
    r = load(name)
    n, off, pins, ns, w = O.read(os.path.join(GOLDEN, name))
    assert n == int(r["raw_n"])
    np.testing.assert_array_equal(off, r["raw_off"])
    np.testing.assert_array_equal(pins, r["raw_pins"])
    np.testing.assert_array_equal(ns, r["raw_nsrc"])
    np.testing.assert_array_equal(w, r["raw_w"])


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_rule2_dedupe_matches_reference(name):
    r = load(name)
    off, pins, ns = O.dedupe(r["raw_off"], r["raw_pins"], r["raw_nsrc"])
    np.testing.assert_array_equal(off, r["ded_off"])
    np.testing.assert_array_equal(pins, r["ded_pins"])
    np.testing.assert_array_equal(ns, r["ded_nsrc"])


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_incidence_csr_matches_reference(name):
    r = load(name)
    toff, touch, nin = O.touching(int(r["ded_n"]), r["ded_off"], r["ded_pins"], r["ded_nsrc"])
    np.testing.assert_array_equal(toff, r["toff"])
    np.testing.assert_array_equal(touch, r["touch"])
    np.testing.assert_array_equal(nin, r["nin"])


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_metrics_and_validity_match_grader(name):
    r = load(name)
    cases = json.load(open(os.path.join(GOLDEN, name + ".grade.json")))
    n = int(r["raw_n"])
    for c in cases:
        part = np.array(c["part"], np.uint32)
        ev = O.evaluate(n, r["raw_off"], r["raw_pins"], r["raw_nsrc"], r["raw_w"], part,
                        c["omega"], c["delta"], c["kmax"])
        g = c["grade"]
        assert bool(ev["valid"]) == bool(g["valid"])
        # the grader prints float sums with three decimals
        for key, fx in (("Connectivity", "connectivity_fx"), ("Cut-net", "cutnet_fx"), ("SOED", "soed_fx")):
            assert abs(ev[fx] / 262144.0 - g[key]) <= 1e-3 + 1e-6 * abs(g[key]), (key, ev[fx] / 262144.0, g[key])
        t = c["tight"]
        ev2 = O.evaluate(n, r["raw_off"], r["raw_pins"], r["raw_nsrc"], r["raw_w"], part,
                         t["omega"], t["delta"], t["kmax"])
        assert bool(ev2["valid"]) == bool(t["grade"]["valid"])


def test_rating_is_symmetric():
    # score(u, v) == score(v, u) whenever both list each other (kernels/coarsening.cu:39-44)
    r = load("snn_4x64.snn")
    n = int(r["ded_n"])
    w = O.wfx(r["ded_w"])
    cnc = 8
    pairs, scores = O.rating(n, r["ded_off"], r["ded_pins"], r["ded_nsrc"], w, np.ones(n), 1 << 20, 1 << 20, cnc)
    P = pairs.reshape(n, cnc)
    S = scores.reshape(n, cnc)
    seen = 0
    for u in range(n):
        for j in range(cnc):
            v = P[u, j]
            if v == O.NONE:
                continue
            hit = np.where(P[v] == u)[0]
            if len(hit):
                assert S[v, hit[0]] == S[u, j]
                seen += 1
    assert seen > 0


@pytest.mark.parametrize("length,rated", [(128, True), (129, False)])
def test_rating_skips_hyperedges_over_the_length_limit(length, rated):
    """Hyperedges of more than 128 pins (AXC_RATE_MAX_LEN) take no part in the rating: with such a
    hyperedge alone no node has a candidate; at exactly 128 pins every node has some."""
    n = length
    off = np.array([0, length], np.uint64)
    pins = np.arange(length, dtype=np.uint32)
    nsrc = np.array([1], np.uint32)
    w = O.wfx(np.ones(1, np.float32))
    pairs, _ = O.rating(n, off, pins, nsrc, w, np.ones(n, np.uint32), 1 << 20, 1 << 20, 4)
    has = (pairs.reshape(n, 4)[:, 0] != O.NONE)
    assert has.all() if rated else not has.any()


@pytest.mark.parametrize("name", ["snn_4x64.snn", "circ_2k.hgr", "snn_5x40_ln.snn"])
def test_oracle_partitioner_valid_and_deterministic(name):
    r = load(name)
    n = int(r["raw_n"])
    args = (n, r["raw_off"], r["raw_pins"], r["raw_nsrc"], r["raw_w"])
    p1, K1, _, _ = O.partition(*args, 0, omega=16, delta=64, max_parts=1 << 20, cnc=4, rfr=8, ipm=1)
    p2, K2, _, _ = O.partition(*args, 0, omega=16, delta=64, max_parts=1 << 20, cnc=4, rfr=8, ipm=1)
    np.testing.assert_array_equal(p1, p2)
    ev = O.evaluate(*args, p1, 16, 64, 1 << 20)
    assert ev["valid"] == 1 and ev["num_parts"] == K1
    q1, Kq, _, _ = O.partition(*args, 1, k=4, eps=0.05, cnc=4, rfr=8)
    om = int(np.ceil(np.float32(1.05) * np.float32(n) / np.float32(4)))
    ev = O.evaluate(*args, q1, om, 0x7FFFFFFF, 4)
    assert ev["valid"] == 1


# ---- the reference's own coarsening stages (oracle/refstages.cu run on a GPU; fixtures made by
# tests/golden/make_refstages.py) --------------------------------------------------------------
REFSTAGE = sorted(f[: -len(".refstage.npz")] for f in os.listdir(GOLDEN) if f.endswith(".refstage.npz"))


def refstage(case):
    name = case.rsplit(".", 1)[0]
    return name, np.load(os.path.join(GOLDEN, case + ".refstage.npz"))


def test_refstage_fixtures_present():
    """Every input of make_refstages.py has its fixture (loose and tight limits for the synthetic ones)."""
    assert len(REFSTAGE) >= 9, REFSTAGE


@pytest.mark.parametrize("case", REFSTAGE)
def test_rating_matches_reference_stage(case):
    """The oracle's rating equals the reference's candidatesProposal (sources/coarsening.cu:17-68,
    kernels/coarsening.cu:10-213) pair for pair and score for score: same neighbours, same size
    and inbound filters, same symmetric noise, same top-cnc order. The reference rates through
    every hyperedge, so the oracle runs without its length limit here."""
    name, s = refstage(case)
    r = load(name)
    n, cnc = int(s["n"]), int(s["cnc"])
    assert n == int(r["ded_n"]) and int(s["P"]) == len(r["ded_pins"])
    pairs, scores = O.rating(n, r["ded_off"], r["ded_pins"], r["ded_nsrc"], O.wfx(r["ded_w"]),
                             np.ones(n, np.uint32), int(s["omega"]), int(s["delta"]), cnc, max_len=O.NO_LEN_LIMIT)
    np.testing.assert_array_equal(pairs, s["pairs"])
    ok = s["pairs"] != O.NONE  # the reference leaves the score of an empty slot unwritten
    np.testing.assert_array_equal(scores[ok], s["scores"][ok])


@pytest.mark.parametrize("case", REFSTAGE)
def test_rating_length_limit_is_inert_below_128(case):
    """On inputs whose hyperedges all have at most 128 pins, the length limit changes nothing."""
    name, s = refstage(case)
    r = load(name)
    n, cnc = int(s["n"]), int(s["cnc"])
    off = r["ded_off"].astype(np.int64)
    if len(off) > 1 and int((off[1:] - off[:-1]).max()) > O.RATE_MAX_LEN:
        pytest.skip("input has hyperedges above the rating length limit")
    args = (n, r["ded_off"], r["ded_pins"], r["ded_nsrc"], O.wfx(r["ded_w"]), np.ones(n, np.uint32),
            int(s["omega"]), int(s["delta"]), cnc)
    a, _ = O.rating(*args)
    b, _ = O.rating(*args, max_len=O.NO_LEN_LIMIT)
    np.testing.assert_array_equal(a, b)


def _hedge_sets(off, pins, nsrc):
    out = []
    for h in range(len(nsrc)):
        seg = pins[int(off[h]): int(off[h + 1])]
        k = int(nsrc[h])
        out.append((tuple(sorted(seg[:k].tolist())), tuple(sorted(seg[k:].tolist()))))
    return out


@pytest.mark.parametrize("case", REFSTAGE)
def test_contract_matches_reference_stage(case):
    """The oracle's contraction of the reference's own grouping equals the reference's
    coarsenHedges (sources/construction.cu:563-676): the same hyperedge offsets and source counts,
    and per hyperedge the same source set and destination set (a group that is also a destination
    leaves the sources; size-1 hyperedges stay). The reference lists destinations descending,
    the oracle ascending, so the segments are compared as sets."""
    name, s = refstage(case)
    r = load(name)
    off, pins, nsrc = O.contract(r["ded_off"], r["ded_pins"], r["ded_nsrc"], s["groups"])
    np.testing.assert_array_equal(off, s["coff"])
    np.testing.assert_array_equal(nsrc, s["cnsrc"])
    assert _hedge_sets(off, pins, nsrc) == _hedge_sets(s["coff"], s["cpins"], s["cnsrc"])


@pytest.mark.parametrize("case", REFSTAGE)
def test_coarse_incidence_matches_reference_stage(case):
    """Incidence sets of the contracted graph equal the reference's coarsenTouching
    (sources/construction.cu:678-789): per coarse node the same inbound hyperedges and the same
    outbound ones (an edge in both stays inbound only), both in ascending order."""
    name, s = refstage(case)
    r = load(name)
    off, pins, nsrc = O.contract(r["ded_off"], r["ded_pins"], r["ded_nsrc"], s["groups"])
    toff, touch, nin = O.touching(int(s["ngroups"]), off, pins, nsrc)
    np.testing.assert_array_equal(nin, s["cinb"])
    np.testing.assert_array_equal(toff, s["ctoff"])
    for v in range(int(s["ngroups"])):
        a, b = int(toff[v]), int(toff[v + 1])
        k = int(nin[v])
        assert sorted(touch[a:a + k].tolist()) == sorted(s["ctouch"][a:a + k].tolist())
        assert sorted(touch[a + k:b].tolist()) == sorted(s["ctouch"][a + k:b].tolist())
