"""Generates the golden fixtures under tests/golden/ from the reference's own code.

Inputs: small hand-written hypergraphs (edge cases of the reference readers and the rule-2 dedupe)
plus small seeded synthetic ones. Outputs, per input:
  <name>.ref.npz   what the reference's HyperGraph code computes (oracle/_ref/refharness.exe):
                   the graph as loaded, after deduplicateHyperedges(2), and its incidence sets
  <name>.grade.json  metrics and validity printed by the reference grader (oracle/_ref/hgrade.exe)
                   for a few partitions, together with those partitions

Run from the repository root after `make -C oracle ref` (which compiles the reference tools here):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# ---- hand-written inputs ------------------------------------------------------------------
HGR = {
    # duplicate pins, a singleton net (skipped), comments, CRLF, blank lines
    "tiny_dups.hgr": "% comment line\n5 6\n1 2 3 2\n\n4 4 5\r\n6\n% another\n1 6 1 6 2\n3 4 5 6\n",
    # weighted nets (fmt 1)
    "tiny_w.hgr": "4 5 1\n2 1 2 3\n1 3 4\n3 4 5 1\n5 2 5\n",
    # vertex weights flagged (fmt 11): vertex weight lines are not read
    "tiny_vw.hgr": "3 4 11\n1 1 2\n2 2 3 4\n1 1 4\n",
}


def snn_bytes(n, hedges):
    out = [np.array([n, len(hedges)], np.uint32).tobytes()]
    for src, dsts, w in hedges:
        out.append(np.array([len(dsts), src] + list(dsts), np.uint32).tobytes())
        out.append(np.array([w], np.float32).tobytes())
    return b"".join(out)


def axh_bytes(n, hedges):
    out = [np.array([n, len(hedges)], np.uint32).tobytes()]
    for srcs, dsts, w in hedges:
        out.append(np.array([len(srcs) + len(dsts), len(srcs)] + list(srcs) + list(dsts), np.uint32).tobytes())
        out.append(np.array([w], np.float32).tobytes())
    return b"".join(out)


BIN = {
    # a destination equal to the source (dropped by rule 2), repeated destinations
    "tiny_self.snn": snn_bytes(6, [(0, [1, 2, 0, 2], 1.0), (3, [4, 5, 4], 2.5), (5, [0], 1.0), (1, [2], 0.5)]),
    # multi-source hyperedges with duplicates across sources and destinations
    "tiny_multi.axh": axh_bytes(7, [([0, 1, 0], [1, 2, 3, 2], 1.0), ([4], [5, 6], 3.0), ([2, 3], [3, 6, 0], 1.5),
                                    ([6, 6], [6, 5], 1.0)]),
}


def synthetic():
    import axoncuda_b200 as ax
    ax.write(os.path.join(HERE, "snn_4x64.snn"), ax.gen_snn(4, 64, 8, 0.0, 0, 1.0, 7))
    ax.write(os.path.join(HERE, "snn_5x40_ln.snn"), ax.gen_snn(5, 40, 6, 0.6, 20, 0.7, 8))
    ax.write(os.path.join(HERE, "circ_2k.hgr"), ax.gen_circuit(2000, 2200, 2, 32, 2.5, 0.9, 0.02, 9))


def main():
    for name, text in HGR.items():
        with open(os.path.join(HERE, name), "w", newline="") as f:
            f.write(text)
    for name, data in BIN.items():
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)
    synthetic()
    inputs = sorted(list(HGR) + list(BIN) + ["snn_4x64.snn", "snn_5x40_ln.snn", "circ_2k.hgr"])
    rng = np.random.default_rng(42)
    for name in inputs:
        path = os.path.join(HERE, name)
        raw, ded, tch = O.ref_dump(path)
        np.savez(os.path.join(HERE, name + ".ref.npz"),
                 raw_n=raw[0], raw_off=raw[1], raw_pins=raw[2], raw_nsrc=raw[3], raw_w=raw[4],
                 ded_n=ded[0], ded_off=ded[1], ded_pins=ded[2], ded_nsrc=ded[3], ded_w=ded[4],
                 toff=tch[0], touch=tch[1], nin=tch[2])
        n = raw[0]
        cases = []
        for K in (1, 2, 3, 7):
            part = (np.arange(n) * K // max(n, 1)).astype(np.uint32) if K < 7 else rng.integers(0, 7, n).astype(np.uint32)
            # make ids dense (the grader rejects gaps)
            _, part = np.unique(part, return_inverse=True)
            part = part.astype(np.uint32)
            pf = os.path.join(HERE, "_tmp.part")
            np.savetxt(pf, part, fmt="%d")
            omega, delta, kmax = n, 1 << 30, max(K, 1)
            g = O.ref_grade(path, pf, "incc", omega, delta, kmax)
            # a tight constraint set to exercise the invalid path
            g2 = O.ref_grade(path, pf, "incc", max(1, n // (K + 1)), 2, kmax)
            cases.append({"part": part.tolist(), "omega": omega, "delta": delta, "kmax": kmax, "grade": g,
                          "tight": {"omega": max(1, n // (K + 1)), "delta": 2, "kmax": kmax, "grade": g2}})
            os.remove(pf)
        with open(os.path.join(HERE, name + ".grade.json"), "w") as f:
            json.dump(cases, f)
        print("golden:", name)


if __name__ == "__main__":
    main()
