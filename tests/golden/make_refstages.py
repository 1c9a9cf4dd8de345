"""Generates tests/golden/<input>.<case>.refstage.npz from the reference's own coarsening stages.

oracle/_ref/refstages.exe (oracle/refstages.cu, linked with the reference's objects compiled from
its sources by `make -C oracle ref`) runs, on the GPU, the reference's candidatesProposal,
groupNodes, coarsenHedges and coarsenTouching once on level 0 of a golden input and dumps their
outputs; this script stores them as small fixtures that the CPU tests compare the oracle against
(tests/test_oracle_pins.py). It needs a CUDA GPU, so it runs on the GPU box:

    python tests/golden/make_refstages.py <out_dir>

and the .npz files it writes are then copied into tests/golden/.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "refstages.exe")

# (input, case name, omega, delta, cnc): loose limits rate every neighbour; tight ones make the
# size and inbound filters of the rating bind.
CASES = [
    ("snn_4x64.snn", "loose", 1 << 20, 1 << 20, 16),
    ("snn_4x64.snn", "tight", 4, 40, 4),
    ("snn_5x40_ln.snn", "loose", 1 << 20, 1 << 20, 8),
    ("snn_5x40_ln.snn", "tight", 3, 24, 4),
    ("circ_2k.hgr", "loose", 1 << 20, 1 << 20, 16),
    ("circ_2k.hgr", "tight", 4, 12, 4),
    ("tiny_multi.axh", "loose", 1 << 20, 1 << 20, 4),
    ("tiny_self.snn", "loose", 1 << 20, 1 << 20, 4),
    ("tiny_w.hgr", "loose", 1 << 20, 1 << 20, 4),
]


def parse(buf: bytes) -> dict:
    pos = 0

    def take(dt, cnt):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=cnt, offset=pos).copy()
        pos += a.nbytes
        return a

    n, e = (int(x) for x in take(np.uint32, 2))
    P = int(take(np.uint64, 1)[0])
    cnc = int(take(np.uint32, 1)[0])
    out = {"n": n, "e": e, "P": P, "cnc": cnc}
    out["pairs"] = take(np.uint32, n * cnc)
    out["scores"] = take(np.uint32, n * cnc)
    ng = int(take(np.uint32, 1)[0])
    out["ngroups"] = ng
    out["groups"] = take(np.uint32, n)
    cP = int(take(np.uint64, 1)[0])
    out["coff"] = take(np.uint64, e + 1)
    out["cpins"] = take(np.uint32, cP)
    out["cnsrc"] = take(np.uint32, e)
    out["ctoff"] = take(np.uint64, ng + 1)
    out["ctouch"] = take(np.uint32, int(out["ctoff"][-1]) if ng else 0)
    out["cinb"] = take(np.uint32, ng)
    assert pos == len(buf), "trailing bytes in the refstages dump"
    return out


def main() -> int:
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    for name, case, omega, delta, cnc in CASES:
        with tempfile.NamedTemporaryFile(suffix=".bin") as t:
            r = subprocess.run([EXE, os.path.join(HERE, name), str(omega), str(delta), str(cnc), t.name],
                               capture_output=True, text=True)
            if r.returncode != 0:
                print(f"{name} {case}: refstages.exe exited {r.returncode}: {r.stderr[-400:]}", file=sys.stderr)
                return 1
            d = parse(open(t.name, "rb").read())
        np.savez(os.path.join(out_dir, f"{name}.{case}.refstage.npz"), omega=omega, delta=delta, **d)
        print(f"{name} {case}: {r.stdout.strip()}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
