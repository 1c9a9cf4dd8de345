"""The drop-in command line (axoncuda_b200/axc_hgraph_gpu) run the way the reference's scripts run
hgraph_gpu.exe: INCC with `-rfr 16 -cnc 4 -dtc -ipm -v 0` (hgraphs/run_snns.sh:20), k-way with
`-rfr 16 -cnc 4 -dtc -v 0 -smh 0` (hgraphs/run_ispd.sh:20). Its result lines parse as the
reference's (sources/main.cu:908-928), its -p file is accepted by the reference grader with the
same lambda-1 as the library reports, and its -s file reads back as the quotient hypergraph."""
import os
import re
import subprocess

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN, ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "axoncuda_b200", "axc_hgraph_gpu")

CASES = [
    ("snn_4x64.snn", ["-m", "16", "64", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"],
     ax.params_incc(16, 64, 1048576, cnc=4, rfr=16, ipm=1), ("incc", 16, 64, 1048576)),
    ("circ_2k.hgr", ["-k", "8", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"],
     ax.params_kway(8, 0.03, cnc=4, rfr=16), ("kway", 8, 0.03)),
    ("snn_5x40_ln.snn", ["-c", "loihi64", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"], None, None),
]


def run_cli(tmp_path, name, flags):
    pf, sf = tmp_path / "out.part", tmp_path / ("out" + os.path.splitext(name)[1])
    r = subprocess.run([CLI, "-r", os.path.join(GOLDEN, name), *flags, "-p", str(pf), "-s", str(sf)],
                       capture_output=True, text=True, timeout=300)
    return r, pf, sf


@pytest.mark.parametrize("i", range(len(CASES)))
def test_cli_result_lines_grader_and_quotient(tmp_path, i):
    name, flags, params, grade_args = CASES[i]
    r, pf, sf = run_cli(tmp_path, name, flags)
    assert r.returncode == 0, r.stderr[-2000:]
    # the reference's result lines
    m = re.search(r"Total host execution time: ([0-9.]+) ms", r.stdout)
    assert m and float(m.group(1)) > 0
    for key in ("Total device core execution time:", "Total device execution time:", "Partitioned hypergraph:",
                "Nodes:", "Hyperedges:", "Total pins:", "Cut-net:", "Connectivity:", "SOED:"):
        assert key in r.stdout, key
    res = r.stdout[r.stdout.index("Partitioned hypergraph:"):]  # the result block, after the input's summary
    conn = float(re.search(r"Connectivity:\s+([0-9.eE+-]+)", res).group(1))
    nodes = int(float(re.search(r"Nodes:\s+([0-9.]+)", res).group(1)))
    g = ax.read(os.path.join(GOLDEN, name))
    part = ax.read_partition(str(pf), g.n)
    assert int(part.max()) + 1 == nodes
    if params is not None:
        # the same partition and lambda-1 as the library, and the grader agrees
        with ax.Context(0, 1 << 30) as ctx:
            lib_part, st = ctx.partition(g, params)
        np.testing.assert_array_equal(part, lib_part)
        assert abs(conn - st.connectivity) <= 1e-3 * max(1.0, st.connectivity)
        gr = O.ref_grade(os.path.join(GOLDEN, name), str(pf), *grade_args)
        assert gr["valid"] and abs(gr["Connectivity"] - st.connectivity) <= 1e-3 * max(1.0, st.connectivity)
    # -s: the quotient hypergraph as written reads back equal to the library's construction
    q = ax.read(str(sf))
    qr = ax.quotient(g, part)
    if name.endswith(".hgr"):
        qr = as_hmetis(qr)
    assert q.n == qr.n and q.e == qr.e
    np.testing.assert_array_equal(q.off, qr.off)
    np.testing.assert_array_equal(q.pins, qr.pins)
    np.testing.assert_array_equal(q.nsrc, qr.nsrc)
    np.testing.assert_allclose(q.w, qr.w, rtol=1e-6)


def as_hmetis(q):
    """What an .hgr file keeps of a hypergraph (savehMETIS, includes/hgraph.hpp:1016-1051, read back
    by loadhMETIS): weights as uint32(w * 1024) when any weight is not 1, no sources, and nets of
    one pin dropped by the reader."""
    lens = (q.off[1:] - q.off[:-1]).astype(np.int64)
    keep = lens >= 2
    scaled = (q.w != 1.0).any()
    segs = [q.pins[int(q.off[h]):int(q.off[h + 1])] for h in range(q.e) if keep[h]]
    off = np.zeros(int(keep.sum()) + 1, np.uint64)
    off[1:] = np.cumsum(lens[keep])
    w = q.w[keep]
    w = np.floor(w * np.float32(1024.0)).astype(np.float32) if scaled else np.ones(len(w), np.float32)
    pins = np.concatenate(segs).astype(np.uint32) if segs else np.zeros(0, np.uint32)
    return ax.Hypergraph(q.n, off, pins, np.zeros(len(w), np.uint32), w)


def test_cli_reports_errors_like_the_reference(tmp_path):
    """A missing input file ends with a non-zero status and a message, as the reference's
    loadHgraph does (sources/runconfig.cpp:175-178)."""
    r = subprocess.run([CLI, "-r", str(tmp_path / "missing.snn")], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and r.stderr.strip()
