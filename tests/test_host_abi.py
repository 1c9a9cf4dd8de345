"""The C-ABI library without a GPU: it loads, exports every symbol include/axc.h declares, and its
host-side readers, writers and generators agree with the oracle. No kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import axoncuda_b200 as ax
from conftest import GOLDEN, GOLDEN_INPUTS, ROOT
from oracle import oracle as O


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "axc.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(axc_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = ax.lib()
    declared = header_symbols()
    assert declared, "no declarations parsed"
    for s in declared:
        assert hasattr(L, s), s
    assert set(ax.EXPORTS) <= set(declared)


@pytest.mark.parametrize("name", GOLDEN_INPUTS)
def test_host_reader_matches_oracle(name):
    path = os.path.join(GOLDEN, name)
    g = ax.read(path)
    n, off, pins, ns, w = O.read(path)
    assert g.n == n
    np.testing.assert_array_equal(g.off, off)
    np.testing.assert_array_equal(g.pins, pins)
    np.testing.assert_array_equal(g.nsrc, ns)
    np.testing.assert_array_equal(g.w, w)


@pytest.mark.parametrize("ext", [".snn", ".axh", ".hgr"])
def test_writer_roundtrip(tmp_path, ext):
    g = ax.gen_snn(4, 32, 5, 0.0, 0, 1.0, 3)
    p = str(tmp_path / ("x" + ext))
    ax.write(p, g)
    h = ax.read(p)
    np.testing.assert_array_equal(h.pins, g.pins)
    np.testing.assert_array_equal(h.off, g.off)
    if ext == ".hgr":  # hMETIS has no sources
        assert (h.nsrc == 0).all()
    else:
        np.testing.assert_array_equal(h.nsrc, g.nsrc)


@pytest.mark.parametrize("fmt", [0, 1, 11])
def test_parallel_hgr_parse_matches_line_reader(tmp_path, fmt):
    """The .hgr reader splits the text over threads; a large file with comments, blank and
    CRLF lines, tabs, singleton nets, weights and trailing lines must read exactly as the
    oracle's line-by-line restatement of the reference reader reads it."""
    rng = np.random.default_rng(fmt)
    g = ax.gen_circuit(40000, 44000, 2, 64, 2.5, 0.9, 0.02, 9)
    lines = [f"% generated\n", f"{g.e + 50} {g.n} {fmt}\n" if fmt else f"{g.e + 50} {g.n}\n"]
    nets = [g.pins[g.off[i]:g.off[i + 1]] + 1 for i in range(g.e)]
    nets += [np.array([rng.integers(1, g.n + 1)]) for _ in range(50)]  # singletons: skipped
    order = rng.permutation(len(nets))
    for i in order:
        toks = " ".join(map(str, nets[i].tolist()))
        if fmt in (1, 11):
            toks = f"{rng.integers(1, 9) * 0.5} " + toks
        r = rng.random()
        if r < 0.05:
            lines.append("\n")
        elif r < 0.08:
            lines.append("  % a comment line\n")
        if r < 0.3:
            toks = "\t " + toks.replace(" ", "\t", 3)
        lines.append(toks + ("\r\n" if r > 0.9 else "\n"))
    lines += [f"{i + 1}\n" for i in range(5)]  # vertex weights (fmt 10/11) or junk: ignored
    p = tmp_path / "big.hgr"
    p.write_text("".join(lines))
    h = ax.read(str(p))
    n, off, pins, ns, w = O.read(str(p))
    assert h.n == n and h.e == len(off) - 1
    np.testing.assert_array_equal(h.off, off)
    np.testing.assert_array_equal(h.pins, pins)
    np.testing.assert_array_equal(h.nsrc, ns)
    np.testing.assert_array_equal(h.w, w)
    # one net short: the reader fails as the line reader does
    q = tmp_path / "short.hgr"
    body = "".join(lines[:-5])
    q.write_text(body.replace(f"{g.e + 50} {g.n}", f"{g.e + 56} {g.n}", 1))
    with pytest.raises(ax.AxcError) as e:
        ax.read(str(q))
    assert e.value.code == 5


def test_partition_file_roundtrip(tmp_path):
    part = np.array([0, 3, 2, 2, 1], np.uint32)
    p = str(tmp_path / "p.txt")
    L = ax.lib()
    assert L.axc_write_partition(p.encode(), part.ctypes.data_as(C.POINTER(C.c_uint32)), 5) == 0
    assert open(p).read() == "0\n3\n2\n2\n1\n"
    out = np.zeros(5, np.uint32)
    assert L.axc_read_partition(p.encode(), 5, out.ctypes.data_as(C.POINTER(C.c_uint32))) == 0
    np.testing.assert_array_equal(out, part)
    # more entries than nodes / trailing data are rejected (includes/hgraph.hpp:1070-1080)
    assert L.axc_read_partition(p.encode(), 4, out.ctypes.data_as(C.POINTER(C.c_uint32))) == 5
    open(p, "w").write("1 2\n")
    assert L.axc_read_partition(p.encode(), 1, out.ctypes.data_as(C.POINTER(C.c_uint32))) == 5


def test_malformed_inputs_are_rejected(tmp_path):
    bad = tmp_path / "bad.hgr"
    bad.write_text("2 3\n1 4\n")  # node 4 > V
    with pytest.raises(ax.AxcError) as e:
        ax.read(str(bad))
    assert e.value.code == 5
    with pytest.raises(ax.AxcError) as e:
        ax.read(str(tmp_path / "missing.snn"))
    assert e.value.code == 4
    trunc = tmp_path / "t.snn"
    trunc.write_bytes(np.array([3, 1, 2, 0], np.uint32).tobytes())
    with pytest.raises(ax.AxcError):
        ax.read(str(trunc))


def test_generators_follow_the_workload_shapes():
    g0 = ax.gen_snn(8, 512, 64, 0.0, 0, 1.0, 0)
    assert (g0.n, g0.e, g0.P) == (4096, 3584, 3584 * 65)
    h = np.diff(g0.off.astype(np.int64))
    assert (h == 65).all() and (g0.nsrc == 1).all()
    # destinations of neuron i's hyperedge lie in the next layer, without repeats
    for i in (0, 777, 3583):
        d = g0.pins[g0.off[i] + 1:g0.off[i + 1]]
        assert len(set(d.tolist())) == 64
        assert ((d // 512) == (i // 512 + 1)).all()
    g1 = ax.gen_circuit(20000, 22000, 2, 64, 2.5, 0.9, 0.02, 1)
    s = np.diff(g1.off.astype(np.int64))
    assert s.min() >= 2 and s.max() <= 64 and 3.5 < s.mean() < 4.5
    assert (g1.nsrc == 0).all()
    a = ax.gen_circuit(5000, 5000, 2, 64, 2.5, 0.9, 0.02, 5)
    b = ax.gen_circuit(5000, 5000, 2, 64, 2.5, 0.9, 0.02, 5)
    c = ax.gen_circuit(5000, 5000, 2, 64, 2.5, 0.9, 0.02, 6)
    np.testing.assert_array_equal(a.pins, b.pins)
    assert not np.array_equal(a.pins[:1000], c.pins[:1000])


def test_quotient_hypergraph_connectivity_matches_metric():
    g = ax.gen_circuit(3000, 3300, 2, 16, 2.5, 0.9, 0.02, 4)
    part = (np.arange(g.n) * 5 // g.n).astype(np.uint32)
    L = ax.lib()
    q = ax.HGraph()
    assert L.axc_quotient_hgraph(C.byref(g.c()), part.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(q)) == 0
    Q = ax.Hypergraph.from_c(q)
    L.axc_free_hgraph(C.byref(q))
    lam_minus_1 = float(np.sum(Q.w.astype(np.float64) * (np.diff(Q.off.astype(np.int64)) - 1)))
    ev = O.evaluate(g.n, g.off, g.pins, g.nsrc, g.w, part, g.n, 1 << 30, 5)
    assert abs(lam_minus_1 - ev["connectivity_fx"] / 262144.0) < 1e-6


def test_context_entry_points_reject_missing_arguments():
    """Calls that need a context return AXC_EINVAL for a missing one before touching a GPU."""
    g = ax.gen_circuit(100, 110, 2, 8, 2.5, 0.9, 0.02, 1)
    part = np.zeros(g.n, np.uint32)
    L = ax.lib()
    q = ax.HGraph()
    pp = part.ctypes.data_as(C.POINTER(C.c_uint32))
    assert L.axc_quotient_hgraph_device(None, C.byref(g.c()), pp, C.byref(q)) == 1
    p = ax.params_kway(2, 0.03)
    st = ax.Stats()
    assert L.axc_partition(None, C.byref(g.c()), C.byref(p), pp, C.byref(st)) == 1
    assert L.axc_evaluate(None, C.byref(g.c()), C.byref(p), pp, C.byref(st)) == 1
    assert L.axc_serve_configure(None, 2, 0) == 1


def test_kway_omega_matches_reference_rule():
    # ceil((1 + eps) * n / k) in float (sources/runconfig.cpp:190)
    for n, k, e in ((200000, 2, 0.03), (200000, 64, 0.03), (1000000, 128, 0.03), (4097, 3, 0.1)):
        want = int(np.ceil(np.float32(1 + np.float32(e)) * np.float32(n) / np.float32(k)))
        assert ax.kway_omega(n, k, e) == want
