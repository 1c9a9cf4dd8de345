"""ctypes binding of oracle/liboracle.so — TEST INFRASTRUCTURE ONLY.

The oracle is the CPU restatement of the partitioner's stages (oracle/oracle.cpp). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, as the checker or as
the timed CPU port; the product path (axoncuda_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
NONE = 0xFFFFFFFF

_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def read(path: str):
    """Returns (n, off, pins, nsrc, w) as loaded by the restated readers."""
    L = lib()
    n, e, P = C.c_uint32(), C.c_uint32(), C.c_uint64()
    rc = L.or_read(path.encode(), C.byref(n), C.byref(e), C.byref(P), None, None, None, None)
    if rc:
        raise IOError(f"or_read failed ({rc})")
    off = np.zeros(e.value + 1, np.uint64)
    pins = np.zeros(max(P.value, 1), np.uint32)
    ns = np.zeros(max(e.value, 1), np.uint32)
    w = np.zeros(max(e.value, 1), np.float32)
    L.or_read(path.encode(), C.byref(n), C.byref(e), C.byref(P), _p(off, C.c_uint64), _p(pins, C.c_uint32),
              _p(ns, C.c_uint32), _p(w, C.c_float))
    return n.value, off, pins[: P.value], ns[: e.value], w[: e.value]


def wfx(w):
    L = lib()
    L.or_wfx.restype = C.c_uint32
    L.or_wfx.argtypes = [C.c_float]
    return np.array([L.or_wfx(float(x)) for x in w], np.uint32)


def dedupe(off, pins, nsrc):
    off, pins, nsrc = _u64(off), _u32(pins), _u32(nsrc)
    e = len(nsrc)
    o2 = np.zeros(e + 1, np.uint64); p2 = np.zeros(max(len(pins), 1), np.uint32); n2 = np.zeros(max(e, 1), np.uint32)
    L = lib()
    L.or_dedupe.restype = C.c_uint64
    P = L.or_dedupe(C.c_uint32(e), _p(off, C.c_uint64), _p(pins, C.c_uint32), _p(nsrc, C.c_uint32),
                    _p(o2, C.c_uint64), _p(p2, C.c_uint32), _p(n2, C.c_uint32))
    return o2, p2[:P], n2[:e]


def touching(n, off, pins, nsrc):
    off, pins, nsrc = _u64(off), _u32(pins), _u32(nsrc)
    toff = np.zeros(n + 1, np.uint64); touch = np.zeros(max(len(pins), 1), np.uint32)
    nin = np.zeros(max(n, 1), np.uint32)
    lib().or_touching(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                      _p(nsrc, C.c_uint32), _p(toff, C.c_uint64), _p(touch, C.c_uint32), _p(nin, C.c_uint32))
    return toff, touch[: len(pins)], nin[:n]


RATE_MAX_LEN = 128  # include/axc.h AXC_RATE_MAX_LEN
NO_LEN_LIMIT = (1 << 64) - 1


def rating(n, off, pins, nsrc, wfx_, node_size, omega, delta, cnc, max_len=RATE_MAX_LEN):
    """Top-cnc candidates per node; hyperedges longer than max_len pins take no part (NO_LEN_LIMIT
    rates through all of them, as the reference does)."""
    off, pins, nsrc, wfx_, ns = _u64(off), _u32(pins), _u32(nsrc), _u32(wfx_), _u32(node_size)
    toff, touch, nin = touching(n, off, pins, nsrc)
    pairs = np.zeros(max(n * cnc, 1), np.uint32); scores = np.zeros(max(n * cnc, 1), np.uint32)
    lib().or_rating_len(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                        _p(nsrc, C.c_uint32), _p(wfx_, C.c_uint32), _p(toff, C.c_uint64), _p(touch, C.c_uint32),
                        _p(nin, C.c_uint32), _p(ns, C.c_uint32), C.c_uint32(omega), C.c_uint32(delta),
                        C.c_uint32(cnc), C.c_uint64(max_len), _p(pairs, C.c_uint32), _p(scores, C.c_uint32))
    return pairs[: n * cnc], scores[: n * cnc]


def matching(n, cnc, pairs, scores, node_size, inbound, omega, delta, rounds=32):
    pairs, scores, ns, nin = _u32(pairs), _u32(scores), _u32(node_size), _u32(inbound)
    groups = np.zeros(max(n, 1), np.uint32)
    L = lib()
    L.or_matching.restype = C.c_uint32
    ng = L.or_matching(C.c_uint32(n), C.c_uint32(cnc), _p(pairs, C.c_uint32), _p(scores, C.c_uint32),
                       _p(ns, C.c_uint32),
                       _p(nin, C.c_uint32), C.c_uint32(omega), C.c_uint32(delta), C.c_uint32(rounds),
                       _p(groups, C.c_uint32))
    return groups[:n], ng


def contract(off, pins, nsrc, groups):
    off, pins, nsrc, groups = _u64(off), _u32(pins), _u32(nsrc), _u32(groups)
    e = len(nsrc)
    o2 = np.zeros(e + 1, np.uint64); p2 = np.zeros(max(len(pins), 1), np.uint32); n2 = np.zeros(max(e, 1), np.uint32)
    L = lib()
    L.or_contract.restype = C.c_uint64
    P = L.or_contract(C.c_uint32(e), _p(off, C.c_uint64), _p(pins, C.c_uint32), _p(nsrc, C.c_uint32),
                      _p(groups, C.c_uint32), _p(o2, C.c_uint64), _p(p2, C.c_uint32), _p(n2, C.c_uint32))
    return o2, p2[:P], n2[:e]


def gains(n, off, pins, nsrc, wfx_, node_size, part, num_parts, omega, delta, encourage, discount, rnd=0, seed=0):
    off, pins, nsrc, wfx_, ns, part = _u64(off), _u32(pins), _u32(nsrc), _u32(wfx_), _u32(node_size), _u32(part)
    toff, touch, nin = touching(n, off, pins, nsrc)
    tgt = np.zeros(max(n, 1), np.uint32); gain = np.zeros(max(n, 1), np.int64)
    lib().or_gains(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                   _p(nsrc, C.c_uint32), _p(wfx_, C.c_uint32), _p(toff, C.c_uint64), _p(touch, C.c_uint32),
                   _p(nin, C.c_uint32), _p(ns, C.c_uint32), _p(part, C.c_uint32), C.c_uint32(num_parts),
                   C.c_uint32(omega), C.c_uint32(delta), C.c_int(int(encourage)), C.c_uint32(discount),
                   C.c_uint32(rnd), C.c_uint64(seed), _p(tgt, C.c_uint32), _p(gain, C.c_int64))
    return tgt[:n], gain[:n]


def refine(n, off, pins, nsrc, wfx_, node_size, part, num_parts, omega, delta, encourage, rounds, seed=0):
    off, pins, nsrc, wfx_, ns = _u64(off), _u32(pins), _u32(nsrc), _u32(wfx_), _u32(node_size)
    toff, touch, nin = touching(n, off, pins, nsrc)
    pv = np.array(part, dtype=np.uint32, copy=True)
    if len(pv) == 0:
        pv = np.zeros(1, np.uint32)
    lib().or_refine(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                    _p(nsrc, C.c_uint32), _p(wfx_, C.c_uint32), _p(toff, C.c_uint64), _p(touch, C.c_uint32),
                    _p(nin, C.c_uint32), _p(ns, C.c_uint32), _p(pv, C.c_uint32), C.c_uint32(num_parts),
                    C.c_uint32(omega), C.c_uint32(delta), C.c_int(int(encourage)), C.c_uint32(rounds),
                    C.c_uint64(seed))
    return pv[:n]


def evaluate(n, off, pins, nsrc, w, part, omega, delta, max_parts):
    off, pins, nsrc, part = _u64(off), _u32(pins), _u32(nsrc), _u32(part)
    w = np.ascontiguousarray(w, dtype=np.float32)
    out = np.zeros(8, np.int64)
    lib().or_evaluate(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                      _p(nsrc, C.c_uint32), _p(w, C.c_float), _p(part, C.c_uint32), C.c_uint32(omega),
                      C.c_uint32(delta), C.c_uint32(max_parts), _p(out, C.c_int64))
    keys = ["connectivity_fx", "cutnet_fx", "soed_fx", "num_parts", "max_size", "max_inbound", "valid", "dense"]
    return dict(zip(keys, (int(x) for x in out)))


def partition(n, off, pins, nsrc, w, mode, omega=0, delta=0, max_parts=0, k=0, eps=0.0, cnc=4, rfr=16, ipm=1,
              seed=0):
    """The whole partitioner on the CPU (single thread). Returns (part, num_parts, levels, pins)."""
    off, pins, nsrc = _u64(off), _u32(pins), _u32(nsrc)
    w = np.ascontiguousarray(w, dtype=np.float32)
    part = np.zeros(max(n, 1), np.uint32)
    stats = np.zeros(2, np.uint64)
    L = lib()
    L.or_partition.restype = C.c_uint32
    K = L.or_partition(C.c_uint32(n), C.c_uint32(len(nsrc)), _p(off, C.c_uint64), _p(pins, C.c_uint32),
                       _p(nsrc, C.c_uint32), _p(w, C.c_float), C.c_int(mode), C.c_uint32(omega), C.c_uint32(delta),
                       C.c_uint32(max_parts), C.c_uint32(k), C.c_float(eps), C.c_uint32(cnc), C.c_uint32(rfr),
                       C.c_int(ipm), C.c_uint64(seed), _p(part, C.c_uint32), _p(stats, C.c_uint64))
    return part[:n], int(K), int(stats[0]), int(stats[1])


# ---- the reference's own tools, compiled here from its sources (oracle/Makefile `ref`) ----
def ref_tool(name: str) -> str:
    return os.path.join(REF_DIR, name)


def ref_dump(path: str):
    """Runs refharness.exe (reference HyperGraph code) and parses its three sections."""
    import tempfile
    with tempfile.NamedTemporaryFile(suffix=".bin") as t:
        subprocess.run([ref_tool("refharness.exe"), "dump", path, t.name], check=True, capture_output=True)
        buf = open(t.name, "rb").read()
    pos = 0

    def take(dt, cnt):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=cnt, offset=pos).copy()
        pos += a.nbytes
        return a

    def graph():
        n, e = take(np.uint32, 2)
        P = int(take(np.uint64, 1)[0])
        off = take(np.uint64, int(e) + 1)
        pins = take(np.uint32, P)
        ns = take(np.uint32, int(e))
        w = take(np.float32, int(e))
        return int(n), off, pins, ns, w

    raw = graph()
    ded = graph()
    n = ded[0]
    toff = take(np.uint64, n + 1)
    touch = take(np.uint32, int(toff[-1]))
    nin = take(np.uint32, n)
    return raw, ded, (toff, touch, nin)


def ref_grade(hg_path: str, part_path: str, mode: str, *args) -> dict:
    """Runs the reference grader (grading/grade.cpp) and parses its metric lines."""
    flag = {"incc": "-m-prt", "kway": "-k-prt"}[mode]
    r = subprocess.run([ref_tool("hgrade.exe"), "-r", hg_path, "-prt", part_path, flag, *map(str, args)],
                       capture_output=True, text=True)
    out = {"rc": r.returncode, "valid": "invalid partitioning" not in r.stderr and r.returncode == 0}
    for line in r.stdout.splitlines():
        s = line.strip()
        for key in ("Cut-net", "Connectivity", "SOED", "Nodes", "Hyperedges", "Total pins"):
            if s.startswith(key + ":"):
                out.setdefault(key, float(s.split(":", 1)[1].split()[0]))
    return out
