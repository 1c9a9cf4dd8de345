"""axoncuda_b200 — Python binding of the B200-native hypergraph partitioner's C ABI.

The product is the native library ``libaxc.so`` (include/axc.h); this module is a thin ctypes
client used by the tests and the benchmark, mirroring the reference's process surface
(``hgraph_gpu.exe -r <file> -m Ω Δ K | -k k ε``, sources/runconfig.cpp:25-46). There is no CPU
fallback: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaxc.so")

MODE_INCC = 0
MODE_KWAY = 1
MAX_CANDIDATES = 16
FIXED_POINT_SCALE = 262144
RATE_MAX_LEN = 128  # AXC_RATE_MAX_LEN: longer hyperedges take no part in the rating

STATUS = {
    0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error", 4: "I/O error",
    5: "malformed input", 6: "infeasible", 7: "timed out", 8: "unknown job", 9: "admission refused",
    10: "internal device check failed", 11: "size exceeds limit", 12: "canceled at shutdown",
}


class AxcError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        super().__init__(f"axc status {code} ({STATUS.get(code, '?')}){': ' + msg if msg else ''}")
        self.code = code


class HGraph(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("e", C.c_uint32),
        ("hedge_off", C.POINTER(C.c_uint64)), ("pins", C.POINTER(C.c_uint32)),
        ("src_count", C.POINTER(C.c_uint32)), ("hedge_w", C.POINTER(C.c_float)),
        ("_owner", C.c_void_p),
    ]


class Params(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("omega", C.c_uint32), ("delta", C.c_uint32), ("max_parts", C.c_uint32),
        ("k", C.c_uint32), ("eps", C.c_float), ("cnc", C.c_uint32), ("rfr", C.c_uint32),
        ("smh", C.c_uint32), ("ipm", C.c_int), ("om", C.c_float), ("seed", C.c_uint64),
        ("verbose", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("num_parts", C.c_uint32), ("levels", C.c_uint32), ("pins", C.c_uint64),
        ("connectivity_fx", C.c_int64), ("cutnet_fx", C.c_int64), ("soed_fx", C.c_int64),
        ("connectivity", C.c_double), ("cutnet", C.c_double), ("soed", C.c_double),
        ("max_part_size", C.c_uint32), ("max_part_inbound", C.c_uint32), ("valid", C.c_int),
        ("ms_device", C.c_double), ("ms_core", C.c_double), ("kernel_launches", C.c_uint32),
        ("level_pins", C.c_uint64 * 64), ("level_nodes", C.c_uint32 * 64),
        ("refine_rounds", C.c_uint32 * 64), ("rating_pin_visits", C.c_uint64),
        ("device_bytes_peak", C.c_uint64), ("ms_queued", C.c_double), ("ms_run", C.c_double),
    ]


class KernelTiming(C.Structure):
    """axc_kernel_timing: launches, summed event-timed duration and algorithmic bytes of one kernel."""
    _fields_ = [("launches", C.c_uint32), ("ms_total", C.c_double), ("bytes", C.c_uint64)]


# Every symbol include/axc.h declares (tests check the library exports all of them).
EXPORTS = [
    "axc_create", "axc_destroy", "axc_strerror", "axc_last_error", "axc_params_default",
    "axc_params_preset", "axc_kway_omega", "axc_partition", "axc_partition_device", "axc_evaluate",
    "axc_read_hgr", "axc_read_snn", "axc_read_axh", "axc_read_auto", "axc_free_hgraph",
    "axc_write_hgraph", "axc_write_partition", "axc_read_partition", "axc_quotient_hgraph",
    "axc_quotient_hgraph_device",
    "axc_gen_snn", "axc_gen_circuit", "axc_submit", "axc_poll", "axc_partition_batch",
    "axc_stage_construct", "axc_stage_rating", "axc_stage_matching", "axc_stage_contract",
    "axc_stage_gains", "axc_stage_refine", "axc_profile_kernel", "axc_profile_read", "axc_connectivity_noalloc",
    "axc_serve_configure", "axc_selftest_bounded_wait", "axc_tune_set",
]

_lib = None


def lib() -> C.CDLL:
    """Load libaxc.so (built in-tree by ``make -C axoncuda_b200``); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C axoncuda_b200`")
        L = C.CDLL(LIB_PATH)
        P, H, S = C.POINTER(Params), C.POINTER(HGraph), C.POINTER(Stats)
        u32p, u64p, i64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_int64)
        sig = {
            "axc_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
            "axc_destroy": (None, [C.c_void_p]),
            "axc_strerror": (C.c_char_p, [C.c_int]),
            "axc_last_error": (C.c_char_p, [C.c_void_p]),
            "axc_params_default": (None, [P, C.c_int]),
            "axc_params_preset": (C.c_int, [P, C.c_char_p]),
            "axc_kway_omega": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_float]),
            "axc_partition": (C.c_int, [C.c_void_p, H, P, u32p, S]),
            "axc_partition_device": (C.c_int, [C.c_void_p, H, P, u32p, S]),
            "axc_evaluate": (C.c_int, [C.c_void_p, H, P, u32p, S]),
            "axc_read_auto": (C.c_int, [C.c_char_p, H]),
            "axc_read_hgr": (C.c_int, [C.c_char_p, H]),
            "axc_read_snn": (C.c_int, [C.c_char_p, H]),
            "axc_read_axh": (C.c_int, [C.c_char_p, H]),
            "axc_free_hgraph": (None, [H]),
            "axc_write_hgraph": (C.c_int, [C.c_char_p, H]),
            "axc_write_partition": (C.c_int, [C.c_char_p, u32p, C.c_uint32]),
            "axc_read_partition": (C.c_int, [C.c_char_p, C.c_uint32, u32p]),
            "axc_quotient_hgraph": (C.c_int, [H, u32p, H]),
            "axc_quotient_hgraph_device": (C.c_int, [C.c_void_p, H, u32p, H]),
            "axc_gen_snn": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32,
                                      C.c_double, C.c_uint64, H]),
            "axc_gen_circuit": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                          C.c_double, C.c_double, C.c_uint64, H]),
            "axc_submit": (C.c_int, [C.c_void_p, H, P, u64p]),
            "axc_poll": (C.c_int, [C.c_void_p, C.c_uint64, u32p, S, C.c_int]),
            "axc_stage_construct": (C.c_int, [C.c_void_p, H, u64p, u32p, u32p, u64p, u32p, u32p, u64p]),
            "axc_stage_rating": (C.c_int, [C.c_void_p, H, u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                                           C.c_uint64, u32p, u32p]),
            "axc_stage_matching": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p,
                                             C.c_uint32, C.c_uint32, u32p, u32p]),
            "axc_stage_contract": (C.c_int, [C.c_void_p, H, u32p, C.c_uint32, u64p, u32p, u32p, u64p]),
            "axc_stage_gains": (C.c_int, [C.c_void_p, H, u32p, C.c_uint32, u32p, C.c_uint32, C.c_uint32,
                                          C.c_int, C.c_uint32, u32p, i64p]),
            "axc_stage_refine": (C.c_int, [C.c_void_p, H, u32p, C.c_uint32, u32p, C.c_uint32, C.c_uint32,
                                           C.c_int, C.c_uint32, C.c_uint64, u32p, u32p]),
        }
        sig["axc_profile_kernel"] = (C.c_int, [C.c_void_p, C.c_char_p])
        sig["axc_profile_read"] = (C.c_int, [C.c_void_p, C.POINTER(KernelTiming)])
        sig["axc_connectivity_noalloc"] = (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.c_void_p, C.POINTER(C.c_int64)])
        sig["axc_serve_configure"] = (C.c_int, [C.c_void_p, C.c_uint32, C.c_size_t])
        sig["axc_partition_batch"] = (C.c_int, [C.c_void_p, C.c_uint32, H, P, C.POINTER(u32p), S])
        sig["axc_tune_set"] = (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint64])
        sig["axc_selftest_bounded_wait"] = (C.c_int, [C.c_void_p, C.c_uint32])
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


@dataclass
class Hypergraph:
    """Host hypergraph in the reference layout (sources first per hyperedge)."""
    n: int
    off: np.ndarray      # uint64 [e+1]
    pins: np.ndarray     # uint32 [P]
    nsrc: np.ndarray     # uint32 [e]
    w: np.ndarray        # float32 [e]

    @property
    def e(self) -> int:
        return len(self.nsrc)

    @property
    def P(self) -> int:
        return int(self.off[-1]) if len(self.off) else 0

    def c(self) -> HGraph:
        self.off = np.ascontiguousarray(self.off, dtype=np.uint64)
        self.pins = np.ascontiguousarray(self.pins, dtype=np.uint32)
        self.nsrc = np.ascontiguousarray(self.nsrc, dtype=np.uint32)
        self.w = np.ascontiguousarray(self.w, dtype=np.float32)
        return HGraph(self.n, self.e, _ptr(self.off, C.c_uint64), _ptr(self.pins, C.c_uint32),
                      _ptr(self.nsrc, C.c_uint32), _ptr(self.w, C.c_float), None)

    @staticmethod
    def from_c(g: HGraph) -> "Hypergraph":
        e = g.e
        off = np.ctypeslib.as_array(g.hedge_off, shape=(e + 1,)).copy() if e else np.zeros(1, np.uint64)
        P = int(off[-1])
        pins = np.ctypeslib.as_array(g.pins, shape=(P,)).copy() if P else np.zeros(0, np.uint32)
        nsrc = np.ctypeslib.as_array(g.src_count, shape=(e,)).copy() if e else np.zeros(0, np.uint32)
        w = (np.ctypeslib.as_array(g.hedge_w, shape=(e,)).copy() if (e and g.hedge_w)
             else np.ones(e, np.float32))
        return Hypergraph(int(g.n), off, pins, nsrc, w)


def _owned(fn, *args) -> Hypergraph:
    g = HGraph()
    rc = fn(*args, C.byref(g))
    if rc:
        raise AxcError(rc)
    try:
        return Hypergraph.from_c(g)
    finally:
        lib().axc_free_hgraph(C.byref(g))


def read(path: str) -> Hypergraph:
    """HyperGraph::loadhMETIS / loadSNN / loadAXH by extension (sources/runconfig.cpp:153-184)."""
    return _owned(lib().axc_read_auto, path.encode())


def write(path: str, g: Hypergraph) -> None:
    rc = lib().axc_write_hgraph(path.encode(), C.byref(g.c()))
    if rc:
        raise AxcError(rc)


def read_partition(path: str, n: int) -> np.ndarray:
    """HyperGraph::loadPartitioning (includes/hgraph.hpp:1062-1083): n partition ids."""
    out = np.zeros(max(n, 1), np.uint32)
    rc = lib().axc_read_partition(path.encode(), n, _ptr(out, C.c_uint32))
    if rc:
        raise AxcError(rc, path)
    return out[:n]


def quotient(g: Hypergraph, part: np.ndarray) -> Hypergraph:
    """The quotient hypergraph of `-s` built on the host (axc_quotient_hgraph)."""
    part = np.ascontiguousarray(part, dtype=np.uint32)
    return _owned(lib().axc_quotient_hgraph, C.byref(g.c()), _ptr(part, C.c_uint32))


def gen_snn(layers, width, fanout, sigma=0.0, cap=0, p_next=1.0, seed=0) -> Hypergraph:
    return _owned(lib().axc_gen_snn, layers, width, float(fanout), float(sigma), cap, float(p_next), seed)


def gen_circuit(n, e, smin=2, smax=64, alpha=2.5, p_local=0.9, local_frac=0.02, seed=1) -> Hypergraph:
    return _owned(lib().axc_gen_circuit, n, e, smin, smax, float(alpha), float(p_local),
                  float(local_frac), seed)


# The workloads: layered SNN (8 x 512, fan-out 64), circuit netlist (200k nodes, 220k nets),
# large SNN (20 x 50k, lognormal fan-out) and its 20 x 5k version, each with its run parameters.
def workload(name: str) -> tuple[Hypergraph, "Params"]:
    if name == "snn-8x512":
        return gen_snn(8, 512, 64, 0.0, 0, 1.0, 0), params_incc(128, 1024, 1048576, cnc=4, rfr=16, ipm=1)
    if name in ("circuit-200k-k2", "circuit-200k-k64"):
        k = 2 if name.endswith("k2") else 64
        return gen_circuit(200000, 220000, 2, 64, 2.5, 0.9, 0.02, 1), params_kway(k, 0.03, cnc=4, rfr=16)
    if name == "snn-100k-incc":  # the large SNN's generator at 20 x 5k: a profiling-size INCC case
        g = gen_snn(20, 5000, 256, 0.8, 2048, 0.7, 2)
        return g, params_incc(1024, 4096, 1048576, cnc=4, rfr=16, ipm=1)
    if name in ("snn-1m-incc", "snn-1m-k128"):
        g = gen_snn(20, 50000, 256, 0.8, 2048, 0.7, 2)
        if name.endswith("incc"):
            return g, params_incc(1024, 4096, 1048576, cnc=4, rfr=16, ipm=1)
        return g, params_kway(128, 0.03, cnc=4, rfr=16)
    raise KeyError(name)


def params_incc(omega, delta, max_parts, cnc=4, rfr=16, ipm=1, seed=0) -> Params:
    p = Params()
    lib().axc_params_default(C.byref(p), MODE_INCC)
    p.omega, p.delta, p.max_parts, p.cnc, p.rfr, p.ipm, p.seed = omega, delta, max_parts, cnc, rfr, ipm, seed
    return p


def params_kway(k, eps, cnc=4, rfr=16, seed=0) -> Params:
    p = Params()
    lib().axc_params_default(C.byref(p), MODE_KWAY)
    p.k, p.eps, p.cnc, p.rfr, p.seed = k, eps, cnc, rfr, seed
    return p


def kway_omega(n: int, k: int, eps: float) -> int:
    return int(lib().axc_kway_omega(n, k, eps))


class Context:
    """One device context (include/axc.h axc_create / axc_destroy)."""

    def __init__(self, device: int = 0, arena_bytes: int = 0):
        self._h = C.c_void_p()
        rc = lib().axc_create(device, arena_bytes, C.byref(self._h))
        if rc:
            raise AxcError(rc, "axc_create")

    def close(self):
        if self._h:
            lib().axc_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int, what: str):
        if rc:
            raise AxcError(rc, f"{what}: {lib().axc_last_error(self._h).decode(errors='replace')}")

    def profile_kernel(self, name: str | None):
        """Time every launch of the named kernel with CUDA events on the context stream."""
        self._check(lib().axc_profile_kernel(self._h, name.encode() if name else None), "axc_profile_kernel")

    def profile_read(self) -> KernelTiming:
        """Launches, summed duration (ms) and algorithmic bytes since the last read; resets them."""
        t = KernelTiming()
        self._check(lib().axc_profile_read(self._h, C.byref(t)), "axc_profile_read")
        return t

    def partition(self, g: Hypergraph, p: Params) -> tuple[np.ndarray, Stats]:
        out = np.zeros(max(g.n, 1), np.uint32)
        st = Stats()
        self._check(lib().axc_partition(self._h, C.byref(g.c()), C.byref(p), _ptr(out, C.c_uint32),
                                        C.byref(st)), "axc_partition")
        return out[: g.n], st

    def evaluate(self, g: Hypergraph, p: Params, part: np.ndarray) -> Stats:
        part = np.ascontiguousarray(part, dtype=np.uint32)
        st = Stats()
        self._check(lib().axc_evaluate(self._h, C.byref(g.c()), C.byref(p), _ptr(part, C.c_uint32),
                                       C.byref(st)), "axc_evaluate")
        return st

    def quotient(self, g: Hypergraph, part: np.ndarray) -> Hypergraph:
        """The quotient hypergraph written by `-s` (axc_quotient_hgraph_device)."""
        part = np.ascontiguousarray(part, dtype=np.uint32)
        q = HGraph()
        self._check(lib().axc_quotient_hgraph_device(self._h, C.byref(g.c()), _ptr(part, C.c_uint32), C.byref(q)),
                    "axc_quotient_hgraph_device")
        try:
            return Hypergraph.from_c(q)
        finally:
            lib().axc_free_hgraph(C.byref(q))

    def submit(self, g: Hypergraph, p: Params) -> int:
        jid = C.c_uint64()
        self._check(lib().axc_submit(self._h, C.byref(g.c()), C.byref(p), C.byref(jid)), "axc_submit")
        return jid.value

    def poll(self, jid: int, n: int, timeout_ms: int = -1) -> tuple[np.ndarray, Stats]:
        out = np.zeros(max(n, 1), np.uint32)
        st = Stats()
        self._check(lib().axc_poll(self._h, jid, _ptr(out, C.c_uint32), C.byref(st), timeout_ms), "axc_poll")
        return out[:n], st

    def tune(self, key: str, value: int):
        """axc_tune_set: a tile or table size, or an executor setting (see include/axc.h)."""
        self._check(lib().axc_tune_set(self._h, key.encode(), C.c_uint64(value)), "axc_tune_set " + key)

    def serve_configure(self, lanes: int, device_budget: int = 0):
        """Lanes and device-memory budget of the batching / serving executor (before any submit)."""
        self._check(lib().axc_serve_configure(self._h, lanes, device_budget), "axc_serve_configure")

    def partition_batch(self, jobs: list[tuple[Hypergraph, Params]]) -> list[tuple[np.ndarray, Stats]]:
        """All jobs through the executor's lanes in one call (axc_partition_batch)."""
        k = len(jobs)
        hg = (HGraph * k)(*[g.c() for g, _ in jobs])
        ps = (Params * k)(*[p for _, p in jobs])
        outs = [np.zeros(max(g.n, 1), np.uint32) for g, _ in jobs]
        ptrs = (C.POINTER(C.c_uint32) * k)(*[_ptr(o, C.c_uint32) for o in outs])
        sts = (Stats * k)()
        self._check(lib().axc_partition_batch(self._h, k, hg, ps, ptrs, sts), "axc_partition_batch")
        return [(outs[i][: jobs[i][0].n], sts[i]) for i in range(k)]

    # ---- stages (host buffers in/out) ----
    def stage_construct(self, g: Hypergraph):
        P, e, n = g.P, g.e, g.n
        off = np.zeros(e + 1, np.uint64); pins = np.zeros(max(P, 1), np.uint32)
        ns = np.zeros(max(e, 1), np.uint32); toff = np.zeros(n + 1, np.uint64)
        touch = np.zeros(max(P, 1), np.uint32); nin = np.zeros(max(n, 1), np.uint32)
        pa = C.c_uint64()
        self._check(lib().axc_stage_construct(
            self._h, C.byref(g.c()), _ptr(off, C.c_uint64), _ptr(pins, C.c_uint32), _ptr(ns, C.c_uint32),
            _ptr(toff, C.c_uint64), _ptr(touch, C.c_uint32), _ptr(nin, C.c_uint32), C.byref(pa)),
            "axc_stage_construct")
        Pa = pa.value
        return off, pins[:Pa], ns[:e], toff, touch[:Pa], nin[:n]

    def stage_rating(self, g: Hypergraph, node_size, omega, delta, cnc):
        n = g.n
        ns = np.ascontiguousarray(node_size, dtype=np.uint32)
        pairs = np.zeros(max(n * cnc, 1), np.uint32); scores = np.zeros(max(n * cnc, 1), np.uint32)
        self._check(lib().axc_stage_rating(self._h, C.byref(g.c()), _ptr(ns, C.c_uint32), omega, delta, cnc,
                                           0, _ptr(pairs, C.c_uint32), _ptr(scores, C.c_uint32)),
                    "axc_stage_rating")
        return pairs[: n * cnc], scores[: n * cnc]

    def stage_matching(self, n, cnc, pairs, scores, node_size, inbound, omega, delta):
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
        scores = np.ascontiguousarray(scores, dtype=np.uint32)
        ns = np.ascontiguousarray(node_size, dtype=np.uint32)
        nin = np.ascontiguousarray(inbound, dtype=np.uint32)
        out = np.zeros(max(n, 1), np.uint32); ng = C.c_uint32()
        self._check(lib().axc_stage_matching(self._h, n, cnc, _ptr(pairs, C.c_uint32), _ptr(scores, C.c_uint32),
                                             _ptr(ns, C.c_uint32), _ptr(nin, C.c_uint32), omega, delta,
                                             _ptr(out, C.c_uint32), C.byref(ng)), "axc_stage_matching")
        return out[:n], ng.value

    def stage_contract(self, g: Hypergraph, groups):
        groups = np.ascontiguousarray(groups, dtype=np.uint32)
        off = np.zeros(g.e + 1, np.uint64); pins = np.zeros(max(g.P, 1), np.uint32)
        ns = np.zeros(max(g.e, 1), np.uint32); pa = C.c_uint64()
        self._check(lib().axc_stage_contract(self._h, C.byref(g.c()), _ptr(groups, C.c_uint32),
                                             int(groups.max()) + 1 if len(groups) else 0,
                                             _ptr(off, C.c_uint64), _ptr(pins, C.c_uint32),
                                             _ptr(ns, C.c_uint32), C.byref(pa)), "axc_stage_contract")
        return off, pins[: pa.value], ns[: g.e]

    def stage_gains(self, g: Hypergraph, part, num_parts, node_size, omega, delta, encourage, discount):
        part = np.ascontiguousarray(part, dtype=np.uint32)
        ns = np.ascontiguousarray(node_size, dtype=np.uint32)
        tgt = np.zeros(max(g.n, 1), np.uint32); gain = np.zeros(max(g.n, 1), np.int64)
        self._check(lib().axc_stage_gains(self._h, C.byref(g.c()), _ptr(part, C.c_uint32), num_parts,
                                          _ptr(ns, C.c_uint32), omega, delta, int(encourage), discount,
                                          _ptr(tgt, C.c_uint32), _ptr(gain, C.c_int64)), "axc_stage_gains")
        return tgt[: g.n], gain[: g.n]

    def stage_refine(self, g: Hypergraph, part, num_parts, node_size, omega, delta, encourage, rounds, seed=0):
        part = np.ascontiguousarray(part, dtype=np.uint32)
        ns = np.ascontiguousarray(node_size, dtype=np.uint32)
        out = np.zeros(max(g.n, 1), np.uint32); ran = C.c_uint32()
        self._check(lib().axc_stage_refine(self._h, C.byref(g.c()), _ptr(part, C.c_uint32), num_parts,
                                           _ptr(ns, C.c_uint32), omega, delta, int(encourage), rounds, seed,
                                           _ptr(out, C.c_uint32), C.byref(ran)), "axc_stage_refine")
        return out[: g.n], ran.value
