"""Benchmark: pins/s of the whole multilevel partitioner (end to end, at the reference's metric).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step partitions one seeded synthetic hypergraph of the named workload end to end:
  value  pins/s with the raw hypergraph already resident in HBM (axc_partition_device), the L2
         flushed between steps (outside the timed step);
  e2e    pins/s through axc_partition with pinned host buffers: the upload of the step's input and
         the download of its partition are inside the timed region.
Every partition is also scored by the reference grader (grading/grade.cpp, built from the
reference sources as oracle/_ref/hgrade.exe) from its partition file; that evaluation, timed, is
the CPU baseline. The other configurations (--configs) follow as sub-results of the same line.
`--impl reference` times the reference's own implementation of the path on this box, its GPU
build compiled from the reference sources (oracle/_ref/hgraph_gpu.exe; for k-way, the same
sources with the reference's dormant GPU initial partitioner in place of the absent Mt-KaHyPar),
over the span it reports as "Total host execution time". That arm loads none of this
repository's libraries: its inputs come from the host-only generator binary axoncuda_b200/axc_gen.
Multi-GPU (torchrun): one partition job does not shard, so every rank runs a replica; timing is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# name: description, axc_gen arguments (kind, seed) for the input file, the reference scripts'
# flags (hgraphs/run_snns.sh:20 for INCC, hgraphs/run_ispd.sh:20 for k-way) and the grader's
# constraint flags (grading/grade.cpp -m-prt / -k-prt)
WORKLOADS = {
    "snn-8x512": dict(
        desc="layered SNN 8x512 fan-out 64 seed 0, INCC omega=128 delta=1024 Kmax=1048576",
        gen=("snn-layered", "0", ".snn"), kway=False,
        ref=["-m", "128", "1024", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"],
        grade=["-m-prt", "128", "1024", "1048576"]),
    "circuit-200k-k2": dict(
        desc="circuit .hgr 200k nodes 220k nets seed 1, k-way k=2 eps=0.03",
        gen=("circuit", "1", ".hgr"), kway=True,
        ref=["-k", "2", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"],
        grade=["-k-prt", "2", "0.03"]),
    "circuit-200k-k64": dict(
        desc="circuit .hgr 200k nodes 220k nets seed 1, k-way k=64 eps=0.03",
        gen=("circuit", "1", ".hgr"), kway=True,
        ref=["-k", "64", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"],
        grade=["-k-prt", "64", "0.03"]),
    "snn-1m-incc": dict(
        desc="large SNN 20x50k lognormal fan-out seed 2, INCC omega=1024 delta=4096 Kmax=1048576",
        gen=("snn-large", "2", ".snn"), kway=False,
        ref=["-m", "1024", "4096", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"],
        grade=["-m-prt", "1024", "4096", "1048576"]),
    "snn-100k-incc": dict(
        desc="SNN 20x5k lognormal fan-out seed 2 (the large SNN's generator at a tenth of the width), INCC "
             "omega=1024 delta=4096 Kmax=1048576: a profiling-size case",
        gen=("snn-mid", "2", ".snn"), kway=False,
        ref=["-m", "1024", "4096", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"],
        grade=["-m-prt", "1024", "4096", "1048576"]),
    "snn-1m-k128": dict(
        desc="large SNN 20x50k lognormal fan-out seed 2, k-way k=128 eps=0.03",
        gen=("snn-large", "2", ".snn"), kway=True,
        ref=["-k", "128", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"],
        grade=["-k-prt", "128", "0.03"]),
}
DEFAULT_WORKLOAD = "circuit-200k-k2"
# the other configurations, measured in the same run as per-config sub-results of the line
DEFAULT_CONFIGS = ["snn-8x512", "circuit-200k-k64", "snn-1m-k128", "snn-1m-incc"]
METRIC = "pins/s end-to-end at equal lambda-1"
L2_NOTE = "cold between timed steps: a 256 MiB write flushes L2 (the reference arm runs a fresh process per step)"
GEN = os.path.join(ROOT, "axoncuda_b200", "axc_gen")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def gen_file(name: str, td: str):
    """Writes the workload's input file with the host-only generator binary (no library loaded in
    this process) and returns (path, nodes, hyperedges, pins)."""
    kind, seed, ext = WORKLOADS[name]["gen"]
    path = os.path.join(td, name + ext)
    r = subprocess.run([GEN, kind, path, seed], capture_output=True, text=True, check=True)
    m = re.search(r"(\d+) nodes, (\d+) hyperedges, (\d+) pins", r.stdout)
    return path, int(m.group(1)), int(m.group(2)), int(m.group(3))


def config_of(name: str, nodes: int, hedges: int, pins: int, world: int) -> dict:
    """The line's config: the same keys and values on both arms."""
    return {"workload": name, "description": WORKLOADS[name]["desc"], "pins": pins, "nodes": nodes,
            "hyperedges": hedges, "parallelism": f"replicas x{world}", "l2": L2_NOTE}


def grade(path: str, part_path: str, name: str, timeout: float) -> dict:
    """lambda-1 and validity of a partition file by the reference grader (grading/grade.cpp, built
    from the reference sources as oracle/_ref/hgrade.exe), with its wall time."""
    exe = os.path.join(REF_DIR, "hgrade.exe")
    if not os.path.exists(exe):
        return {"grader": "unavailable: oracle/_ref/hgrade.exe not built"}
    t0 = time.perf_counter()
    try:
        r = subprocess.run([exe, "-r", path, "-prt", part_path, *WORKLOADS[name]["grade"]], capture_output=True,
                           text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"grader": f"did not finish within {timeout:.0f} s"}
    dt = time.perf_counter() - t0
    out = {"valid": int(r.returncode == 0 and "invalid partitioning" not in r.stderr), "grader_s": dt}
    for line in r.stdout.splitlines():
        s = line.strip()
        for key, nm in (("Connectivity:", "connectivity"), ("Cut-net:", "cutnet"), ("Nodes:", "num_parts")):
            if s.startswith(key):
                out[nm] = float(s.split(":", 1)[1].split()[0])
    return out


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self.proc = None
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the sampler's start-up takes a host core for a moment; let it pass before timing
            t0 = time.time()
            while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier_max(world, value: float) -> float:
    """The maximum of `value` over all ranks (the slowest replica sets the job's time)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_jobs(sizes, world: int) -> list[list[int]]:
    """Independent jobs spread over ranks: the largest job first to the least-loaded rank (ties to
    the lower rank), so every rank sees the same deterministic assignment."""
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        shards[r].append(i)
        load[r] += sizes[i]
    return [sorted(s) for s in shards]


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# the kernel with the largest share of device time (ncu launch lists in profiles/) per workload
ROOFLINE_KERNELS = {"circuit-200k-k2": "k_census_inc_warp", "circuit-200k-k64": "k_census_inc_warp",
                    "snn-8x512": "k_rate_block", "snn-1m-k128": "k_rate_block"}
# algorithmic bytes per launch of the kernels the library's timer has a byte model for
BYTE_MODELS = {
    "k_rate_block": "4 B per pin visit of the listed nodes (the pin id) + 8 B per candidate slot written",
    "k_gain_warp": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_block": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_mask_warp": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_mask_block": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_cascade_warp": "per listed hyperedge (those holding a mover), counted by the kernel: 24 B (list entry, "
                      "offsets, source count) + 8 B per pin (id, rank) + 4 B (census size), then 4 B (hand-off "
                      "to the block kernel) or 12 B per census entry + 16 B per mover (partition, target, "
                      "cascaded gain) + 4 B (weight); inbound transitions not counted",
    "k_census_direct_warp": "per hyperedge, counted by the kernel: 20 B (offsets, source count) + 8 B per pin (id, "
                            "partition) + 12 B per census entry written + 4 B (its count) + 8 B per mask word pair "
                            "+ 4 B (weight) + 8 B per nonzero saving added to a pin's node",
    "k_census_inc_warp": "per recomputed hyperedge, counted by the kernel: 24 B (list entry, offsets, source count) "
                         "+ 12 B per pin (id, partition, move stamp) + 8 B per old census entry read + 12 B per "
                         "entry written + 4 B (its count) + 8 B per mask word pair + 4 B (weight) + 8 B per "
                         "nonzero saving change",
}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch from one ncu capture of the
# kernel on the workload, recorded with its capture command in profiles/<kernel>-<workload>.md
PROFILED_TRAFFIC = {("k_rate_block", "snn-8x512"): 616456, ("k_census_direct_warp", "circuit-200k-k2"): 67656819,
                    ("k_census_inc_warp", "circuit-200k-k2"): 22632375}
STEP_MODEL = ("construction 8P+8(n+E); per rated level 4 B per rating pin visit + 4P_l + 16 n_l C (matching); "
              "per contraction 8P_l + 12P_(l+1); per refinement round 16P_l + 16n_l (moves not counted)")


def sub_configs(arg: str | None, world: int) -> list[str]:
    """The other configurations measured as sub-results: the given comma-separated list ('none'
    for none), or by default DEFAULT_CONFIGS on one GPU and none under torchrun, where the
    scaling runs time the line's workload alone."""
    if arg is None:
        return list(DEFAULT_CONFIGS) if world == 1 else []
    return [] if arg == "none" else [x for x in arg.split(",") if x]


def hbm_peak() -> tuple[float, str]:
    """Measured copy bandwidth of this pool's B200s (GB/s), else the stated fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def step_bytes(st, n0: int, e: int, cnc: int) -> int:
    """Algorithmic bytes of one whole partition from its per-level sizes (no credit for reuse):
    level 0 construction, the rating, matching and contraction of every coarsened level, and each
    refinement round actually run."""
    L = int(st.levels)
    P = [int(st.level_pins[l]) for l in range(min(L, 64))]
    n = [int(st.level_nodes[l]) for l in range(min(L, 64))]
    total = 8 * P[0] + 8 * (n0 + e) + 4 * int(st.rating_pin_visits)
    for l in range(len(P)):
        total += 4 * P[l] + 16 * n[l] * cnc
        if l + 1 < len(P):
            total += 8 * P[l] + 12 * P[l + 1]
        total += int(st.refine_rounds[l]) * (16 * P[l] + 16 * n[l])
    return total


def measure_ours(ctx, name: str, steps: int, warmup: int, world: int, td: str, clocks: bool = True,
                 roofline_kernel: str | None = None, grade_timeout: float = 120.0) -> dict:
    """One workload on our arm: `value` from device-resident input, `e2e` through the host-buffer
    call, quality from the library and from the reference grader on the partition file."""
    import ctypes as C

    import torch

    import axoncuda_b200 as ax
    g, p = ax.workload(name)
    P = g.P
    dev = torch.device("cuda", torch.cuda.current_device())
    d_off = torch.from_numpy(g.off.astype(np.uint64).view(np.int64)).to(dev)
    d_pins = torch.from_numpy(g.pins.view(np.int32)).to(dev)
    d_ns = torch.from_numpy(g.nsrc.view(np.int32)).to(dev)
    d_w = torch.from_numpy(g.w).to(dev)
    d_out = torch.empty(max(g.n, 1), dtype=torch.int32, device=dev)
    dg = ax.HGraph(g.n, g.e, C.cast(d_off.data_ptr(), C.POINTER(C.c_uint64)),
                   C.cast(d_pins.data_ptr(), C.POINTER(C.c_uint32)), C.cast(d_ns.data_ptr(), C.POINTER(C.c_uint32)),
                   C.cast(d_w.data_ptr(), C.POINTER(C.c_float)), None)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    st = ax.Stats()

    def dev_step():
        rc = ax.lib().axc_partition_device(ctx._h, C.byref(dg), C.byref(p),
                                           C.cast(d_out.data_ptr(), C.POINTER(C.c_uint32)), C.byref(st))
        if rc:
            raise ax.AxcError(rc, ax.lib().axc_last_error(ctx._h).decode())

    for _ in range(warmup):
        dev_step()
    torch.cuda.synchronize()
    total_ms, launches = 0.0, 0
    if roofline_kernel:
        ctx.profile_kernel(roofline_kernel)
        ctx.profile_read()
    k_launches, k_ms, k_bytes = 0, 0.0, 0
    clk = Clocks(torch.cuda.current_device()) if clocks else None
    if clk:
        clk.__enter__()
    try:
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            barrier(world)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dev_step()
            e1.record()
            torch.cuda.synchronize()
            total_ms += e0.elapsed_time(e1)
            launches += int(st.kernel_launches)
            if roofline_kernel:
                kt = ctx.profile_read()
                k_launches += kt.launches
                k_ms += kt.ms_total
                k_bytes += kt.bytes
    finally:
        if clk:
            clk.__exit__(None, None, None)
    if roofline_kernel:
        ctx.profile_kernel(None)
    total_ms = barrier_max(world, total_ms)
    ms_step = total_ms / steps
    sbytes = step_bytes(st, g.n, g.e, int(p.cnc))
    # ---- end to end through the host-buffer C-ABI call (pinned buffers) ----
    h_off = torch.from_numpy(g.off.view(np.int64)).pin_memory()
    h_pins = torch.from_numpy(g.pins.view(np.int32)).pin_memory()
    h_ns = torch.from_numpy(g.nsrc.view(np.int32)).pin_memory()
    h_w = torch.from_numpy(g.w).pin_memory()
    h_out = torch.empty(max(g.n, 1), dtype=torch.int32).pin_memory()
    hg = ax.HGraph(g.n, g.e, C.cast(h_off.data_ptr(), C.POINTER(C.c_uint64)),
                   C.cast(h_pins.data_ptr(), C.POINTER(C.c_uint32)), C.cast(h_ns.data_ptr(), C.POINTER(C.c_uint32)),
                   C.cast(h_w.data_ptr(), C.POINTER(C.c_float)), None)
    st2 = ax.Stats()

    def e2e_step():
        rc = ax.lib().axc_partition(ctx._h, C.byref(hg), C.byref(p),
                                    C.cast(h_out.data_ptr(), C.POINTER(C.c_uint32)), C.byref(st2))
        if rc:
            raise ax.AxcError(rc, ax.lib().axc_last_error(ctx._h).decode())

    for _ in range(max(1, min(warmup, 3))):
        e2e_step()
    e2e_ms = 0.0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms += (time.perf_counter() - t0) * 1e3
    e2e_ms = barrier_max(world, e2e_ms)
    e2e_step_ms = e2e_ms / steps
    part = h_out.numpy()[: g.n].view(np.uint32).copy()
    h2d = g.off.nbytes + g.pins.nbytes + g.nsrc.nbytes + g.w.nbytes
    peak, peak_kind = hbm_peak()
    out = {
        "value": world * P / (ms_step / 1e3), "ms_per_step": ms_step, "steps": steps, "warmup": warmup,
        "config": config_of(name, g.n, g.e, P, world),
        "e2e": {"value": world * P / (e2e_step_ms / 1e3), "unit": "pins/s", "ms_per_step": e2e_step_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4 * g.n},
        "gpu_launches": launches,
        "quality": {"connectivity": st2.connectivity, "cutnet": st2.cutnet, "num_parts": int(st2.num_parts),
                    "valid": int(st2.valid), "levels": int(st2.levels)},
        "step_bytes": sbytes, "step_gbs": sbytes / (ms_step / 1e3) / 1e9,
        "step_frac": sbytes / (ms_step / 1e3) / 1e9 / peak,
        "peak_device_gb": int(st.device_bytes_peak) / 1e9,
    }
    if clk:
        out["clocks"] = clk.summary()
    if roofline_kernel:
        achieved = (k_bytes / (k_ms / 1e3)) / 1e9 if k_ms > 0 else 0.0
        out["kernel"] = {"achieved": achieved, "k_launches": k_launches, "k_ms": k_ms, "k_bytes": k_bytes,
                         "peak": peak, "peak_kind": peak_kind}
    # the reference grader's verdict on this partition (outside every timed region)
    path, _, _, _ = gen_file(name, td)
    pf = os.path.join(td, name + ".part")
    np.savetxt(pf, part, fmt="%d")
    out["graded"] = grade(path, pf, name, grade_timeout)
    out["_partfile"] = (path, pf)
    return out


def run_ours(args, world, rank, local):
    import torch

    import axoncuda_b200 as ax
    torch.cuda.set_device(local)
    ctx = ax.Context(local, int(args.arena_gb * (1 << 30)))
    td = tempfile.mkdtemp(prefix="axc_bench_")
    kname = args.roofline_kernel or ROOFLINE_KERNELS.get(args.workload, "k_rate_block")
    head = measure_ours(ctx, args.workload, args.steps, args.warmup, world, td, roofline_kernel=kname)
    peak, peak_kind = hbm_peak()
    kt = head.pop("kernel")
    P = head["config"]["pins"]
    out = {"metric": METRIC, "value": head["value"], "unit": "pins/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator)",
           "config": head["config"], "e2e": head["e2e"], "gpu_launches": head["gpu_launches"],
           "quality": dict(head["quality"], grader=head["graded"]), "clocks": head["clocks"]}
    out["roofline"] = {
        "bound": "hbm", "kernel": kname, "achieved": kt["achieved"], "peak": peak, "unit": "GB/s",
        "frac": kt["achieved"] / peak if peak else None, "peak_source": peak_kind,
        "traffic": PROFILED_TRAFFIC.get((kname, args.workload)),
        "bytes_per_launch": kt["k_bytes"] / kt["k_launches"] if kt["k_launches"] else 0,
        "ms_per_launch": kt["k_ms"] / kt["k_launches"] if kt["k_launches"] else 0,
        "launches_per_step": kt["k_launches"] / args.steps,
        "share_of_step": (kt["k_ms"] / args.steps) / head["ms_per_step"] if head["ms_per_step"] else None,
        "model": BYTE_MODELS.get(kname, "none: achieved is 0"),
        "step_bytes": head["step_bytes"], "step_achieved": head["step_gbs"], "step_frac": head["step_frac"],
        "step_model": STEP_MODEL,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        path, pf = head["_partfile"]
        out["cpu_baseline"] = grader_baseline(path, pf, args.workload, P)
    # the other configurations, fewer steps each (the step count is in each entry)
    subs = {}
    for name in sub_configs(args.configs, world):
        if name == args.workload:
            continue
        large = name.startswith("snn-1m")
        try:
            r = measure_ours(ctx, name, 1 if large else 3, 1 if large else 3, world, td, clocks=True,
                             grade_timeout=300.0 if large else 60.0)
        except Exception as exc:  # a failing configuration is reported, not fatal to the line
            subs[name] = {"unavailable": f"{type(exc).__name__}: {exc}"[:300]}
            continue
        r.pop("_partfile")
        subs[name] = {k: r[k] for k in ("value", "ms_per_step", "steps", "warmup", "e2e", "quality", "graded",
                                       "step_bytes", "step_frac", "peak_device_gb", "clocks", "gpu_launches")}
        subs[name]["config"] = r["config"]
    if subs:
        out["configs"] = subs
    ctx.close()
    return out


def grader_baseline(path: str, pf: str, name: str, pins: int) -> dict:
    """The CPU path of the metric: the reference grader's evaluation (grading/grade.cpp, compiled
    here as oracle/_ref/hgrade.exe; Mt-KaHyPar is not installable offline) of this run's partition,
    timed around the process. It is single-threaded."""
    reps, total, last = 0, 0.0, {}
    while reps < 50 and total < 15.0:
        last = grade(path, pf, name, 300.0)
        if "grader_s" not in last:
            return {"value": None, "unit": "pins/s", "cores": 1, "kind": "reference",
                    "sample": f"grade.cpp evaluation: {last.get('grader')}"}
        total += last["grader_s"]
        reps += 1
    return {"value": pins * reps / total, "unit": "pins/s", "cores": 1, "kind": "reference",
            "host_cores": os.cpu_count(),
            "sample": f"grade.cpp evaluation (oracle/_ref/hgrade.exe: read, constraint check, lambda-1) of this "
                      f"run's partition of the full workload ({pins} pins), {reps} runs in {total:.2f} s, "
                      f"1 thread of {os.cpu_count()} host cores"}


def run_reference_one(name: str, steps: int, warmup: int, td: str, timeout: float) -> dict:
    """The reference GPU build on one workload: its own executable and stdout, this box's B200.
    INCC runs hgraph_gpu.exe; k-way runs hgraph_gpu_gpuinit.exe, the same sources with the
    reference's dormant GPU initial partitioner in place of Mt-KaHyPar (absent offline)."""
    w = WORKLOADS[name]
    exe = os.path.join(REF_DIR, "hgraph_gpu_gpuinit.exe" if w["kway"] else "hgraph_gpu.exe")
    path, nodes, hedges, pins = gen_file(name, td)
    res = {"config": config_of(name, nodes, hedges, pins, 1),
           "variant": ("reference GPU build with its in-tree GPU initial partitioner (sources/init_part.cu:186-727) "
                       "in place of Mt-KaHyPar: reference-family, not the Mt-KaHyPar result") if w["kway"]
           else "reference GPU build (hgraph_gpu.exe, sm_100a, -dlto)"}
    if not os.path.exists(exe):
        res["unavailable"] = f"{os.path.relpath(exe, ROOT)} not built"
        return res
    times, conn_stdout = [], None
    pf = os.path.join(td, name + ".ref.part")
    for i in range(warmup + steps):
        try:
            r = subprocess.run([exe, "-r", path, *w["ref"], "-p", pf], capture_output=True, text=True, cwd=td,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            res["unavailable"] = f"reference did not finish one partition within {timeout:.0f} s"
            return res
        if r.returncode != 0:
            tail = " ".join((r.stderr.strip() or r.stdout.strip()).split())[-240:]
            res["unavailable"] = f"reference exited {r.returncode}: {tail}"
            return res
        m = re.search(r"Total host execution time: ([0-9.]+) ms", r.stdout)
        if m is None:
            res["unavailable"] = "reference printed no 'Total host execution time'"
            return res
        if i >= warmup:
            times.append(float(m.group(1)))
        mc = re.search(r"Connectivity:\s+([0-9.eE+]+)", r.stdout)
        conn_stdout = float(mc.group(1)) if mc else None
    ms = sum(times) / len(times)
    res.update({"value": pins / (ms / 1e3), "ms_per_step": ms, "steps": steps, "warmup": warmup,
                "graded": grade(path, pf, name, 600.0), "stdout_connectivity": conn_stdout})
    return res


def run_reference(args):
    """The reference's own implementation of the path, timed on this box. This process loads none
    of the repository's libraries: inputs come from the host-only generator binary, the reference
    runs as its own executables, and its partitions are scored by its own grader."""
    td = tempfile.mkdtemp(prefix="axc_ref_")
    line = {"metric": METRIC, "unit": "pins/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded generator)", "impl": "reference"}
    with Clocks(0) as clk:
        head = run_reference_one(args.workload, args.steps, args.warmup, td, args.ref_timeout)
    line["config"] = head.pop("config")
    if "unavailable" in head:
        line["unavailable"] = head["unavailable"]
        return line
    v = head["value"]
    line.update({"value": v, "ms_per_step": head["ms_per_step"], "variant": head["variant"],
                 "cpu_baseline": {"value": v, "unit": "pins/s", "cores": 1, "kind": "reference",
                                  "sample": f"the full workload through {head['variant']}: its 'Total host execution "
                                            f"time' (upload to partition download), one host thread driving one B200"},
                 "e2e": {"value": v, "unit": "pins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "quality": {"grader": head["graded"], "stdout_connectivity": head["stdout_connectivity"]},
                 "clocks": clk.summary()})
    subs = {}
    for name in sub_configs(args.configs, int(os.environ.get("WORLD_SIZE", "1"))):
        if name == args.workload:
            continue
        large = name.startswith("snn-1m")
        r = run_reference_one(name, 1 if large else 2, 0 if large else 1, td, args.ref_timeout)
        subs[name] = r
    if subs:
        line["configs"] = subs
    return line


def batch_jobs(count: int = 256, seed0: int = 100):
    """The batched workload: `count` hypergraphs, seeds seed0.., alternately from the circuit and the
    layered-SNN generator, nodes log-uniform in [1e3, 1e5] (nets in proportion), k-way with k drawn
    from {2, 8, 32}, eps 0.03."""
    import axoncuda_b200 as ax
    rng = np.random.default_rng(seed0)
    jobs = []
    for i in range(count):
        s = seed0 + i
        n = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e5)))))
        k = int(rng.choice([2, 8, 32]))
        if i % 2 == 0:
            g = ax.gen_circuit(n, int(1.1 * n), 2, 64, 2.5, 0.9, 0.02, s)
        else:
            g = ax.gen_snn(8, max(n // 8, 65), 64, 0.0, 0, 1.0, s)
        jobs.append((g, ax.params_kway(k, 0.03, cnc=4, rfr=16)))
    return jobs


def serve_requests(count: int, max_pins: float, seed: int = 7):
    """The served workload: requests with pin counts log-uniform in [1e4, max_pins], half from the
    circuit generator and half from the lognormal-fan-out SNN generator; half INCC (omega 256,
    delta 2048), half k-way with k in {2, 16, 64}, eps 0.03."""
    import axoncuda_b200 as ax
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        pins = float(np.exp(rng.uniform(np.log(1e4), np.log(max_pins))))
        if i % 2 == 0:  # circuit: about 4.4 pins per net, 1.1 nets per node
            n = max(int(pins / 4.85), 1000)
            g = ax.gen_circuit(n, int(1.1 * n), 2, 64, 2.5, 0.9, 0.02, 1000 + i)
        else:  # SNN, 20 layers, fan-out median 256: about 350 pins per neuron
            width = max(int(pins / (20 * 350)), 64)
            g = ax.gen_snn(20, width, 256, 0.8, 2048, 0.7, 1000 + i)
        if rng.random() < 0.5:
            p = ax.params_incc(256, 2048, 1048576, cnc=4, rfr=16)
        else:
            p = ax.params_kway(int(rng.choice([2, 16, 64])), 0.03, cnc=4, rfr=16)
        reqs.append((g, p))
    return reqs


def percentiles(xs):
    xs = np.asarray(xs, dtype=np.float64)
    return {"p50_ms": float(np.percentile(xs, 50)), "p99_ms": float(np.percentile(xs, 99)),
            "mean_ms": float(xs.mean())}


def tuning_table(args):
    """The autotuner's table for the batch and serve modes, when there is one."""
    return args.tune if args.tune != "none" and os.path.exists(args.tune) else None


def run_batch(args) -> dict:
    """jobs/s of the batched workload through the executor's lanes (axc_partition_batch) against a
    one-at-a-time loop of axc_partition over the same jobs; both from host buffers to host results."""
    import axoncuda_b200 as ax
    world, rank, local = dist_setup(args)
    all_jobs = batch_jobs(args.batch_jobs)
    mine = shard_jobs([g.P for g, _ in all_jobs], world)[rank]  # independent jobs: no collective
    jobs = [all_jobs[i] for i in mine]
    pins = sum(g.P for g, _ in all_jobs)
    with ax.Context(local, 2 << 30) as seq:
        for g, p in jobs[:4]:
            seq.partition(g, p)  # warm-up: module load, first allocations
        barrier(world)
        t0 = time.perf_counter()
        solo = [seq.partition(g, p)[0] for g, p in jobs]
        t_seq = barrier_max(world, time.perf_counter() - t0)
    tuning = tuning_table(args)
    with ax.Context(local, 256 << 20) as srv:
        lanes = args.lanes
        if tuning:  # the autotuner's table: size classes, exclusive threshold, lane count
            from axoncuda_b200 import tune as T
            lanes = lanes or T.apply(srv, tuning)
        lanes = lanes or 8
        srv.serve_configure(lanes, int(args.budget_gb * (1 << 30)))
        srv.partition_batch(jobs[:lanes])  # warm-up: lanes, graphs of the first levels
        with Clocks(local) as clk:
            barrier(world)
            t0 = time.perf_counter()
            res = srv.partition_batch(jobs)
            t_bat = barrier_max(world, time.perf_counter() - t0)
    same = sum(int(np.array_equal(r[0], s)) for r, s in zip(res, solo))
    lat = [st.ms_queued + st.ms_run for _, st in res]
    return {"metric": f"jobs/s batched ({len(all_jobs)} mixed k-way jobs)", "value": len(all_jobs) / t_bat,
            "unit": "jobs/s", "n_gpus": world, "higher_is_better": True, "scaling": "strong", "dtype": "u32",
            "data": "synthetic (seeded generators)",
            "config": {"workload": f"batch-{len(all_jobs)}", "jobs": len(all_jobs), "pins": pins,
                       "lanes_per_gpu": lanes, "budget_gb": args.budget_gb,
                       "tuning": os.path.relpath(tuning, ROOT) if tuning else "defaults",
                       "parallelism": f"jobs sharded over {world} GPU(s), no collective"},
            "sequential": {"value": len(all_jobs) / t_seq, "unit": "jobs/s", "seconds": t_seq},
            "speedup_vs_sequential": t_seq / t_bat, "seconds": t_bat, "pins_per_s": pins / t_bat,
            "identical_to_sequential_rank0": f"{same}/{len(jobs)}",
            "valid_rank0": f"{sum(int(st.valid) for _, st in res)}/{len(jobs)}",
            "latency_in_batch_rank0": percentiles(lat), "clocks": clk.summary()}


def run_serve(args) -> dict:
    """A Poisson stream of requests through axc_submit / axc_poll with continuous batching, against a
    FIFO single server running the same requests one at a time (its latencies follow from the
    measured service times and the same arrival times)."""
    import axoncuda_b200 as ax
    reqs = serve_requests(args.serve_requests, args.serve_max_pins)
    pins = sum(g.P for g, _ in reqs)
    with ax.Context(0, int(args.seq_arena_gb * (1 << 30))) as seq:
        seq.partition(*reqs[0])  # warm-up
        service = []
        for g, p in reqs:
            t0 = time.perf_counter()
            seq.partition(g, p)
            service.append(time.perf_counter() - t0)
    cap = len(reqs) / sum(service)
    rate = args.serve_load * cap  # arrivals per second, a multiple of the sequential capacity
    rng = np.random.default_rng(11)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    # the single server: FIFO, one request at a time
    t, seq_lat = 0.0, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        seq_lat.append((t - a) * 1e3)
    seq_span = t - arrivals[0]
    tuning = tuning_table(args)
    with ax.Context(0, 256 << 20) as srv:
        lanes = args.lanes
        if tuning:
            from axoncuda_b200 import tune as T
            lanes = lanes or T.apply(srv, tuning)
        lanes = lanes or 8
        srv.serve_configure(lanes, int(args.budget_gb * (1 << 30)))
        srv.partition_batch(reqs[:lanes])  # warm-up
        done = {}
        ids = []
        with Clocks(0) as clk:
            t0 = time.perf_counter()
            for a, (g, p) in zip(arrivals, reqs):
                wait = t0 + (a - arrivals[0]) - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                ids.append(srv.submit(g, p))
            for i, (jid, (g, _)) in enumerate(zip(ids, reqs)):
                done[i] = srv.poll(jid, g.n)
            span = time.perf_counter() - t0
    lat = [done[i][1].ms_queued + done[i][1].ms_run for i in range(len(reqs))]
    return {"metric": "jobs/s served (Poisson stream, continuous batching)", "value": len(reqs) / span,
            "unit": "jobs/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u32",
            "data": "synthetic (seeded generators)",
            "config": {"workload": "serve-poisson", "requests": len(reqs), "pins": pins,
                       "pins_per_request": f"log-uniform in [1e4, {args.serve_max_pins:.0e}]",
                       "arrival_rate_per_s": rate, "load_vs_sequential_capacity": args.serve_load,
                       "lanes": lanes, "budget_gb": args.budget_gb,
                       "tuning": os.path.relpath(tuning, ROOT) if tuning else "defaults"},
            "latency": percentiles(lat), "seconds": span,
            "sequential": {"value": len(reqs) / seq_span, "unit": "jobs/s", "capacity_jobs_per_s": cap,
                           "latency": percentiles(seq_lat)},
            "speedup_vs_sequential": (len(reqs) / span) / (len(reqs) / seq_span),
            "valid": f"{sum(int(done[i][1].valid) for i in range(len(reqs)))}/{len(reqs)}",
            "clocks": clk.summary()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--roofline-kernel", default=None,
                    help="kernel timed for the roofline (default: the workload's largest, ROOFLINE_KERNELS)")
    ap.add_argument("--ref-timeout", type=float, default=900.0,
                    help="seconds one reference partition may take before its arm reports unavailable")
    ap.add_argument("--mode", default="partition", choices=["partition", "batch", "serve"],
                    help="partition: one hypergraph per step (the headline); batch / serve: many jobs")
    ap.add_argument("--lanes", type=int, default=0, help="executor lanes (0: the tuning table's, else 8)")
    ap.add_argument("--tune", default=os.path.join(ROOT, "axoncuda_b200", "tuned_b200.json"),
                    help="the autotuner's table (python -m axoncuda_b200.tune) for the batch and serve modes, "
                         "or 'none'")
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--batch-jobs", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=120)
    ap.add_argument("--serve-max-pins", type=float, default=2e7)
    ap.add_argument("--serve-load", type=float, default=2.0)
    ap.add_argument("--seq-arena-gb", type=float, default=24.0)
    ap.add_argument("--arena-gb", type=float, default=0.0,
                    help="device arena of the partition context in GiB (0: the library default, 60%% of free memory)")
    ap.add_argument("--configs", default=None,
                    help="comma-separated other workloads measured as sub-results of the line, or 'none' "
                         f"(default: {','.join(DEFAULT_CONFIGS)} on one GPU, none under torchrun)")
    args = ap.parse_args()
    if args.mode == "batch":
        out = run_batch(args)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(out), flush=True)
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.mode == "serve":
        print(json.dumps(run_serve(args)), flush=True)
        return
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    world, rank, local = dist_setup(args)
    out = run_ours(args, world, rank, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
