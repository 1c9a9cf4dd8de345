"""Benchmark: pins/s of the whole multilevel partitioner (end to end, at the reference's metric).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step partitions one seeded synthetic hypergraph of the named workload end to end:
  value  pins/s with the raw hypergraph already resident in HBM (axc_partition_device), the L2
         flushed between steps (outside the timed step);
  e2e    pins/s through axc_partition with pinned host buffers: the upload of the step's input and
         the download of its partition are inside the timed region.
`--impl reference` times the reference's own implementation of the path on this box: its GPU
build compiled from the reference sources (oracle/_ref/hgraph_gpu.exe, the span it reports as
"Total host execution time"), or the CPU port of the oracle where the reference cannot run the
mode (k-way needs the external Mt-KaHyPar binary).
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

WORKLOADS = {
    # name: (description, reference CLI flags)
    "snn-8x512": ("layered SNN 8x512 fan-out 64 seed 0, INCC omega=128 delta=1024 Kmax=1048576",
                  ["-m", "128", "1024", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"]),
    "circuit-200k-k2": ("circuit .hgr 200k nodes 220k nets seed 1, k-way k=2 eps=0.03",
                        ["-k", "2", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"]),
    "circuit-200k-k64": ("circuit .hgr 200k nodes 220k nets seed 1, k-way k=64 eps=0.03",
                         ["-k", "64", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"]),
    "snn-1m-incc": ("large SNN 20x50k lognormal fan-out seed 2, INCC omega=1024 delta=4096 Kmax=1048576",
                    ["-m", "1024", "4096", "1048576", "-rfr", "16", "-cnc", "4", "-dtc", "-ipm", "-v", "0"]),
    "snn-1m-k128": ("large SNN 20x50k lognormal fan-out seed 2, k-way k=128 eps=0.03",
                    ["-k", "128", "0.03", "-rfr", "16", "-cnc", "4", "-dtc", "-v", "0", "-smh", "0"]),
}
DEFAULT_WORKLOAD = "snn-8x512"
METRIC = "pins/s end-to-end at equal lambda-1"


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


ROOFLINE_KERNEL = "k_rate_block"  # the kernel with the largest share of device time (profiles/)
# algorithmic bytes per launch of the kernels the library's timer has a byte model for
BYTE_MODELS = {
    "k_rate_block": "4 B per pin visit of the listed nodes (the pin id) + 8 B per candidate slot written",
    "k_gain_warp": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_block": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_mask_warp": "8 B per incidence entry of the listed nodes + 16 B per listed node",
    "k_gain_mask_block": "8 B per incidence entry of the listed nodes + 16 B per listed node",
}


def hbm_peak() -> tuple[float, str]:
    """Measured copy bandwidth of this pool's B200s (GB/s), else the stated fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of the kernel from its committed ncu summary, if there is one."""
    path = os.path.join(ROOT, "profiles", f"{kernel}-{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                m = re.match(r"\s*traffic_bytes_per_launch:\s*([0-9]+)", line)
                if m:
                    return int(m.group(1))
    except OSError:
        pass
    return None


def run_ours(args, world, rank, local):
    import torch

    import axoncuda_b200 as ax
    g, p = ax.workload(args.workload)
    P = g.P
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = ax.Context(local, 0)
    # ---- device-resident input (value) ----
    d_off = torch.from_numpy(g.off.astype(np.uint64).view(np.int64)).to(dev)
    d_pins = torch.from_numpy(g.pins.view(np.int32)).to(dev)
    d_ns = torch.from_numpy(g.nsrc.view(np.int32)).to(dev)
    d_w = torch.from_numpy(g.w).to(dev)
    d_out = torch.empty(max(g.n, 1), dtype=torch.int32, device=dev)
    import ctypes as C
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

    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize()
    total_ms = 0.0
    launches = 0
    # the dominant kernel is timed with events on the library's own stream, launch by launch
    kname = args.roofline_kernel
    ctx.profile_kernel(kname)
    ctx.profile_read()
    k_launches, k_ms, k_bytes = 0, 0.0, 0
    with Clocks(local) as clk:
        for _ in range(args.steps):
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
            kt = ctx.profile_read()
            k_launches += kt.launches
            k_ms += kt.ms_total
            k_bytes += kt.bytes
    ctx.profile_kernel(None)
    total_ms = barrier_max(world, total_ms)
    ms_step = total_ms / args.steps
    value = world * P / (ms_step / 1e3)
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

    for _ in range(max(1, args.warmup)):
        e2e_step()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms += (time.perf_counter() - t0) * 1e3
    e2e_ms = barrier_max(world, e2e_ms)
    e2e_step_ms = e2e_ms / args.steps
    part = h_out.numpy()[: g.n].view(np.uint32).copy()
    h2d = g.off.nbytes + g.pins.nbytes + g.nsrc.nbytes + g.w.nbytes
    d2h = 4 * g.n
    out = {
        "metric": METRIC, "value": value, "unit": "pins/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload][0], "pins": P,
                   "nodes": g.n, "hyperedges": g.e, "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) between timed steps"},
        "e2e": {"value": world * P / (e2e_step_ms / 1e3), "unit": "pins/s", "ms_per_step": e2e_step_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "quality": {"connectivity": st2.connectivity, "cutnet": st2.cutnet, "num_parts": int(st2.num_parts),
                    "valid": int(st2.valid), "levels": int(st2.levels)},
        "clocks": clk.summary(),
    }
    peak, peak_kind = hbm_peak()
    achieved = (k_bytes / (k_ms / 1e3)) / 1e9 if k_ms > 0 else 0.0
    traffic = profiled_traffic(kname, args.workload)
    out["roofline"] = {
        "bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak if peak else None, "peak_source": peak_kind,
        "traffic": traffic,
        "bytes_per_launch": k_bytes / k_launches if k_launches else 0,
        "ms_per_launch": k_ms / k_launches if k_launches else 0,
        "launches_per_step": k_launches / args.steps,
        "share_of_step": (k_ms / args.steps) / ms_step if ms_step else None,
        "model": BYTE_MODELS.get(kname, "none: achieved is 0"),
    }
    ctx.close()
    return out, g, p, part


CPU_SAMPLE_PINS = 5_000_000  # above this the CPU baseline times a smaller instance of the generator


def cpu_sample(name: str, g, p):
    """The workload itself when the oracle finishes it in seconds, else a smaller instance of the same
    generator with the same parameters (the large SNN at 20 x 500 neurons), with its description."""
    import axoncuda_b200 as ax
    if g.P > CPU_SAMPLE_PINS and name.startswith("snn-1m"):
        gs = ax.gen_snn(20, 500, 256, 0.8, 2048, 0.7, 2)
        return gs, (f"one full step of the same generator at 20 x 500 neurons ({gs.P} pins; the workload has "
                    f"{g.P}), same parameters")
    return g, f"one full step of the workload ({g.P} pins)"


def cpu_port_baseline(g, p, name: str) -> dict:
    from oracle import oracle as O
    gs, what = cpu_sample(name, g, p)
    t0 = time.perf_counter()
    if p.mode == 0:
        O.partition(gs.n, gs.off, gs.pins, gs.nsrc, gs.w, 0, omega=p.omega, delta=p.delta, max_parts=p.max_parts,
                    cnc=p.cnc, rfr=p.rfr, ipm=p.ipm, seed=p.seed)
    else:
        O.partition(gs.n, gs.off, gs.pins, gs.nsrc, gs.w, 1, k=p.k, eps=p.eps, cnc=p.cnc, rfr=p.rfr, seed=p.seed)
    dt = time.perf_counter() - t0
    return {"value": gs.P / dt, "unit": "pins/s", "cores": 1, "kind": "port",
            "sample": f"{what} through the oracle's single-threaded C++ restatement of the whole partitioner, "
                      f"{dt:.2f} s"}


def run_reference(args):
    """The reference's own implementation of the path, timed on this box."""
    import axoncuda_b200 as ax
    g, p = ax.workload(args.workload)
    exe = os.path.join(ROOT, "oracle", "_ref", "hgraph_gpu.exe")
    flags = WORKLOADS[args.workload][1]
    kway = p.mode == ax.MODE_KWAY
    line = {"metric": METRIC, "unit": "pins/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded generator)", "impl": "reference",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload][0], "pins": g.P}}
    if not kway and os.path.exists(exe):
        with tempfile.TemporaryDirectory() as td:
            ext = ".hgr" if "circuit" in args.workload else ".snn"
            path = os.path.join(td, "in" + ext)
            ax.write(path, g)
            times = []
            conn = None
            for i in range(args.warmup + args.steps):
                pf = os.path.join(td, "out.part")
                try:
                    r = subprocess.run([exe, "-r", path, *flags, "-p", pf], capture_output=True, text=True, cwd=td,
                                       timeout=args.ref_timeout)
                except subprocess.TimeoutExpired:
                    line["unavailable"] = f"reference did not finish one partition within {args.ref_timeout:.0f} s"
                    return line
                if r.returncode != 0:
                    tail = (r.stderr.strip() or r.stdout.strip())[-200:]
                    line["unavailable"] = f"reference exited {r.returncode}: {tail}"
                    return line
                m = re.search(r"Total host execution time: ([0-9.]+) ms", r.stdout)
                if m is None:
                    line["unavailable"] = "reference printed no 'Total host execution time'"
                    return line
                if i >= args.warmup:
                    times.append(float(m.group(1)))
                mc = re.search(r"Connectivity:\s+([0-9.]+)", r.stdout)
                conn = float(mc.group(1)) if mc else None
            ms = sum(times) / len(times)
            v = g.P / (ms / 1e3)
            line.update({"value": v, "ms_per_step": ms,
                         "cpu_baseline": {"value": v, "unit": "pins/s", "cores": 0, "kind": "reference",
                                          "sample": "full workload through the reference GPU build "
                                                    "(hgraph_gpu.exe, sm_100a), its 'Total host execution time'"},
                         "e2e": {"value": v, "unit": "pins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                         "quality": {"connectivity": conn}})
            return line
    # k-way: the reference needs the external Mt-KaHyPar binary (sources/init_part.cu:891-906), which
    # is not installable offline; time the oracle's CPU port instead.
    cb = cpu_port_baseline(g, p, args.workload)
    line.update({"value": cb["value"], "ms_per_step": g.P / cb["value"] * 1e3, "cpu_baseline": cb,
                 "e2e": {"value": cb["value"], "unit": "pins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "note": "reference k-way needs mtkahypar (absent); CPU port of the oracle timed instead"})
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
    with ax.Context(local, 256 << 20) as srv:
        srv.serve_configure(args.lanes, int(args.budget_gb * (1 << 30)))
        srv.partition_batch(jobs[:args.lanes])  # warm-up: lanes, graphs of the first levels
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
                       "lanes_per_gpu": args.lanes, "budget_gb": args.budget_gb,
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
    with ax.Context(0, 256 << 20) as srv:
        srv.serve_configure(args.lanes, int(args.budget_gb * (1 << 30)))
        srv.partition_batch(reqs[:args.lanes])  # warm-up
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
                       "lanes": args.lanes, "budget_gb": args.budget_gb},
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
    ap.add_argument("--roofline-kernel", default=ROOFLINE_KERNEL)
    ap.add_argument("--ref-timeout", type=float, default=900.0,
                    help="seconds one reference partition may take before its arm reports unavailable")
    ap.add_argument("--mode", default="partition", choices=["partition", "batch", "serve"],
                    help="partition: one hypergraph per step (the headline); batch / serve: many jobs")
    ap.add_argument("--lanes", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--batch-jobs", type=int, default=256)
    ap.add_argument("--serve-requests", type=int, default=120)
    ap.add_argument("--serve-max-pins", type=float, default=2e7)
    ap.add_argument("--serve-load", type=float, default=2.0)
    ap.add_argument("--seq-arena-gb", type=float, default=24.0)
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
    out, g, p, part = run_ours(args, world, rank, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_port_baseline(g, p, args.workload)
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
