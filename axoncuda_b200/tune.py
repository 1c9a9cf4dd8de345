"""Autotuner for the tile and table sizes and the executor settings of axc_tune_set.

    python -m axoncuda_b200.tune [--jobs 64] [--out axoncuda_b200/tuned_b200.json]

None of the tuned values changes a partition, only the time it takes; the tuner checks that every
candidate gives the same partitions as the defaults, and refuses a candidate that does not.

1. Calibration jobs: a sample drawn by the batched workload's rule (circuit-style and layered-SNN
   hypergraphs, node counts log-uniform in [1e3, 1e5], k-way with k in {2, 8, 32}, eps 0.03),
   from seeds of their own.
2. Size classes by pins: [0, 2^17), [2^17, 2^20), [2^20, 2^23), [2^23, inf). Per class, coordinate
   descent over the block rating's first-try table (rate.try_slots), its second try
   (rate.mid_slots) and the cascade block kernel's movers (cascade.block_movers): each candidate
   is timed as a sequential loop over the class's jobs on one warm context, best of `reps`.
3. The executor: lanes x serve.exclusive_pins over the whole sample through axc_partition_batch
   with the chosen class settings.

The result is a JSON table; `apply(ctx, path)` sets it on a context (before its first submit) and
returns its lane count.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import Context, gen_circuit, gen_snn, lib, params_kway

CLASS_EDGES = [0, 1 << 17, 1 << 20, 1 << 23]
DEFAULTS = {"rate.try_slots": 2048, "rate.mid_slots": 8192, "cascade.block_movers": 0}
CANDIDATES = (("rate.try_slots", [512, 1024, 2048, 4096]), ("rate.mid_slots", [4096, 8192, 16384]),
              ("cascade.block_movers", [0, 512, 1024]))  # 0: the kernel's default of 2048 movers
LANES = [1, 2, 4, 8, 16]
EXCLUSIVE = [0, 1 << 20, 1 << 22]


def calibration_jobs(count: int, seed0: int = 9000):
    """`count` jobs by the batched workload's rule, from seeds of their own."""
    rng = np.random.default_rng(seed0)
    jobs = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e5)))))
        k = int(rng.choice([2, 8, 32]))
        s = seed0 + i
        g = gen_circuit(n, int(1.1 * n), 2, 64, 2.5, 0.9, 0.02, s) if i % 2 == 0 else \
            gen_snn(8, max(n // 8, 65), 64, 0.0, 0, 1.0, s)
        jobs.append((g, params_kway(k, 0.03, cnc=4, rfr=16)))
    return jobs


def size_class(pins: int) -> int:
    return max(i for i, lo in enumerate(CLASS_EDGES) if pins >= lo)


def time_loop(ctx: Context, jobs, reps: int):
    """Best-of-reps seconds of a sequential loop over the jobs, and the partitions."""
    best, parts = float("inf"), None
    for _ in range(reps):
        t0 = time.perf_counter()
        parts = [ctx.partition(g, p)[0] for g, p in jobs]
        best = min(best, time.perf_counter() - t0)
    return best, parts


def tune_class(jobs, reps: int, device: int) -> tuple[dict, dict]:
    """Coordinate descent over the three kernel sizes for one class's jobs."""
    cur, log = dict(DEFAULTS), {}
    with Context(device, 8 << 30) as ctx:
        for g, p in jobs[:2]:
            ctx.partition(g, p)  # warm-up
        best_t, ref = time_loop(ctx, jobs, reps)
        log["defaults"] = best_t
        for key, values in CANDIDATES:
            for v in values:
                trial = dict(cur, **{key: v})
                if trial == cur:
                    continue
                for k2, v2 in trial.items():
                    ctx.tune(k2, v2)
                t, parts = time_loop(ctx, jobs, reps)
                if not all(np.array_equal(a, b) for a, b in zip(parts, ref)):
                    raise RuntimeError(f"tuning {key}={v} changed a partition")
                log[f"{key}={v}"] = t
                if t < best_t:
                    best_t, cur = t, trial
            for k2, v2 in cur.items():
                ctx.tune(k2, v2)
    log["chosen"] = best_t
    return cur, log


def tune_executor(jobs, classes: list[dict], device: int) -> tuple[dict, dict]:
    """Lanes and the exclusive-job threshold over the whole sample."""
    log, best = {}, (float("inf"), None)
    for lanes in LANES:
        for excl in EXCLUSIVE:
            with Context(device, 256 << 20) as srv:
                srv.serve_configure(lanes, 120 << 30)
                srv.tune("serve.exclusive_pins", excl)
                for i, c in enumerate(classes):
                    for k, v in c.items():
                        srv.tune(f"class.{i}.{k}", v)
                srv.partition_batch(jobs[:lanes])  # warm-up: the lanes
                t0 = time.perf_counter()
                srv.partition_batch(jobs)
                t = time.perf_counter() - t0
            log[f"lanes={lanes},exclusive_pins={excl}"] = t
            if t < best[0]:
                best = (t, {"lanes": lanes, "serve.exclusive_pins": excl})
    return best[1], log


def apply(ctx: Context, path: str) -> int:
    """Sets a tuning table on a context (before its first submit); returns its lane count."""
    with open(path) as f:
        t = json.load(f)
    for i, c in enumerate(t["classes"]):
        for k, v in c.items():
            ctx.tune(f"class.{i}.{k}", int(v))
    ctx.tune("serve.exclusive_pins", int(t["serve.exclusive_pins"]))
    return int(t["lanes"])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json"))
    a = ap.parse_args()
    lib()
    jobs = calibration_jobs(a.jobs)
    by_class: dict[int, list] = {}
    for g, p in jobs:
        by_class.setdefault(size_class(g.P), []).append((g, p))
    classes, sweep = [], {}
    for ci, lo in enumerate(CLASS_EDGES):
        cj = by_class.get(ci, [])
        chosen, log = tune_class(cj[:16], a.reps, a.device) if cj else (dict(DEFAULTS), {})
        classes.append(dict({"min_pins": lo}, **chosen))
        sweep[f"class {ci} (>= {lo} pins, {len(cj)} jobs)"] = log
        print(f"class {ci}: {chosen}", flush=True)
    ex, exlog = tune_executor(jobs, classes, a.device)
    sweep["executor"] = exlog
    print(f"executor: {ex}", flush=True)
    out = {"device": "B200", "calibration_jobs": a.jobs, "classes": classes, **ex, "sweep_seconds": sweep,
           "command": f"python -m axoncuda_b200.tune --jobs {a.jobs} --reps {a.reps}"}
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
    print(f"written {a.out}", flush=True)


if __name__ == "__main__":
    main()
