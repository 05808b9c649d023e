#!/usr/bin/env python
"""Throughput of the nricp wrapping path on B200: wraps per second.

Workload (N = 1): the large single wrap -- a 25,000-vertex ellipsoid template
with 20 bumps onto a 400,000-triangle deformed, holed, outlier-laden target;
graph 250/500/1000/2000 nodes, k = 6, 4 levels (nricp_b200.synthetic.config2,
seeded synthetic data).  One step is one whole wrap: the target's hierarchy
rebuilt, then the coarse-to-fine schedule run to completion.

Lines printed (one JSON line on rank 0):
* ``value``      wraps/s with every input resident in HBM (CUDA events on the
                 solver's stream, max over ranks),
* ``e2e``        wraps/s through the public API (nricp_dp.solve_route_b) from
                 host arrays, host<->device copies inside the timed region,
* ``roofline``   the dominant kernel's algorithmic bytes / its event time,
* ``cpu_baseline`` the reference's own FP64 route A (compiled from its
                 sources, oracle/_ref) on the host's cores.

``--impl reference`` times that reference CPU route instead (the reference has
no other implementation of this path that runs here).  With torchrun (N > 1)
every rank wraps its own target: replicas, no collective on the data path.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "wraps/sec"
WORKLOAD = ("config 2: 25k-vertex template -> 400k-triangle target, "
            "2,000 nodes (250/500/1000/2000), k=6, 4 levels, route B")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-profile", action="store_true")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------

def Ranks(gpus: int):
    """One process per GPU under torchrun (NCCL for the host bookkeeping:
    barrier, max of the times, sum of the work); a single process otherwise."""
    from nricp_b200.replicas import ReplicaGroup

    return ReplicaGroup(backend="nccl", timeout_s=600.0)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, max_sm, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                max_sm.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(max_sm) if max_sm else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference CPU route (oracle/_ref) on all host cores
# ---------------------------------------------------------------------------

def _reference_wrap(args):
    """One wrap through the reference's own route A, in a worker process."""
    seed, kind = args
    sys.path.insert(0, str(ROOT))
    from nricp_b200 import synthetic as S
    from oracle.oracle import Oracle

    case = S.config2(seed)
    options = dict(case.options)
    if kind == "reference":
        # the reference's data model caps the binding at four nodes and its
        # graph at 4-NN edges (src/core/sampling.h:17, graph.h:52-53)
        options["max_nodes_per_vertex"] = 4
        options["edge_neighbours"] = 4
    t0 = time.perf_counter()
    Oracle(kind).solve(*case.args(), **options)
    return time.perf_counter() - t0


def cpu_reference_sample(cores: int, seed: int) -> dict:
    """`cores` independent wraps, one per process (route A is single-threaded
    by construction), all at once: wraps/s of the host."""
    import multiprocessing as mp

    from oracle.oracle import reference_available

    kind = "reference" if reference_available() else "restatement"
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        times = pool.map(_reference_wrap, [(seed + i, kind) for i in range(cores)])
    elapsed = time.perf_counter() - t0
    return {"value": cores / elapsed, "unit": METRIC, "cores": cores,
            "kind": "reference" if kind == "reference" else "port",
            "sample": (f"{cores} config-2 wraps (k=4, 4-NN: the reference's caps), one per "
                       f"process on {cores} host cores, run to completion; "
                       f"per-wrap {min(times):.1f}-{max(times):.1f} s"),
            "seconds": elapsed}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, ranks):
    if ranks.rank != 0:
        return
    cores = min(host_cores(), 64)
    for _ in range(args.warmup):
        cpu_reference_warmup()
    samples = []
    for _ in range(args.steps):
        samples.append(cpu_reference_sample(cores, args.seed))
    value = statistics.median(s["value"] for s in samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * statistics.median(s["seconds"] for s in samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy generator, nricp_b200.synthetic.config2)",
        "config": {"workload": WORKLOAD, "model": None, "inputs": "host memory"},
        "cpu_baseline": {k: samples[-1][k] for k in ("kind", "cores", "sample")} | {"value": value,
                                                                                    "unit": METRIC},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_reference_warmup():
    sys.path.insert(0, str(ROOT))
    from nricp_b200 import synthetic as S
    from oracle.oracle import Oracle, reference_available

    case = S.small_case()
    Oracle("reference" if reference_available() else "restatement").solve(*case.args(), **case.options)


# ---------------------------------------------------------------------------
# algorithmic bytes per launch (the formulas of the design's roofline table)
# ---------------------------------------------------------------------------

def query_bytes(s: dict) -> float:
    # V (24 in + 33 out) + one read of the tree (2F x 32) + mesh (F x 12 + Vt x 24)
    return s["vertices"] * 57 + s["target_triangles"] * 76 + s["target_vertices"] * 24


def pcg_bytes(s: dict, iterations: int) -> float:
    # per iteration N x 504 + (E + G) x 248
    return iterations * (s["nodes"] * 504 + (s["edges"] + s["pairs"]) * 248)


def assembly_bytes(s: dict) -> float:
    # S x 98 + P x 106 + V x 98 + N x 168 + (E + G) x 144
    return (s["entries"] * 98 + s["pair_entries"] * 106 + s["vertices"] * 98 +
            s["nodes"] * 168 + (s["edges"] + s["pairs"]) * 144)


def roofline(batch, peak_gbs: float) -> tuple[dict, dict]:
    records = batch.profile()
    levels = batch.level_sizes(0, 0)["levels"]
    sizes = [batch.level_sizes(0, l) for l in range(levels)]
    kernels = {"query": [0.0, 0.0, 0], "pcg": [0.0, 0.0, 0], "assembly": [0.0, 0.0, 0]}
    for r in records:
        s = sizes[min(r["level"], levels - 1)]
        if r["phase"] in (0, 1, 3):  # transfer / refresh / final: the query works
            kernels["query"][0] += r["query_ms"]
            kernels["query"][1] += query_bytes(s)
            kernels["query"][2] += 1
        if r["phase"] == 2 and r["pcg_iterations"] > 0:
            kernels["pcg"][0] += r["pcg_ms"]
            kernels["pcg"][1] += pcg_bytes(s, r["pcg_iterations"])
            kernels["pcg"][2] += 1
        if r["phase"] in (0, 1, 2):
            kernels["assembly"][0] += r["assemble_ms"]
            kernels["assembly"][1] += assembly_bytes(s)
            kernels["assembly"][2] += 1
    total_tick = sum(r["tick_ms"] for r in records)
    dominant = max(kernels, key=lambda k: kernels[k][0])
    ms, nbytes, launches = kernels[dominant]
    achieved = (nbytes / launches) / (ms / launches * 1e-3) / 1e9 if ms > 0 else 0.0
    detail = {k: {"ms": v[0], "launches": v[2], "share_of_ticks": v[0] / total_tick if total_tick else 0,
                  "gbs": (v[1] / (v[0] * 1e-3) / 1e9) if v[0] > 0 else 0.0}
              for k, v in kernels.items()}
    by_level = {}
    for r in records:
        if r["phase"] == 2:
            entry = by_level.setdefault(r["level"], {"solves": 0, "iterations": 0, "pcg_ms": 0.0,
                                                     "max_iterations": 0})
            entry["solves"] += 1
            entry["iterations"] += r["pcg_iterations"]
            entry["pcg_ms"] += r["pcg_ms"]
            entry["max_iterations"] = max(entry["max_iterations"], r["pcg_iterations"])
    detail["pcg_by_level"] = by_level
    detail["ticks"] = len(records)
    detail["tick_ms_total"] = total_tick
    line = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak_gbs,
            "unit": "GB/s", "frac": achieved / peak_gbs if peak_gbs else None,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": None, "algorithmic_bytes_per_launch": nbytes / max(1, launches),
            "avg_launch_us": 1000.0 * ms / max(1, launches)}
    return line, detail


def measured_peak() -> float:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def flush_l2():
    """Writes a buffer larger than the 126 MB L2 between timed steps."""
    import torch

    buf = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    buf.fill_(1)
    torch.cuda.synchronize()
    del buf


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, ranks):
    import torch

    from nricp_b200 import nricp_dp as dp
    from nricp_b200 import synthetic as S

    torch.cuda.set_device(ranks.local)
    case = S.config2(args.seed + ranks.rank)
    batch = dp.WrapBatch([(*case.args(), case.options)])

    # ---- value: device-resident steps ----
    for _ in range(max(3, args.warmup)):
        batch.step()
    step_ms = []
    launches = 0
    ranks.barrier()
    torch.cuda.synchronize()
    with ClockSampler(ranks.local) as clocks:
        for _ in range(args.steps):
            flush_l2()
            step_ms.append(batch.step())
            launches += batch.counters()[1]
    torch.cuda.synchronize()
    ranks.barrier()
    total_ms = ranks.max(sum(step_ms))
    wraps = ranks.sum(float(args.steps))
    value = wraps / (total_ms * 1e-3)

    # ---- e2e: the public API from host arrays ----
    dp.solve_route_b(*case.args(), **case.options)  # warm
    dp.transfer_counters(reset=True)
    ranks.barrier()
    e2e_steps = max(2, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dp.solve_route_b(*case.args(), **case.options)
    torch.cuda.synchronize()
    e2e_s = ranks.max(time.perf_counter() - t0)
    h2d, d2h = dp.transfer_counters(reset=True)
    result_bytes = case.template_points.nbytes + 8 * 12 * batch.level_sizes(0, 3)["nodes"]
    e2e = {"value": ranks.sum(float(e2e_steps)) / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(h2d / e2e_steps),
           "d2h_bytes_per_step": int(d2h / e2e_steps + result_bytes)}

    # ---- roofline of the dominant kernel ----
    roof, detail = (None, None)
    if not args.no_profile:
        roof, detail = roofline(batch, measured_peak())

    result = batch.result(0)
    report = json.loads(result["report"])

    cpu = None
    if ranks.rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(min(host_cores(), 64), args.seed)
        cpu.pop("seconds", None)

    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ranks.world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded numpy generator, nricp_b200.synthetic.config2)",
        "config": {"workload": WORKLOAD, "model": None, "global_batch": ranks.world,
                   "template_vertices": int(len(case.template_points)),
                   "target_triangles": int(len(case.target_faces)),
                   "parallelism": f"replicas x{ranks.world}",
                   "l2": "flushed (256 MB write) between timed steps",
                   "precision": "FP32 assembly/matvec/traversal, FP64 state/energies/dots/Horn"},
        "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                       "steps": [round(x, 3) for x in step_ms]},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "e2e": e2e,
        "roofline": roof,
        "kernels": detail,
        "cpu_baseline": cpu,
        "fit": {"energy": report["energy"]["total"],
                "levels": [(l["outer_iterations"], l["inner_iterations"]) for l in report["levels"]]},
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    ranks = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, ranks)
        else:
            run_ours(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
