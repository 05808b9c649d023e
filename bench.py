#!/usr/bin/env python
"""Throughput of the nricp wrapping path on B200: wraps per second, batched
against one wrap at a time, at equal fit error.

Workload (N = 1): 64 uneven wraps solved as one batch -- template vertices
log-uniform in [5k, 50k] (ellipsoid grids with 20 bumps), graph nodes = V/15
over 4 levels, k = 6, targets log-uniform in [50k, 500k] triangles (deformed,
holed, 1 % outliers); seeded synthetic data (nricp_b200.synthetic.config3).
One step is the whole batch: every target's hierarchy rebuilt, then every
wrap's coarse-to-fine schedule run to completion, all wraps advancing
together (one launch sequence per tick, replayed as a CUDA graph).

Printed (one JSON line on rank 0):
* ``value``        batched wraps/s, inputs resident in HBM (CUDA events on
                   the batch's stream; the 64 wraps' data, ~3 GB, exceeds L2
                   and a 256 MB write flushes it between steps as well),
* ``plain``        the same 64 wraps one at a time through the same engine,
                   and ``batched_vs_plain``,
* ``latency_ms``   per-wrap latency one at a time (p50/p99 over the wraps)
                   and the batch's step time (p50/p99 over the steps),
* ``e2e``          wraps/s through the public API (nricp_dp.solve_batch) from
                   host arrays: host graph builds, uploads, hierarchy builds,
                   the solve and the result download all inside the clock,
* ``roofline``     the dominant kernel's algorithmic bytes over the batch
                   run / its CUDA-event time, against the measured HBM peak,
* ``fit``          max vertex error and final-energy error of the GPU route
                   against the reference's FP64 route A on a sample,
* ``cpu_baseline`` the reference's own route A (compiled from its sources,
                   oracle/_ref) on the host cores, on a bounded sample,
* ``served``       the same wraps as requests arriving in Poisson windows
                   (config 4's 5, 20 and 80 per second by default; 5 is below
                   the server's capacity) served with continuous batching:
                   throughput, p50/p99 latency and p50/p99 of each phase of
                   a request's latency per window,
* ``single_wrap``  the large single wrap of config 2 (25k vertices onto a
                   393k-triangle target, 2,000 nodes) one at a time.

``--impl reference`` times that reference CPU route instead.
``--precision OUT.npz`` solves config 5 (100k-vertex template onto a
2M-triangle target, 10,000 nodes) with the shipped library and with its
variant whose solve reductions are FP32; ``--precision-compare OUT.npz`` then
runs the reference's FP64 route A on the same problem on the CPU and reports
max/RMS vertex error over the diagonal and the energy per level.  With torchrun
(N > 1) every rank solves its own 64-wrap batch: replicas, no collective on
the data path.
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
WORKLOAD = ("config 3: 64 uneven wraps batched (template 5k-50k vertices log-uniform, "
            "nodes = V/15 over 4 levels, k=6, target 50k-500k triangles log-uniform), route B")
INSTANCES = 64
REFERENCE_SAMPLE = 16   # wraps per CPU-reference sample
# DRAM traffic of a seeded closest-point query over its algorithmic bytes,
# measured with ncu on one config-2 wrap (median of 15 seeded launches)
QUERY_TRAFFIC_RATIO = 1.22
SAME_CONFIG_REASON = (
    "the reference arm times the reference's FP64 route A on the 16 smallest of config 3's 64 wraps "
    "at its own caps (k=4 bindings, 4-NN edges; src/core/sampling.h:17, graph.h:52-53), one process "
    "per wrap: the reference cannot bind k=6, and its largest wraps take minutes each on one core. "
    "Our line's value is all 64 wraps at k=6; its same_sample_as_reference field times this engine "
    "on exactly the reference arm's sample and settings")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-profile", action="store_true")
    p.add_argument("--instances", type=int, default=INSTANCES,
                   help="wraps in the batch (config 3 has 64; fewer for profiling captures)")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--batch-only", action="store_true",
                   help="only the batched value (for profiler captures of its launches)")
    p.add_argument("--precision", metavar="OUT.npz",
                   help="config 5 on the GPU with the shipped library and its FP32-reductions "
                        "variant; writes both results to OUT.npz")
    p.add_argument("--precision-variant", metavar="OUT.npz", help=argparse.SUPPRESS)
    p.add_argument("--capture-steps", type=int, default=0,
                   help="profiler captures: the config-2 wrap through RouteBSession for this many "
                        "ticks, eager launches, nothing timed")
    p.add_argument("--capture-batch", type=int, default=0, metavar="N",
                   help="profiler captures: one step of a batch of config 3's first N wraps with "
                        "eager launches (the kernel-group re-run, branches one after the other), "
                        "nothing timed")
    p.add_argument("--precision-compare", metavar="IN.npz",
                   help="CPU only: the reference's FP64 route A on config 5 and its spread under "
                        "perturbations, against the GPU results of --precision ('-': none)")
    p.add_argument("--perturb-seeds", type=int, default=5,
                   help="--precision-compare: independent perturbation draws per size")
    p.add_argument("--perturb-sigmas", default="1e-12,1e-9",
                   help="--precision-compare: perturbation sizes, relative to the target diagonal")
    p.add_argument("--precision-cache", default=None, metavar="DIR",
                   help="--precision-compare: store each route-A run here and reuse it")
    p.add_argument("--precision-workers", type=int, default=0,
                   help="--precision-compare: processes (default: the host's cores)")
    p.add_argument("--serve-rates", default="5,20,80",
                   help="Poisson arrival rates (requests/s) of the serving windows")
    p.add_argument("--serve-seconds", type=float, default=6.0,
                   help="length of each serving window (the full protocol: 60)")
    p.add_argument("--serve-large", type=float, default=0.1,
                   help="fraction of requests drawn from the large (100k-vertex, 2M-triangle) cases")
    return p.parse_args()


def Ranks(gpus: int):
    """One process per GPU under torchrun (NCCL for the host bookkeeping:
    barrier, max of the times, sum of the work); a single process otherwise."""
    from nricp_b200.replicas import ReplicaGroup

    return ReplicaGroup(backend="nccl", timeout_s=600.0)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def make_cases(seed: int, instances: int = INSTANCES):
    from nricp_b200 import synthetic as S

    return S.config3(seed, instances=instances, workers=min(16, host_cores()))


def reference_options(options: dict) -> dict:
    """The reference's data model caps the binding at four nodes and its graph
    at 4-NN edges (src/core/sampling.h:17, graph.h:52-53)."""
    out = dict(options)
    out["max_nodes_per_vertex"] = 4
    out["edge_neighbours"] = 4
    return out


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
# the reference CPU route (oracle/_ref) on the host's cores
# ---------------------------------------------------------------------------

def _reference_wrap(args):
    """One config-3 wrap through the reference's own route A, in a worker."""
    spec, kind = args
    sys.path.insert(0, str(ROOT))
    from nricp_b200 import synthetic as S
    from oracle.oracle import Oracle

    case = S.config3_case(spec)
    t0 = time.perf_counter()
    result = Oracle(kind).solve(*case.args(), **reference_options(case.options))
    seconds = time.perf_counter() - t0
    return seconds, result["vertices"], json.loads(result["report"])["energy"]["total"]


def reference_gpu_sample(dp, cases, idx, route_a_vertices):
    """The reference's own GPU route B (its src/cuda, compiled for sm_100a in
    oracle/_ref) one wrap at a time on the CPU sample's wraps, beside this
    engine on the same wraps and settings (the reference's caps), one at a
    time and as one batch -- each through its public call from host arrays --
    with both routes' errors against route A."""
    from oracle.oracle import Oracle

    try:
        ref = Oracle("reference_gpu")
    except (FileNotFoundError, OSError) as error:
        return {"unavailable": str(error)}
    same = [(*cases[i].args(), reference_options(cases[i].options)) for i in idx]
    ref.solve(*same[0][:5], **same[0][5])  # warm: the reference's device set-up
    t0 = time.perf_counter()
    theirs = [ref.solve(*c[:5], **c[5]) for c in same]
    ref_s = time.perf_counter() - t0
    dp.solve_route_b(*same[0][:5], **same[0][5])
    t0 = time.perf_counter()
    ours_one = [dp.solve_route_b(*c[:5], **c[5]) for c in same]
    ours_one_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    dp.solve_batch(same)
    ours_batch_s = time.perf_counter() - t0

    def worst(results):
        out = 0.0
        for i, r, a in zip(idx, results, route_a_vertices):
            p = cases[i].target_points
            out = max(out, float(np.abs(r["vertices"] - a).max()) / float(np.linalg.norm(p.max(0) - p.min(0))))
        return out

    n = len(same)
    return {"sample": f"the CPU sample's {n} wraps, the reference's caps (k=4, 4-NN), host arrays in and out",
            "reference_route_b_one_at_a_time": n / ref_s,
            "ours_one_at_a_time": n / ours_one_s,
            "ours_batched": n / ours_batch_s,
            "unit": METRIC,
            "max_vertex_error_over_diag_vs_route_a": {"reference_route_b": worst(theirs),
                                                      "ours": worst(ours_one)}}


def cpu_reference_sample(seed: int, cores: int) -> dict:
    """The sample's wraps, one per process (route A is single-threaded by
    construction), all at once: wraps/s of the host on that sample."""
    import multiprocessing as mp

    from nricp_b200 import synthetic as S
    from oracle.oracle import reference_available

    kind = "reference" if reference_available() else "restatement"
    specs = S.config3_specs(seed, INSTANCES)
    order = sorted(range(INSTANCES), key=lambda i: (specs[i][1], i))
    picked = sorted(order[:REFERENCE_SAMPLE])
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(min(cores, len(picked))) as pool:
        out = pool.map(_reference_wrap, [(specs[i], kind) for i in picked])
    elapsed = time.perf_counter() - t0
    times = [o[0] for o in out]
    sizes = [specs[i][1] for i in picked]
    return {"value": len(picked) / elapsed, "unit": METRIC, "cores": min(cores, len(picked)),
            "kind": "reference" if kind == "reference" else "port",
            "sample": (f"the {len(picked)} smallest of the 64 config-3 wraps ({min(sizes)}-"
                       f"{max(sizes)} template vertices; k=4, 4-NN: the reference's caps), one "
                       f"per process, run to completion; per wrap {min(times):.1f}-"
                       f"{max(times):.1f} s"),
            "seconds": elapsed, "indices": picked,
            "vertices": [o[1] for o in out], "energies": [o[2] for o in out]}


def run_reference_arm(args, ranks):
    if ranks.rank != 0:
        return
    cores = host_cores()
    for _ in range(args.warmup):
        cpu_reference_warmup()
    samples = [cpu_reference_sample(args.seed, cores) for _ in range(args.steps)]
    value = statistics.median(s["value"] for s in samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * statistics.median(s["seconds"] for s in samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy generator, nricp_b200.synthetic.config3)",
        "config": {"workload": WORKLOAD, "inputs": "host memory"},
        "same_config": False,
        "same_config_reason": SAME_CONFIG_REASON,
        "cpu_baseline": {k: samples[-1][k] for k in ("kind", "cores", "sample")} | {
            "value": value, "unit": METRIC},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_reference_warmup():
    from nricp_b200 import synthetic as S
    from oracle.oracle import Oracle, reference_available

    case = S.small_case()
    Oracle("reference" if reference_available() else "restatement").solve(*case.args(), **case.options)


# ---------------------------------------------------------------------------
# algorithmic bytes (the formulas of the design's roofline table)
# ---------------------------------------------------------------------------

def query_bytes(s: dict) -> float:
    # per pass: V (24 in + 33 out) + one read of the tree (2F x 32) + mesh (F x 12 + Vt x 24)
    return s["vertices"] * 57 + s["target_triangles"] * 76 + s["target_vertices"] * 24


def pcg_bytes(s: dict) -> float:
    # per iteration: N x 504 + B x 248 (B off-diagonal blocks, one per coupled node pair)
    return s["nodes"] * 504 + s["offdiag_blocks"] * 248


def assembly_bytes(s: dict) -> float:
    # per pass: S x 98 + P x 106 + V x 98 + N x 168 + (E + G) x 144
    return (s["entries"] * 98 + s["pair_entries"] * 106 + s["vertices"] * 98 +
            s["nodes"] * 168 + (s["edges"] + s["pairs"]) * 144)


def roofline(batch, peak_gbs: float) -> tuple[dict, dict]:
    """Re-runs the batch with CUDA events around the query, the solve and the
    assembly of every tick, then divides each kernel group's algorithmic bytes
    over every wrap (per-level work counters of that run) by its event time."""
    records = batch.profile()
    ms = {"query": sum(r["query_ms"] for r in records), "pcg": sum(r["pcg_ms"] for r in records),
          "assembly": sum(r["assemble_ms"] for r in records)}
    nbytes = {"query": 0.0, "pcg": 0.0, "assembly": 0.0}
    launches = len(records)
    work = {"pcg_iterations": 0, "solves": 0, "queries": 0, "assemblies": 0}
    for i in range(len(batch)):
        levels = batch.level_sizes(i, 0)["levels"]
        for level in range(levels):
            s = batch.level_sizes(i, level)
            nbytes["query"] += s["queries"] * query_bytes(s)
            nbytes["pcg"] += s["pcg_iterations"] * pcg_bytes(s)
            nbytes["assembly"] += s["assemblies"] * assembly_bytes(s)
            for k in work:
                work[k] += s[k]
    total_tick = sum(r["tick_ms"] for r in records)
    dominant = max(ms, key=lambda k: ms[k])
    achieved = nbytes[dominant] / (ms[dominant] * 1e-3) / 1e9 if ms[dominant] > 0 else 0.0
    detail = {k: {"ms": ms[k], "share_of_ticks": ms[k] / total_tick if total_tick else 0.0,
                  "algorithmic_gb": nbytes[k] / 1e9,
                  "gbs": nbytes[k] / (ms[k] * 1e-3) / 1e9 if ms[k] > 0 else 0.0} for k in ms}
    detail["ticks"] = launches
    detail["timing"] = ("CUDA events per kernel group on a re-run whose ticks run the solve and refresh "
                        "branches one after the other; the timed step runs them side by side")
    detail["tick_ms_total"] = total_tick
    # how the step's time is spread over its ticks: the share of each tenth of
    # the ticks, in order (late tenths carry only the wraps still running)
    tenth = max(1, len(records) // 10)
    detail["tick_ms_by_tenth"] = [round(sum(r["tick_ms"] for r in records[i:i + tenth]), 1)
                                  for i in range(0, len(records), tenth)]
    detail["work"] = work
    per_launch = nbytes[dominant] / max(1, launches)
    traffic = QUERY_TRAFFIC_RATIO * per_launch if dominant == "query" else None
    line = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak_gbs,
            "unit": "GB/s", "frac": achieved / peak_gbs if peak_gbs else None,
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)", "traffic": traffic,
            "traffic_source": (f"{QUERY_TRAFFIC_RATIO} x the algorithmic bytes per launch: the DRAM "
                               "read+write of seeded query launches of one config-2 wrap over their "
                               "algorithmic bytes (ncu, profiles/k_query_dram_config2_wrap.md)")
                              if traffic is not None else None,
            "algorithmic_bytes_per_launch": nbytes[dominant] / max(1, launches),
            "avg_launch_us": 1000.0 * ms[dominant] / max(1, launches)}
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


def serve_window(server, cases, rate: float, seconds: float, rng, large=(), large_fraction=0.0) -> dict:
    """Requests drawn from `cases` (a `large_fraction` of them from `large`)
    arriving as a Poisson process at `rate` per second for `seconds`; latency
    is submit to result ready."""
    submitted = []
    large_count = 0
    t0 = time.perf_counter()
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            break
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        if large and rng.random() < large_fraction:
            c = large[int(rng.integers(len(large)))]
            large_count += 1
        else:
            c = cases[int(rng.integers(len(cases)))]
        submitted.append((time.perf_counter(), server.submit(*c.args(), **c.options)))
    latencies, finished, phases = [], [], {k: [] for k in server.PHASES}
    for ts, rid in submitted:
        state, latency = server.wait(rid, timeout=900.0)
        if state != "done":
            raise RuntimeError(f"served request {rid} ended {state}")
        for k, v in server.phases(rid).items():
            phases[k].append(1000.0 * v)
        server.result(rid)
        latencies.append(1000.0 * latency)
        finished.append(ts + latency)
    span = max(finished) - submitted[0][0] if submitted else 0.0
    out = {"rate_per_s": rate, "seconds": seconds, "requests": len(submitted), "large_requests": large_count,
           "wraps_per_second": len(submitted) / span if span > 0 else 0.0}
    out.update({f"latency_{k}_ms": v for k, v in percentiles(latencies).items() if k != "n"})
    out["phase_ms"] = {k: {q: round(x, 2) for q, x in percentiles(v).items() if q != "n"}
                       for k, v in phases.items()}
    return out


def large_requests(seed: int, count: int = 2):
    """Config 4's large requests: 100k-vertex templates onto 2M-triangle
    targets with 10,000 nodes, generated as in config 2."""
    from nricp_b200 import synthetic as S

    return [S.config2(seed=10_000 + seed * 10 + i, vertex_count=100_000, triangle_count=2_000_000,
                      nodes_finest=10_000, k=6, levels=4) for i in range(count)]


def run_serving(dp, cases, rates, seconds, seed, large=(), large_fraction=0.0) -> dict:
    budget = 120 * 10**9
    with dp.WrapServer(memory_budget_bytes=budget, max_slots=64) as server:
        # warm: every template's graph cached, the launch shape captured
        for rid in [server.submit(*c.args(), **c.options) for c in list(cases) + list(large)]:
            server.result(rid, timeout=900.0)
        rng = np.random.default_rng(seed)
        windows = []
        for r in rates:
            before = server.stats()
            windows.append(serve_window(server, cases, r, seconds, rng, large, large_fraction))
            after = server.stats()
            windows[-1]["ticks"] = after["ticks"] - before["ticks"]
            windows[-1]["tick_device_s"] = after["busy_seconds"] - before["busy_seconds"]
        stats = server.stats()
    return {"workload": ("Poisson arrivals drawn from the 64 config-3 wraps" +
                         (f" and, with probability {large_fraction:g}, from {len(large)} large requests "
                          "(100k-vertex template, 2M-triangle target, 10,000 nodes)" if large else "") +
                         ", continuous batching, 64 resident slots, 120 GB admission budget"),
            "windows": windows, "graph_captures": stats["captures"],
            "peak_resident_gb": stats["peak_resident_bytes"] / 1e9}


def percentiles(values) -> dict:
    v = sorted(values)
    if not v:
        return {}
    pick = lambda q: v[min(len(v) - 1, int(math.ceil(q * len(v))) - 1)]  # noqa: E731
    return {"p50": pick(0.50), "p99": pick(0.99), "n": len(v)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, ranks):
    import torch

    from nricp_b200 import nricp_dp as dp
    from nricp_b200 import synthetic as S

    torch.cuda.set_device(ranks.local)
    cases = make_cases(args.seed + ranks.rank, args.instances)
    tuples = [(*c.args(), c.options) for c in cases]

    # ---- value: the batch, device-resident ----
    batch = dp.WrapBatch(tuples)
    tuning = batch.autotune()  # measured; every setting gives the same bits
    cluster = tuning["largest_cluster"]
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
    wraps = ranks.sum(float(args.steps * len(cases)))
    value = wraps / (total_ms * 1e-3)
    if args.batch_only:
        if ranks.rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ranks.world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                              "gpu_launches": launches, "batch_only": True}), flush=True)
        return

    # ---- plain: the same wraps one at a time through the same engine ----
    plain_ms = []
    plain_results = []
    for t in tuples:
        one = dp.WrapBatch([t])
        one.step()
        plain_ms.append(one.step())
        plain_results.append(one.result(0)["vertices"])
        del one
    plain_total = ranks.max(sum(plain_ms))
    plain = ranks.sum(float(len(cases))) / (plain_total * 1e-3)
    identical = sum(int(np.array_equal(plain_results[i], batch.result(i)["vertices"]))
                    for i in range(len(cases)))

    # ---- e2e: the public API from host arrays ----
    for _ in range(2):  # warm-up: the process's page-locked staging, device pool and host heap
        dp.solve_batch(tuples)
    dp.transfer_counters(reset=True)
    ranks.barrier()
    e2e_steps = 5  # calls of ~0.9 s each; host outliers of one call weigh less over five
    call_s, prep_s, solve_s = [], [], []
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        results = dp.solve_batch(tuples)
        call_s.append(time.perf_counter() - t1)
        reports = [json.loads(r["report"]) for r in results]
        prep_s.append(sum(r["setup_seconds"] for r in reports))
        solve_s.append(max(r["solve_seconds"] for r in reports))
    torch.cuda.synchronize()
    e2e_s = ranks.max(time.perf_counter() - t0)
    h2d, d2h = dp.transfer_counters(reset=True)
    e2e = {"value": ranks.sum(float(e2e_steps * len(cases))) / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(h2d / e2e_steps), "d2h_bytes_per_step": int(d2h / e2e_steps),
           "call_seconds": [round(x, 3) for x in call_s],
           "preparation_seconds": [round(x, 3) for x in prep_s],
           "solve_seconds": [round(x, 3) for x in solve_s],
           "how": "nricp_dp.solve_batch on the 64 wraps from host arrays, five calls after two untimed "
                  "calls; preparation = input checks, graphs, layouts, uploads and hierarchies (the "
                  "reports' setup_seconds summed), solve = the device schedule"}

    # ---- roofline of the dominant kernel over the batch ----
    roof, detail = (None, None)
    if not args.no_profile:
        roof, detail = roofline(batch, measured_peak())

    # ---- CPU reference sample and the fit against it ----
    cpu, fit, reference_gpu, same_sample = None, None, None, None
    if ranks.rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(args.seed, host_cores())
        idx = cpu.pop("indices")
        ref_vertices, ref_energies = cpu.pop("vertices"), cpu.pop("energies")
        cpu.pop("seconds", None)
        same = [(*cases[i].args(), reference_options(cases[i].options)) for i in idx]
        ours = dp.solve_batch(same)
        errors, energy_errors = [], []
        for i, mine, rv, re in zip(idx, ours, ref_vertices, ref_energies):
            p = cases[i].target_points
            diag = float(np.linalg.norm(p.max(0) - p.min(0)))
            errors.append(float(np.abs(mine["vertices"] - rv).max()) / diag)
            e = json.loads(mine["report"])["energy"]["total"]
            energy_errors.append(abs(e - re) / abs(re) if re else abs(e))
        order = sorted(range(len(errors)), key=lambda k: errors[k])
        fit = {"against": "the reference's FP64 route A (oracle/_ref) on the CPU sample, "
                          "same settings (k=4, 4-NN)",
               "wraps": len(idx), "max_vertex_error_over_diag": max(errors),
               "median_vertex_error_over_diag": errors[order[len(order) // 2]],
               "max_final_energy_rel_error": max(energy_errors),
               "wraps_within_1e-4": sum(1 for e in errors if e <= 1e-4)}
        reference_gpu = reference_gpu_sample(dp, cases, idx, ref_vertices)
        same_sample = {
            "sample": cpu["sample"], "unit": METRIC,
            "reference_cpu_route_a": cpu["value"],
            "ours_batched_from_host_arrays": reference_gpu.get("ours_batched"),
            "ours_over_reference": (reference_gpu["ours_batched"] / cpu["value"]
                                    if reference_gpu.get("ours_batched") and cpu["value"] else None)}

    # ---- serving: continuous batching under Poisson arrivals ----
    served = None
    if ranks.rank == 0 and not args.no_serve:
        rates = [float(x) for x in args.serve_rates.split(",") if x]
        large = large_requests(args.seed) if args.serve_large > 0 else []
        served = run_serving(dp, cases, rates, args.serve_seconds, args.seed, large, args.serve_large)
        served["vs_plain"] = {f"{w['rate_per_s']:g}/s": w["wraps_per_second"] / plain
                              for w in served["windows"]}

    # ---- the large single wrap (config 2), one at a time ----
    single = None
    if ranks.rank == 0:
        c2 = S.config2(args.seed)
        one = dp.WrapBatch([(*c2.args(), c2.options)])
        one.step()
        ms2 = [one.step() for _ in range(3)]
        single = {"workload": "config 2: 25k-vertex template -> 393k-triangle target, 2,000 nodes, "
                              "k=6, 4 levels, route B",
                  "value": 1000.0 / statistics.median(ms2), "unit": METRIC,
                  "ms": [round(x, 2) for x in ms2]}
        del one

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ranks.world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded numpy generator, nricp_b200.synthetic.config3)",
        "config": {"workload": WORKLOAD, "wraps_per_gpu": len(cases),
                   "template_vertices": [int(min(len(c.template_points) for c in cases)),
                                         int(max(len(c.template_points) for c in cases))],
                   "target_triangles": [int(min(len(c.target_faces) for c in cases)),
                                        int(max(len(c.target_faces) for c in cases))],
                   "parallelism": f"replicas x{ranks.world}",
                   "solve_cluster": {"autotuned": tuning["choice"], "largest": cluster,
                                     "candidates_ms": tuning["ms"]},
                   "l2": "inputs larger than L2 (~3 GB per batch), plus a 256 MB write between steps",
                   "precision": "FP32 assembly/matvec/traversal, FP64 state/energies/dots/Horn",
                   "host_allocator": " ".join(f"{k}={os.environ.get(k)}" for k in ALLOCATOR)},
        "plain": {"value": plain, "unit": METRIC,
                  "how": "the same 64 wraps one at a time (a batch of one each), device-resident"},
        "batched_vs_plain": value / plain if plain else None,
        "same_config_as_reference": False,
        "same_config_reason": SAME_CONFIG_REASON,
        "same_sample_as_reference": same_sample,
        "bit_identical_alone_and_batched": f"{identical}/{len(cases)}",
        "latency_ms": {"plain_wrap": percentiles(plain_ms), "batch_step": percentiles(step_ms)},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "e2e": e2e,
        "roofline": roof,
        "kernels": detail,
        "served": served,
        "fit": fit,
        "reference_gpu": reference_gpu,
        "cpu_baseline": cpu,
        "single_wrap": single,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# config 5: precision stress
# ---------------------------------------------------------------------------

def _level_energies(report: str) -> list:
    return [lv["energy_end"] for lv in json.loads(report)["levels"]]


def _precision_solve(seed: int) -> dict:
    """Config 5 through solve_route_b at the reference's caps (k=4, 4-NN, so
    that its FP64 route A can run the same problem), and at the config's own
    k=8 for the time."""
    from nricp_b200 import nricp_dp as dp
    from nricp_b200 import synthetic as S

    case = S.config5(seed)
    out = {}
    for name, opts in (("capped", reference_options(case.options)), ("k8", case.options)):
        dp.solve_route_b(*case.args(), **opts)  # warm: library, pools
        t0 = time.perf_counter()
        r = dp.solve_route_b(*case.args(), **opts)
        out[f"{name}_seconds"] = time.perf_counter() - t0
        out[f"{name}_vertices"] = r["vertices"]
        out[f"{name}_report"] = r["report"]
    return out


def run_precision(args) -> None:
    from nricp_b200 import build as native

    shipped = _precision_solve(args.seed)
    variant_out = Path(args.precision).with_suffix(".variant.npz")
    env = dict(os.environ, NRICP_B200_LIBRARY=str(native.FP32_REDUCTIONS_LIB))
    subprocess.run([sys.executable, str(Path(__file__).resolve()), "--precision-variant",
                    str(variant_out), "--seed", str(args.seed)], check=True, env=env)
    variant = dict(np.load(variant_out, allow_pickle=False))
    np.savez(args.precision, seed=args.seed,
             **{f"fp64_reductions_{k}": v for k, v in shipped.items()},
             **{f"fp32_reductions_{k}": v for k, v in variant.items()})
    p = np.asarray(shipped["capped_vertices"])
    q = np.asarray(variant["capped_vertices"])
    print(json.dumps({
        "workload": "config 5: 100k-vertex template, 2M-triangle target, 10,000 nodes, route B",
        "fp64_reductions": {"seconds_capped": shipped["capped_seconds"], "seconds_k8": shipped["k8_seconds"],
                            "level_energies": _level_energies(str(shipped["capped_report"]))},
        "fp32_reductions": {"seconds_capped": float(variant["capped_seconds"]),
                            "seconds_k8": float(variant["k8_seconds"]),
                            "level_energies": _level_energies(str(variant["capped_report"]))},
        "max_difference_between_them": float(np.abs(p - q).max()),
        "written": str(args.precision)}), flush=True)


def run_precision_variant(args) -> None:
    out = _precision_solve(args.seed)
    np.savez(args.precision_variant, **out)


def _route_a_config5(job):
    """The reference's FP64 route A on config 5 at its caps, in a worker; with
    `sigma` > 0 the template is first perturbed by N(0, sigma) per coordinate
    (relative to the target's diagonal), drawn from generator `draw` -- the
    problem's own sensitivity.  With a cache directory, a finished run is
    stored there and read back instead of being solved again."""
    seed, sigma, draw, cache = job
    sys.path.insert(0, str(ROOT))
    path = Path(cache) / f"route_a_c5_seed{seed}_sigma{sigma:g}_draw{draw}.npz" if cache else None
    if path is not None and path.exists():
        done = np.load(path, allow_pickle=False)
        return float(done["seconds"]), done["vertices"], str(done["report"])
    from nricp_b200 import synthetic as S
    from oracle.oracle import Oracle

    case = S.config5(seed)
    points = case.template_points
    if sigma > 0.0:
        p = case.target_points
        diag = float(np.linalg.norm(p.max(0) - p.min(0)))
        points = points + np.random.default_rng(draw).normal(0.0, sigma * diag, size=points.shape)
    t0 = time.perf_counter()
    ref = Oracle("reference").solve(points, case.template_faces, case.target_points, case.target_faces,
                                    case.level_settings, **reference_options(case.options))
    seconds = time.perf_counter() - t0
    if path is not None:
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez(path, seconds=seconds, vertices=ref["vertices"], report=ref["report"])
    return seconds, ref["vertices"], ref["report"]


def _against(vertices, report, ref_vertices, ref_report, diag) -> dict:
    err = np.linalg.norm(np.asarray(vertices) - ref_vertices, axis=1) / diag
    e, ref_e = json.loads(report)["energy"]["total"], json.loads(ref_report)["energy"]["total"]
    levels, ref_levels = _level_energies(report), _level_energies(ref_report)
    return {"max_vertex_error_over_diag": float(err.max()),
            "rms_vertex_error_over_diag": float(np.sqrt(np.mean(err ** 2))),
            "final_energy_rel_error": abs(e - ref_e) / abs(ref_e) if ref_e else abs(e),
            "level_energy_rel_error": [abs(a - b) / abs(b) if b else abs(a)
                                       for a, b in zip(levels, ref_levels)],
            "level_energies": levels}


def run_precision_compare(args) -> None:
    """The reference's FP64 route A (oracle/_ref) on config 5 at its caps, on
    this host's CPU; route A again on templates perturbed by each of
    --perturb-sigmas of the diagonal, each with --perturb-seeds independent
    draws (the spread a perturbation of that size produces on its own); and,
    unless IN.npz is '-', the GPU results of --precision placed in that
    spread."""
    import multiprocessing as mp

    from nricp_b200 import synthetic as S

    seed = args.seed
    gpu = None
    if args.precision_compare != "-":
        gpu = np.load(args.precision_compare, allow_pickle=False)
        seed = int(gpu["seed"])
    sigmas = [float(x) for x in args.perturb_sigmas.split(",") if x]
    jobs = [(seed, 0.0, 0, args.precision_cache)]
    jobs += [(seed, sigma, 1000 + k, args.precision_cache) for sigma in sigmas for k in range(args.perturb_seeds)]
    workers = max(1, min(args.precision_workers or host_cores(), len(jobs)))
    with mp.get_context("spawn").Pool(workers) as pool:
        runs = pool.map(_route_a_config5, jobs, chunksize=1)
    case = S.config5(seed)
    p = case.target_points
    diag = float(np.linalg.norm(p.max(0) - p.min(0)))
    seconds, ref_v, ref_report = runs[0]
    line = {"workload": "config 5 at the reference's caps (k=4, 4-NN): GPU route B against the "
                        "reference's FP64 route A, and route A's own spread under perturbations "
                        "of the template",
            "route_a": {"seconds": seconds, "level_energies": _level_energies(ref_report),
                        "final_energy": json.loads(ref_report)["energy"]["total"]},
            "perturbed": {}}
    for sigma in sigmas:
        members = [_against(v, r, ref_v, ref_report, diag)
                   for (_, sg, _, _), (_, v, r) in zip(jobs, runs) if sg == sigma]
        spread = {k: [m[k] for m in members] for k in ("max_vertex_error_over_diag",
                                                       "rms_vertex_error_over_diag",
                                                       "final_energy_rel_error")}
        spread["level_energy_rel_error"] = [list(x) for x in zip(*[m["level_energy_rel_error"]
                                                                    for m in members])]
        line["perturbed"][f"{sigma:g}"] = {"draws": len(members), **spread}
    if gpu is not None:
        for name in ("fp64_reductions", "fp32_reductions"):
            line[name] = _against(gpu[f"{name}_capped_vertices"], str(gpu[f"{name}_capped_report"]),
                                  ref_v, ref_report, diag)
    print(json.dumps(line), flush=True)


def run_capture(args) -> None:
    """A few hundred eager launches (one config-2 wrap, a few ticks) for
    ncu: the tick graphs of the timed runs make every launch slow under a
    profiler."""
    import torch

    from nricp_b200 import nricp_dp as dp
    from nricp_b200 import synthetic as S

    case = S.config2(args.seed)
    session = dp.RouteBSession(*case.args(), **case.options)
    for _ in range(args.capture_steps):
        if session.finished():
            break
        session.step()
    torch.cuda.synchronize()
    print(json.dumps({"capture_steps": args.capture_steps, "ticks": session.ticks()[0]}), flush=True)


def run_capture_batch(args) -> None:
    """One batch step of config 3's first N wraps with eager launches, for
    an ncu launch list of the batch's kernels: the re-run that times the
    kernel groups (reset, hierarchy builds, every tick with its solve and
    refresh branches one after the other) and nothing else."""
    import torch

    from nricp_b200 import nricp_dp as dp
    from nricp_b200 import synthetic as S

    cases = [S.config3_case(spec) for spec in S.config3_specs(args.seed)[: args.capture_batch]]
    batch = dp.WrapBatch([(*c.args(), c.options) for c in cases])
    batch.tune(-1)
    records = batch.profile()
    torch.cuda.synchronize()
    print(json.dumps({"capture_batch": args.capture_batch, "ticks": len(records)}), flush=True)


# Host allocator settings of a long-running caller: glibc keeps freed memory
# instead of returning it to the system after every batch, so the next batch
# does not fault it in again (without them an end-to-end call of the 64-wrap
# batch took 1.15-1.95 s, with them 1.13-1.17 s; the device part is the same).
ALLOCATOR = {"MALLOC_MMAP_THRESHOLD_": str(1 << 30), "MALLOC_TRIM_THRESHOLD_": str(16 << 30)}


def main():
    args = parse_args()
    if args.impl == "ours" and any(k not in os.environ for k in ALLOCATOR):
        os.environ.update({k: v for k, v in ALLOCATOR.items() if k not in os.environ})
        os.execv(sys.executable, [sys.executable, *sys.argv])  # the same process, the settings in force
    if args.capture_steps:
        return run_capture(args)
    if args.capture_batch:
        return run_capture_batch(args)
    if args.precision_variant:
        return run_precision_variant(args)
    if args.precision_compare:
        return run_precision_compare(args)
    if args.precision:
        return run_precision(args)
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
