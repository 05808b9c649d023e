"""Drop-in for the reference's `nricp_dp` extension module (route B / route C).

Same function names, positional and keyword arguments, defaults, result
dictionaries and error types as src/python/bindings.cpp:714-1623 for the
device routes:

* ``solve_route_b`` / ``solve_route_c`` (bindings.cpp:1422-1492)
* ``RouteBSession`` with ``step``, ``finished``, ``vertices``, ``report``,
  ``result`` (bindings.cpp:1510-1612)
* ``device_info``, ``build_info``, ``build_template_graph``, ``closest_points``,
  ``find_correspondences``, ``fit_rigid``, ``normalization``, ``bounding_box_diagonal``, ``validate_*``,
  ``clean_mesh``, ``farthest_point_seeds``, ``bind_vertices``,
  ``vertex_normals``, ``evaluate_deformation``, ``transfer_level``,
  ``retract_deformation``, ``tangent_difference``, ``robust_weights``,
  ``serialize_report``

plus, beyond the reference, ``solve_batch`` (many uneven wraps advanced by the
same kernel launches) and the keyword extensions ``max_nodes_per_vertex``
(k <= 8 bindings) and ``edge_neighbours`` (k-NN graph edges).

The solves, the graph build, the closest-point query and the rigid fit run
in the CUDA library through its C ABI; the small host helpers (deformation
algebra, cleaning, report text) are numpy restatements, bit-exact with the
reference's own functions.  The FP64 route A lives only in the test oracle.
"""

from __future__ import annotations

import ctypes as C
import json
import math
import os

import numpy as np

from . import _abi
from ._lib import check, load

__version__ = "0.1.0"

_ROUTES = {"route_b": _abi.ROUTE_B, "route_c": _abi.ROUTE_C}


def _plan(desc: _abi.Desc) -> list[int]:
    counts = (C.c_int32 * 64)()
    levels = C.c_int()
    check(load().nricp_plan(C.byref(desc.struct), counts, 64, C.byref(levels)))
    return [counts[i] for i in range(levels.value)]


def _solve(route: str, template_points, template_faces, target_points, target_faces,
           level_settings, **kwargs) -> dict:
    desc = _abi.Desc(template_points, template_faces, target_points, target_faces,
                     level_settings, route=_ROUTES[route], **kwargs)
    out = _abi.ResultBuffers(desc.template_points.shape[0], _plan(desc))
    check(load().nricp_solve(C.byref(desc.struct), C.byref(out.struct)))
    return out.to_dict()


def solve_route_b(template_points, template_faces, target_points, target_faces,
                  level_settings, **kwargs) -> dict:
    """Fit the template onto the target and return the result plus the run
    report.  Distances (distance_threshold, robust_threshold) are given in the
    caller's units and converted into the solver's normalized frame
    internally; the caller hands in the template and target already aligned to
    each other."""
    return _solve("route_b", template_points, template_faces, target_points, target_faces,
                  level_settings, **kwargs)


def solve_route_c(template_points, template_faces, target_points, target_faces,
                  level_settings, **kwargs) -> dict:
    """Route C: the same schedule solved by the global/local alternation."""
    return _solve("route_c", template_points, template_faces, target_points, target_faces,
                  level_settings, **kwargs)


def _descs(cases, route: str) -> list:
    """The cases' descriptors; the array conversions (numpy copies, which
    release the GIL) run on a few threads when there are many cases."""
    def one(case):
        return _abi.Desc(*case[:5], route=_ROUTES[route], **(case[5] if len(case) > 5 else {}))

    cases = list(cases)
    if len(cases) < 8:
        return [one(c) for c in cases]
    import concurrent.futures as cf

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        return list(pool.map(one, cases))


def solve_batch(cases, route: str = "route_b") -> list[dict]:
    """Many wraps at once: every case is ``(template_points, template_faces,
    target_points, target_faces, level_settings, kwargs)``.  The wraps may
    differ in every size; they share the device launches."""
    descs = _descs(cases, route)
    outs = [_abi.ResultBuffers(d.template_points.shape[0], _plan(d)) for d in descs]
    array = (_abi.SolveDesc * len(descs))(*[d.struct for d in descs])
    results = (_abi.Result * len(outs))(*[o.struct for o in outs])
    check(load().nricp_batch_solve(array, len(descs), results))
    return [o.to_dict() for o in outs]


class WrapBatch:
    """Many wraps resident on the device, advanced together by the same
    launches (no reference counterpart: the reference solves one wrap per
    call).  `cases` as for solve_batch."""

    def __init__(self, cases, route: str = "route_b"):
        self._descs = _descs(cases, route)
        self._plans = [_plan(d) for d in self._descs]
        array = (_abi.SolveDesc * len(self._descs))(*[d.struct for d in self._descs])
        self._handle = C.c_void_p()
        check(load().nricp_batch_create(array, len(self._descs), C.byref(self._handle)))

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            load().nricp_batch_destroy(handle)
            self._handle = None

    def __len__(self):
        return len(self._descs)

    def run(self) -> None:
        check(load().nricp_batch_run(self._handle))

    def step(self) -> float:
        """Reset every wrap and run all of them to completion; returns the
        device time in milliseconds (CUDA events on the batch's stream)."""
        ms = C.c_double()
        check(load().nricp_batch_step(self._handle, C.byref(ms)))
        return ms.value

    def tune(self, pcg_cluster: int = 0) -> int:
        """Cluster size of the linear solve: a power of two up to 16 for every
        wrap, 0 for each wrap's own size in per-class launches, -s for those
        sizes halved s times (a new batch starts at the smallest s whose
        classes need at most three CTAs per SM).  Returns the largest size in
        effect; results are bit-identical for every choice."""
        out = C.c_int()
        check(load().nricp_batch_tune(self._handle, int(pcg_cluster), C.byref(out)))
        return out.value

    # Candidate cluster settings of the linear solve that autotune() times:
    # per-wrap classes halved once, unhalved, halved twice, and uniform sizes.
    TUNE_CANDIDATES = (-1, 0, -2, 8, 16, 4)

    def autotune(self, candidates=TUNE_CANDIDATES) -> dict:
        """Picks the linear solve's cluster setting by measurement: one batch
        step (device time) per candidate, the two fastest timed once more, the
        fastest kept.  Every setting gives bit-identical results, so the
        choice trades nothing but speed.  Returns the choice, the largest
        cluster in effect and each candidate's best time in milliseconds."""
        times = {}
        for c in candidates:
            self.tune(c)
            times[c] = self.step()
        for c in sorted(times, key=times.get)[:2]:  # one step is noisy
            self.tune(c)
            times[c] = min(times[c], self.step())
        choice = min(times, key=times.get)
        return {"choice": choice, "largest_cluster": self.tune(choice),
                "ms": {str(c): round(t, 2) for c, t in times.items()}}

    def result(self, index: int) -> dict:
        out = _abi.ResultBuffers(self._descs[index].template_points.shape[0], self._plans[index])
        check(load().nricp_batch_result(self._handle, index, C.byref(out.struct)))
        return out.to_dict()

    def counters(self) -> tuple[int, int]:
        t, l = C.c_long(), C.c_long()
        check(load().nricp_batch_counters(self._handle, C.byref(t), C.byref(l)))
        return t.value, l.value

    def profile(self) -> list[dict]:
        """Re-runs the batch with CUDA events around the closest-point query,
        the linear solve and the assembly of every tick; per-tick records of
        the first wrap."""
        q, p, a = C.c_double(), C.c_double(), C.c_double()
        ticks = C.c_long()
        check(load().nricp_batch_profile(self._handle, C.byref(q), C.byref(p), C.byref(a),
                                         C.byref(ticks)))
        records = (_abi.TickRecord * max(1, ticks.value))()
        count = C.c_int()
        check(load().nricp_batch_tick_records(self._handle, records, ticks.value, C.byref(count)))
        return [{"phase": r.phase, "level": r.level, "pcg_iterations": r.pcg_iterations,
                 "query_ms": r.query_ms, "pcg_ms": r.pcg_ms, "assemble_ms": r.assemble_ms,
                 "tick_ms": r.tick_ms} for r in records[:count.value]]

    def level_sizes(self, index: int, level: int) -> dict:
        sizes = (C.c_int32 * 15)()
        check(load().nricp_batch_level_sizes(self._handle, index, level, sizes))
        keys = ("nodes", "edges", "pairs", "entries", "pair_entries", "vertices",
                "target_triangles", "target_vertices", "template_triangles", "levels",
                "solves", "pcg_iterations", "queries", "assemblies", "offdiag_blocks")
        return dict(zip(keys, list(sizes)))


class WrapServer:
    """Continuous batching on one device (no reference counterpart: the
    reference solves one wrap per call).  ``submit`` copies and validates a
    request and returns at once; the request's graph is built on a host
    thread (cached per template), it is admitted into a free resident slot
    as soon as the device-memory budget allows, advanced together with
    every other running wrap, and its result is kept until ``result`` takes
    it.  Each result is bit-identical to the same wrap solved alone."""

    def __init__(self, memory_budget_bytes: int = 0, max_slots: int = 64,
                 prep_threads: int = 0, pcg_cluster: int = 0, ticks_per_poll: int = 8,
                 large_face_threshold: int = 1_000_000, large_slots: int = 8):
        cfg = _abi.ServerConfig()
        load().nricp_server_default_config(C.byref(cfg))
        cfg.memory_budget_bytes = int(memory_budget_bytes)
        cfg.max_slots = int(max_slots)
        cfg.prep_threads = int(prep_threads)
        cfg.pcg_cluster = int(pcg_cluster)
        cfg.ticks_per_poll = int(ticks_per_poll)
        cfg.large_face_threshold = int(large_face_threshold)
        cfg.large_slots = int(large_slots)
        self._handle = C.c_void_p()
        check(load().nricp_server_create(C.byref(cfg), C.byref(self._handle)))
        self._plans: dict[int, tuple[int, list[int]]] = {}

    def close(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle:
            load().nricp_server_destroy(handle)
            self._handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, template_points, template_faces, target_points, target_faces,
               level_settings, route: str = "route_b", **kwargs) -> int:
        if route not in _ROUTES:
            raise ValueError(f"the device session runs 'route_b' or 'route_c', not '{route}'")
        desc = _abi.Desc(template_points, template_faces, target_points, target_faces,
                         level_settings, route=_ROUTES[route], **kwargs)
        rid = C.c_long()
        check(load().nricp_server_submit(self._handle, C.byref(desc.struct), C.byref(rid)))
        self._plans[rid.value] = (desc.template_points.shape[0], _plan(desc))
        return rid.value

    def poll(self, request: int) -> tuple[str, float]:
        """('waiting' | 'running' | 'done' | 'failed', latency in seconds once done)."""
        status, latency = C.c_int(), C.c_double()
        check(load().nricp_server_poll(self._handle, request, C.byref(status), C.byref(latency)))
        return _abi.REQUEST_STATES[status.value], latency.value

    PHASES = ("prepare", "load", "wait_for_slot", "device", "compose")

    def phases(self, request: int) -> dict:
        """Where the request's latency went so far, in seconds: host preparation
        (graph, level layouts), loading (memory budget, uploads, target
        hierarchy), waiting for a slot, on the device, composing the result.
        Read it before ``result`` takes the request."""
        out = (C.c_double * 5)()
        check(load().nricp_server_phases(self._handle, request, out))
        return dict(zip(self.PHASES, list(out)))

    def wait(self, request: int, timeout: float | None = None) -> tuple[str, float]:
        """Blocks until the request is done or failed; returns poll()."""
        check(load().nricp_server_wait(self._handle, request, float(timeout or 0.0)))
        return self.poll(request)

    def result(self, request: int, timeout: float | None = None) -> dict:
        """Waits for the request and returns its result dict (as solve_route_b)."""
        check(load().nricp_server_wait(self._handle, request, float(timeout or 0.0)))
        vertices, levels = self._plans[request]
        out = _abi.ResultBuffers(vertices, levels)
        check(load().nricp_server_result(self._handle, request, C.byref(out.struct)))
        del self._plans[request]
        return out.to_dict()

    def stats(self) -> dict:
        s = _abi.ServerStats()
        check(load().nricp_server_stats(self._handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}


def transfer_counters(reset: bool = False) -> tuple[int, int]:
    """Bytes copied host->device and device->host by this thread's calls."""
    h2d, d2h = C.c_ulonglong(), C.c_ulonglong()
    check(load().nricp_transfer_counters(C.byref(h2d), C.byref(d2h), int(reset)))
    return h2d.value, d2h.value


class RouteBSession:
    """The device schedule with the caller holding the loop: construct the
    session, then call step() until finished().  `route` selects 'route_b'
    (the default) or 'route_c'."""

    def __init__(self, template_points, template_faces, target_points, target_faces,
                 level_settings, route: str = "route_b", **kwargs):
        if route not in _ROUTES:
            raise ValueError(f"the device session runs 'route_b' or 'route_c', not '{route}'")
        self._desc = _abi.Desc(template_points, template_faces, target_points, target_faces,
                               level_settings, route=_ROUTES[route], **kwargs)
        self._levels = _plan(self._desc)
        self._handle = C.c_void_p()
        check(load().nricp_session_create(C.byref(self._desc.struct), C.byref(self._handle)))

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle:
            load().nricp_session_destroy(handle)
            self._handle = None

    def step(self) -> dict:
        """Advance the schedule by one unit of work and report where it got to."""
        p = _abi.Progress()
        check(load().nricp_session_step(self._handle, C.byref(p)))
        return {"level": p.level, "outer": p.outer, "inner": p.inner,
                "finished": bool(p.finished), "level_converged": bool(p.level_converged),
                "energy": p.energy, "correspondence_mean": p.correspondence_mean}

    def finished(self) -> bool:
        done = C.c_int()
        check(load().nricp_session_finished(self._handle, C.byref(done)))
        return bool(done.value)

    def run(self) -> None:
        """Steps until finished without a host round trip between steps."""
        check(load().nricp_session_run(self._handle))

    def vertices(self) -> np.ndarray:
        """The template as it currently stands, for redrawing between steps."""
        out = np.zeros_like(self._desc.template_points)
        check(load().nricp_session_vertices(self._handle, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def result(self) -> dict:
        out = _abi.ResultBuffers(self._desc.template_points.shape[0], self._levels)
        check(load().nricp_session_result(self._handle, C.byref(out.struct)))
        return out.to_dict()

    def report(self) -> str:
        return self.result()["report"]

    def ticks(self) -> tuple[int, int]:
        t, l = C.c_long(), C.c_long()
        check(load().nricp_session_ticks(self._handle, C.byref(t), C.byref(l)))
        return t.value, l.value

    def target(self) -> dict:
        """The target as the device holds it (no reference counterpart; for
        checking its ingestion): points in the normalised frame and their
        area-weighted vertex normals."""
        vt = self._desc.target_points.shape[0]
        out = {"points": np.zeros((vt, 3)), "normals": np.zeros((vt, 3))}
        s = _abi.Inspect()
        s.off_capacity = 1 << 30  # nothing else is read
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        s.target_points, s.target_normals = P(out["points"], C.c_double), P(out["normals"], C.c_double)
        check(load().nricp_session_inspect(self._handle, C.byref(s)))
        return out

    def inspect(self) -> dict:
        """The current linear system and the state it was assembled at (no
        reference counterpart; for checking the assembly): phase, level,
        accepted rotations / translations, correspondences in the solver's
        normalised frame, the FP32 diagonal blocks, right-hand side and
        off-diagonal (a, b) blocks, the accepted energy parts, the
        correspondences' distances and the last linear solve's outcome
        (converged, iterations, relative residual)."""
        n_max = max(self._levels)
        v = self._desc.template_points.shape[0]
        cap = max(1, n_max * 64)
        out = {"rotations": np.zeros((n_max, 3, 3)), "translations": np.zeros((n_max, 3)),
               "corr_points": np.zeros((v, 3)), "corr_normals": np.zeros((v, 3)),
               "corr_robust": np.zeros(v), "corr_codes": np.zeros(v, np.uint8),
               "diag": np.zeros((n_max, 6, 6), np.float32), "rhs": np.zeros((n_max, 6), np.float32),
               "off_nodes": np.zeros((cap, 2), np.int32), "off_blocks": np.zeros((cap, 6, 6), np.float32),
               "delta": np.zeros((n_max, 6)), "corr_distances": np.zeros(v)}
        s = _abi.Inspect()
        s.off_capacity = cap
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        s.rotations, s.translations = P(out["rotations"], C.c_double), P(out["translations"], C.c_double)
        s.corr_points, s.corr_normals = P(out["corr_points"], C.c_double), P(out["corr_normals"], C.c_double)
        s.corr_robust, s.corr_codes = P(out["corr_robust"], C.c_double), P(out["corr_codes"], C.c_uint8)
        s.diag, s.rhs = P(out["diag"], C.c_float), P(out["rhs"], C.c_float)
        s.off_nodes, s.off_blocks = P(out["off_nodes"], C.c_int32), P(out["off_blocks"], C.c_float)
        s.delta = P(out["delta"], C.c_double)
        s.corr_distances = P(out["corr_distances"], C.c_double)
        check(load().nricp_session_inspect(self._handle, C.byref(s)))
        n, k = s.node_count, s.off_count
        for key in ("rotations", "translations", "diag", "rhs", "delta"):
            out[key] = out[key][:n]
        out["off_nodes"], out["off_blocks"] = out["off_nodes"][:k], out["off_blocks"][:k]
        out.update(level=s.level, node_count=n, phase=s.phase, energies=list(s.energies),
                   damping=s.damping, pcg_ok=bool(s.pcg_ok), pcg_iterations=s.pcg_iterations,
                   pcg_residual=s.pcg_residual)
        return out


def device_info() -> dict:
    """Report whether the accelerated path can run here, and on what."""
    available = C.c_int()
    text = C.create_string_buffer(256)
    check(load().nricp_device_info(C.byref(available), text, 256))
    return {"available": bool(available.value), "device": text.value.decode()}


def build_info() -> dict:
    """The reference's keys (bindings.cpp:723-737); pybind11_version names the
    binding layer, here ctypes over the C ABI."""
    import platform

    return {"version": __version__, "build_type": "Release", "cxx_compiler": "GNU (via nvcc)",
            "cuda_toolkit": "12.9", "cuda_architectures": "100a",
            "accelerated_precision": "float", "python_version": platform.python_version(),
            "pybind11_version": "none (ctypes over the C ABI)"}


def _points(a, name):
    out = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if out.ndim != 2 or out.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    return out


def _faces(a, name):
    out = np.asarray(a)
    if out.ndim != 2 or out.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    return np.ascontiguousarray(out.astype(np.int64).astype(np.int32))


def bounding_box_diagonal(points) -> float:
    """|max - min| of the bounding box, summed as the reference sums it
    (mesh.cpp:48-69, vec3.h:62-72)."""
    p = _points(points, "points")
    if not len(p):
        return 0.0
    d = p.max(0) - p.min(0)
    return math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])


def normalization(points) -> dict:
    """Centering and scaling that puts the bounding-box diagonal at 1
    (src/core/mesh.cpp:174-181)."""
    p = _points(points, "points")
    if len(p) == 0:
        return {"center": np.zeros((1, 3)), "scale": 1.0}
    lo, hi = p.min(0), p.max(0)
    center = (lo + hi) * 0.5
    d = hi - lo
    diagonal = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    return {"center": center[None, :], "scale": 1.0 / diagonal if diagonal > 0 else 1.0}


def validate_mesh(points, faces) -> dict:
    """Structural validation (src/core/mesh.cpp:90-116)."""
    p, f = _points(points, "points"), np.asarray(faces)
    problems = []
    if len(p) == 0:
        problems.append("mesh has no vertices")
    if len(f) == 0:
        problems.append("mesh has no faces; closest-point queries need a surface")
    for i in np.nonzero(~np.isfinite(p).all(1))[0]:
        problems.append(f"vertex {i} is not finite")
    if len(f):
        bad = (f < 0) | (f >= len(p))
        for i, k in zip(*np.nonzero(bad)):
            problems.append(f"face {i} corner {k} index {f[i, k]} is out of range")
    return {"ok": not problems, "problems": problems}


def clean_mesh(points, faces) -> dict:
    """Drops degenerate faces -- a repeated corner, or a squared cross product
    of at most 1e-12 of the squared bounding-box diagonal -- then faces whose
    three corners repeat an earlier face's in any order (the first is kept,
    winding and all), then the vertices no face uses, renumbering the rest in
    order (bindings.cpp:762-778, mesh.cpp:118-173)."""
    p = _points(points, "points")
    f = np.asarray(faces)
    if f.ndim != 2 or f.shape[1] != 3:
        raise ValueError("faces must have shape (n, 3)")
    f = np.ascontiguousarray(f.astype(np.int64))
    check = validate_mesh(p, f)
    if not check["ok"]:
        raise ValueError("invalid mesh: " + "; ".join(check["problems"]))
    diagonal = bounding_box_diagonal(p)
    floor = 1e-12 * max(diagonal * diagonal, 1e-300)
    a, b, c = f[:, 0], f[:, 1], f[:, 2]
    u, v = p[b] - p[a], p[c] - p[a]
    x = u[:, 1] * v[:, 2] - u[:, 2] * v[:, 1]
    y = u[:, 2] * v[:, 0] - u[:, 0] * v[:, 2]
    z = u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]
    degenerate = (a == b) | (b == c) | (a == c) | (x * x + y * y + z * z <= floor)
    candidates = np.nonzero(~degenerate)[0]
    first = np.unique(np.sort(f[candidates], axis=1), axis=0, return_index=True)[1] if len(candidates) else []
    kept = candidates[np.sort(np.asarray(first, dtype=np.int64))]
    used = np.zeros(len(p), dtype=bool)
    used[f[kept].reshape(-1)] = True
    renumber = np.cumsum(used) - 1
    return {"points": p[used], "faces": renumber[f[kept]].astype(np.int64).reshape(-1, 3),
            "duplicate_faces": int(len(candidates) - len(kept)), "degenerate_faces": int(degenerate.sum()),
            "isolated_vertices": int(len(p) - used.sum())}


# ---- deformation helpers on the host (the reference's component functions) ----

def _matrices(array, name: str) -> np.ndarray:
    m = np.asarray(array, dtype=np.float64)
    if m.ndim != 3 or m.shape[1:] != (3, 3):
        raise ValueError(f"{name} must have shape (n, 3, 3)")
    return m


def _deformation(rotations, translations, node_positions=None):
    r = _matrices(rotations, "rotations")
    t = np.asarray(translations, dtype=np.float64)
    if t.ndim != 2 or t.shape[1:] != (3,) or t.shape[0] != r.shape[0]:
        raise ValueError("translations must have shape (n, 3)")
    if node_positions is not None:
        g = np.asarray(node_positions, dtype=np.float64)
        if g.ndim != 2 or g.shape[1:] != (3,) or g.shape[0] != r.shape[0]:
            raise ValueError("node_positions must have shape (n, 3)")
        return r, t, g
    return r, t, None


def _libm(fn, *args) -> np.ndarray:
    """fn applied elementwise through the C library's own function (Python's
    math module), which the reference's std:: calls resolve to; numpy's
    vectorised transcendentals can round the last bit differently."""
    return np.frompyfunc(fn, len(args), 1)(*args).astype(np.float64)


def _mat_vec(m: np.ndarray, v: np.ndarray) -> np.ndarray:
    """m v per row, each dot summed left to right (mat3.h:17-22)."""
    return np.stack([m[:, i, 0] * v[:, 0] + m[:, i, 1] * v[:, 1] + m[:, i, 2] * v[:, 2] for i in range(3)], 1)


def _mat_mat(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a b per pair of matrices, each entry summed left to right (mat3.h:24-36)."""
    out = np.empty((max(len(a), len(b)), 3, 3))
    for i in range(3):
        for j in range(3):
            out[:, i, j] = a[:, i, 0] * b[:, 0, j] + a[:, i, 1] * b[:, 1, j] + a[:, i, 2] * b[:, 2, j]
    return out


def _exp_so3(omega: np.ndarray) -> np.ndarray:
    """Rodrigues: R = I + (a [w] + b [w]^2), a = sin(th)/th,
    b = (1 - cos(th))/th^2, and the second-order series below th^2 = 1e-24
    (rotation.h:28-46)."""
    w = np.asarray(omega, dtype=np.float64).reshape(-1, 3)
    hat = np.zeros((len(w), 3, 3))
    hat[:, 0, 1], hat[:, 0, 2], hat[:, 1, 2] = -w[:, 2], w[:, 1], -w[:, 0]
    hat[:, 1, 0], hat[:, 2, 0], hat[:, 2, 1] = w[:, 2], -w[:, 1], w[:, 0]
    hat2 = _mat_mat(hat, hat)
    th2 = w[:, 0] * w[:, 0] + w[:, 1] * w[:, 1] + w[:, 2] * w[:, 2]
    small = th2 < 1e-24
    th = np.sqrt(np.where(small, 1.0, th2))
    a = np.where(small, 1.0, _libm(math.sin, th) / th)
    b = np.where(small, 0.5, (1.0 - _libm(math.cos, th)) / np.where(small, 1.0, th2))
    return np.eye(3) + (a[:, None, None] * hat + b[:, None, None] * hat2)


def _quaternions(m: np.ndarray) -> np.ndarray:
    """(w, x, y, z) of each rotation matrix by Shepperd's branches, unnormalised
    (quaternion.h:48-75)."""
    q = np.empty((len(m), 4))
    d0, d1, d2 = m[:, 0, 0], m[:, 1, 1], m[:, 2, 2]
    trace = d0 + d1 + d2
    b0 = trace > 0.0
    b1 = ~b0 & (d0 > d1) & (d0 > d2)
    b2 = ~b0 & ~b1 & (d1 > d2)
    b3 = ~(b0 | b1 | b2)
    r = lambda sel, i, j: m[sel, i, j]  # noqa: E731
    s = np.sqrt(trace[b0] + 1.0) * 2.0
    q[b0] = np.stack([0.25 * s, (r(b0, 2, 1) - r(b0, 1, 2)) / s, (r(b0, 0, 2) - r(b0, 2, 0)) / s,
                      (r(b0, 1, 0) - r(b0, 0, 1)) / s], 1)
    s = np.sqrt(1.0 + d0[b1] - d1[b1] - d2[b1]) * 2.0
    q[b1] = np.stack([(r(b1, 2, 1) - r(b1, 1, 2)) / s, 0.25 * s, (r(b1, 0, 1) + r(b1, 1, 0)) / s,
                      (r(b1, 0, 2) + r(b1, 2, 0)) / s], 1)
    s = np.sqrt(1.0 + d1[b2] - d0[b2] - d2[b2]) * 2.0
    q[b2] = np.stack([(r(b2, 0, 2) - r(b2, 2, 0)) / s, (r(b2, 0, 1) + r(b2, 1, 0)) / s, 0.25 * s,
                      (r(b2, 1, 2) + r(b2, 2, 1)) / s], 1)
    s = np.sqrt(1.0 + d2[b3] - d0[b3] - d1[b3]) * 2.0
    q[b3] = np.stack([(r(b3, 1, 0) - r(b3, 0, 1)) / s, (r(b3, 0, 2) + r(b3, 2, 0)) / s,
                      (r(b3, 1, 2) + r(b3, 2, 1)) / s, 0.25 * s], 1)
    return q


def _qdot(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2] + a[:, 3] * b[:, 3]


def _unit(q: np.ndarray) -> np.ndarray:
    """q / |q|, the identity for a zero quaternion (quaternion.h:38-44)."""
    length = np.sqrt(_qdot(q, q))
    zero = length <= 0.0
    out = q / np.where(zero, 1.0, length)[:, None]
    out[zero] = (1.0, 0.0, 0.0, 0.0)
    return out


def _matrices_of(q: np.ndarray) -> np.ndarray:
    """Rotation matrix of each unit quaternion (quaternion.h:77-93)."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack([1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
                     2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
                     2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)],
                    1).reshape(-1, 3, 3)


def _log_so3(rotations: np.ndarray) -> np.ndarray:
    """The rotation vector of each matrix, through its unit quaternion (w >= 0)
    so that it stays accurate up to a half turn (rotation.h:48-62)."""
    q = _unit(_quaternions(rotations))
    q[q[:, 0] < 0.0] *= -1.0
    v = q[:, 1:]
    length = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
    tiny = length < 1e-12
    safe = np.where(tiny, 1.0, length)
    out = v * ((2.0 * _libm(math.atan2, length, q[:, 0])) / safe)[:, None]
    out[tiny] = 0.0
    return out


def _applied(r: np.ndarray, t: np.ndarray, g: np.ndarray, p: np.ndarray) -> np.ndarray:
    """R (p - g) + g + t for node transforms and points paired row by row
    (deformation.h:39-43)."""
    return _mat_vec(r, p - g) + g + t


def robust_weights(kernel: str, squared_residuals, threshold: float) -> np.ndarray:
    """IRLS weights of a robust kernel, 'none', 'huber' or 'geman_mcclure'
    (bindings.cpp:1077-1092, src/energy/robust.cpp:7-58); negative squared
    residuals count as zero."""
    r = np.maximum(np.asarray(squared_residuals, dtype=np.float64).reshape(-1), 0.0)
    t = float(threshold)
    if kernel in ("huber", "Huber"):
        if t <= 0.0:
            return np.ones_like(r)
        return np.where(r <= t * t, 1.0, t / np.sqrt(np.where(r > 0.0, r, 1.0)))
    if kernel in ("geman_mcclure", "geman-mcclure", "GemanMcClure"):
        if t <= 0.0:
            return np.ones_like(r)
        d = 1.0 + r / (t * t)
        return 1.0 / (d * d)
    return np.ones_like(r)


def evaluate_deformation(points, binding_nodes, binding_weights, binding_counts, rotations, translations,
                         node_positions) -> np.ndarray:
    """The embedded deformation at the points: sum over a point's bound nodes
    of w (R (p - g) + g + t), skipping node indices out of range
    (bindings.cpp:817-838, 338-367, deformation.cpp:55-85)."""
    r, t, g = _deformation(rotations, translations, node_positions)
    n_idx = np.asarray(binding_nodes)
    w = np.asarray(binding_weights, dtype=np.float64)
    c = np.asarray(binding_counts)
    if n_idx.ndim != 2 or n_idx.shape[1] != 4:
        raise ValueError("binding nodes must have shape (n, 4)")
    if w.ndim != 2 or w.shape != n_idx.shape:
        raise ValueError("binding weights must have shape (n, 4)")
    if c.ndim != 1 or c.shape[0] != n_idx.shape[0]:
        raise ValueError("binding counts must have shape (n,)")
    bad = np.nonzero((c < 1) | (c > 4))[0]
    if len(bad):
        raise ValueError(f"binding count out of range at vertex {bad[0]}")
    p = _points(points, "points")
    if len(p) != len(n_idx):
        raise ValueError(f"points and bindings must have the same length ({len(p)} vs {len(n_idx)})")
    out = np.zeros_like(p)
    for s in range(4):
        j = n_idx[:, s]
        ok = (s < c) & (j >= 0) & (j < len(r))
        jj = np.where(ok, j, 0)
        out += np.where(ok[:, None], _applied(r[jj], t[jj], g[jj], p) * w[:, s:s + 1], 0.0)
    return out


def retract_deformation(rotations, translations, node_positions, delta) -> dict:
    """R <- exp([w]) R, t <- t + dt per node, delta = (w, dt) per node
    (bindings.cpp:1026-1049, deformation.cpp:19-32)."""
    r, t, _ = _deformation(rotations, translations, node_positions)
    d = np.asarray(delta, dtype=np.float64)
    if d.ndim != 1 or d.shape[0] != 6 * len(r):
        raise ValueError("delta must have shape (6 * node_count,): rotation increment then translation "
                         "increment per node")
    d = d.reshape(-1, 6)
    return {"rotations": _mat_mat(_exp_so3(d[:, :3]), r), "translations": t + d[:, 3:]}


def tangent_difference(rotations_from, translations_from, rotations_to, translations_to) -> np.ndarray:
    """The tangent increment taking one deformation to the other:
    w = log(R_to R_from^T), dt = t_to - t_from, per node
    (bindings.cpp:1051-1075, deformation.cpp:34-54)."""
    ra, ta, _ = _deformation(rotations_from, translations_from)
    rb, tb, _ = _deformation(rotations_to, translations_to)
    n = min(len(ra), len(rb))
    w = _log_so3(_mat_mat(rb[:n], np.transpose(ra[:n], (0, 2, 1))))
    return np.concatenate([w, tb[:n] - ta[:n]], axis=1).reshape(-1)


def transfer_level(from_nodes, rotations, translations, to_nodes, max_nodes: int = 4) -> dict:
    """Sample a deformation at new node positions (bindings.cpp:840-856,
    deformation.cpp:141-203): each new node binds to its nearest source nodes
    (support clamped to 4 slots, as the reference's binding has), blends their
    rotations as quaternions with signs aligned to the heaviest contributor --
    falling back to that contributor's rotation when the blend is shorter than
    1e-8 -- and takes the field's own value at its rest position."""
    src = _points(from_nodes, "from_nodes")
    r, t, g = _deformation(rotations, translations, src)
    dst = _points(to_nodes, "to_nodes")
    n = len(dst)
    rot = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()
    shift = np.zeros((n, 3))
    if len(src) == 0 or n == 0:
        return {"rotations": rot, "translations": shift}
    b = bind_vertices(dst, src, min(int(max_nodes), 4))
    nodes, w, c = b["nodes"], b["weights"], b["counts"]
    q_src = _quaternions(r)
    heaviest, heavy_w = nodes[:, 0].copy(), w[:, 0].copy()
    for s in range(1, 4):
        take = (s < c) & (w[:, s] > heavy_w)
        heaviest[take], heavy_w[take] = nodes[take, s], w[take, s]
    q_ref = q_src[heaviest]
    blended = np.zeros((n, 4))
    position = np.zeros((n, 3))
    for s in range(4):
        ok = (s < c)[:, None]
        j = np.where(s < c, nodes[:, s], 0)
        q = q_src[j]
        q = np.where((_qdot(q, q_ref) < 0.0)[:, None], q * -1.0, q)
        blended += np.where(ok, q * w[:, s:s + 1], 0.0)
        position += np.where(ok, _applied(r[j], t[j], g[j], dst) * w[:, s:s + 1], 0.0)
    spread = np.sqrt(_qdot(blended, blended)) > 1e-8
    rot = _matrices_of(np.where(spread[:, None], _unit(blended), q_ref))
    return {"rotations": rot, "translations": position - dst}


def validate_mask(mask, template_vertex_count: int) -> int:
    """Validate a participation mask and return how many vertices stay active
    (bindings.cpp:955-973, src/core/constraints.cpp:33-58).  Entries are
    read as true or false, so only the length and an all-false mask can fail."""
    m = np.asarray(mask).reshape(-1) != 0
    if m.size == 0:
        return 0  # no mask (every vertex takes part); the reference counts none (constraints.cpp:60-63)
    if m.size != int(template_vertex_count):
        raise ValueError(f"invalid mask: mask has {m.size} entries but the template has "
                         f"{int(template_vertex_count)} vertices")
    active = int(m.sum())
    if active == 0:
        raise ValueError("invalid mask: mask excludes every vertex; the fit would be unconstrained")
    return active


def validate_landmarks(indices, targets, template_vertex_count: int) -> None:
    """Raise with a descriptive message when landmarks are unusable
    (bindings.cpp:926-953, src/core/constraints.cpp:8-31)."""
    idx, tgt = np.asarray(indices), np.asarray(targets, dtype=np.float64)
    if idx.ndim != 1:
        raise ValueError("landmark indices must have shape (n,)")
    if tgt.ndim != 2 or tgt.shape[1] != 3 or tgt.shape[0] != idx.shape[0]:
        raise ValueError("landmark targets must have shape (n, 3), matching indices")
    problems, seen, n = [], set(), int(template_vertex_count)
    for i, (v, t) in enumerate(zip(idx.astype(np.int64).astype(np.int32).tolist(), tgt)):
        if v < 0 or v >= n:
            problems.append(f"landmark {i} points at template vertex {v} but the template has {n} vertices")
            continue
        if not np.isfinite(t).all():
            problems.append(f"landmark {i} has a non-finite target")
        if v in seen:
            problems.append(f"landmark {i} marks template vertex {v} twice")
        seen.add(v)
    if problems:
        raise ValueError("invalid landmarks: " + "; ".join(problems))


def build_template_graph(points, faces, levels: int = 4, nodes_initial: int = 100,
                         growth: int = 2, max_nodes_per_vertex: int = 4,
                         use_device: bool = False, edge_neighbours: int = 4) -> dict:
    """The cached template side: nodes, bindings and edges per level
    (bindings.cpp:886-925).  Built with the reference's FP64 rules on the
    host, or with `use_device` on the GPU -- bit-identical either way, as
    the reference requires of its device build (tests/test_graph_parity.py)."""
    p, f = _points(points, "points"), _faces(faces, "faces")
    report = validate_mesh(p, f)
    if not report["ok"]:
        raise ValueError("invalid mesh: " + "; ".join(report["problems"]))
    lib = load()
    n = len(p)
    level_count = max(1, int(levels))
    out_levels = []
    center = np.zeros(3)
    scale = C.c_double()
    for level in range(level_count):
        g = float(max(1, growth)) ** level
        nodes = min(max(1, int(math.floor(nodes_initial * g + 0.5))), n)
        idx = np.zeros(nodes, dtype=np.int32)
        pos = np.zeros((nodes, 3))
        bn = np.zeros((n, _abi.MAX_SLOTS), dtype=np.int32)
        bw = np.zeros((n, _abi.MAX_SLOTS))
        bc = np.zeros(n, dtype=np.int32)
        cap = max(1, nodes * max(1, edge_neighbours))
        edges = np.zeros((cap, 2), dtype=np.int32)
        count = C.c_int()
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        check(lib.nricp_template_graph_level(
            P(p, C.c_double), n, level_count, nodes_initial, growth, max_nodes_per_vertex,
            edge_neighbours, level, P(center, C.c_double), C.byref(scale), P(idx, C.c_int32),
            P(pos, C.c_double), P(bn, C.c_int32), P(bw, C.c_double), P(bc, C.c_int32),
            P(edges, C.c_int32), cap, C.byref(count), int(bool(use_device))))
        support = max(4, int(max_nodes_per_vertex))
        out_levels.append({
            "node_positions": pos,
            "node_template_indices": idx.astype(np.int64),
            "bindings": {"nodes": bn[:, :support].astype(np.int64), "weights": bw[:, :support],
                         "counts": bc.astype(np.int64)},
            "edges": edges[:count.value].astype(np.int64),
        })
    return {"normalization": {"center": center[None, :].copy(), "scale": scale.value},
            "levels": out_levels}


def closest_points(target_points, target_faces, query_points) -> dict:
    """Closest point and interpolated normal on the target surface, through
    the device hierarchy."""
    p, f, q = _points(target_points, "target_points"), _faces(target_faces, "target_faces"), \
        _points(query_points, "query_points")
    n = len(q)
    out = {"points": np.zeros((n, 3)), "normals": np.zeros((n, 3)), "distances": np.zeros(n),
           "triangles": np.zeros(n, dtype=np.int32)}
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    check(load().nricp_closest_points(P(p, C.c_double), len(p), P(f, C.c_int32), len(f),
                                      P(q, C.c_double), n, P(out["points"], C.c_double),
                                      P(out["normals"], C.c_double),
                                      P(out["distances"], C.c_double),
                                      P(out["triangles"], C.c_int32)))
    out["triangles"] = out["triangles"].astype(np.int64)
    return out


def find_correspondences(target_points, target_faces, query_points, query_normals,
                         distance_threshold: float = math.inf, min_normal_cosine: float = -1.0,
                         min_slope: float = 0.0, mask=None) -> dict:
    """Closest-point correspondences with the reference's filters and
    rejection breakdown (bindings.cpp:1187-1251, correspondence.cpp:18-97).
    The closest points come from the device query (``closest_points``); a
    query is then, in this order, masked (mask 0, or beyond a non-empty
    mask), rejected for distance, for its normal against the surface's
    (queries past the end of ``query_normals`` skip this test) or for slope
    (|n . (q - p)| / distance below ``min_slope``), else accepted.  Rejection
    codes: 0 accepted, 1 distance, 2 normal, 3 slope, 4 masked."""
    tp, q = _points(target_points, "target_points"), _points(query_points, "query_points")
    tf = np.asarray(target_faces)
    if tf.ndim != 2 or tf.shape[1] != 3:
        raise ValueError("target_faces must have shape (n, 3)")
    check_target = validate_mesh(tp, tf)
    if not check_target["ok"]:
        raise ValueError("invalid target mesh: " + "; ".join(check_target["problems"]))
    qn = _points(query_normals, "query_normals")
    active = np.ones(len(q), dtype=bool)
    if mask is not None:
        m = np.asarray(mask)
        if m.ndim != 1:
            raise ValueError("mask must have shape (n,)")
        if len(m):
            active = np.zeros(len(q), dtype=bool)
            k = min(len(m), len(q))
            active[:k] = m[:k].astype(np.int64) != 0
    n = len(q)
    points, normals, distances = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    triangles = np.full(n, -1, dtype=np.int64)
    rejection = np.full(n, 4, dtype=np.int64)
    idx = np.nonzero(active)[0]
    if len(idx):
        found = closest_points(tp, tf, q[idx])
        points[idx], normals[idx] = found["points"], found["normals"]
        distances[idx], triangles[idx] = found["distances"], found["triangles"]
        p, cn, d = points[idx], normals[idx], distances[idx]
        code = np.zeros(len(idx), dtype=np.int64)
        far = d > float(distance_threshold)
        code[far] = 1
        has_normal = idx < len(qn)
        qni = qn[np.minimum(idx, max(len(qn) - 1, 0))] if len(qn) else np.zeros((len(idx), 3))
        cos = qni[:, 0] * cn[:, 0] + qni[:, 1] * cn[:, 1] + qni[:, 2] * cn[:, 2]
        turned = ~far & has_normal & (cos < float(min_normal_cosine))
        code[turned] = 2
        off = q[idx] - p
        along = np.abs(cn[:, 0] * off[:, 0] + cn[:, 1] * off[:, 1] + cn[:, 2] * off[:, 2])
        with np.errstate(divide="ignore", invalid="ignore"):
            slope = along / d
        sliding = ~far & ~turned & (d > 0.0) & (slope < float(min_slope))
        code[sliding] = 3
        rejection[idx] = code
    accepted = rejection == 0
    counts = {"total": n, "accepted": int(accepted.sum()),
              "rejected_distance": int((rejection == 1).sum()), "rejected_normal": int((rejection == 2).sum()),
              "rejected_slope": int((rejection == 3).sum()), "rejected_masked": int((rejection == 4).sum()),
              "distance_mean": 0.0, "distance_p95": 0.0, "distance_max": 0.0}
    if accepted.any():
        kept = np.sort(distances[accepted])
        counts["distance_mean"] = float(np.cumsum(kept)[-1] / len(kept))  # summed in sorted order
        counts["distance_p95"] = float(kept[int(min(len(kept) - 1, 0.95 * (len(kept) - 1)))])
        counts["distance_max"] = float(kept[-1])
    return {"points": points, "normals": normals, "distances": distances, "triangles": triangles,
            "rejection": rejection, "accepted": accepted.astype(np.int64), "counts": counts}


def farthest_point_seeds(points, count: int, first_index: int = 0) -> np.ndarray:
    """Deterministic farthest-point sampling; ties break to the lower index
    (bindings.cpp:796-804, sampling.cpp:47-88)."""
    p = _points(points, "points")
    out = np.zeros(max(0, min(int(count), len(p))), dtype=np.int32)
    written = C.c_int()
    check(load().nricp_farthest_point_seeds(p.ctypes.data_as(C.POINTER(C.c_double)), len(p), int(count),
                                            int(first_index),
                                            (out if len(out) else np.zeros(1, np.int32)).ctypes.data_as(
                                                C.POINTER(C.c_int32)), C.byref(written)))
    return out[:written.value].astype(np.int64)


def bind_vertices(points, nodes, max_nodes: int = 4) -> dict:
    """Bind every vertex to its nearest nodes with distance-ratio weights
    (bindings.cpp:806-815, sampling.cpp:90-143): nodes (n, 4) -- (n, 8) when
    max_nodes > 4 -- with -1 past the count, weights likewise, counts (n,)."""
    p, q = _points(points, "points"), _points(nodes, "nodes")
    n = len(p)
    nodes_out = np.full((max(1, n), 8), -1, dtype=np.int32)
    weights_out = np.zeros((max(1, n), 8))
    counts_out = np.zeros(max(1, n), dtype=np.int32)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    check(load().nricp_bind_vertices(P(p, C.c_double), n, P(q, C.c_double), len(q), int(max_nodes),
                                     P(nodes_out, C.c_int32), P(weights_out, C.c_double),
                                     P(counts_out, C.c_int32)))
    width = 4 if int(max_nodes) <= 4 else 8
    return {"nodes": nodes_out[:n, :width].astype(np.int64), "weights": weights_out[:n, :width].copy(),
            "counts": counts_out[:n].astype(np.int64)}


def vertex_normals(points, faces) -> np.ndarray:
    """Area-weighted vertex normals (bindings.cpp:1014-1024, mesh.cpp:71-88)."""
    p, f = _points(points, "points"), _faces(faces, "faces")
    out = np.zeros((len(p), 3))
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    check(load().nricp_vertex_normals(P(p, C.c_double) if len(p) else P(np.zeros(3), C.c_double), len(p),
                                      P(f, C.c_int32) if len(f) else P(np.zeros(3, np.int32), C.c_int32),
                                      len(f), P(out, C.c_double) if len(p) else P(np.zeros(3), C.c_double)))
    return out


def fit_rigid(source_points, target_points, weights) -> dict:
    """Weighted rigid fit (reflection excluded) between point pairs, on the
    device (bindings.cpp:857-883, deformation.cpp:86-139): the rotation (1, 3,
    3) and translation (1, 3) that best map the sources onto the targets."""
    s = np.ascontiguousarray(source_points, dtype=np.float64)
    t = np.ascontiguousarray(target_points, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    if (s.ndim != 2 or s.shape[1:] != (3,) or t.shape != s.shape or w.ndim != 1
            or w.shape[0] != s.shape[0]):
        raise ValueError("fit_rigid expects (n, 3) point pairs and (n,) weights")
    rotation, translation = np.zeros((1, 3, 3)), np.zeros((1, 3))
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    check(load().nricp_fit_rigid(P(s), P(t), P(w), len(s), P(rotation), P(translation)))
    return {"rotation": rotation, "translation": translation}


def _escape(text: str) -> str:
    return text.replace("\\", "\\\\").replace('"', '\\"').replace("\n", "\\n").replace("\t", "\\t")


def _number(value) -> str:
    """%.17g, or null for a non-finite value (report.cpp:35-42)."""
    value = float(value)
    return "%.17g" % value if math.isfinite(value) else "null"


def serialize_report(route: str, precision: str, setup_seconds: float, solve_seconds: float, energy: dict,
                     correspondence: dict, levels: list, settings: dict) -> str:
    """A run report as JSON, carrying this artifact's version, in the
    reference's exact text (bindings.cpp:1253-1312, report.cpp:44-106): the
    energy total is the five terms summed in order, non-finite numbers are
    null, settings keep their order."""
    e = [float(energy[k]) for k in ("point_to_point", "point_to_plane", "smoothness", "anchor", "landmark")]
    c = correspondence
    out = ["{\n",
           f'  "version": "{_escape(__version__)}",\n',
           f'  "route": "{_escape(route)}",\n',
           f'  "precision": "{_escape(precision)}",\n',
           f'  "setup_seconds": {_number(setup_seconds)},\n',
           f'  "solve_seconds": {_number(solve_seconds)},\n',
           '  "energy": {\n',
           f'    "point_to_point": {_number(e[0])},\n',
           f'    "point_to_plane": {_number(e[1])},\n',
           f'    "smoothness": {_number(e[2])},\n',
           f'    "anchor": {_number(e[3])},\n',
           f'    "landmark": {_number(e[4])},\n',
           f'    "total": {_number(e[0] + e[1] + e[2] + e[3] + e[4])}\n',
           "  },\n",
           '  "correspondence": {\n']
    for key in ("total", "accepted", "rejected_distance", "rejected_normal", "rejected_slope", "rejected_masked"):
        out.append(f'    "{key}": {int(c[key])},\n')
    out += [f'    "distance_mean": {_number(c["distance_mean"])},\n',
            f'    "distance_p95": {_number(c["distance_p95"])},\n',
            f'    "distance_max": {_number(c["distance_max"])}\n',
            "  },\n",
            '  "levels": [']
    for i, level in enumerate(levels):
        out.append("\n" if i == 0 else ",\n")
        out.append(f'    {{"level": {int(level["level"])}, "nodes": {int(level["nodes"])}, '
                   f'"outer_iterations": {int(level["outer_iterations"])}, '
                   f'"inner_iterations": {int(level["inner_iterations"])}, '
                   f'"energy_start": {_number(level["energy_start"])}, '
                   f'"energy_end": {_number(level["energy_end"])}, '
                   f'"correspondence_mean": {_number(level["correspondence_mean"])}, '
                   f'"converged": {"true" if level["converged"] else "false"}}}')
    out.append("],\n" if not levels else "\n  ],\n")
    out.append('  "settings": {')
    for i, (name, value) in enumerate(settings.items()):
        out.append("\n" if i == 0 else ",\n")
        out.append(f'    "{_escape(str(name))}": {_number(value)}')
    out.append("}\n" if not settings else "\n  }\n")
    out.append("}\n")
    return "".join(out)


# The reference module's entry points that this module does not provide, each
# with the reason.  Reaching one raises AttributeError with that reason, so a
# caller learns why instead of meeting a bare missing name.
_NOT_PROVIDED = {
    "solve_route_a": "the reference's FP64 CPU route (bindings.cpp:1490) is its parity reference, not "
                     "a device route; this module runs the device routes: use solve_route_b or "
                     "solve_route_c",
    "energy_blocks": "the reference's CPU teaching interface (bindings.cpp:1094) is not provided",
    "assemble_normal_equations": "the reference's CPU teaching interface (bindings.cpp:1314) is not "
                                 "provided",
    "solve_normal_equations": "the reference's CPU teaching interface (bindings.cpp:1371) is not "
                              "provided",
    "fused_system": "the reference's FP64 CPU assembly (bindings.cpp:1328) is not provided; the "
                    "device assembly is reachable through nricp_session_inspect",
}


def __getattr__(name: str):
    if name in _NOT_PROVIDED:
        raise AttributeError(f"nricp_dp.{name} is not provided by this module: {_NOT_PROVIDED[name]}")
    raise AttributeError(f"module 'nricp_dp' has no attribute {name!r}")
