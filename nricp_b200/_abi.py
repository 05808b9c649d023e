"""ctypes mirror of include/nricp_b200.h and the argument parsing of the
reference's route functions (src/python/bindings.cpp:181-196, 584-672).

Everything here is plain data marshalling: numpy arrays in, descriptor structs
out.  The descriptor keeps references to the arrays it points into, so they stay
alive as long as the descriptor does.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import Any

import numpy as np

MAX_SLOTS = 8

OK = 0
ERR_INVALID = 1
ERR_CUDA = 2
ERR_NO_DEVICE = 3
ERR_CAPACITY = 4
ERR_STATE = 5
ERR_TIMEOUT = 6

ROBUST_NONE = 0
ROBUST_HUBER = 1
ROBUST_GEMAN_MCCLURE = 2

ROUTE_B = 0
ROUTE_C = 1


class LevelSettings(C.Structure):
    _fields_ = [
        ("point_to_point", C.c_double),
        ("point_to_plane", C.c_double),
        ("smoothness", C.c_double),
        ("anchor", C.c_double),
        ("landmark", C.c_double),
        ("robust_kernel", C.c_int),
        ("robust_threshold", C.c_double),
        ("max_outer_iterations", C.c_int),
        ("max_inner_iterations", C.c_int),
        ("outer_tolerance", C.c_double),
        ("inner_tolerance", C.c_double),
    ]


class SolveDesc(C.Structure):
    _fields_ = [
        ("template_points", C.POINTER(C.c_double)),
        ("template_vertex_count", C.c_int),
        ("template_faces", C.POINTER(C.c_int32)),
        ("template_face_count", C.c_int),
        ("target_points", C.POINTER(C.c_double)),
        ("target_vertex_count", C.c_int),
        ("target_faces", C.POINTER(C.c_int32)),
        ("target_face_count", C.c_int),
        ("levels", C.POINTER(LevelSettings)),
        ("level_setting_count", C.c_int),
        ("mask", C.POINTER(C.c_uint8)),
        ("landmark_indices", C.POINTER(C.c_int32)),
        ("landmark_targets", C.POINTER(C.c_double)),
        ("landmark_count", C.c_int),
        ("distance_threshold", C.c_double),
        ("min_normal_cosine", C.c_double),
        ("min_slope", C.c_double),
        ("initial_damping", C.c_double),
        ("damping_decrease", C.c_double),
        ("damping_increase", C.c_double),
        ("max_damping_attempts", C.c_int),
        ("diagonal_damping", C.c_int),
        ("graph_levels", C.c_int),
        ("nodes_initial", C.c_int),
        ("growth", C.c_int),
        ("pcg_tolerance", C.c_double),
        ("pcg_max_iterations", C.c_int),
        ("max_nodes_per_vertex", C.c_int),
        ("edge_neighbours", C.c_int),
        ("route", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("vertices", C.POINTER(C.c_double)),
        ("rotations", C.POINTER(C.c_double)),
        ("translations", C.POINTER(C.c_double)),
        ("node_positions", C.POINTER(C.c_double)),
        ("level_nodes", C.POINTER(C.c_int32)),
        ("report_json", C.c_char_p),
        ("report_capacity", C.c_size_t),
        ("report_length", C.c_size_t),
    ]


class Progress(C.Structure):
    _fields_ = [
        ("level", C.c_int),
        ("outer", C.c_int),
        ("inner", C.c_int),
        ("finished", C.c_int),
        ("level_converged", C.c_int),
        ("energy", C.c_double),
        ("correspondence_mean", C.c_double),
    ]


class TickRecord(C.Structure):
    _fields_ = [
        ("phase", C.c_int), ("level", C.c_int), ("pcg_iterations", C.c_int), ("pad", C.c_int),
        ("query_ms", C.c_float), ("pcg_ms", C.c_float), ("assemble_ms", C.c_float),
        ("tick_ms", C.c_float),
    ]


class Inspect(C.Structure):
    P = C.POINTER
    _fields_ = [
        ("level", C.c_int), ("node_count", C.c_int), ("phase", C.c_int), ("off_count", C.c_int),
        ("off_capacity", C.c_int), ("energies", C.c_double * 5),
        ("rotations", P(C.c_double)), ("translations", P(C.c_double)),
        ("corr_points", P(C.c_double)), ("corr_normals", P(C.c_double)),
        ("corr_robust", P(C.c_double)), ("corr_codes", P(C.c_uint8)),
        ("diag", P(C.c_float)), ("rhs", P(C.c_float)),
        ("off_nodes", P(C.c_int32)), ("off_blocks", P(C.c_float)),
        ("damping", C.c_double), ("delta", P(C.c_double)),
        ("corr_distances", P(C.c_double)), ("pcg_ok", C.c_int), ("pcg_iterations", C.c_int),
        ("pcg_residual", C.c_double), ("target_points", P(C.c_double)), ("target_normals", P(C.c_double)),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("memory_budget_bytes", C.c_size_t), ("max_slots", C.c_int), ("prep_threads", C.c_int),
        ("pcg_cluster", C.c_int), ("ticks_per_poll", C.c_int),
        ("large_face_threshold", C.c_int), ("large_slots", C.c_int),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_long), ("completed", C.c_long), ("failed", C.c_long),
        ("waiting", C.c_long), ("running", C.c_long),
        ("latency_p50_ms", C.c_double), ("latency_p99_ms", C.c_double),
        ("latency_mean_ms", C.c_double), ("queue_p50_ms", C.c_double),
        ("wraps_per_second", C.c_double),
        ("ticks", C.c_long), ("launches", C.c_long), ("captures", C.c_long),
        ("busy_seconds", C.c_double),
        ("resident_bytes", C.c_size_t), ("peak_resident_bytes", C.c_size_t),
        ("slots_used", C.c_int),
    ]


REQUEST_STATES = {0: "waiting", 1: "running", 2: "done", 3: "failed"}


# Defaults of the route functions, src/python/bindings.cpp:1470-1481.
ROUTE_DEFAULTS: dict[str, Any] = dict(
    mask=None,
    landmark_indices=None,
    landmark_targets=None,
    distance_threshold=math.inf,
    min_normal_cosine=-1.0,
    min_slope=0.0,
    initial_damping=1e-3,
    damping_decrease=0.3,
    damping_increase=4.0,
    max_damping_attempts=6,
    diagonal_damping=True,
    graph_levels=4,
    nodes_initial=100,
    growth=2,
    pcg_tolerance=1e-5,
    pcg_max_iterations=60,
    # extensions beyond the reference's keyword set
    max_nodes_per_vertex=4,
    edge_neighbours=4,
)


def robust_kernel_code(name: str) -> int:
    """robust_kernel_from_string, src/energy/robust.cpp:7-17."""
    if name in ("huber", "Huber"):
        return ROBUST_HUBER
    if name in ("geman_mcclure", "geman-mcclure", "GemanMcClure"):
        return ROBUST_GEMAN_MCCLURE
    return ROBUST_NONE


def level_settings(values: dict) -> LevelSettings:
    """to_level_settings, src/python/bindings.cpp:181-196 (same defaults)."""
    return LevelSettings(
        point_to_point=float(values.get("point_to_point", 1.0)),
        point_to_plane=float(values.get("point_to_plane", 1.0)),
        smoothness=float(values.get("smoothness", 1.0)),
        anchor=float(values.get("anchor", 0.0)),
        landmark=float(values.get("landmark", 1.0)),
        robust_kernel=robust_kernel_code(str(values.get("robust_kernel", "huber"))),
        robust_threshold=float(values.get("robust_threshold", 0.0)),
        max_outer_iterations=int(values.get("max_outer_iterations", 10)),
        max_inner_iterations=int(values.get("max_inner_iterations", 10)),
        outer_tolerance=float(values.get("outer_tolerance", 1e-3)),
        inner_tolerance=float(values.get("inner_tolerance", 1e-4)),
    )


def _points(array, name: str) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(array, dtype=np.float64))
    if out.ndim != 2 or out.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    return out


def _faces(array, name: str) -> np.ndarray:
    out = np.asarray(array)
    if out.ndim != 2 or out.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    if out.dtype == np.int32:  # as the cast below would give, without copies
        return np.ascontiguousarray(out)
    # any other type through int64 (the reference's forcecast), then narrowed
    return np.ascontiguousarray(np.asarray(out, dtype=np.int64).astype(np.int32))


def _ptr(array: np.ndarray | None, ctype):
    if array is None:
        return C.POINTER(ctype)()
    return array.ctypes.data_as(C.POINTER(ctype))


class Desc:
    """A SolveDesc plus the arrays it points into."""

    def __init__(self, template_points, template_faces, target_points, target_faces,
                 level_settings_list, route: int = ROUTE_B, **kwargs):
        unknown = set(kwargs) - set(ROUTE_DEFAULTS)
        if unknown:
            raise TypeError(f"unexpected keyword arguments: {sorted(unknown)}")
        options = dict(ROUTE_DEFAULTS)
        options.update(kwargs)
        self.template_points = _points(template_points, "template_points")
        self.template_faces = _faces(template_faces, "template_faces")
        self.target_points = _points(target_points, "target_points")
        self.target_faces = _faces(target_faces, "target_faces")
        levels = list(level_settings_list)
        self.levels = (LevelSettings * max(1, len(levels)))()
        for i, entry in enumerate(levels):
            self.levels[i] = level_settings(dict(entry))
        self.mask = None
        if options["mask"] is not None:
            mask = np.asarray(options["mask"])
            if mask.ndim != 1:
                raise ValueError("mask must have shape (n,)")
            self.mask = np.ascontiguousarray((mask != 0).astype(np.uint8))
        self.landmark_indices = None
        self.landmark_targets = None
        landmark_count = 0
        if options["landmark_indices"] is not None and options["landmark_targets"] is not None:
            self.landmark_indices = np.ascontiguousarray(
                np.asarray(options["landmark_indices"]).astype(np.int64).astype(np.int32))
            self.landmark_targets = _points(options["landmark_targets"], "landmark_targets")
            if self.landmark_indices.shape[0] != self.landmark_targets.shape[0]:
                raise ValueError("landmark indices and targets must agree in length")
            landmark_count = int(self.landmark_indices.shape[0])
        self.options = options
        self.route = route
        d = SolveDesc()
        d.template_points = _ptr(self.template_points, C.c_double)
        d.template_vertex_count = self.template_points.shape[0]
        d.template_faces = _ptr(self.template_faces, C.c_int32)
        d.template_face_count = self.template_faces.shape[0]
        d.target_points = _ptr(self.target_points, C.c_double)
        d.target_vertex_count = self.target_points.shape[0]
        d.target_faces = _ptr(self.target_faces, C.c_int32)
        d.target_face_count = self.target_faces.shape[0]
        d.levels = C.cast(self.levels, C.POINTER(LevelSettings))
        d.level_setting_count = len(levels)
        d.mask = _ptr(self.mask, C.c_uint8)
        d.landmark_indices = _ptr(self.landmark_indices, C.c_int32)
        d.landmark_targets = _ptr(self.landmark_targets, C.c_double)
        d.landmark_count = landmark_count
        d.distance_threshold = float(options["distance_threshold"])
        d.min_normal_cosine = float(options["min_normal_cosine"])
        d.min_slope = float(options["min_slope"])
        d.initial_damping = float(options["initial_damping"])
        d.damping_decrease = float(options["damping_decrease"])
        d.damping_increase = float(options["damping_increase"])
        d.max_damping_attempts = int(options["max_damping_attempts"])
        d.diagonal_damping = 1 if options["diagonal_damping"] else 0
        d.graph_levels = int(options["graph_levels"])
        d.nodes_initial = int(options["nodes_initial"])
        d.growth = int(options["growth"])
        d.pcg_tolerance = float(options["pcg_tolerance"])
        d.pcg_max_iterations = int(options["pcg_max_iterations"])
        d.max_nodes_per_vertex = int(options["max_nodes_per_vertex"])
        d.edge_neighbours = int(options["edge_neighbours"])
        d.route = int(route)
        self.struct = d

    def level_node_counts(self) -> list[int]:
        """Node count per level, src/core/graph.cpp:52-57."""
        count = self.template_points.shape[0]
        levels = max(1, int(self.options["graph_levels"]))
        out = []
        for level in range(levels):
            growth = float(max(1, int(self.options["growth"]))) ** level
            requested = max(1, int(_lround(self.options["nodes_initial"] * growth)))
            out.append(min(requested, count))
        return out


def _lround(value: float) -> int:
    """C lround: halves away from zero."""
    return int(math.floor(abs(value) + 0.5)) * (1 if value >= 0 else -1)


class ResultBuffers:
    """Caller-allocated outputs for one wrap, as route_result_to_dict lays them
    out (src/python/bindings.cpp:674-710)."""

    def __init__(self, vertex_count: int, level_nodes: list[int], report_capacity: int = 1 << 16):
        finest = level_nodes[-1]
        self.vertices = np.zeros((vertex_count, 3))
        self.rotations = np.zeros((finest, 3, 3))
        self.translations = np.zeros((finest, 3))
        self.node_positions = np.zeros((finest, 3))
        self.level_nodes = np.zeros(len(level_nodes), dtype=np.int32)
        self.report = C.create_string_buffer(report_capacity)
        r = Result()
        r.vertices = _ptr(self.vertices, C.c_double)
        r.rotations = _ptr(self.rotations, C.c_double)
        r.translations = _ptr(self.translations, C.c_double)
        r.node_positions = _ptr(self.node_positions, C.c_double)
        r.level_nodes = _ptr(self.level_nodes, C.c_int32)
        r.report_json = C.cast(self.report, C.c_char_p)
        r.report_capacity = report_capacity
        r.report_length = 0
        self.struct = r

    def to_dict(self) -> dict:
        return {
            "vertices": self.vertices,
            "rotations": self.rotations,
            "translations": self.translations,
            "node_positions": self.node_positions,
            "report": self.report.value.decode(),
            "level_nodes": self.level_nodes.astype(np.int64),
        }
