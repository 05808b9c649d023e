"""Python access to the oracle -- TEST INFRASTRUCTURE ONLY.

Two interchangeable checkers with one interface:

* ``Oracle("restatement")`` -- the plain-C restatement (oracle/nricp_oracle.c),
  built on demand with gcc.  Always available.
* ``Oracle("reference")`` -- the reference's own route A compiled from its
  sources (oracle/_ref/libnricp_ref.so, see oracle/build.py); available where
  that library was built.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.
"""

from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from nricp_b200 import _abi  # noqa: E402

from . import build  # noqa: E402

ROUTE_A = 0
ROUTE_C = 1

_LIBS: dict[str, C.CDLL] = {}


def _load(kind: str) -> C.CDLL:
    if kind in _LIBS:
        return _LIBS[kind]
    if kind == "restatement":
        path = build.build_oracle()
        prefix = "oracle_"
    elif kind == "reference":
        path = build.REF_LIB
        if not path.exists():
            built = build.build_reference()
            if built is None:
                raise FileNotFoundError("the reference's route A is not built here")
        prefix = "ref_"
    elif kind == "reference_gpu":  # the reference's own GPU route B: a timed comparison, not a checker
        path = build.REF_GPU_LIB
        if not path.exists():
            raise FileNotFoundError("the reference's GPU route B is not built here")
        prefix = "ref_"
    else:
        raise ValueError(kind)
    lib = C.CDLL(str(path))
    lib._prefix = prefix  # type: ignore[attr-defined]
    _LIBS[kind] = lib
    return lib


def reference_available() -> bool:
    try:
        _load("reference")
        return True
    except (FileNotFoundError, OSError):
        return False


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a).astype(np.int32))


def _p(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


class Oracle:
    def __init__(self, kind: str = "restatement"):
        self.kind = kind
        self.lib = _load(kind)
        self._prefix = self.lib._prefix

    def _fn(self, name: str):
        return getattr(self.lib, self._prefix + name)

    # ---- whole wrap ------------------------------------------------------
    def solve(self, template_points, template_faces, target_points, target_faces,
              level_settings, route: int = ROUTE_A, **kwargs) -> dict:
        """route_a (or the FP64 route C restatement) with the route functions'
        signature (src/python/bindings.cpp:1426-1481); returns the same dict."""
        desc = _abi.Desc(template_points, template_faces, target_points, target_faces,
                         level_settings, route=0, **kwargs)
        out = _abi.ResultBuffers(desc.template_points.shape[0], desc.level_node_counts())
        if self.kind in ("reference", "reference_gpu"):
            if route != ROUTE_A and self.kind == "reference":
                raise ValueError("the reference has no CPU route C")
            # the GPU build runs the reference's device routes instead: route B
            # in place of route A, and its own route C
            if self.kind == "reference_gpu":
                fn = self.lib.ref_solve_route_c if route == ROUTE_C else self.lib.ref_solve_route_b
            else:
                fn = self.lib.ref_solve_route_a
            fn.argtypes = [C.POINTER(_abi.SolveDesc), C.POINTER(_abi.Result)]
            status = fn(C.byref(desc.struct), C.byref(out.struct))
            if status:
                self.lib.ref_last_error.restype = C.c_char_p
                raise (ValueError if status == _abi.ERR_INVALID else RuntimeError)(
                    self.lib.ref_last_error().decode())
        else:
            fn = self.lib.oracle_solve
            fn.argtypes = [C.POINTER(_abi.SolveDesc), C.c_int, C.POINTER(_abi.Result)]
            status = fn(C.byref(desc.struct), route, C.byref(out.struct))
            if status:
                self.lib.oracle_last_error.restype = C.c_char_p
                raise (ValueError if status == _abi.ERR_INVALID else RuntimeError)(
                    self.lib.oracle_last_error().decode())
        return out.to_dict()

    # ---- graph pieces ----------------------------------------------------
    def normalization(self, points):
        pts = _f64(points)
        center = np.zeros(3)
        scale = C.c_double()
        self._fn("normalization")(_p(pts), C.c_int(len(pts)), _p(center), C.byref(scale))
        return center, scale.value

    def farthest_point_seeds(self, points, count: int, first_index: int = 0) -> np.ndarray:
        pts = _f64(points)
        out = np.zeros(max(1, count), dtype=np.int32)
        n = self._fn("farthest_point_seeds")(_p(pts), C.c_int(len(pts)), C.c_int(count),
                                             C.c_int(first_index), _p(out, C.c_int32))
        return out[:n].astype(np.int64)

    def bind_vertices(self, points, nodes, max_nodes: int = 4):
        pts, nds = _f64(points), _f64(nodes)
        n = len(pts)
        out_nodes = np.zeros((n, _abi.MAX_SLOTS), dtype=np.int32)
        out_weights = np.zeros((n, _abi.MAX_SLOTS))
        out_counts = np.zeros(n, dtype=np.int32)
        self._fn("bind_vertices")(_p(pts), C.c_int(n), _p(nds), C.c_int(len(nds)),
                                  C.c_int(max_nodes), _p(out_nodes, C.c_int32),
                                  _p(out_weights), _p(out_counts, C.c_int32))
        return out_nodes, out_weights, out_counts

    def node_edges(self, nodes, neighbours: int = 4) -> np.ndarray:
        nds = _f64(nodes)
        cap = max(1, len(nds) * neighbours)
        out = np.zeros((cap, 2), dtype=np.int32)
        n = self._fn("node_edges")(_p(nds), C.c_int(len(nds)), C.c_int(neighbours),
                                   _p(out, C.c_int32), C.c_int(cap))
        return out[:max(n, 0)].astype(np.int64)

    def vertex_normals(self, points, faces) -> np.ndarray:
        pts, fcs = _f64(points), _i32(faces)
        out = np.zeros_like(pts)
        self._fn("vertex_normals")(_p(pts), C.c_int(len(pts)), _p(fcs, C.c_int32),
                                   C.c_int(len(fcs)), _p(out))
        return out

    def closest_points(self, points, faces, queries, brute: bool = False) -> dict:
        pts, fcs, q = _f64(points), _i32(faces), _f64(queries)
        n = len(q)
        out = dict(points=np.zeros((n, 3)), normals=np.zeros((n, 3)),
                   distances=np.zeros(n), triangles=np.zeros(n, dtype=np.int32))
        self._fn("closest_points")(_p(pts), C.c_int(len(pts)), _p(fcs, C.c_int32),
                                   C.c_int(len(fcs)), _p(q), C.c_int(n), C.c_int(int(brute)),
                                   _p(out["points"]), _p(out["normals"]),
                                   _p(out["distances"]), _p(out["triangles"], C.c_int32))
        return out

    # ---- assembly and solve ----------------------------------------------
    def fused_system(self, template_points, binding_nodes, binding_weights, binding_counts,
                     node_positions, rotations, translations, corr_points, corr_normals,
                     corr_robust, corr_accepted, edges, landmark_indices, landmark_targets,
                     weights, mask=None) -> dict:
        keep = []

        def hold(a):
            keep.append(a)
            return a

        class Inputs(C.Structure):
            _fields_ = [
                ("template_points", C.POINTER(C.c_double)), ("vertex_count", C.c_int),
                ("binding_nodes", C.POINTER(C.c_int32)), ("binding_weights", C.POINTER(C.c_double)),
                ("binding_counts", C.POINTER(C.c_int32)),
                ("node_positions", C.POINTER(C.c_double)), ("node_count", C.c_int),
                ("rotations", C.POINTER(C.c_double)), ("translations", C.POINTER(C.c_double)),
                ("corr_points", C.POINTER(C.c_double)), ("corr_normals", C.POINTER(C.c_double)),
                ("corr_robust", C.POINTER(C.c_double)), ("corr_accepted", C.POINTER(C.c_uint8)),
                ("edges", C.POINTER(C.c_int32)), ("edge_count", C.c_int),
                ("landmark_indices", C.POINTER(C.c_int32)),
                ("landmark_targets", C.POINTER(C.c_double)), ("landmark_count", C.c_int),
                ("mask", C.POINTER(C.c_uint8)), ("weights", C.c_double * 5),
            ]

        tp = hold(_f64(template_points))
        bn = hold(_i32(binding_nodes))
        bw = hold(_f64(binding_weights))
        bc = hold(_i32(binding_counts))
        npos = hold(_f64(node_positions))
        rot = hold(_f64(rotations).reshape(-1, 9))
        tr = hold(_f64(translations))
        cp, cn, cr = hold(_f64(corr_points)), hold(_f64(corr_normals)), hold(_f64(corr_robust))
        ca = hold(np.ascontiguousarray(np.asarray(corr_accepted).astype(np.uint8)))
        ed = hold(_i32(edges).reshape(-1, 2))
        li = hold(_i32(landmark_indices).reshape(-1))
        lt = hold(_f64(landmark_targets).reshape(-1, 3))
        mk = hold(np.ascontiguousarray(np.asarray(mask).astype(np.uint8))) if mask is not None else None
        x = Inputs()
        x.template_points, x.vertex_count = _p(tp), len(tp)
        x.binding_nodes, x.binding_weights = _p(bn, C.c_int32), _p(bw)
        x.binding_counts = _p(bc, C.c_int32)
        x.node_positions, x.node_count = _p(npos), len(npos)
        x.rotations, x.translations = _p(rot), _p(tr)
        x.corr_points, x.corr_normals, x.corr_robust = _p(cp), _p(cn), _p(cr)
        x.corr_accepted = _p(ca, C.c_uint8)
        x.edges, x.edge_count = _p(ed, C.c_int32), len(ed)
        x.landmark_indices, x.landmark_targets = _p(li, C.c_int32), _p(lt)
        x.landmark_count = len(li)
        x.mask = _p(mk, C.c_uint8) if mk is not None else C.POINTER(C.c_uint8)()
        for i in range(5):
            x.weights[i] = float(weights[i])
        n = len(npos)
        cap = max(16, len(tp) * 16 + len(ed) + 16)
        diag = np.zeros((n, 6, 6))
        rhs = np.zeros((n, 6))
        oa = np.zeros(cap, dtype=np.int32)
        ob = np.zeros(cap, dtype=np.int32)
        ob_blocks = np.zeros((cap, 6, 6))
        count = C.c_int()
        energies = np.zeros(5)
        status = self._fn("fused_system")(C.byref(x), _p(diag), _p(rhs), _p(oa, C.c_int32),
                                          _p(ob, C.c_int32), _p(ob_blocks), C.c_int(cap),
                                          C.byref(count), _p(energies))
        if status:
            raise RuntimeError("fused_system capacity")
        k = count.value
        return dict(diagonal=diag, rhs=rhs, edges=np.stack([oa[:k], ob[:k]], 1).astype(np.int64),
                    edge_blocks=ob_blocks[:k].copy(), energies=energies)

    def solve_direct(self, diagonal, edges, edge_blocks, rhs, damping=0.0,
                     diagonal_scaling=True):
        lib = _load("restatement")
        d = _f64(diagonal).reshape(-1, 36)
        e = _i32(edges).reshape(-1, 2)
        a, b = np.ascontiguousarray(e[:, 0]), np.ascontiguousarray(e[:, 1])
        blocks = _f64(edge_blocks).reshape(-1, 36)
        r = _f64(rhs).reshape(-1)
        delta = np.zeros_like(r)
        ok = lib.oracle_solve_direct(C.c_int(len(d)), _p(d), C.c_int(len(a)), _p(a, C.c_int32),
                                     _p(b, C.c_int32), _p(blocks), _p(r), C.c_double(damping),
                                     C.c_int(int(diagonal_scaling)), _p(delta))
        return bool(ok), delta.reshape(-1, 6)

    def summarize(self, codes, distances) -> dict:
        """The correspondence statistics (correspondence.cpp:59-94) of
        per-vertex outcome codes and distances, with the report's keys."""
        lib = _load("restatement")
        cd = np.ascontiguousarray(np.asarray(codes, dtype=np.uint8))
        d = _f64(distances)
        counts, stats = np.zeros(6, dtype=np.int32), np.zeros(3)
        lib.oracle_summarize(C.c_int(len(cd)), _p(cd, C.c_uint8), _p(d), _p(counts, C.c_int32), _p(stats))
        keys = ("total", "accepted", "rejected_distance", "rejected_normal", "rejected_slope", "rejected_masked")
        return {**dict(zip(keys, counts.tolist())), "distance_mean": float(stats[0]),
                "distance_p95": float(stats[1]), "distance_max": float(stats[2])}

    def reference_lbvh(self, points, faces) -> dict:
        """The reference's own device hierarchy (Lbvh::build, src/cuda/lbvh.cu:
        553-668), read back: sorted codes, permutation and Karras children in
        the export's numbering.  Needs the GPU build (kind "reference_gpu")."""
        if self.kind != "reference_gpu":
            raise ValueError("the reference's hierarchy needs Oracle('reference_gpu')")
        pts, fcs = _f64(points), _i32(faces)
        n = len(fcs)
        out = dict(codes=np.zeros(n, np.uint32), order=np.zeros(n, np.uint32),
                   left=np.zeros(max(1, n - 1), np.int32), right=np.zeros(max(1, n - 1), np.int32))
        status = self.lib.ref_lbvh_build(_p(pts), C.c_int(len(pts)), _p(fcs, C.c_int32), C.c_int(n),
                                         _p(out["codes"], C.c_uint32), _p(out["order"], C.c_uint32),
                                         _p(out["left"], C.c_int32), _p(out["right"], C.c_int32))
        if status:
            self.lib.ref_lbvh_last_error.restype = C.c_char_p
            raise RuntimeError(self.lib.ref_lbvh_last_error().decode())
        out["left"], out["right"] = out["left"][: n - 1], out["right"][: n - 1]
        return out

    def lbvh_build(self, points_f32, faces):
        lib = _load("restatement")
        pts = np.ascontiguousarray(np.asarray(points_f32, dtype=np.float32))
        fcs = _i32(faces)
        n = len(fcs)
        codes = np.zeros(n, dtype=np.uint32)
        order = np.zeros(n, dtype=np.uint32)
        left = np.zeros(max(1, n - 1), dtype=np.int32)
        right = np.zeros(max(1, n - 1), dtype=np.int32)
        bounds = np.zeros(6, dtype=np.float32)
        lib.oracle_lbvh_build(pts.ctypes.data_as(C.POINTER(C.c_float)), C.c_int(len(pts)),
                              _p(fcs, C.c_int32), C.c_int(n), _p(codes, C.c_uint32),
                              _p(order, C.c_uint32), _p(left, C.c_int32), _p(right, C.c_int32),
                              bounds.ctypes.data_as(C.POINTER(C.c_float)))
        return dict(codes=codes, order=order, left=left[: max(0, n - 1)],
                    right=right[: max(0, n - 1)], bounds=bounds)

    def horn_rotation(self, correlation) -> np.ndarray:
        lib = _load("restatement")
        c = _f64(correlation).reshape(9)
        out = np.zeros(9)
        lib.oracle_horn_rotation(_p(c), _p(out))
        return out.reshape(3, 3)

    # ---- deformation pieces (the reference's own functions only) ----------
    def _reference_only(self, what: str):
        if self.kind not in ("reference", "reference_gpu"):
            raise NotImplementedError(f"{what} is pinned to the reference's own function only")

    def retract(self, rotations, translations, delta) -> tuple[np.ndarray, np.ndarray]:
        self._reference_only("retract")
        r, t, d = _f64(rotations).copy(), _f64(translations).copy(), _f64(delta)
        self.lib.ref_retract(C.c_int(len(r)), _p(r), _p(t), _p(d))
        return r, t

    def tangent_difference(self, rotations_from, translations_from, rotations_to, translations_to):
        self._reference_only("tangent_difference")
        ra, ta, rb, tb = map(_f64, (rotations_from, translations_from, rotations_to, translations_to))
        out = np.zeros(len(ra) * 6)
        self.lib.ref_tangent_difference(C.c_int(len(ra)), _p(ra), _p(ta), _p(rb), _p(tb), _p(out))
        return out

    def evaluate_deformation(self, points, binding_nodes, binding_weights, binding_counts,
                             rotations, translations, node_positions) -> np.ndarray:
        self._reference_only("evaluate_deformation")
        pts = _f64(points)
        n, w, c = _i32(binding_nodes), _f64(binding_weights), _i32(binding_counts)
        r, t, g = _f64(rotations), _f64(translations), _f64(node_positions)
        out = np.zeros_like(pts)
        self.lib.ref_evaluate_deformation(_p(pts), C.c_int(len(pts)), _p(n, C.c_int32), _p(w),
                                          _p(c, C.c_int32), C.c_int(len(r)), _p(r), _p(t), _p(g),
                                          _p(out))
        return out

    def robust_weights(self, kernel: str, squared_residuals, threshold: float) -> np.ndarray:
        self._reference_only("robust_weights")
        r = _f64(squared_residuals)
        out = np.zeros(len(r))
        self.lib.ref_robust_weights(kernel.encode(), _p(r), C.c_int(len(r)), C.c_double(threshold),
                                    _p(out))
        return out

    def transfer_level(self, from_nodes, rotations, translations, to_nodes, max_nodes: int = 4):
        self._reference_only("transfer_level")
        src, r, t, dst = _f64(from_nodes), _f64(rotations), _f64(translations), _f64(to_nodes)
        out_r, out_t = np.zeros((len(dst), 3, 3)), np.zeros((len(dst), 3))
        self.lib.ref_transfer_level(C.c_int(len(src)), _p(src), _p(r), _p(t), C.c_int(len(dst)), _p(dst),
                                    C.c_int(max_nodes), _p(out_r), _p(out_t))
        return out_r, out_t

    def clean_mesh(self, points, faces) -> dict:
        self._reference_only("clean_mesh")
        pts, fcs = _f64(points), _i32(faces)
        out_p, out_f = np.zeros_like(pts), np.zeros_like(fcs)
        counts = np.zeros(4, dtype=np.int32)
        kept = self.lib.ref_clean_mesh(_p(pts), C.c_int(len(pts)), _p(fcs, C.c_int32), C.c_int(len(fcs)),
                                       _p(out_p), _p(out_f, C.c_int32), _p(counts, C.c_int32))
        return {"points": out_p[:kept], "faces": out_f[:counts[3]].astype(np.int64),
                "duplicate_faces": int(counts[0]), "degenerate_faces": int(counts[1]),
                "isolated_vertices": int(counts[2])}

    def find_correspondences(self, target_points, target_faces, query_points, query_normals,
                             distance_threshold=np.inf, min_normal_cosine=-1.0, min_slope=0.0, mask=None):
        self._reference_only("find_correspondences")
        tp, tf, q, qn = _f64(target_points), _i32(target_faces), _f64(query_points), _f64(query_normals)
        m = np.zeros(0, dtype=np.uint8) if mask is None else (np.asarray(mask) != 0).astype(np.uint8)
        n = len(q)
        out = dict(points=np.zeros((n, 3)), normals=np.zeros((n, 3)), distances=np.zeros(n),
                   triangles=np.zeros(n, dtype=np.int32), rejection=np.zeros(n, dtype=np.int32))
        ints, stats = np.zeros(6, dtype=np.int32), np.zeros(3)
        self.lib.ref_find_correspondences(
            _p(tp), C.c_int(len(tp)), _p(tf, C.c_int32), C.c_int(len(tf)), _p(q), C.c_int(n), _p(qn),
            C.c_int(len(qn)), C.c_double(distance_threshold), C.c_double(min_normal_cosine),
            C.c_double(min_slope), _p(np.ascontiguousarray(m), C.c_uint8), C.c_int(len(m)), _p(out["points"]),
            _p(out["normals"]), _p(out["distances"]), _p(out["triangles"], C.c_int32),
            _p(out["rejection"], C.c_int32), _p(ints, C.c_int32), _p(stats))
        keys = ("total", "accepted", "rejected_distance", "rejected_normal", "rejected_slope", "rejected_masked")
        out["counts"] = {**dict(zip(keys, ints.tolist())), "distance_mean": stats[0], "distance_p95": stats[1],
                         "distance_max": stats[2]}
        return out
