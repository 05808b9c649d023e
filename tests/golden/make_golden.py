"""Regenerates the golden fixtures in this folder from the reference itself.

The reference's own host code (its FP64 route A, template graph, closest-point
queries and fused assembly) is compiled from its sources by oracle/build.py
into oracle/_ref/libnricp_ref.so; this script runs it on small seeded inputs
and stores inputs and outputs together as .npz files, so that the tests can
pin the oracle restatement and the library's host code without the reference
being present.

    python tests/golden/make_golden.py          # needs the reference sources

Each fixture is a few hundred KB at most.
"""

from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from nricp_b200 import synthetic as S  # noqa: E402
from oracle.oracle import ROUTE_A, Oracle, _load  # noqa: E402

MAX_SLOTS = 8


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def template_mesh(seed: int = 3):
    points, faces = S.icosphere(3)
    rng = np.random.default_rng(seed)
    points = points * np.array([1.0, 0.8, 1.2]) + rng.normal(scale=0.01, size=points.shape)
    return np.ascontiguousarray(points), np.ascontiguousarray(faces.astype(np.int32))


def reference_graph(points, levels, nodes_initial, growth, max_nodes):
    """The reference's build_template_graph, one level at a time."""
    lib = _load("reference")
    fn = lib.ref_template_graph_level
    n = len(points)
    out = {}
    for level in range(levels):
        cap = n * 8
        center, scale = np.zeros(3), C.c_double()
        idx = np.zeros(n, np.int32)
        pos = np.zeros((n, 3))
        bn = np.zeros((n, MAX_SLOTS), np.int32)
        bw = np.zeros((n, MAX_SLOTS))
        bc = np.zeros(n, np.int32)
        edges = np.zeros((cap, 2), np.int32)
        nodes, count = C.c_int(), C.c_int()
        status = fn(_p(points), n, levels, nodes_initial, growth, max_nodes, level, _p(center),
                    C.byref(scale), _p(idx, C.c_int32), _p(pos), _p(bn, C.c_int32), _p(bw),
                    _p(bc, C.c_int32), _p(edges, C.c_int32), cap, C.byref(nodes),
                    C.byref(count))
        assert status == 0, status
        k = nodes.value
        out.update({
            "center": center, "scale": np.array(scale.value),
            f"l{level}_node_indices": idx[:k], f"l{level}_node_positions": pos[:k],
            f"l{level}_binding_nodes": bn[:, :4], f"l{level}_binding_weights": bw[:, :4],
            f"l{level}_binding_counts": bc, f"l{level}_edges": edges[:count.value],
        })
    return out


def make_graph():
    points, faces = template_mesh()
    settings = dict(levels=3, nodes_initial=20, growth=2, max_nodes=4)
    out = reference_graph(points, **settings)
    np.savez_compressed(HERE / "graph_icosphere3.npz", points=points, faces=faces,
                        **{k: np.array(v) for k, v in settings.items()}, **out)


def make_closest():
    ref = Oracle("reference")
    rng = np.random.default_rng(5)
    points, faces = S.icosphere(3)
    points = points + 0.05 * rng.normal(size=points.shape)
    faces = faces.astype(np.int32)
    queries = rng.normal(size=(400, 3)) * 0.8
    queries[:100] *= 2.0   # some far outside, some well inside
    got = ref.closest_points(points, faces, queries)
    normals = ref.vertex_normals(points, faces)
    np.savez_compressed(HERE / "closest_points.npz", points=points, faces=faces, queries=queries,
                        vertex_normals=normals, **{f"out_{k}": v for k, v in got.items()})


def make_fused():
    ref = Oracle("reference")
    rng = np.random.default_rng(9)
    points, faces = template_mesh(seed=4)
    graph = reference_graph(points, levels=1, nodes_initial=30, growth=2, max_nodes=4)
    center, scale = graph["center"], float(graph["scale"])
    template = (points - center) * scale
    nodes = graph["l0_node_positions"]
    n = len(nodes)
    rotations = np.stack([S.random_rotation(rng, 10.0) for _ in range(n)])
    translations = rng.normal(scale=0.02, size=(n, 3))
    target_points = template * 1.03 + rng.normal(scale=0.003, size=template.shape)
    corr = ref.closest_points(target_points, faces, template + 0.01)
    robust = rng.uniform(0.3, 1.0, size=len(template))
    accepted = (rng.uniform(size=len(template)) > 0.1).astype(np.uint8)
    mask = (rng.uniform(size=len(template)) > 0.05).astype(np.uint8)
    landmark_indices = np.array([3, 77, 150, 400, 600], np.int32)
    landmark_targets = template[landmark_indices] + rng.normal(scale=0.02, size=(5, 3))
    weights = np.array([1.0, 0.5, 3.0, 0.1, 2.0])
    inputs = dict(template_points=template, binding_nodes=graph["l0_binding_nodes"],
                  binding_weights=graph["l0_binding_weights"],
                  binding_counts=graph["l0_binding_counts"], node_positions=nodes,
                  rotations=rotations, translations=translations,
                  corr_points=corr["points"], corr_normals=corr["normals"], corr_robust=robust,
                  corr_accepted=accepted, edges=graph["l0_edges"],
                  landmark_indices=landmark_indices, landmark_targets=landmark_targets,
                  weights=weights, mask=mask)
    padded = dict(inputs)
    for key in ("binding_nodes", "binding_weights"):
        full = np.full((len(template), MAX_SLOTS), -1 if key == "binding_nodes" else 0.0,
                       dtype=inputs[key].dtype)
        full[:, :4] = inputs[key]
        padded[key] = full
    out = ref.fused_system(**padded)
    np.savez_compressed(HERE / "fused_system.npz", **{f"in_{k}": v for k, v in inputs.items()},
                        **{f"out_{k}": v for k, v in out.items()})


def make_route_a():
    ref = Oracle("reference")
    case = S.small_case(seed=11)
    result = ref.solve(*case.args(), route=ROUTE_A, **case.options)
    np.savez_compressed(
        HERE / "route_a_small.npz",
        template_points=case.template_points, template_faces=case.template_faces,
        target_points=case.target_points, target_faces=case.target_faces,
        level_settings=np.array(json.dumps(case.level_settings)),
        options=np.array(json.dumps(case.options)),
        **{f"out_{k}": np.asarray(v) for k, v in result.items()})


if __name__ == "__main__":
    make_graph()
    make_closest()
    make_fused()
    make_route_a()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)
