"""The oracle and the library's host code, pinned to the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference's own host code
(tests/golden/make_golden.py over oracle/_ref).  These tests need no GPU and
no reference checkout:

* the oracle restatement reproduces the reference's template graph, closest
  points, vertex normals, fused FP64 assembly and whole route-A wrap;
* the library's host graph build (nricp_template_graph_level, the graph every
  device wrap uses) is bit-identical to the reference's build_template_graph
  (src/core/graph.cpp:43-76);
* where the reference library is built here, it still reproduces the
  fixtures (so they are current).
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _load(name):
    return np.load(GOLDEN / name)


def _level_count(level, nodes_initial, growth, vertices):
    return min(max(1, int(math.floor(nodes_initial * float(growth) ** level + 0.5))), vertices)


def _graph_checks(g, level, node_indices, positions, bnodes, bweights, bcounts, edges):
    assert np.array_equal(node_indices, g[f"l{level}_node_indices"])
    assert np.array_equal(positions, g[f"l{level}_node_positions"])
    assert np.array_equal(bnodes, g[f"l{level}_binding_nodes"])
    assert np.array_equal(bweights, g[f"l{level}_binding_weights"])  # bitwise
    assert np.array_equal(bcounts, g[f"l{level}_binding_counts"])
    assert np.array_equal(edges, g[f"l{level}_edges"])


def test_restatement_template_graph_is_bit_exact(oracle):
    g = _load("graph_icosphere3.npz")
    points = g["points"]
    center, scale = oracle.normalization(points)
    assert np.array_equal(center, g["center"]) and scale == float(g["scale"])
    normalized = (points - center) * scale            # mesh.cpp:183-187
    for level in range(int(g["levels"])):
        count = _level_count(level, int(g["nodes_initial"]), int(g["growth"]), len(points))
        idx = oracle.farthest_point_seeds(normalized, count)
        nodes = normalized[idx]
        bn, bw, bc = oracle.bind_vertices(normalized, nodes, int(g["max_nodes"]))
        edges = oracle.node_edges(nodes, 4)
        _graph_checks(g, level, idx, nodes, bn[:, :4], bw[:, :4], bc, edges)


def test_library_template_graph_is_bit_exact(dp):
    g = _load("graph_icosphere3.npz")
    graph = dp.build_template_graph(g["points"], g["faces"], levels=int(g["levels"]),
                                    nodes_initial=int(g["nodes_initial"]),
                                    growth=int(g["growth"]),
                                    max_nodes_per_vertex=int(g["max_nodes"]))
    assert np.array_equal(graph["normalization"]["center"][0], g["center"])
    assert graph["normalization"]["scale"] == float(g["scale"])
    for level, L in enumerate(graph["levels"]):
        b = L["bindings"]
        _graph_checks(g, level, L["node_template_indices"], L["node_positions"], b["nodes"],
                      b["weights"], b["counts"], L["edges"])


@pytest.mark.parametrize("brute", [False, True])
def test_restatement_closest_points(oracle, brute):
    f = _load("closest_points.npz")
    got = oracle.closest_points(f["points"], f["faces"], f["queries"], brute=brute)
    # same closest point and distance everywhere (FP64, 1e-12 absolute on a unit mesh)
    assert np.abs(got["points"] - f["out_points"]).max() < 1e-12
    assert np.abs(got["distances"] - f["out_distances"]).max() < 1e-12
    assert np.abs(got["normals"] - f["out_normals"]).max() < 1e-12
    # a different triangle only where both give the same closest point: a
    # query whose nearest point lies on an edge or vertex the two share
    differ = np.nonzero(got["triangles"] != f["out_triangles"])[0]
    faces = f["faces"]
    for q in differ:
        shared = set(faces[got["triangles"][q]]) & set(faces[f["out_triangles"][q]])
        assert shared, f"query {q}: triangles share no corner"


def test_restatement_vertex_normals(oracle):
    f = _load("closest_points.npz")
    assert np.array_equal(oracle.vertex_normals(f["points"], f["faces"]), f["vertex_normals"])


def test_restatement_fused_system_is_exact(oracle):
    f = _load("fused_system.npz")
    inputs = {k[3:]: f[k] for k in f.files if k.startswith("in_")}
    v = len(inputs["template_points"])
    for key, fill in (("binding_nodes", -1), ("binding_weights", 0.0)):
        full = np.full((v, 8), fill, dtype=inputs[key].dtype)
        full[:, :4] = inputs[key]
        inputs[key] = full
    got = oracle.fused_system(**inputs)
    for key in ("diagonal", "rhs", "edges", "edge_blocks", "energies"):
        assert np.array_equal(got[key], f["out_" + key]), key


def test_restatement_route_a_wrap(oracle):
    from oracle.oracle import ROUTE_A

    f = _load("route_a_small.npz")
    got = oracle.solve(f["template_points"], f["template_faces"], f["target_points"],
                       f["target_faces"], json.loads(str(f["level_settings"])), route=ROUTE_A,
                       **json.loads(str(f["options"])))
    p = f["target_points"]
    diag = float(np.linalg.norm(p.max(0) - p.min(0)))
    assert np.abs(got["vertices"] - f["out_vertices"]).max() <= 1e-12 * diag
    assert np.array_equal(got["level_nodes"], f["out_level_nodes"])
    mine, theirs = json.loads(got["report"]), json.loads(str(f["out_report"]))
    for key, value in theirs["energy"].items():
        assert mine["energy"][key] == pytest.approx(value, rel=1e-12, abs=1e-300), key
    assert [lv["outer_iterations"] for lv in mine["levels"]] == \
        [lv["outer_iterations"] for lv in theirs["levels"]]
    assert mine["correspondence"]["accepted"] == theirs["correspondence"]["accepted"]


def test_fixtures_are_current_with_the_reference(reference):
    """Where the reference library is built here, it reproduces the fixtures."""
    import sys

    sys.path.insert(0, str(GOLDEN))
    import make_golden

    g = _load("graph_icosphere3.npz")
    again = make_golden.reference_graph(g["points"], int(g["levels"]), int(g["nodes_initial"]),
                                        int(g["growth"]), int(g["max_nodes"]))
    for key, value in again.items():
        assert np.array_equal(np.asarray(value), g[key]), key
    f = _load("closest_points.npz")
    got = reference.closest_points(f["points"], f["faces"], f["queries"])
    assert np.array_equal(got["triangles"], f["out_triangles"])
    assert np.array_equal(got["points"], f["out_points"])
