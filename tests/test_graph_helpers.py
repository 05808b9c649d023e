"""The graph helpers of the drop-in module on the host -- farthest-point
seeds, vertex bindings and vertex normals (bindings.cpp:796-815, 1014-1024)
-- bit for bit against the reference's own functions (oracle/_ref) where they
are built, and against the oracle's C restatement."""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import nricp_dp as dp
from nricp_b200 import synthetic as S


def _checkers(oracle):
    from oracle.oracle import Oracle, reference_available

    out = [oracle]
    if reference_available():
        out.append(Oracle("reference"))
    return out


def _cloud(seed, n=400):
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3))
    p[n // 2:n // 2 + 20] = p[:20]  # duplicates: ties in every distance
    return p


@pytest.mark.parametrize("count,first", [(1, 0), (37, 0), (37, 11), (500, 3), (5, -4), (5, 10_000)])
def test_farthest_point_seeds_are_the_references(oracle, count, first):
    p = _cloud(1)
    mine = dp.farthest_point_seeds(p, count, first)
    assert mine.dtype == np.int64
    for checker in _checkers(oracle):
        assert np.array_equal(mine, checker.farthest_point_seeds(p, count, first))


def test_farthest_point_seeds_of_nothing():
    assert len(dp.farthest_point_seeds(np.zeros((0, 3)), 4)) == 0
    assert len(dp.farthest_point_seeds(np.ones((3, 3)), 0)) == 0


@pytest.mark.parametrize("max_nodes", [1, 3, 4])
def test_bindings_are_the_references(oracle, max_nodes):
    p = _cloud(2, 300)
    nodes = p[dp.farthest_point_seeds(p, 25)]
    mine = dp.bind_vertices(p, nodes, max_nodes)
    assert mine["nodes"].shape == (300, 4) and mine["weights"].shape == (300, 4)
    for checker in _checkers(oracle):
        n, w, c = checker.bind_vertices(p, nodes, max_nodes)
        assert np.array_equal(mine["counts"], c)
        assert np.array_equal(mine["nodes"], n[:, :4])
        assert np.array_equal(mine["weights"], w[:, :4])


def test_vertex_normals_are_the_references(oracle):
    case = S.small_case(seed=4)
    mine = dp.vertex_normals(case.target_points, case.target_faces)
    for checker in _checkers(oracle):
        assert np.array_equal(mine, checker.vertex_normals(case.target_points, case.target_faces))
    with pytest.raises(ValueError, match="missing vertex"):
        dp.vertex_normals(case.target_points[:3], case.target_faces)


# Above a million (query, node) pairs the library searches a uniform grid over
# the nodes instead of scanning them all; the k nearest it keeps must be the
# scan's, ties and all.
@pytest.mark.parametrize("shape", ["cloud", "plane", "outside", "far"])
def test_bindings_through_the_grid_are_the_references(oracle, shape):
    rng = np.random.default_rng(11)
    p = rng.uniform(-1.0, 1.0, size=(20_000, 3))
    if shape == "plane":
        p[:, 2] = 0.0
    p[-2000:] = p[:2000]                       # duplicates: equal distances
    nodes = p[dp.farthest_point_seeds(p, 500)]
    if shape == "outside":                     # a few cells beyond the nodes' box
        p = p + np.array([2.5, -1.0, 0.0])
    if shape == "far":                         # beyond twice the box: the plain scan
        p = p * 7.0 + np.array([30.0, -5.0, 2.0])
    mine = dp.bind_vertices(p, nodes, 4)
    for checker in _checkers(oracle):
        n, w, c = checker.bind_vertices(p, nodes, 4)
        assert np.array_equal(mine["counts"], c)
        assert np.array_equal(mine["nodes"], n[:, :4])
        assert np.array_equal(mine["weights"], w[:, :4])
    # eight slots (beyond the reference's four): the nearest eight by
    # (squared distance, index), from every distance, rounded as the library does
    eight = dp.bind_vertices(p, nodes, 8)["nodes"]
    for rows in np.array_split(np.arange(len(p)), 10):
        d = p[rows, None, :] - nodes[None, :, :]
        sq = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
        order = np.lexsort((np.broadcast_to(np.arange(len(nodes)), sq.shape), sq), axis=1)[:, :8]
        assert np.array_equal(eight[rows], order)


def test_graph_levels_through_the_grid_are_the_references(oracle):
    points, faces = S.latlong_ellipsoid(120, 220, (1.0, 0.8, 1.2))[:2]
    graph = dp.build_template_graph(points, faces, levels=2, nodes_initial=1100, growth=2,
                                    max_nodes_per_vertex=4, edge_neighbours=6)
    center, scale = oracle.normalization(points)
    normalized = (points - center) * scale
    for level in graph["levels"]:
        nodes = np.asarray(level["node_positions"])
        assert len(nodes) > 1024               # edges: more than a million node pairs
        for checker in _checkers(oracle):
            assert np.array_equal(np.asarray(level["edges"]), checker.node_edges(nodes, 6))
            n, w, c = checker.bind_vertices(normalized, nodes, 4)
            b = level["bindings"]
            assert np.array_equal(np.asarray(b["counts"]), c)
            assert np.array_equal(np.asarray(b["nodes"])[:, :4], n[:, :4])
            assert np.array_equal(np.asarray(b["weights"])[:, :4], w[:, :4])


@pytest.mark.parametrize("shape", ["cloud", "plane", "lattice"])
def test_seeds_through_the_grid_are_the_references(oracle, shape):
    """Farthest-point sampling of more than a million (point, seed) pairs
    updates only the grid cells a new seed can reach; ties (duplicates, a
    lattice's equal distances) must still go to the first point."""
    rng = np.random.default_rng(12)
    p = rng.uniform(-1.0, 1.0, size=(20_000, 3))
    if shape == "plane":
        p[:, 2] = 0.0
    if shape == "lattice":
        p = np.round(p * 6.0) / 6.0
    p[-3000:] = p[:3000]
    mine = dp.farthest_point_seeds(p, 700, 5)
    for checker in _checkers(oracle):
        assert np.array_equal(mine, checker.farthest_point_seeds(p, 700, 5))


def test_seeds_of_the_chunked_scan_are_the_references(oracle):
    """From 20,000 points up to a million (point, seed) pairs the sampling
    scans the points in parallel chunks, each keeping its first maximum."""
    rng = np.random.default_rng(13)
    p = rng.normal(size=(25_000, 3))
    p[-500:] = p[:500]
    mine = dp.farthest_point_seeds(p, 36, 17)
    assert len(p) * len(mine) <= 1 << 20
    for checker in _checkers(oracle):
        assert np.array_equal(mine, checker.farthest_point_seeds(p, 36, 17))
