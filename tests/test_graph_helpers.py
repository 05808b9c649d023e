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
