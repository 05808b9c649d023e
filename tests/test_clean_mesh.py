"""clean_mesh (bindings.cpp:762-778, mesh.cpp:118-173) against the
reference's own cleaning where oracle/_ref is built, and by the answers the
reference's tests expect (test_core_geometry.py:92-149)."""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import nricp_dp as dp
from nricp_b200 import synthetic as S


def _messy(seed: int):
    """A closed surface with planted repeated corners, collinear and tiny
    faces, duplicates in both windings and vertices no face uses."""
    rng = np.random.default_rng(seed)
    points, faces = S.icosphere(3)
    points = points * rng.uniform(0.5, 2.0, size=3)
    extra = rng.normal(size=(40, 3))                          # unused vertices
    points = np.vstack([points, extra])
    n = len(points)
    f = [faces]
    f.append(faces[rng.choice(len(faces), 60)][:, ::-1])      # reversed duplicates
    f.append(faces[rng.choice(len(faces), 30)][:, [1, 2, 0]])  # rotated duplicates
    rep = faces[rng.choice(len(faces), 25)].copy()
    rep[:, 2] = rep[:, 0]                                      # a repeated corner
    f.append(rep)
    # collinear: a new vertex on an edge's line, and a face of a sliver whose
    # squared area sits just around 1e-12 of the squared diagonal
    a, b = faces[0, 0], faces[0, 1]
    mid = points[a] + 0.37 * (points[b] - points[a])
    d = np.linalg.norm(points.max(0) - points.min(0))
    off = np.array([0.0, 0.0, 1.0]) * 1e-6 * d / np.linalg.norm(points[b] - points[a]) * 2.0
    points = np.vstack([points, mid, mid + off * 0.999, mid + off * 1.001])
    f.append(np.array([[a, b, n], [a, b, n + 1], [a, b, n + 2]]))
    faces = np.vstack(f)
    return points, faces[rng.permutation(len(faces))]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cleaning_is_the_references(reference, seed):
    points, faces = _messy(seed)
    mine = dp.clean_mesh(points, faces)
    ref = reference.clean_mesh(points, faces)
    for key in ("duplicate_faces", "degenerate_faces", "isolated_vertices"):
        assert mine[key] == ref[key], key
    assert mine["faces"].dtype == np.int64
    assert np.array_equal(mine["faces"], ref["faces"])
    assert np.array_equal(mine["points"], ref["points"])
    assert mine["duplicate_faces"] >= 60 and mine["degenerate_faces"] >= 26 and mine["isolated_vertices"] >= 40


def test_cleaning_reports_what_it_dropped():
    points = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [2, 0, 0], [0, 3, 0]])
    faces = np.array([[0, 1, 2], [1, 3, 2], [0, 2, 1], [0, 1, 0], [0, 1, 4]])
    out = dp.clean_mesh(points, faces)
    assert (out["duplicate_faces"], out["degenerate_faces"], out["isolated_vertices"]) == (1, 2, 2)
    assert out["faces"].tolist() == [[0, 1, 2], [1, 3, 2]] and out["points"].shape == (4, 3)
    # faces sharing only an edge are not duplicates
    tet = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    sides = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
    assert dp.clean_mesh(tet, sides)["duplicate_faces"] == 0
    assert dp.clean_mesh(tet, np.vstack([sides, sides[:, ::-1]]))["duplicate_faces"] == 4


def test_cleaning_rejects_an_invalid_mesh():
    with pytest.raises(ValueError, match=r"^invalid mesh: face 0 corner 2 index 9 is out of range$"):
        dp.clean_mesh(np.zeros((3, 3)), [[0, 1, 9]])
    with pytest.raises(ValueError, match=r"^faces must have shape \(n, 3\)$"):
        dp.clean_mesh(np.zeros((3, 3)), [0, 1, 2])
