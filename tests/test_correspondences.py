"""find_correspondences (bindings.cpp:1187-1251, correspondence.cpp:18-97):
the filters, rejection codes and statistics on the host, the closest points
from the device query.  On the CPU the filters run on the reference's own
closest points and must reproduce the reference's function bit for bit; on
the GPU the whole call runs against the oracle's FP64 closest points."""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import nricp_dp as dp
from nricp_b200 import synthetic as S


def _case(seed: int):
    rng = np.random.default_rng(seed)
    points, faces = S.icosphere(3)
    points = points * np.array([1.0, 0.8, 1.2])
    queries = rng.normal(size=(600, 3)) * 0.7
    queries[:40] = points[:40] * 1.0                     # on the surface: distance 0
    normals = rng.normal(size=(550, 3))                  # fewer normals than queries
    normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    mask = (rng.uniform(size=580) > 0.15).astype(np.int64)  # shorter than the queries
    return points, faces, queries, normals, mask


SETTINGS = [dict(), dict(distance_threshold=0.4), dict(min_normal_cosine=0.2),
            dict(min_slope=0.6), dict(distance_threshold=0.5, min_normal_cosine=-0.3, min_slope=0.3)]


@pytest.mark.parametrize("settings", SETTINGS)
@pytest.mark.parametrize("masked", [False, True])
def test_filters_and_statistics_are_the_references(reference, monkeypatch, settings, masked):
    points, faces, queries, normals, mask = _case(3)
    mask = mask if masked else None
    # the reference's own closest points stand in for the device query here
    monkeypatch.setattr(dp, "closest_points",
                        lambda p, f, q: {k: np.asarray(v) for k, v in reference.closest_points(p, f, q).items()})
    mine = dp.find_correspondences(points, faces, queries, normals, mask=mask, **settings)
    ref = reference.find_correspondences(points, faces, queries, normals, mask=mask, **settings)
    for key in ("points", "normals", "distances", "triangles", "rejection"):
        assert np.array_equal(mine[key], ref[key]), key
    assert np.array_equal(mine["accepted"], (ref["rejection"] == 0).astype(np.int64))
    assert mine["counts"] == ref["counts"]
    assert mine["triangles"].dtype == np.int64 and mine["rejection"].dtype == np.int64


def test_messages_are_the_references():
    points, faces, queries, normals, _ = _case(4)
    with pytest.raises(ValueError, match=r"^invalid target mesh: face 0 corner 0 index -1 is out of range$"):
        bad = faces.copy()
        bad[0, 0] = -1
        dp.find_correspondences(points, bad, queries, normals)
    with pytest.raises(ValueError, match=r"^mask must have shape \(n,\)$"):
        dp.find_correspondences(points, faces, queries, normals, mask=np.ones((3, 2)))
    with pytest.raises(ValueError, match=r"^query_normals must have shape \(n, 3\)$"):
        dp.find_correspondences(points, faces, queries, normals[:, :2])


@pytest.mark.gpu
def test_device_correspondences_match_fp64(dp, device, oracle, monkeypatch):
    """The device query against the FP64 brute force through the same
    filters: wherever the two pick the same triangle, the points, normals,
    distances and rejection codes agree; a different triangle only at a tie
    (distances within 1e-6 of the diagonal), as in the closest-point tests."""
    points, faces, queries, normals, mask = _case(5)
    settings = dict(distance_threshold=0.5, min_normal_cosine=-0.3, min_slope=0.3, mask=mask)
    mine = dp.find_correspondences(points, faces, queries, normals, **settings)
    with monkeypatch.context() as m:
        m.setattr(dp, "closest_points", lambda p, f, q: {
            k: np.asarray(v) for k, v in oracle.closest_points(p, f, q, brute=True).items()})
        exact = dp.find_correspondences(points, faces, queries, normals, **settings)
    diag = float(np.linalg.norm(points.max(0) - points.min(0)))
    same = mine["triangles"] == exact["triangles"]
    assert np.all(np.abs(mine["distances"] - exact["distances"]) <= 1e-6 * diag)
    # shared edges and vertices tie often for queries off a convex surface;
    # most queries still pick one triangle and are compared in full
    assert same.sum() >= len(queries) // 2
    for key in ("points", "normals"):
        assert np.allclose(mine[key][same], exact[key][same], rtol=0, atol=1e-12), key
    assert np.array_equal(mine["rejection"][same], exact["rejection"][same])
    assert np.all(mine["rejection"][len(mask):] == 4) and mine["counts"]["total"] == len(queries)
