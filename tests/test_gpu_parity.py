"""The CUDA path against the oracle, on a B200.

* LBVH: Morton codes, sort order and Karras topology bit-exact with the FP32
  restatement of the reference's build (src/cuda/lbvh.cu:33-352).
* Closest points: triangle ids identical to an FP64 brute-force scan except at
  stated ties (distances within 1e-6 of the bounding-box diagonal).
* Whole wraps: route B against the FP64 route A, route C against the FP64
  restatement of the device route C -- wrapped vertices within 1e-4 of the
  target's bounding-box diagonal (max), final energy within 1e-5 relative.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from nricp_b200 import synthetic as S

from conftest import diagonal

pytestmark = pytest.mark.gpu

VERTEX_TOL = 1e-4   # of the target's bounding-box diagonal, max over vertices
ENERGY_TOL = 1e-5   # relative, final energy


def _lbvh(dp, points, faces):
    import ctypes as C

    from nricp_b200._lib import check, load

    p = np.ascontiguousarray(points, dtype=np.float64)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    n = len(f)
    codes = np.zeros(n, np.uint32)
    order = np.zeros(n, np.uint32)
    left = np.zeros(max(1, n - 1), np.int32)
    right = np.zeros(max(1, n - 1), np.int32)
    bounds = np.zeros(6, np.float32)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    check(load().nricp_lbvh_export(P(p, C.c_double), len(p), P(f, C.c_int32), n,
                                   P(codes, C.c_uint32), P(order, C.c_uint32),
                                   P(left, C.c_int32), P(right, C.c_int32),
                                   P(bounds, C.c_float)))
    return dict(codes=codes, order=order, left=left[: n - 1], right=right[: n - 1], bounds=bounds)


@pytest.mark.parametrize("subdivisions", [1, 3, 5])
def test_lbvh_codes_order_and_topology_are_bit_exact(dp, device, oracle, subdivisions):
    points, faces = S.icosphere(subdivisions)
    rng = np.random.default_rng(subdivisions)
    points = points * rng.uniform(0.5, 2.0, size=3) + rng.normal(size=3)
    gpu = _lbvh(dp, points, faces)
    cpu = oracle.lbvh_build(points.astype(np.float32), faces)
    assert np.array_equal(gpu["bounds"], cpu["bounds"])
    assert np.array_equal(gpu["codes"], cpu["codes"])
    assert np.array_equal(gpu["order"], cpu["order"])
    assert np.array_equal(gpu["left"], cpu["left"])
    assert np.array_equal(gpu["right"], cpu["right"])


def test_lbvh_with_duplicate_codes_and_a_single_triangle(dp, device, oracle):
    # many triangles with the same centroid cell: ties broken by index
    base = np.array([[0, 0, 0], [1e-9, 0, 0], [0, 1e-9, 0], [1, 1, 1]], dtype=np.float64)
    faces = np.array([[0, 1, 2]] * 37 + [[0, 1, 3], [1, 2, 3]], dtype=np.int32)
    gpu = _lbvh(dp, base, faces)
    cpu = oracle.lbvh_build(base.astype(np.float32), faces)
    for key in ("codes", "order", "left", "right"):
        assert np.array_equal(gpu[key], cpu[key]), key
    one = _lbvh(dp, base, faces[:1])
    assert one["codes"].shape == (1,) and one["order"][0] == 0


def _tie_aware_triangle_check(points, faces, queries, gpu, oracle):
    brute = oracle.closest_points(points, faces, queries, brute=True)
    diag = diagonal(points)
    mismatch = np.nonzero(gpu["triangles"] != brute["triangles"])[0]
    # a different triangle is acceptable only at a tie: both triangles are
    # within 1e-6 of the diagonal of the nearest distance
    for q in mismatch:
        assert abs(gpu["distances"][q] - brute["distances"][q]) <= 1e-6 * diag, q
    same = gpu["triangles"] == brute["triangles"]
    assert np.allclose(gpu["points"][same], brute["points"][same], rtol=0, atol=1e-12)
    assert np.allclose(gpu["normals"][same], brute["normals"][same], rtol=0, atol=1e-12)
    return len(mismatch)


def test_closest_triangles_match_the_fp64_brute_force(dp, device, oracle):
    case = S.config1(0)
    rng = np.random.default_rng(1)
    queries = case.target_points[rng.choice(len(case.target_points), 3000)] + \
        rng.normal(scale=0.05, size=(3000, 3))
    gpu = dp.closest_points(case.target_points, case.target_faces, queries)
    ties = _tie_aware_triangle_check(case.target_points, case.target_faces, queries, gpu, oracle)
    assert ties <= 3


def test_closest_points_on_an_open_surface_far_queries(dp, device, oracle):
    t, f = S.uv_sphere(16, 24)
    keep = f[t[f].mean(1)[:, 2] > -0.3]
    rng = np.random.default_rng(2)
    queries = rng.normal(size=(800, 3)) * 3.0
    gpu = dp.closest_points(t, keep, queries)
    _tie_aware_triangle_check(t, keep, queries, gpu, oracle)


def _compare_wraps(result, expected, target_points):
    diag = diagonal(target_points)
    error = np.abs(np.asarray(result["vertices"]) - np.asarray(expected["vertices"]))
    max_error = float(np.linalg.norm(error.reshape(-1, 3), axis=1).max()) / diag
    e_gpu = json.loads(result["report"])["energy"]["total"]
    e_ref = json.loads(expected["report"])["energy"]["total"]
    return max_error, abs(e_gpu - e_ref) / abs(e_ref)


def test_route_b_matches_route_a_on_the_reference_fixture(dp, device, oracle):
    case = S.small_case()
    gpu = dp.solve_route_b(*case.args(), **case.options)
    ref = oracle.solve(*case.args(), **case.options)
    vertex_error, energy_error = _compare_wraps(gpu, ref, case.target_points)
    assert vertex_error <= VERTEX_TOL, vertex_error
    assert energy_error <= ENERGY_TOL, energy_error
    rg, rr = json.loads(gpu["report"]), json.loads(ref["report"])
    assert rg["route"] == "route_b" and rg["precision"] == "float"
    assert [l["nodes"] for l in rg["levels"]] == [l["nodes"] for l in rr["levels"]]
    assert [l["outer_iterations"] for l in rg["levels"]] == [l["outer_iterations"] for l in rr["levels"]]
    assert rg["correspondence"]["accepted"] == rr["correspondence"]["accepted"]


def test_route_b_matches_route_a_on_config_1(dp, device, oracle):
    case = S.config1(0)
    gpu = dp.solve_route_b(*case.args(), **case.options)
    ref = oracle.solve(*case.args(), **case.options)
    vertex_error, energy_error = _compare_wraps(gpu, ref, case.target_points)
    assert vertex_error <= VERTEX_TOL, vertex_error
    assert energy_error <= ENERGY_TOL, energy_error


def test_route_c_matches_its_fp64_restatement(dp, device, oracle):
    from oracle.oracle import ROUTE_C

    case = S.small_case()
    gpu = dp.solve_route_c(*case.args(), **case.options)
    ref = oracle.solve(*case.args(), route=ROUTE_C, **case.options)
    vertex_error, energy_error = _compare_wraps(gpu, ref, case.target_points)
    assert vertex_error <= VERTEX_TOL, vertex_error
    assert energy_error <= ENERGY_TOL, energy_error
    assert json.loads(gpu["report"])["route"] == "route_c"
