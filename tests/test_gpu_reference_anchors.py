"""The two restatements that the reference has no CPU code for, anchored to the
reference's own compiled device code (oracle/_ref/libnricp_ref_gpu.so, built
from its src/cuda by oracle/build.py).

* The hierarchy: the reference's Lbvh::build (src/cuda/lbvh.cu:553-668), run on
  the device and read back, against this library's hierarchy export -- sorted
  Morton codes, the sort permutation and every internal node's Karras children
  bit for bit, on icosphere, duplicate-code, pole-sliver and config-1 target
  meshes.  (tests/test_lbvh_oracle.py and tests/test_gpu_parity.py hold the
  C restatement to the same arrays, so all three agree.)
* Route C: the reference's own device route C (src/cuda/local_global.cu:
  188-302) against the FP64 restatement (oracle/nricp_oracle.c).  The
  reference's route C is FP32 throughout -- FP32 closest points, a Horn fit
  by a fixed 12 sweeps of FP32 Jacobi, assembly with atomics -- and its
  replace-not-step rotation update carries those differences forward, so it
  is held here the way the reference's own tests hold a route
  (tests/test_route_c.py:126-148): the same schedule (outer iterations within
  1 and inner iterations within 2 per level), fit quality within 10 % (mean
  distance to the ground truth, which is the target's vertex of the same
  index), and final energy within 10 %.  The reference's route C sums its
  assembly with FP32 atomics, so its own schedule is not the same from run
  to run: on the session fixture its second level took 4 outer iterations in
  four runs of this test and 3 in a fifth.  The largest vertex gap is printed:
  measured, 1.3e-2 to 2.2e-2 of unit-scale coordinates on the mirror-symmetric
  fixtures, 1e-3 on the asymmetric one.  On the asymmetric fixture, which has
  no exact closest-point ties, this library's route C must lie within 1e-4 of
  the diagonal of the restatement.

  The reference's device session does not cap the inner iterations: its inner
  loop stops only when an attempt is not accepted or the improvement falls to
  the inner tolerance (src/cuda/session.cu:277-326); `max_inner_iterations`
  is honoured by its route A only.  The restatement follows route A's
  schedule, as this library does, so the comparison runs with a cap that
  never binds (1000 inner iterations), where the two schedules agree.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from nricp_b200 import synthetic as S

from conftest import diagonal

pytestmark = pytest.mark.gpu

VERTEX_TOL = 1e-4               # of the target diagonal


@pytest.fixture(scope="module")
def reference_gpu():
    from oracle import build
    from oracle.oracle import Oracle

    if not build.REF_GPU_LIB.exists():
        pytest.skip("the reference's device code is not built here (oracle/_ref/libnricp_ref_gpu.so)")
    return Oracle("reference_gpu")


def _ours(points, faces):
    from test_gpu_parity import _lbvh

    return _lbvh(None, points, faces)


def _meshes():
    out = {}
    for sub in (3, 5):
        points, faces = S.icosphere(sub)
        rng = np.random.default_rng(sub)
        out[f"icosphere{sub}"] = (points * rng.uniform(0.5, 2.0, size=3) + rng.normal(size=3), faces)
    base = np.array([[0, 0, 0], [1e-9, 0, 0], [0, 1e-9, 0], [1, 1, 1]], dtype=np.float64)
    out["duplicate_codes"] = (base, np.array([[0, 1, 2]] * 37 + [[0, 1, 3], [1, 2, 3]]))
    out["pole_slivers"] = S.uv_sphere(40, 64)  # coincident pole vertices, zero-area pole faces
    case = S.config1(0)
    out["config1_target"] = (case.target_points, case.target_faces)
    return out


@pytest.mark.parametrize("name", ["icosphere3", "icosphere5", "duplicate_codes", "pole_slivers",
                                  "config1_target"])
def test_hierarchy_is_the_references_bit_for_bit(device, reference_gpu, name):
    points, faces = _meshes()[name]
    points = np.ascontiguousarray(points, np.float64)
    faces = np.ascontiguousarray(faces, np.int32)
    ours = _ours(points, faces)
    theirs = reference_gpu.reference_lbvh(points, faces)
    for key in ("codes", "order", "left", "right"):
        assert np.array_equal(ours[key], theirs[key]), key


def test_single_triangle_hierarchy(device, reference_gpu):
    points = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    faces = np.array([[0, 1, 2]], np.int32)
    ours = _ours(points, faces)
    theirs = reference_gpu.reference_lbvh(points, faces)
    assert np.array_equal(ours["codes"], theirs["codes"]) and np.array_equal(ours["order"], theirs["order"])


UNCAPPED = 1000  # inner iterations: never reached, as in the reference's device session


def _route_c_cases():
    t1, f1 = S.uv_sphere(10, 14)
    t2, f2 = S.uv_sphere(14, 18)
    small = S.small_case(seed=3)
    levels = S.reference_settings(2, max_inner_iterations=UNCAPPED)
    return {
        "session_fixture": (t1, f1, S.bulge(t1, 0.07), f1, levels,
                            dict(graph_levels=2, nodes_initial=50, growth=2)),
        "route_a_fixture": (t2, f2, S.bulge(t2, 0.09), f2, levels,
                            dict(graph_levels=2, nodes_initial=80, growth=2)),
        "asymmetric": (small.template_points, small.template_faces, small.target_points,
                       small.target_faces, levels, small.options),
    }


@pytest.mark.parametrize("name", ["session_fixture", "route_a_fixture", "asymmetric"])
def test_route_c_restatement_agrees_with_the_references_route_c(dp, device, oracle, reference_gpu, name):
    from oracle.oracle import ROUTE_C

    tp, tf, gp, gf, levels, options = _route_c_cases()[name]
    theirs = reference_gpu.solve(tp, tf, gp, gf, levels, route=ROUTE_C, **options)
    restated = oracle.solve(tp, tf, gp, gf, levels, route=ROUTE_C, **options)
    ours = dp.solve_route_c(tp, tf, gp, gf, levels, **options)
    t_rep, r_rep = json.loads(theirs["report"]), json.loads(restated["report"])
    t_iter = [(lv["outer_iterations"], lv["inner_iterations"]) for lv in t_rep["levels"]]
    r_iter = [(lv["outer_iterations"], lv["inner_iterations"]) for lv in r_rep["levels"]]
    truth = np.asarray(gp)  # the target shares the template's faces: vertex i's ground truth
    t_fit = np.linalg.norm(np.asarray(theirs["vertices"]) - truth, axis=1).mean()
    r_fit = np.linalg.norm(np.asarray(restated["vertices"]) - truth, axis=1).mean()
    t_e, r_e = t_rep["energy"]["total"], r_rep["energy"]["total"]
    gap = np.abs(np.asarray(theirs["vertices"]) - np.asarray(restated["vertices"])).max()
    print(f"{name}: iterations {t_iter} (reference) {r_iter} (restatement); mean fit {t_fit:.4e} / "
          f"{r_fit:.4e}; energy {t_e:.6e} / {r_e:.6e}; largest vertex gap {gap:.2e}")
    assert len(t_iter) == len(r_iter)
    assert all(abs(a - b) <= 1 for (a, _), (b, _) in zip(t_iter, r_iter))
    assert all(abs(a - b) <= 2 for (_, a), (_, b) in zip(t_iter, r_iter))
    assert abs(r_fit - t_fit) <= 0.10 * t_fit
    assert abs(r_e - t_e) <= 0.10 * abs(t_e)
    if name == "asymmetric":
        # the mirror-symmetric fixtures hold exact closest-point ties, which two
        # query structures may break differently; without ties this library's
        # route C is held to the restatement at the parity bar
        assert np.linalg.norm(np.asarray(ours["vertices"]) - np.asarray(restated["vertices"]), axis=1).max() \
            <= VERTEX_TOL * diagonal(gp)
