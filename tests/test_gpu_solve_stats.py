"""The damped linear solve and the correspondence statistics against the oracle.

A session is stepped through whole wraps (nricp_session_inspect between steps):

* every converged solve attempt's increment against the oracle's FP64
  block-Cholesky solve (the reference's damped system, normal_equations.cpp:
  81-96, with a direct solve in place of direct_solve.cpp:10-64) of the same
  damped system -- the FP32 blocks and right-hand side the device assembled,
  the damping of that attempt.  The device iterates in FP32 matvecs with FP64
  dot products and residual norms (pcg_solver.cu:63-241 semantics) and stops
  at |r| / |b| <= the PCG tolerance, so its increment must satisfy the FP64
  system to a small multiple of that tolerance;
* the final correspondence statistics the device reports (counts per outcome,
  mean, 95th percentile and maximum of the accepted distances; deform_ops.cu:
  135-278 semantics) against the oracle's summary (correspondence.cpp:59-94)
  of the same per-vertex outcomes and distances.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu

# The device's recursive residual is FP64 but its matvecs are FP32: the true
# FP64 residual of the increment it returns may exceed the tolerance it
# stopped at by the rounding of those matvecs.  Bar: 10 x the tolerance.
RESIDUAL_FACTOR = 10.0
MEAN_TOL = 1e-12  # the mean is summed in another order than the sorted host sum


def _damped_matvec(diag, pairs, blocks, damping, x):
    """(A + damping * diag-scale) x in FP64 from the FP32 blocks: the
    off-diagonal block B of pair (a, b) is A[a, b]; A[b, a] = B^T."""
    n = len(diag)
    d = diag.astype(np.float64).reshape(n, 6, 6).copy()
    idx = np.arange(6)
    d[:, idx, idx] += damping * np.maximum(d[:, idx, idx], 1e-12)
    y = np.einsum("nij,nj->ni", d, x)
    b = blocks.astype(np.float64).reshape(-1, 6, 6)
    a_side, b_side = pairs[:, 0], pairs[:, 1]
    np.add.at(y, a_side, np.einsum("kij,kj->ki", b, x[b_side]))
    np.add.at(y, b_side, np.einsum("kji,kj->ki", b, x[a_side]))
    return y


def _summed_pairs(pairs, blocks):
    """The oracle's solve takes one block per node pair: sum the device's
    entries (a smoothness edge and a shared-vertex group may share a pair)."""
    acc = {}
    for (a, b), blk in zip(pairs.tolist(), blocks.astype(np.float64).reshape(-1, 36)):
        acc[(a, b)] = acc.get((a, b), 0.0) + blk
    keys = sorted(acc)
    return np.asarray(keys, np.int32).reshape(-1, 2), np.stack([acc[k] for k in keys]) if keys else np.zeros((0, 36))


def _cases():
    c3 = S.config2(seed=21, vertex_count=4000, triangle_count=40_000, nodes_finest=300, levels=3)
    c3.options = dict(c3.options, edge_neighbours=8)  # config 3's graph: k = 6, 8-NN edges
    return {"small": S.small_case(seed=3), "config1": S.config1(2), "k6_8nn": c3}


@pytest.mark.parametrize("which", ["small", "config1", "k6_8nn"])
def test_converged_solves_satisfy_the_fp64_damped_system(dp, device, oracle, which):
    case = _cases()[which]
    tol = case.options.get("pcg_tolerance", 1e-5)
    session = dp.RouteBSession(*case.args(), **case.options)
    checked, worst_residual, worst_error = 0, 0.0, 0.0
    while not session.finished():
        before = session.inspect()
        session.step()
        if before["phase"] != 2:
            continue
        after = session.inspect()
        if not after["pcg_ok"]:
            continue  # a failed attempt feeds the damping; it leaves no increment
        n = before["node_count"]
        x = after["delta"][:n]
        rhs = before["rhs"].astype(np.float64)
        pairs, blocks = _summed_pairs(before["off_nodes"], before["off_blocks"])
        ok, exact = oracle.solve_direct(before["diag"].astype(np.float64).reshape(n, 36), pairs, blocks,
                                        rhs, damping=before["damping"], diagonal_scaling=True)
        assert ok
        bnorm = np.linalg.norm(rhs)
        residual = np.linalg.norm(rhs - _damped_matvec(before["diag"], before["off_nodes"],
                                                       before["off_blocks"], before["damping"], x)) / bnorm
        exact_residual = np.linalg.norm(rhs - _damped_matvec(before["diag"], before["off_nodes"],
                                                             before["off_blocks"], before["damping"],
                                                             exact)) / bnorm
        assert exact_residual < 1e-10  # the oracle's own solve
        assert after["pcg_residual"] <= tol
        assert residual <= RESIDUAL_FACTOR * tol, (checked, residual, after["pcg_iterations"])
        worst_residual = max(worst_residual, residual)
        worst_error = max(worst_error, np.linalg.norm(x - exact) / max(np.linalg.norm(exact), 1e-300))
        checked += 1
    assert checked >= 5
    print(f"{which}: {checked} solves, worst FP64 residual {worst_residual:.2e} (tolerance {tol:.0e}), "
          f"worst increment error {worst_error:.2e}")


def _stats_cases():
    base = S.small_case(seed=5)
    mask = np.ones(len(base.template_points), np.uint8)
    mask[::9] = 0
    # thresholds under which every outcome occurs at the final state
    filtered = dict(base.options, mask=mask, distance_threshold=0.02, min_normal_cosine=0.999,
                    min_slope=0.99)
    c2 = S.config2(seed=8, vertex_count=3000, triangle_count=50_000, nodes_finest=200, levels=3)
    return {"filters": (base, filtered), "outliers": (c2, dict(c2.options, min_normal_cosine=0.5))}


@pytest.mark.parametrize("which", ["filters", "outliers"])
def test_final_statistics_match_the_oracle_summary(dp, device, oracle, which):
    case, options = _stats_cases()[which]
    session = dp.RouteBSession(case.template_points, case.template_faces, case.target_points,
                               case.target_faces, case.level_settings, **options)
    while not session.finished():
        session.step()
    insp = session.inspect()
    got = json.loads(session.report())["correspondence"]
    want = oracle.summarize(insp["corr_codes"], insp["corr_distances"])
    for key in ("total", "accepted", "rejected_distance", "rejected_normal", "rejected_slope",
                "rejected_masked"):
        assert got[key] == want[key], key
    assert got["distance_p95"] == want["distance_p95"]
    assert got["distance_max"] == want["distance_max"]
    assert got["distance_mean"] == pytest.approx(want["distance_mean"], rel=MEAN_TOL)
    if which == "filters":  # every outcome occurs
        assert min(got[k] for k in ("rejected_distance", "rejected_normal", "rejected_slope",
                                    "rejected_masked")) > 0
