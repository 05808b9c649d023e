"""The FP64 route-C restatement (oracle/nricp_oracle.c) against the reference's
own route-C expectations, on the CPU.

The reference has no CPU route C: its route C is device code
(src/cuda/local_global.cu:188-302).  Its test file tests/test_route_c.py holds
the route to known answers that do not depend on how the device rounds, and
the restatement must meet the same ones:

* identity fixed point: target == template leaves every rotation at the
  identity and every translation and vertex in place (test_route_c.py:44-61);
* every fitted rotation is proper (test_route_c.py:64-83);
* a translated target is carried by the translations (test_route_c.py:86-123);
* route C lands within 10 % of route A's mean fit error and well below the
  start (test_route_c.py:126-148), with route A being the reference's own
  compiled route where it was built here.

The GPU test tests/test_gpu_reference_anchors.py compares the restatement with
the reference's compiled route C itself.
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S
from oracle.oracle import ROUTE_A, ROUTE_C


def _run(oracle, route, template, faces, target, levels, nodes_initial):
    return oracle.solve(template, faces, target, faces, S.reference_settings(levels), route=route,
                        graph_levels=levels, nodes_initial=nodes_initial, growth=2)


def _rotations(result):
    return np.asarray(result["rotations"], dtype=np.float64).reshape(-1, 3, 3)


def test_identity_is_the_fixed_point(oracle):
    template, faces = S.uv_sphere(12, 16)
    result = _run(oracle, ROUTE_C, template, faces, template, 2, 60)
    assert np.abs(_rotations(result) - np.eye(3)[None]).max() < 1e-4
    assert np.abs(np.asarray(result["translations"])).max() < 1e-4
    assert np.abs(np.asarray(result["vertices"]) - template).max() < 1e-4


def test_fitted_rotations_are_proper(oracle):
    template, faces = S.uv_sphere(12, 16)
    rotations = _rotations(_run(oracle, ROUTE_C, template, faces, S.bulge(template, 0.08), 2, 60))
    gram = np.einsum("nij,nkj->nik", rotations, rotations)
    assert np.all(np.isfinite(rotations))
    assert np.abs(gram - np.eye(3)[None]).max() < 1e-4
    det = np.linalg.det(rotations)
    assert det.min() > 0.999 and det.max() < 1.001


def test_a_translated_target_is_carried_by_the_translations(oracle):
    base, faces = S.uv_sphere(14, 18)
    template = base * np.array([1.4, 1.0, 0.75])
    offset = np.array([0.0, 0.05, 0.0])
    result = _run(oracle, ROUTE_C, template, faces, template + offset, 2, 80)
    fitted = np.asarray(result["vertices"])
    moved = fitted.mean(0) - template.mean(0)
    assert np.linalg.norm(moved) > 0.15 * np.linalg.norm(offset)
    assert moved @ offset / np.linalg.norm(moved) / np.linalg.norm(offset) > 0.99
    before = np.sort(np.linalg.eigvalsh(np.cov((template - template.mean(0)).T)))
    after = np.sort(np.linalg.eigvalsh(np.cov((fitted - fitted.mean(0)).T)))
    assert np.all(after / before > 0.95) and np.all(after / before < 1.02)
    r = _rotations(result)
    angles = np.degrees(np.arccos(np.clip((np.trace(r, axis1=1, axis2=2) - 1.0) / 2.0, -1.0, 1.0)))
    assert np.median(angles) < 6.0


def test_route_c_reaches_route_a_fit_quality(oracle, reference):
    template, faces = S.uv_sphere(14, 18)
    truth = S.bulge(template, 0.09)
    route_c = _run(oracle, ROUTE_C, template, faces, truth, 2, 80)
    route_a = _run(reference, ROUTE_A, template, faces, truth, 2, 80)
    error_c = np.linalg.norm(np.asarray(route_c["vertices"]) - truth, axis=1).mean()
    error_a = np.linalg.norm(np.asarray(route_a["vertices"]) - truth, axis=1).mean()
    start = np.linalg.norm(template - truth, axis=1).mean()
    assert error_c < 0.75 * start
    assert error_c < 1.10 * error_a, (error_c, error_a)
