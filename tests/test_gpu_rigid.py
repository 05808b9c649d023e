"""fit_rigid on the device against the reference's rigid-fit test
(tests/test_core_geometry.py:381-413) and against the published weighted
Kabsch solution (an SVD with the reflection corrected, as
src/core/deformation.cpp:86-139 computes it) in numpy."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _kabsch(source, target, weights):
    w = np.maximum(weights, 0.0)
    cp = (source * w[:, None]).sum(0) / w.sum()
    cq = (target * w[:, None]).sum(0) / w.sum()
    cov = ((source - cp) * w[:, None]).T @ (target - cq)
    u, _, vt = np.linalg.svd(cov)
    d = np.eye(3)
    d[2, 2] = -1.0 if np.linalg.det(vt.T @ u.T) < 0.0 else 1.0
    rotation = vt.T @ d @ u.T
    return rotation, cq - rotation @ cp


def _rotation_y(angle):
    return np.array([[np.cos(angle), 0.0, np.sin(angle)], [0.0, 1.0, 0.0],
                     [-np.sin(angle), 0.0, np.cos(angle)]])


def test_recovers_a_known_transform_and_survives_a_degenerate_support(dp, device):
    rng = np.random.default_rng(5)
    source = rng.normal(size=(20, 3))
    rotation, translation = _rotation_y(0.7), np.array([-0.2, 0.6, 0.1])
    target = source @ rotation.T + translation
    fit = dp.fit_rigid(source, target, np.ones(len(source)))
    assert np.allclose(fit["rotation"][0], rotation, atol=1e-12)
    assert np.allclose(fit["translation"][0], translation, atol=1e-12)
    # points on a line leave the rotation about the line free; the fit must
    # stay finite and still land the points
    line = np.stack([np.linspace(-1.0, 1.0, 6), np.zeros(6), np.zeros(6)], axis=1)
    line_target = line @ rotation.T + translation
    degenerate = dp.fit_rigid(line, line_target, np.ones(len(line)))
    r, t = degenerate["rotation"][0], degenerate["translation"][0]
    assert np.all(np.isfinite(r)) and np.all(np.isfinite(t))
    assert np.abs(line @ r.T + t - line_target).max() < 1e-9


@pytest.mark.parametrize("count", [3, 257, 100_000])
def test_matches_weighted_kabsch_with_noise_and_negative_weights(dp, device, count):
    rng = np.random.default_rng(count)
    source = rng.normal(size=(count, 3)) * [1.0, 2.0, 0.5]
    rotation = _rotation_y(-1.1) @ np.array([[1, 0, 0], [0, np.cos(0.4), -np.sin(0.4)],
                                             [0, np.sin(0.4), np.cos(0.4)]])
    target = source @ rotation.T + [0.3, -1.0, 2.0] + rng.normal(0.0, 0.01, size=source.shape)
    # negative weights count as zero; with three points all must count, or
    # the rotation is not determined
    weights = rng.uniform(0.1, 1.0, size=count) if count < 10 else rng.uniform(-0.2, 1.0, size=count)
    fit = dp.fit_rigid(source, target, weights)
    want_r, want_t = _kabsch(source, target, weights)
    assert np.abs(fit["rotation"][0] - want_r).max() < 1e-10
    assert np.abs(fit["translation"][0] - want_t).max() < 1e-10
    assert abs(np.linalg.det(fit["rotation"][0]) - 1.0) < 1e-12


def test_no_weight_gives_the_identity_and_bad_shapes_raise(dp, device):
    p = np.ones((4, 3))
    fit = dp.fit_rigid(p, p, np.zeros(4))
    assert np.array_equal(fit["rotation"][0], np.eye(3))
    assert np.array_equal(fit["translation"][0], np.zeros(3))
    with pytest.raises(ValueError, match="fit_rigid expects"):
        dp.fit_rigid(p, p[:3], np.ones(4))
