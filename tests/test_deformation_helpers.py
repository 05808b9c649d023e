"""The deformation helpers of the drop-in module on the host -- retraction,
tangent difference, deformation evaluation, level transfer and robust weights
(bindings.cpp:817-856, 1026-1092) -- bit for bit against the reference's own
functions where oracle/_ref is built, and by the properties the reference's
tests hold (test_core_geometry.py:243-412, 415-458;
test_energy_blocks.py:255-278)."""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import nricp_dp as dp

KERNELS = ("none", "huber", "Huber", "geman_mcclure", "geman-mcclure", "GemanMcClure", "cauchy")


def _rotations(rng, n, scale=1.0):
    return dp.retract_deformation(np.broadcast_to(np.eye(3), (n, 3, 3)), np.zeros((n, 3)),
                                  np.zeros((n, 3)), rng.normal(scale=scale, size=6 * n))["rotations"]


def _half_turns():
    """One rotation per branch of the matrix-to-quaternion conversion:
    positive trace, and a half turn about each axis (largest diagonal x, y, z),
    plus rotations a hair short of a half turn."""
    out = [np.eye(3), np.diag([1.0, -1.0, -1.0]), np.diag([-1.0, 1.0, -1.0]), np.diag([-1.0, -1.0, 1.0])]
    for axis in np.eye(3):
        w = axis * (np.pi - 1e-4)
        out.append(dp.retract_deformation(np.eye(3)[None], np.zeros((1, 3)), np.zeros((1, 3)),
                                          np.concatenate([w, np.zeros(3)]))["rotations"][0])
    return np.stack(out)


def test_robust_weights_against_the_reference(reference):
    r = np.concatenate([[-1.0, 0.0, 0.25, 0.2500000001], np.linspace(0.0, 10.0, 61)])
    for kernel in KERNELS:
        for threshold in (0.5, 1e-3, 0.0, -1.0):
            mine = dp.robust_weights(kernel, r, threshold)
            assert np.array_equal(mine, reference.robust_weights(kernel, r, threshold)), (kernel, threshold)


def test_robust_weights_are_monotone_and_bounded():
    squared = np.linspace(0.0, 10.0, 50)
    t = 0.5
    for kernel in ("huber", "geman_mcclure"):
        w = dp.robust_weights(kernel, squared, t)
        assert w[0] == 1.0 and np.all(np.diff(w) <= 0.0) and np.all((w > 0.0) & (w <= 1.0))
    huber = dp.robust_weights("huber", squared, t)
    outside = squared > t * t
    assert np.all(huber[~outside] == 1.0)
    assert np.allclose(huber[outside], t / np.sqrt(squared[outside]), rtol=0, atol=1e-15)
    assert np.all(dp.robust_weights("geman_mcclure", squared, t)[outside] < huber[outside])
    assert np.all(dp.robust_weights("none", squared, t) == 1.0)
    assert np.all(dp.robust_weights("huber", [-3.0], t) == 1.0)


def test_retraction_against_the_reference(reference):
    rng = np.random.default_rng(3)
    n = 64
    r = _rotations(rng, n)
    t = rng.normal(size=(n, 3))
    delta = rng.normal(scale=0.7, size=(n, 6))
    delta[0] = 0.0
    delta[1, :3] = 1e-13      # below the series threshold
    delta[2, :3] = [3.0, -1.0, 0.5]
    mine = dp.retract_deformation(r, t, np.zeros((n, 3)), delta.reshape(-1))
    ref_r, ref_t = reference.retract(r, t, delta.reshape(-1))
    assert np.array_equal(mine["rotations"], ref_r.reshape(n, 3, 3))
    assert np.array_equal(mine["translations"], ref_t)


def test_tangent_difference_against_the_reference(reference):
    rng = np.random.default_rng(4)
    special = _half_turns()
    n = 48
    ra = np.concatenate([_rotations(rng, n - len(special)), np.broadcast_to(np.eye(3), special.shape)])
    rb = np.concatenate([_rotations(rng, n - len(special)), special])
    ta, tb = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    mine = dp.tangent_difference(ra, ta, rb, tb)
    ref = reference.tangent_difference(ra, ta, rb, tb)
    assert mine.shape == (6 * n,)
    assert np.array_equal(mine, ref)
    # the two inputs need not be of one length: the shorter one counts
    assert dp.tangent_difference(ra[:5], ta[:5], rb, tb).shape == (30,)


def test_evaluation_against_the_reference(reference):
    rng = np.random.default_rng(5)
    p = rng.normal(size=(500, 3))
    nodes = p[dp.farthest_point_seeds(p, 40)]
    b = dp.bind_vertices(p, nodes, 4)
    idx = np.array(b["nodes"])
    idx[7, 1] = -1                  # skipped slots, as the reference skips them
    idx[9, 0] = len(nodes) + 3
    counts = np.array(b["counts"])
    counts[11] = 1
    r = _rotations(rng, len(nodes), 0.3)
    t = rng.normal(scale=0.1, size=(len(nodes), 3))
    mine = dp.evaluate_deformation(p, idx, b["weights"], counts, r, t, nodes)
    ref = reference.evaluate_deformation(p, idx, b["weights"], counts, r.reshape(-1, 9), t, nodes)
    assert np.array_equal(mine, ref)


@pytest.mark.parametrize("max_nodes", [1, 2, 4, 6])
def test_transfer_against_the_reference(reference, max_nodes):
    rng = np.random.default_rng(8)
    src = rng.normal(size=(40, 3))
    dst = np.concatenate([rng.normal(size=(120, 3)), src[:5], [[0.0, 0.0, 0.0]]])
    r = _rotations(rng, len(src), 2.0)      # angles up to and past a half turn
    r[:4] = _half_turns()[:4]
    t = rng.normal(size=(len(src), 3))
    mine = dp.transfer_level(src, r, t, dst, max_nodes)
    ref_r, ref_t = reference.transfer_level(src, r, t, dst, max_nodes)
    assert np.array_equal(mine["rotations"], ref_r) and np.array_equal(mine["translations"], ref_t)
    # equidistant sources: the support weights tie
    ring = np.array([[1.0, 0, 0], [-1.0, 0, 0], [0, 1.0, 0], [0, -1.0, 0]])
    mine = dp.transfer_level(ring, r[:4], t[:4], np.zeros((1, 3)), max_nodes)
    ref_r, ref_t = reference.transfer_level(ring, r[:4], t[:4], np.zeros((1, 3)), max_nodes)
    assert np.array_equal(mine["rotations"], ref_r) and np.array_equal(mine["translations"], ref_t)


def test_transfer_reproduces_a_rigid_field():
    rng = np.random.default_rng(9)
    src, dst = rng.normal(size=(30, 3)), rng.normal(size=(100, 3))
    c, s = np.cos(0.25), np.sin(0.25)
    rot = np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])
    shift = np.array([0.1, 0.4, -0.3])
    out = dp.transfer_level(src, np.broadcast_to(rot, (30, 3, 3)), src @ rot.T + shift - src, dst)
    assert np.allclose(out["rotations"], rot, rtol=0, atol=1e-12)
    assert np.allclose(out["translations"], dst @ rot.T + shift - dst, rtol=0, atol=1e-12)


def test_transfer_keeps_opposite_neighbours_turned():
    """Neighbours near +170 and -170 degrees about one axis sit in opposite
    quaternion hemispheres; aligned to the heaviest, their blend stays a large
    rotation instead of collapsing to the identity."""
    rng = np.random.default_rng(10)
    src, dst = rng.normal(size=(40, 3)), rng.normal(size=(150, 3))
    a = np.deg2rad(170.0)
    turn = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
    r = np.stack([turn if i % 2 == 0 else turn.T for i in range(len(src))])
    got = dp.transfer_level(src, r, np.zeros((len(src), 3)), dst)["rotations"]
    angles = np.arccos(np.clip((np.trace(got, axis1=1, axis2=2) - 1.0) / 2.0, -1.0, 1.0))
    assert np.all(np.isfinite(got)) and np.all(angles > np.deg2rad(90.0))


def test_transfer_of_nothing_is_the_identity():
    out = dp.transfer_level(np.zeros((0, 3)), np.zeros((0, 3, 3)), np.zeros((0, 3)), np.ones((3, 3)))
    assert np.array_equal(out["rotations"], np.broadcast_to(np.eye(3), (3, 3, 3)))
    assert np.array_equal(out["translations"], np.zeros((3, 3)))
    out = dp.transfer_level(np.ones((2, 3)), np.broadcast_to(np.eye(3), (2, 3, 3)), np.zeros((2, 3)),
                            np.zeros((0, 3)))
    assert out["rotations"].shape == (0, 3, 3) and out["translations"].shape == (0, 3)


def test_deformation_identity_and_global_rigid():
    rng = np.random.default_rng(6)
    p = rng.normal(size=(300, 3))
    nodes = p[::13]
    b = dp.bind_vertices(p, nodes)
    n = len(nodes)
    same = dp.evaluate_deformation(p, b["nodes"], b["weights"], b["counts"],
                                   np.broadcast_to(np.eye(3), (n, 3, 3)), np.zeros((n, 3)), nodes)
    assert np.allclose(same, p, rtol=0, atol=1e-12)
    c, s = np.cos(0.4), np.sin(0.4)
    rot = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    shift = np.array([0.3, -0.2, 0.7])
    moved = dp.evaluate_deformation(p, b["nodes"], b["weights"], b["counts"],
                                    np.broadcast_to(rot, (n, 3, 3)), nodes @ rot.T + shift - nodes, nodes)
    assert np.allclose(moved, p @ rot.T + shift, rtol=0, atol=1e-12)


def test_retraction_round_trips_with_the_tangent_difference():
    rng = np.random.default_rng(7)
    nodes = rng.normal(size=(20, 3))
    n = len(nodes)
    r = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()
    t = np.zeros((n, 3))
    still = dp.retract_deformation(r, t, nodes, np.zeros(6 * n))
    assert np.array_equal(still["rotations"], r) and np.array_equal(still["translations"], t)
    step = rng.normal(scale=1e-3, size=6 * n)
    moved = dp.retract_deformation(r, t, nodes, step)
    assert np.allclose(dp.tangent_difference(r, t, moved["rotations"], moved["translations"]), step,
                       rtol=0, atol=1e-12)
    one = np.zeros((n, 4), dtype=np.int64)
    one[:, 0] = np.arange(n)
    w = np.zeros((n, 4))
    w[:, 0] = 1.0
    at_nodes = dp.evaluate_deformation(nodes, one, w, np.ones(n, dtype=np.int64), moved["rotations"],
                                       moved["translations"], nodes)
    assert np.allclose(at_nodes, nodes + step.reshape(n, 6)[:, 3:], rtol=0, atol=1e-12)


def test_messages_are_the_references():
    r, t, g = np.broadcast_to(np.eye(3), (2, 3, 3)), np.zeros((2, 3)), np.zeros((2, 3))
    with pytest.raises(ValueError, match=r"^rotations must have shape \(n, 3, 3\)$"):
        dp.retract_deformation(np.zeros((2, 3)), t, g, np.zeros(12))
    with pytest.raises(ValueError, match=r"^translations must have shape \(n, 3\)$"):
        dp.retract_deformation(r, np.zeros((3, 3)), g, np.zeros(12))
    with pytest.raises(ValueError, match=r"^node_positions must have shape \(n, 3\)$"):
        dp.retract_deformation(r, t, np.zeros((2, 2)), np.zeros(12))
    with pytest.raises(ValueError, match=r"^delta must have shape \(6 \* node_count,\)"):
        dp.retract_deformation(r, t, g, np.zeros(11))
    p = np.zeros((3, 3))
    nodes = np.zeros((3, 4), dtype=np.int64)
    w = np.zeros((3, 4))
    c = np.ones(3, dtype=np.int64)
    with pytest.raises(ValueError, match=r"^binding nodes must have shape \(n, 4\)$"):
        dp.evaluate_deformation(p, np.zeros((3, 8), dtype=np.int64), w, c, r, t, g)
    with pytest.raises(ValueError, match=r"^binding weights must have shape \(n, 4\)$"):
        dp.evaluate_deformation(p, nodes, np.zeros((2, 4)), c, r, t, g)
    with pytest.raises(ValueError, match=r"^binding counts must have shape \(n,\)$"):
        dp.evaluate_deformation(p, nodes, w, np.ones(4, dtype=np.int64), r, t, g)
    with pytest.raises(ValueError, match=r"^binding count out of range at vertex 1$"):
        dp.evaluate_deformation(p, nodes, w, np.array([1, 0, 5]), r, t, g)
    with pytest.raises(ValueError, match=r"^points and bindings must have the same length \(2 vs 3\)$"):
        dp.evaluate_deformation(p[:2], nodes, w, c, r, t, g)
    with pytest.raises(ValueError, match=r"^from_nodes must have shape \(n, 3\)$"):
        dp.transfer_level(np.zeros((2, 2)), r, t, g)
    with pytest.raises(ValueError, match=r"^node_positions must have shape \(n, 3\)$"):
        dp.transfer_level(np.zeros((3, 3)), r, t, g)
    with pytest.raises(ValueError, match=r"^to_nodes must have shape \(n, 3\)$"):
        dp.transfer_level(g, r, t, np.zeros(3))
