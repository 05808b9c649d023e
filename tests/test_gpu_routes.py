"""Route B / route C behaviour through the drop-in API, on a B200: the
reference's own route tests (tests/test_route_b.py, tests/test_route_c.py)
restated against this implementation, plus batching.
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _run(dp, name, template, faces, target, levels, nodes_initial, **extra):
    return getattr(dp, name)(template, faces, target, faces, S.reference_settings(levels),
                             graph_levels=levels, nodes_initial=nodes_initial, growth=2, **extra)


def test_the_device_is_reported(dp):
    info = dp.device_info()
    assert set(info) == {"available", "device"}
    assert info["available"], info
    assert "B200" in info["device"] or "cc 10" in info["device"]


def test_route_b_matches_route_a_on_the_symmetric_reference_fixture(dp, device, oracle):
    """tests/test_route_b.py:40-66: both improve, and agree within 5 % of the
    mean error (the fixture is mirror-symmetric, so exact closest-point ties
    may be broken differently; see test_gpu_parity for the tight bar)."""
    template, faces = S.uv_sphere(14, 18)
    truth = S.bulge(template, 0.09)
    device_result = _run(dp, "solve_route_b", template, faces, truth, 2, 80)
    host_result = oracle.solve(template, faces, truth, faces, S.reference_settings(2),
                               graph_levels=2, nodes_initial=80, growth=2)
    dv = np.asarray(device_result["vertices"])
    hv = np.asarray(host_result["vertices"])
    initial = np.linalg.norm(template - truth, axis=1).mean()
    de = np.linalg.norm(dv - truth, axis=1).mean()
    he = np.linalg.norm(hv - truth, axis=1).mean()
    assert de < 0.75 * initial and he < 0.75 * initial
    assert abs(de - he) < 0.05 * max(he, 1e-9), (de, he)


def test_the_session_steps_to_the_same_fit_as_the_batch_call(dp, device):
    template, faces = S.uv_sphere(10, 14)
    truth = S.bulge(template, 0.07)
    settings = S.reference_settings(2)
    args = dict(graph_levels=2, nodes_initial=50, growth=2)
    session = dp.RouteBSession(template, faces, truth, faces, settings, **args)
    steps, first_error = 0, None
    while not session.finished():
        progress = session.step()
        steps += 1
        assert progress["level"] < 2
        if steps == 3:
            partial = session.vertices()
            assert partial.shape == template.shape and np.all(np.isfinite(partial))
            first_error = float(np.linalg.norm(partial - truth, axis=1).mean())
        assert steps < 5000
    stepped = np.asarray(session.result()["vertices"])
    batch = np.asarray(dp.solve_route_b(template, faces, truth, faces, settings, **args)["vertices"])
    # the schedule is deterministic: stepping by hand is bit-identical
    assert np.array_equal(stepped, batch)
    final_error = float(np.linalg.norm(stepped - truth, axis=1).mean())
    assert first_error is not None and first_error > final_error
    assert final_error < np.linalg.norm(template - truth, axis=1).mean()


def test_route_b_repeats_bit_for_bit_and_reports_its_trace(dp, device):
    template, faces = S.uv_sphere(12, 16)
    truth = S.bulge(template, 0.08)
    first = _run(dp, "solve_route_b", template, faces, truth, 2, 60)
    second = _run(dp, "solve_route_b", template, faces, truth, 2, 60)
    # fixed-order reductions, no float atomics: runs are identical
    assert np.array_equal(first["vertices"], second["vertices"])
    report = json.loads(first["report"])
    assert report["route"] == "route_b" and report["precision"] == "float"
    assert report["version"] == dp.__version__
    assert [l["nodes"] for l in report["levels"]] == list(first["level_nodes"])
    for level in report["levels"]:
        assert level["energy_end"] <= level["energy_start"]
    for key in ("rejected_normal", "rejected_slope", "rejected_masked"):
        assert key in report["correspondence"]


def test_route_c_identity_fixed_point(dp, device):
    """tests/test_route_c.py:44-61."""
    template, faces = S.uv_sphere(12, 16)
    result = _run(dp, "solve_route_c", template, faces, template, 2, 60)
    rot = np.asarray(result["rotations"]).reshape(-1, 3, 3)
    assert np.abs(rot - np.eye(3)[None]).max() < 1e-4
    assert np.abs(np.asarray(result["translations"])).max() < 1e-4
    assert np.abs(np.asarray(result["vertices"]) - template).max() < 1e-4


def test_route_c_rotations_are_proper(dp, device):
    """tests/test_route_c.py:64-84."""
    template, faces = S.uv_sphere(12, 16)
    truth = S.bulge(template, 0.08)
    rot = np.asarray(_run(dp, "solve_route_c", template, faces, truth, 2, 60)["rotations"]).reshape(-1, 3, 3)
    gram = np.einsum("nij,nkj->nik", rot, rot)
    assert np.abs(gram - np.eye(3)[None]).max() < 1e-6
    det = np.linalg.det(rot)
    assert det.min() > 0.999999 and det.max() < 1.000001


def test_route_c_is_within_ten_percent_of_route_a(dp, device, oracle):
    """tests/test_route_c.py:127-151."""
    template, faces = S.uv_sphere(14, 18)
    truth = S.bulge(template, 0.09)
    native = _run(dp, "solve_route_c", template, faces, truth, 2, 80)
    reference = oracle.solve(template, faces, truth, faces, S.reference_settings(2),
                             graph_levels=2, nodes_initial=80, growth=2)
    ne = np.linalg.norm(np.asarray(native["vertices"]) - truth, axis=1).mean()
    re = np.linalg.norm(np.asarray(reference["vertices"]) - truth, axis=1).mean()
    initial = np.linalg.norm(template - truth, axis=1).mean()
    assert ne < 0.75 * initial and ne < 1.10 * re, (ne, re)


def test_a_batch_gives_each_wrap_the_result_it_gets_alone(dp, device):
    """Batched wraps of uneven sizes share every launch; each one's result must
    be what it gets alone (fixed-order reductions: bit for bit)."""
    cases = [S.small_case(seed=1, rings=10, segments=14, nodes_initial=30),
             S.config1(3),
             S.small_case(seed=2, rings=16, segments=20, nodes_initial=50, levels=3)]
    alone = [dp.solve_route_b(*c.args(), **c.options) for c in cases]
    mixed = dp.solve_batch([(*c.args(), c.options) for c in cases])
    for a, m in zip(alone, mixed):
        assert np.array_equal(a["vertices"], m["vertices"])
        assert a["report"].split('"setup_seconds"')[0] == m["report"].split('"setup_seconds"')[0]
        ja, jm = json.loads(a["report"]), json.loads(m["report"])
        assert ja["energy"] == jm["energy"] and ja["levels"] == jm["levels"]


@pytest.mark.parametrize("route", ["route_b", "route_c"])
def test_every_solve_cluster_size_gives_the_same_bits(dp, device, route):
    """The linear solve's cluster size (1 to 16 CTAs per wrap) only decides
    which CTA computes which 4-node segment, never the order of a sum: the
    wraps' results must be bit-identical for every size, alone and batched."""
    cases = [S.small_case(seed=4, nodes_initial=40),           # 40 / 80 nodes: idle CTAs at 16
             S.config1(5),                                     # 50 / 100 / 200 nodes
             S.small_case(seed=7, rings=40, segments=60, nodes_initial=300)]  # 300 / 600 nodes
    tuples = [(*c.args(), c.options) for c in cases]
    reference = None
    for cluster in (1, 2, 4, 8, 16, 0, -1):
        batch = dp.WrapBatch(tuples, route=route)
        effective = batch.tune(cluster)
        assert effective == cluster if cluster > 0 else effective >= 1
        batch.run()
        got = [batch.result(i) for i in range(len(cases))]
        if reference is None:
            reference = got
            continue
        for a, b in zip(reference, got):
            assert np.array_equal(a["vertices"], b["vertices"]), cluster
            assert np.array_equal(a["rotations"], b["rotations"]), cluster
            ja, jb = json.loads(a["report"]), json.loads(b["report"])
            assert ja["energy"] == jb["energy"] and ja["levels"] == jb["levels"], cluster


def test_solve_cluster_size_is_validated(dp, device):
    case = S.small_case(seed=6)
    batch = dp.WrapBatch([(*case.args(), case.options)])
    with pytest.raises(ValueError, match="power of two"):
        batch.tune(3)
    assert batch.tune(0) >= 1


def test_masks_and_landmarks_reach_the_device(dp, device, oracle):
    case = S.small_case(seed=3)
    mask = np.ones(len(case.template_points), dtype=np.int64)
    mask[:20] = 0
    lm = np.array([5, 77, 150])
    targets = case.target_points[lm] + 0.01
    kwargs = dict(case.options, mask=mask, landmark_indices=lm, landmark_targets=targets)
    gpu = dp.solve_route_b(*case.args(), **kwargs)
    ref = oracle.solve(*case.args(), **kwargs)
    rg, rr = json.loads(gpu["report"]), json.loads(ref["report"])
    assert rg["correspondence"]["rejected_masked"] == rr["correspondence"]["rejected_masked"] == 20
    diag = np.linalg.norm(case.target_points.max(0) - case.target_points.min(0))
    err = np.linalg.norm(gpu["vertices"] - ref["vertices"], axis=1).max() / diag
    assert err <= 1e-4, err
    assert abs(rg["energy"]["landmark"] - rr["energy"]["landmark"]) <= 1e-5 * rr["energy"]["total"]


def test_filters_and_robust_kernels_match_route_a(dp, device, oracle):
    case = S.small_case(seed=4)
    for kernel in ("huber", "geman_mcclure"):
        levels = [dict(l, robust_kernel=kernel, robust_threshold=0.01) for l in case.level_settings]
        kwargs = dict(case.options, distance_threshold=0.2, min_normal_cosine=0.2, min_slope=0.05)
        gpu = dp.solve_route_b(case.template_points, case.template_faces, case.target_points,
                               case.target_faces, levels, **kwargs)
        ref = oracle.solve(case.template_points, case.template_faces, case.target_points,
                           case.target_faces, levels, **kwargs)
        rg, rr = json.loads(gpu["report"]), json.loads(ref["report"])
        for key in ("accepted", "rejected_distance", "rejected_normal", "rejected_slope"):
            assert rg["correspondence"][key] == rr["correspondence"][key], (kernel, key)
        diag = np.linalg.norm(case.target_points.max(0) - case.target_points.min(0))
        err = np.linalg.norm(gpu["vertices"] - ref["vertices"], axis=1).max() / diag
        assert err <= 1e-4, (kernel, err)


def test_k8_bindings_and_8nn_edges(dp, device, oracle):
    case = S.small_case(seed=5)
    kwargs = dict(case.options, max_nodes_per_vertex=8, edge_neighbours=8)
    gpu = dp.solve_route_b(*case.args(), **kwargs)
    ref = oracle.solve(*case.args(), **kwargs)
    diag = np.linalg.norm(case.target_points.max(0) - case.target_points.min(0))
    err = np.linalg.norm(gpu["vertices"] - ref["vertices"], axis=1).max() / diag
    assert err <= 1e-4, err
