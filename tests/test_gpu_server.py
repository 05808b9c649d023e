"""Serving with continuous batching (nricp_server_*, nricp_dp.WrapServer).

Requests arrive while others are on the device; each is admitted into a
resident slot when one is free and the memory budget allows, advanced by the
same launches as every other running wrap, and retired when done.  A wrap's
result must not depend on what shares its launches: served results are
compared bit for bit with the same wraps solved alone.
"""

from __future__ import annotations

import json
import time

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _cases():
    return [S.small_case(seed=1, rings=10, segments=14, nodes_initial=30),
            S.config1(3),
            S.small_case(seed=2, rings=16, segments=20, nodes_initial=50, levels=3),
            S.small_case(seed=7, rings=40, segments=60, nodes_initial=300),
            S.config1(4)]


def _same(a, b):
    assert np.array_equal(a["vertices"], b["vertices"])
    assert np.array_equal(a["rotations"], b["rotations"])
    ja, jb = json.loads(a["report"]), json.loads(b["report"])
    assert ja["energy"] == jb["energy"] and ja["levels"] == jb["levels"]
    assert ja["correspondence"] == jb["correspondence"]


# pcg_cluster: 0 latency classes halved by load (the default), -1 always
# halved once, 4 one cluster size for every slot
@pytest.mark.parametrize("route,cluster", [("route_b", 0), ("route_c", 0), ("route_b", -1), ("route_b", 4)])
def test_served_results_equal_the_wraps_solved_alone(dp, device, route, cluster):
    cases = _cases()
    solve = dp.solve_route_b if route == "route_b" else dp.solve_route_c
    alone = [solve(*c.args(), **c.options) for c in cases]
    with dp.WrapServer(max_slots=8, pcg_cluster=cluster) as server:
        ids = [server.submit(*cases[0].args(), route=route, **cases[0].options),
               server.submit(*cases[1].args(), route=route, **cases[1].options)]
        # later arrivals join while the first ones are running
        while server.poll(ids[0])[0] == "waiting":
            time.sleep(0.001)
        for c in cases[2:]:
            ids.append(server.submit(*c.args(), route=route, **c.options))
            time.sleep(0.005)
        served = [server.result(i, timeout=120.0) for i in ids]
        stats = server.stats()
    for a, s in zip(alone, served):
        _same(a, s)
    assert stats["completed"] == len(cases) and stats["failed"] == 0
    assert stats["latency_p99_ms"] >= stats["latency_p50_ms"] > 0.0


def test_large_requests_run_in_their_own_lane(dp, device):
    # a threshold that sends two of the cases to the large lane: every result
    # is still the wrap solved alone
    cases = _cases()
    alone = [dp.solve_route_b(*c.args(), **c.options) for c in cases]
    faces = sorted(len(c.target_faces) for c in cases)
    with dp.WrapServer(max_slots=8, large_face_threshold=faces[-2], large_slots=2) as server:
        ids = [server.submit(*c.args(), **c.options) for c in cases]
        served = [server.result(i, timeout=120.0) for i in ids]
        stats = server.stats()
    for a, s in zip(alone, served):
        _same(a, s)
    assert stats["completed"] == len(cases) and stats["failed"] == 0
    assert stats["latency_p99_ms"] >= stats["latency_p50_ms"] > 0.0


def test_one_slot_serialises_the_requests(dp, device):
    cases = _cases()[:3]
    alone = [dp.solve_route_b(*c.args(), **c.options) for c in cases]
    with dp.WrapServer(max_slots=1) as server:
        ids = [server.submit(*c.args(), **c.options) for c in cases]
        served = [server.result(i, timeout=120.0) for i in ids]
        stats = server.stats()
    for a, s in zip(alone, served):
        _same(a, s)
    assert stats["slots_used"] == 1 and stats["completed"] == 3


def test_a_wrap_beyond_the_memory_budget_fails_cleanly(dp, device):
    case = S.small_case(seed=3)
    with dp.WrapServer(memory_budget_bytes=4096, max_slots=4) as server:
        rid = server.submit(*case.args(), **case.options)
        with pytest.raises(RuntimeError, match="budget"):
            server.result(rid, timeout=60.0)
        assert server.stats()["failed"] == 1


def test_invalid_requests_are_rejected_at_submit(dp, device):
    case = S.small_case(seed=3)
    bad = case.template_points.copy()
    bad[4, 0] = np.nan
    with dp.WrapServer(max_slots=2) as server:
        with pytest.raises(ValueError, match="vertex 4 is not finite"):
            server.submit(bad, case.template_faces, case.target_points, case.target_faces,
                          case.level_settings, **case.options)
        with pytest.raises(ValueError, match="route"):
            server.submit(*case.args(), route="route_q", **case.options)
