"""The solver's inner pieces against the FP64 oracle, at states of a real run.

A session is stepped through a wrap and inspected at solve attempts
(nricp_session_inspect):

* the FP32 Gauss-Newton system the device assembled (diagonal blocks,
  right-hand side, off-diagonal node-pair blocks) and its FP64 energies
  against the oracle's FP64 fused assembly (src/solver/fused_assembly.cpp:
  159-291) at the same state and correspondences;
* the correspondences the seeded closest-point query found right after each
  refresh against the oracle's FP64 closest points at the same deformed
  template -- on a lat-long target whose pole triangles are thin slivers.
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu

DIAG_TOL = 1e-5    # FP32 blocks: max entry error / max entry of the block
RHS_TOL = 1e-6     # right-hand side error / max entry of the node's diagonal block
ENERGY_TOL = 1e-10  # FP64 energies, relative


def _graph(dp, case, opts):
    return dp.build_template_graph(case.template_points, case.template_faces,
                                   levels=opts.get("graph_levels", 4),
                                   nodes_initial=opts.get("nodes_initial", 100),
                                   growth=opts.get("growth", 2),
                                   max_nodes_per_vertex=opts.get("max_nodes_per_vertex", 4),
                                   edge_neighbours=opts.get("edge_neighbours", 4))


def _deformed(tpl, level, insp):
    b = level["bindings"]
    R, T, rest = insp["rotations"], insp["translations"], level["node_positions"]
    out = np.zeros_like(tpl)
    for k in range(b["nodes"].shape[1]):
        nodes = b["nodes"][:, k]
        ok = (k < b["counts"]) & (nodes >= 0)
        nn = np.where(ok, nodes, 0)
        applied = np.einsum("vij,vj->vi", R[nn], tpl - rest[nn]) + rest[nn] + T[nn]
        out += np.where(ok[:, None], applied * b["weights"][:, k:k + 1], 0.0)
    return out


def _fused(oracle, case, graph, insp):
    level = graph["levels"][insp["level"]]
    center, scale = graph["normalization"]["center"][0], graph["normalization"]["scale"]
    tpl = (case.template_points - center) * scale
    b = level["bindings"]
    v = len(tpl)
    nodes = np.full((v, 8), -1, np.int32)
    nodes[:, :b["nodes"].shape[1]] = b["nodes"]
    weights = np.zeros((v, 8))
    weights[:, :b["weights"].shape[1]] = b["weights"]
    ls = case.level_settings[min(insp["level"], len(case.level_settings) - 1)]
    w = [ls["point_to_point"], ls["point_to_plane"], ls["smoothness"], ls["anchor"], ls["landmark"]]
    return oracle.fused_system(tpl, nodes, weights, b["counts"], level["node_positions"],
                               insp["rotations"], insp["translations"], insp["corr_points"],
                               insp["corr_normals"], insp["corr_robust"], insp["corr_codes"] == 0,
                               level["edges"], np.zeros(0, np.int32), np.zeros((0, 3)), w)


def _check_system(insp, ref):
    n = insp["node_count"]
    diag = insp["diag"].astype(np.float64).reshape(n, 36)
    want = ref["diagonal"].reshape(n, 36)
    scale = np.maximum(np.abs(want).max(1), 1e-30)
    assert (np.abs(diag - want).max(1) / scale).max() <= DIAG_TOL
    assert (np.abs(insp["rhs"].astype(np.float64) - ref["rhs"]).max(1) / scale).max() <= RHS_TOL
    mine = {}
    for (a, b), block in zip(insp["off_nodes"], insp["off_blocks"].astype(np.float64)):
        mine[(int(a), int(b))] = mine.get((int(a), int(b)), 0.0) + block
    theirs = {(int(a), int(b)): blk for (a, b), blk in zip(ref["edges"], ref["edge_blocks"])}
    assert set(mine) == set(theirs)
    for key, block in theirs.items():
        assert np.abs(mine[key] - block).max() <= DIAG_TOL * max(np.abs(block).max(), 1e-30), key
    for got, exp in zip(insp["energies"], ref["energies"]):
        assert got == pytest.approx(exp, rel=ENERGY_TOL, abs=1e-300)


@pytest.mark.parametrize("which", ["small", "config1"])
def test_assembled_system_matches_the_fp64_fused_assembly(dp, device, oracle, which):
    case = S.small_case(seed=3) if which == "small" else S.config1(2)
    graph = _graph(dp, case, case.options)
    session = dp.RouteBSession(*case.args(), **case.options)
    checked = set()
    while not session.finished():
        session.step()
        insp = session.inspect()
        if insp["phase"] != 2 or insp["level"] in checked:
            continue
        checked.add(insp["level"])
        _check_system(insp, _fused(oracle, case, graph, insp))
    assert checked == set(range(len(graph["levels"])))


def test_seeded_correspondences_are_the_fp64_closest_points(dp, device, oracle):
    # a lat-long target: the triangles around its poles are thin slivers
    case = S.config2(seed=4, vertex_count=3000, triangle_count=60_000, nodes_finest=200, levels=3)
    opts = dict(case.options, max_nodes_per_vertex=4)
    graph = _graph(dp, case, opts)
    center, scale = graph["normalization"]["center"][0], graph["normalization"]["scale"]
    tpl = (case.template_points - center) * scale
    tgt = (case.target_points - center) * scale
    session = dp.RouteBSession(case.template_points, case.template_faces, case.target_points,
                               case.target_faces, case.level_settings, **opts)
    refreshes = 0
    while not session.finished():
        phase_before = session.inspect()["phase"]
        session.step()
        insp = session.inspect()
        if phase_before not in (0, 1) or insp["phase"] != 2:
            continue  # only right after a refresh do the correspondences match the state
        refreshes += 1
        deformed = _deformed(tpl, graph["levels"][insp["level"]], insp)
        exact = oracle.closest_points(tgt, case.target_faces, deformed)
        assert np.abs(exact["distances"] - np.linalg.norm(insp["corr_points"] - deformed, axis=1)).max() < 1e-12
        assert np.abs(exact["points"] - insp["corr_points"]).max() < 1e-12
        assert np.abs(exact["normals"] - insp["corr_normals"]).max() < 1e-9
    assert refreshes >= 10
