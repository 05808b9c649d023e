"""Closest points for vertices far from the target (nricp_b200/csrc/lbvh.cu,
`nearest_triangle` and `k_query_queue`).  A template vertex over a hole in
the target is far from every triangle, and its nearest ones are the hole's
rim, all nearly at the same distance, so its seeded walk visits hundreds of
them (replayed on the CPU: 35 of the 544 first queries take more than 256
steps, the longest 357) and its answer rests on many near ties.  The answer
must still be the FP64 brute-force winner (smallest FP64 distance, exact
ties to the lowest triangle index) at every refresh, and the batch must give
the session's bits.

The fixture: a finely tessellated sphere with a wide hole around one pole
as the target, a smaller coarse sphere, rotated off the target's axis, as the
template.
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S

from test_gpu_assembly import _deformed, _graph

pytestmark = pytest.mark.gpu


def _holed_case():
    target, target_faces = S.uv_sphere(120, 240)
    target_faces = target_faces[target[target_faces].mean(1)[:, 2] > -0.8]  # a hole of radius 0.6
    template, template_faces = S.uv_sphere(16, 32)
    # off the target's axis, so that no vertex is equidistant from the whole rim
    rotation = S.random_rotation(np.random.default_rng(5), 20.0)
    template = template @ rotation.T * 0.9 + np.array([0.02, -0.03, 0.01])
    levels = S.reference_settings(2)
    options = dict(graph_levels=2, nodes_initial=40, growth=2)
    return template, template_faces, target, target_faces, levels, options


def test_vertices_over_a_hole_get_the_fp64_closest_points(dp, device, oracle):
    tp, tf, gp, gf, levels, options = _holed_case()
    graph = _graph(dp, S.WrapCase(tp, tf, gp, gf, levels, options), options)
    center, scale = graph["normalization"]["center"][0], graph["normalization"]["scale"]
    tpl = (tp - center) * scale
    tgt = (gp - center) * scale
    session = dp.RouteBSession(tp, tf, gp, gf, levels, **options)
    refreshes = 0
    while not session.finished():
        phase_before = session.inspect()["phase"]
        session.step()
        insp = session.inspect()
        if phase_before not in (0, 1) or insp["phase"] != 2:
            continue  # only right after a refresh do the correspondences match the state
        refreshes += 1
        deformed = _deformed(tpl, graph["levels"][insp["level"]], insp)
        exact = oracle.closest_points(tgt, gf, deformed)
        assert np.abs(exact["distances"] - np.linalg.norm(insp["corr_points"] - deformed, axis=1)).max() < 1e-12
        assert np.abs(exact["points"] - insp["corr_points"]).max() < 1e-12
        assert np.abs(exact["normals"] - insp["corr_normals"]).max() < 1e-9
    assert refreshes >= 4

    batch = dp.WrapBatch([(tp, tf, gp, gf, levels, options)])
    batch.step()
    assert np.array_equal(batch.result(0)["vertices"], session.vertices())
