"""The target's ingestion on the device against the host's.

The target is uploaded in the caller's units; the device normalises it and
computes its area-weighted vertex normals (src/core/mesh.cpp:71-88,
183-187).  Both must be bit-identical to the host's computation -- the
normalisation (p - center) * scale with the template's frame, and the
library's host vertex normals of the normalised target, which are themselves
bit-exact with the reference's (tests/test_graph_helpers.py) -- on a large
target with holes and outlier spikes and on a lat-long target whose pole
vertices have hundreds of faces.
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _cases():
    c3 = S.config2(seed=33, vertex_count=3000, triangle_count=300_000, nodes_finest=200, levels=3)
    pole = S.small_case(seed=2)
    t, f = S.uv_sphere(60, 400)  # 400 faces around each pole vertex ring
    pole.target_points, pole.target_faces = S.bulge(t, 0.05), f
    return {"holes_and_spikes": c3, "poles": pole}


@pytest.mark.parametrize("which", ["holes_and_spikes", "poles"])
def test_device_target_is_the_hosts_bit_for_bit(dp, device, which):
    case = _cases()[which]
    session = dp.RouteBSession(*case.args(), **case.options)
    got = session.target()
    graph = dp.build_template_graph(case.template_points, case.template_faces,
                                    levels=case.options.get("graph_levels", 4),
                                    nodes_initial=case.options.get("nodes_initial", 100),
                                    growth=case.options.get("growth", 2))
    center, scale = graph["normalization"]["center"][0], graph["normalization"]["scale"]
    want_points = (np.asarray(case.target_points, np.float64) - center) * scale
    want_normals = dp.vertex_normals(want_points, case.target_faces)
    assert np.array_equal(got["points"], want_points)
    assert np.array_equal(got["normals"], want_normals)
