"""The template graph built on the device is the host build, bit for bit.

As the reference's own parity test demands of its device builder
(tests/test_graph_parity.py:22-47): node indices, node positions, binding
nodes and weights, and edges compared with exact equality, on templates
below and above the size where the host's sampling runs in parallel, with
several binding sizes and edge counts.  Every batch and solve prepares its
graphs this way, so the route parity tests cover the device graph too.
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _templates():
    sphere_p, sphere_f = S.uv_sphere(rings=12, segments=16)
    ico_p, ico_f = S.icosphere(5)
    big_p, big_f = S.latlong_ellipsoid(120, 220, (1.0, 0.8, 1.2))[:2]
    return [("uv sphere (coincident poles)", sphere_p, sphere_f, dict(levels=3, nodes_initial=10)),
            ("icosphere 5", ico_p, ico_f, dict(levels=4, nodes_initial=60, max_nodes_per_vertex=6,
                                              edge_neighbours=8)),
            ("lat-long 26k", big_p, big_f, dict(levels=2, nodes_initial=400, max_nodes_per_vertex=8,
                                               edge_neighbours=6))]


@pytest.mark.parametrize("index", range(3))
def test_device_graph_is_the_host_graph(dp, device, index):
    name, points, faces, opts = _templates()[index]
    host = dp.build_template_graph(points, faces, use_device=False, **opts)
    dev = dp.build_template_graph(points, faces, use_device=True, **opts)
    assert np.array_equal(host["normalization"]["center"], dev["normalization"]["center"]), name
    assert host["normalization"]["scale"] == dev["normalization"]["scale"], name
    assert len(host["levels"]) == len(dev["levels"])
    for level, (h, d) in enumerate(zip(host["levels"], dev["levels"])):
        assert np.array_equal(h["node_template_indices"], d["node_template_indices"]), (name, level)
        assert np.array_equal(h["node_positions"], d["node_positions"]), (name, level)
        for key in ("nodes", "weights", "counts"):
            assert np.array_equal(h["bindings"][key], d["bindings"][key]), (name, level, key)
        assert np.array_equal(h["edges"], d["edges"]), (name, level)
