"""The library's host graph build on large templates: above a million
(point, seed) pairs farthest-point sampling walks a grid of the points, below
it scans them in parallel chunks from 20,000 vertices up; the bindings run in
parallel over vertices.  The graph must not depend on the thread count (a
batch prepares its wraps side by side, leaving each wrap one thread).
Checked in subprocesses with different OpenMP thread counts against the
oracle's sequential scan (src/core/sampling.cpp)."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from nricp_b200 import nricp_dp as dp
from nricp_b200 import synthetic as S
points, faces = S.latlong_ellipsoid(120, 220, (1.0, 0.8, 1.2))[:2]
g = dp.build_template_graph(points, faces, levels=2, nodes_initial=300, growth=2,
                            max_nodes_per_vertex=6, edge_neighbours=6)
print(json.dumps([l["node_template_indices"].tolist() for l in g["levels"]] +
                 [int(np.asarray(l["edges"]).sum()) for l in g["levels"]]))
"""


def _run(threads: int):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT)], env=env, check=True,
                         capture_output=True, text=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def test_sampling_does_not_depend_on_the_thread_count(oracle):
    one, seven = _run(1), _run(7)
    assert one == seven
    from nricp_b200 import synthetic as S

    points = S.latlong_ellipsoid(120, 220, (1.0, 0.8, 1.2))[0]
    assert len(points) >= 20000
    center, scale = oracle.normalization(points)
    normalized = (points - center) * scale
    sequential = oracle.farthest_point_seeds(normalized, 600)
    assert one[1] == sequential.tolist()
    assert one[0] == sequential[:300].tolist()
