"""Seeded synthetic wraps for the five benchmark configurations.

No dataset is involved: every template/target pair is generated from a
``numpy.random.default_rng(seed)`` stream, with the shapes, sizes and value
distributions the benchmark configurations name.  Choices the configurations
leave open (RBF width, per-level weights) are fixed here and recorded in each
case's ``meta``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class WrapCase:
    template_points: np.ndarray
    template_faces: np.ndarray
    target_points: np.ndarray
    target_faces: np.ndarray
    level_settings: list[dict]
    options: dict
    meta: dict = field(default_factory=dict)

    def args(self):
        return (self.template_points, self.template_faces, self.target_points,
                self.target_faces, self.level_settings)


# ---------------------------------------------------------------------------
# Meshes
# ---------------------------------------------------------------------------


def uv_sphere(rings: int = 32, segments: int = 64, radius: float = 1.0):
    """The reference tests' UV sphere (tests/test_core_geometry.py:26-55):
    a ring of coincident vertices at each pole, faces wound outwards."""
    ring = np.arange(rings + 1)[:, None]
    seg = np.arange(segments)[None, :]
    theta = np.pi * ring / rings
    phi = 2 * np.pi * seg / segments
    vertices = np.stack(np.broadcast_arrays(radius * np.sin(theta) * np.cos(phi),
                                            radius * np.sin(theta) * np.sin(phi),
                                            radius * np.cos(theta) + 0 * phi), -1).reshape(-1, 3)
    r = np.arange(rings)[:, None]
    s = np.arange(segments)[None, :]
    a = r * segments + s
    b = r * segments + (s + 1) % segments
    c = (r + 1) * segments + (s + 1) % segments
    d = (r + 1) * segments + s
    faces = np.stack([np.stack([a, c, b], -1), np.stack([a, d, c], -1)], 2).reshape(-1, 3)
    return vertices, faces.astype(np.int64)


def bulge(points: np.ndarray, amplitude: float = 0.08) -> np.ndarray:
    """The reference tests' smooth displacement (tests/test_route_a.py:18-26)."""
    result = points.copy()
    radius = np.linalg.norm(points, axis=1, keepdims=True)
    direction = points / np.maximum(radius, 1e-12)
    bump = amplitude * np.exp(-((points[:, 2:3] - 0.3) ** 2) / 0.05)
    result = result + direction * bump
    result[:, 0] += 0.02 * points[:, 2]
    return result


def reference_settings(levels: int, **overrides) -> list[dict]:
    """The reference tests' level settings (tests/test_route_a.py:29-44)."""
    base = {
        "point_to_point": 1.0, "point_to_plane": 2.0, "smoothness": 0.05,
        "anchor": 1e-4, "landmark": 10.0, "robust_kernel": "huber",
        "robust_threshold": 0.0, "max_outer_iterations": 6, "max_inner_iterations": 6,
        "outer_tolerance": 1e-4, "inner_tolerance": 1e-5,
    }
    base.update(overrides)
    return [dict(base) for _ in range(levels)]


def icosphere(subdivisions: int, radius: float = 1.0):
    """Loop-free icosahedron subdivision: 10*4^s + 2 vertices, 20*4^s faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9),
             (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2),
             (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
             (8, 6, 7), (9, 8, 1)]
    v = np.asarray(verts, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.asarray(faces, dtype=np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        unique, inverse = np.unique(key, axis=0, return_inverse=True)
        mids = v[unique[:, 0]] + v[unique[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mids])
        m = inverse.reshape(3, -1).T + base
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                            np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return v * radius, f


def latlong_ellipsoid(rings: int, segments: int, axes=(1.0, 1.0, 1.0)):
    """A lat-long grid on an ellipsoid with one vertex per pole (no coincident
    vertices, no zero-area faces); quads split into two triangles."""
    theta = np.pi * np.arange(1, rings) / rings
    phi = 2 * np.pi * np.arange(segments) / segments
    th, ph = np.meshgrid(theta, phi, indexing="ij")
    body = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).reshape(-1, 3)
    unit = np.concatenate([[[0.0, 0.0, 1.0]], body, [[0.0, 0.0, -1.0]]])
    points = unit * np.asarray(axes, dtype=np.float64)
    north, south = 0, len(unit) - 1
    faces = []
    s = np.arange(segments)
    s1 = (s + 1) % segments
    faces.append(np.stack([np.full(segments, north), 1 + s, 1 + s1], 1))
    for r in range(rings - 2):
        a = 1 + r * segments + s
        b = 1 + r * segments + s1
        c = 1 + (r + 1) * segments + s1
        d = 1 + (r + 1) * segments + s
        faces.append(np.stack([a, d, c], 1))
        faces.append(np.stack([a, c, b], 1))
    last = 1 + (rings - 2) * segments
    faces.append(np.stack([last + s, np.full(segments, south), last + s1], 1))
    return points, np.concatenate(faces).astype(np.int64), unit


def vertex_normals(points: np.ndarray, faces: np.ndarray) -> np.ndarray:
    n = np.zeros_like(points)
    w = np.cross(points[faces[:, 1]] - points[faces[:, 0]], points[faces[:, 2]] - points[faces[:, 0]])
    for k in range(3):
        np.add.at(n, faces[:, k], w)
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300)


def real_spherical_harmonics(unit: np.ndarray, lmax: int) -> np.ndarray:
    """Orthonormal real spherical harmonics Y_lm (l <= lmax) at unit vectors,
    columns ordered (l, m) with m = -l..l; associated Legendre recursion."""
    x, y, z = unit[:, 0], unit[:, 1], unit[:, 2]
    ct = np.clip(z, -1.0, 1.0)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    phi = np.arctan2(y, x)
    P = {}
    P[(0, 0)] = np.ones_like(ct)
    for m in range(1, lmax + 1):
        P[(m, m)] = -(2 * m - 1) * st * P[(m - 1, m - 1)]
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * ct * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * ct * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    columns = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                columns.append(norm * P[(l, 0)])
            elif m > 0:
                columns.append(math.sqrt(2) * norm * P[(l, am)] * np.cos(am * phi))
            else:
                columns.append(math.sqrt(2) * norm * P[(l, am)] * np.sin(am * phi))
    return np.stack(columns, 1)


def random_rotation(rng: np.random.Generator, max_degrees: float) -> np.ndarray:
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    angle = math.radians(rng.uniform(0.0, max_degrees))
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * K @ K


# ---------------------------------------------------------------------------
# The configurations
# ---------------------------------------------------------------------------


def config1(seed: int = 0) -> WrapCase:
    """Plain single wrap: icosphere-4 template onto a spherical-harmonic
    displaced icosphere-5 (c_lm ~ N(0, 0.05), l <= 6), scaled U(0.9, 1.1),
    rotated <= 15 degrees, vertex noise sigma 0.002.  Graph 50/100/200 nodes
    (3 levels, growth 2), k = 4, 8-NN edges; stiffness 100/10/1; "10 GN
    iterations per level" = 10 outer iterations of one inner step each, with
    the outer tolerance at zero so that all ten run; PCG tolerance 1e-6."""
    rng = np.random.default_rng(seed)
    template, tfaces = icosphere(4)
    unit, faces = icosphere(5)
    coefficients = rng.normal(0.0, 0.05, size=49)
    radius = 1.0 + real_spherical_harmonics(unit, 6) @ coefficients
    target = unit * radius[:, None]
    target *= rng.uniform(0.9, 1.1)
    target = target @ random_rotation(rng, 15.0).T
    target += rng.normal(0.0, 0.002, size=target.shape)
    levels = [dict(point_to_point=1.0, point_to_plane=1.0, smoothness=s, anchor=1e-4,
                   landmark=1.0, robust_kernel="huber", robust_threshold=0.0,
                   max_outer_iterations=10, max_inner_iterations=1,
                   outer_tolerance=0.0, inner_tolerance=1e-4) for s in (100.0, 10.0, 1.0)]
    options = dict(graph_levels=3, nodes_initial=50, growth=2, max_nodes_per_vertex=4,
                   edge_neighbours=8, pcg_tolerance=1e-6, pcg_max_iterations=400)
    return WrapCase(template, tfaces, target, faces, levels, options,
                    meta=dict(config=1, seed=seed, template_vertices=len(template),
                              target_triangles=len(faces), nodes=[50, 100, 200]))


def _bumpy_ellipsoid(rng, rings, segments, bumps, axes=(1.0, 0.8, 1.2)):
    points, faces, unit = latlong_ellipsoid(rings, segments, axes)
    normals = vertex_normals(points, faces)
    centres = rng.normal(size=(bumps, 3))
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    amplitude = rng.uniform(0.02, 0.1, size=bumps)
    width = rng.uniform(0.05, 0.2, size=bumps)
    d2 = ((unit[:, None, :] - centres[None]) ** 2).sum(-1)
    height = (amplitude[None] * np.exp(-d2 / (2 * width[None] ** 2))).sum(1)
    return points + normals * height[:, None], faces, unit, (centres, amplitude, width)


def _ellipsoid_grid(vertex_count: int):
    segments = max(8, int(round(math.sqrt(2.0 * vertex_count))))
    rings = max(3, int(round(vertex_count / segments)) + 1)
    return rings, segments


def _target_surface(rng, triangle_count, axes, bumps_spec, rbf_centres=30, rbf_sigma=0.08,
                    rbf_width=0.35, holes=5, hole_radius=0.1, outliers=0.01,
                    anisotropy=(1.0, 1.0, 1.0), ridges=None):
    """The template's shape (same bumps) sampled at `triangle_count` triangles,
    deformed by a smooth Gaussian RBF field (centres on the surface, weights
    N(0, rbf_sigma) per axis, width rbf_width), optionally scaled anisotropically
    and ridged, with `holes` patches removed and a fraction of vertices pushed
    off the surface along the normal by U(0.1, 0.3)."""
    segments = max(8, int(round(math.sqrt(triangle_count))))
    rings = max(3, int(round(triangle_count / (2 * segments))) + 1)
    points, faces, unit = latlong_ellipsoid(rings, segments, axes)
    normals = vertex_normals(points, faces)
    centres, amplitude, width = bumps_spec
    d2 = ((unit[:, None, :] - centres[None]) ** 2).sum(-1)
    points = points + normals * (amplitude[None] * np.exp(-d2 / (2 * width[None] ** 2))).sum(1)[:, None]
    if ridges is not None:
        amp, wavelength = ridges
        points = points + normals * (amp * np.sin(2 * np.pi * points[:, 2] / wavelength))[:, None]
    c_idx = rng.choice(len(points), size=rbf_centres, replace=False)
    c = points[c_idx]
    w = rng.normal(0.0, rbf_sigma, size=(rbf_centres, 3))
    d2 = ((points[:, None, :] - c[None]) ** 2).sum(-1)
    points = points + np.exp(-d2 / (2 * rbf_width ** 2)) @ w
    points = points * np.asarray(anisotropy)
    if holes:
        h = unit[rng.choice(len(unit), size=holes, replace=False)]
        centroid_unit = unit[faces].mean(1)
        centroid_unit /= np.linalg.norm(centroid_unit, axis=1, keepdims=True)
        dist = np.sqrt(((centroid_unit[:, None, :] - h[None]) ** 2).sum(-1)).min(1)
        faces = faces[dist > hole_radius]
    if outliers:
        n = vertex_normals(points, faces)
        pick = rng.choice(len(points), size=max(1, int(outliers * len(points))), replace=False)
        points = points.copy()
        points[pick] += n[pick] * rng.uniform(0.1, 0.3, size=(len(pick), 1))
    return points, faces


def _levels_for(level_count: int, smooth0=100.0, ratio=0.3, outer=10, inner=3):
    return [dict(point_to_point=1.0, point_to_plane=1.0, smoothness=smooth0 * ratio ** l,
                 anchor=1e-4, landmark=1.0, robust_kernel="huber", robust_threshold=0.0,
                 max_outer_iterations=outer, max_inner_iterations=inner,
                 outer_tolerance=1e-3, inner_tolerance=1e-4) for l in range(level_count)]


def config2(seed: int = 0, vertex_count: int = 25_000, triangle_count: int = 400_000,
            nodes_finest: int = 2000, k: int = 6, levels: int = 4) -> WrapCase:
    """Large single wrap: a 25,000-vertex quad-grid ellipsoid (1.0/0.8/1.2)
    with 20 Gaussian bumps onto the same shape deformed by a 30-centre RBF
    field, resampled to 400,000 triangles, 5 holes of radius 0.1, 1 % outliers.
    Graph 250/500/1000/2000 nodes, k = 6."""
    rng = np.random.default_rng(seed)
    rings, segments = _ellipsoid_grid(vertex_count)
    template, tfaces, _, bumps = _bumpy_ellipsoid(rng, rings, segments, 20)
    target, faces = _target_surface(rng, triangle_count, (1.0, 0.8, 1.2), bumps)
    nodes_initial = max(1, nodes_finest // 2 ** (levels - 1))
    options = dict(graph_levels=levels, nodes_initial=nodes_initial, growth=2,
                   max_nodes_per_vertex=k, edge_neighbours=4, pcg_tolerance=1e-6,
                   pcg_max_iterations=400)
    return WrapCase(template, tfaces, target, faces, _levels_for(levels), options,
                    meta=dict(config=2, seed=seed, template_vertices=len(template),
                              target_triangles=len(faces), rbf_width=0.35,
                              nodes=[nodes_initial * 2 ** l for l in range(levels)]))


def config3_specs(seed: int, instances: int = 64):
    """(case seed, template vertices, target triangles, finest nodes) of each
    of config 3's instances, in order."""
    rng = np.random.default_rng(seed)
    sizes = []
    for i in range(instances):
        v = int(round(math.exp(rng.uniform(math.log(5_000), math.log(50_000)))))
        f = int(round(math.exp(rng.uniform(math.log(50_000), math.log(500_000)))))
        sizes.append((seed * 1000 + i + 1, v, f, max(8, v // 15)))
    return sizes


def config3_case(spec):
    """One config-3 instance from its spec (see config3_specs)."""
    case_seed, v, f, nodes = spec
    return config2(seed=case_seed, vertex_count=v, triangle_count=f, nodes_finest=nodes,
                   k=6, levels=4)


def config3(seed: int = 0, instances: int = 64, workers: int = 1):
    """64 uneven wraps: template vertices log-uniform in [5k, 50k], nodes =
    verts/15, target triangles log-uniform in [50k, 500k], generated as in
    config 2.  `workers` > 1 generates the instances in that many spawned
    processes (the same cases, in the same order)."""
    specs = config3_specs(seed, instances)
    if workers <= 1:
        return [config3_case(s) for s in specs]
    import concurrent.futures as cf
    import multiprocessing as mp

    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
        return list(pool.map(config3_case, specs))


def config5(seed: int = 0, vertex_count: int = 100_000, triangle_count: int = 2_000_000,
            nodes_finest: int = 10_000) -> WrapCase:
    """Precision stress: 100k-vertex ellipsoid with 100 bumps onto a 2M-triangle
    target scaled (1, 1, 3) with sinusoidal ridges (amplitude 0.05, wavelength
    0.02).  Graph 10,000 nodes, k = 8."""
    rng = np.random.default_rng(seed)
    rings, segments = _ellipsoid_grid(vertex_count)
    template, tfaces, _, bumps = _bumpy_ellipsoid(rng, rings, segments, 100)
    target, faces = _target_surface(rng, triangle_count, (1.0, 0.8, 1.2), bumps,
                                    anisotropy=(1.0, 1.0, 3.0), ridges=(0.05, 0.02),
                                    holes=0, outliers=0.0)
    levels = 4
    nodes_initial = max(1, nodes_finest // 2 ** (levels - 1))
    options = dict(graph_levels=levels, nodes_initial=nodes_initial, growth=2,
                   max_nodes_per_vertex=8, edge_neighbours=4, pcg_tolerance=1e-6,
                   pcg_max_iterations=1000)
    return WrapCase(template, tfaces, target, faces, _levels_for(levels), options,
                    meta=dict(config=5, seed=seed, template_vertices=len(template),
                              target_triangles=len(faces)))


def small_case(seed: int = 0, rings: int = 14, segments: int = 18, levels: int = 2,
               nodes_initial: int = 40, amplitude: float = 0.09,
               asymmetric: bool = True) -> WrapCase:
    """The reference tests' synthetic wrap (a UV sphere onto its bulge), small
    enough for the CPU oracle to finish in well under a second.

    The reference's fixture is mirror-symmetric, so a vertex on the mirror
    plane is exactly equidistant from two mirrored triangles with different
    closest points -- an exact tie that any two closest-point structures may
    break differently.  `asymmetric` adds seeded noise (sigma 1e-3) to both
    meshes so that exact ties have probability zero."""
    template, faces = uv_sphere(rings, segments)
    target = bulge(template, amplitude)
    if asymmetric:
        rng = np.random.default_rng(seed)
        template = template + rng.normal(0.0, 1e-3, size=template.shape)
        target = target + rng.normal(0.0, 1e-3, size=target.shape)
    return WrapCase(template, faces, target, faces, reference_settings(levels),
                    dict(graph_levels=levels, nodes_initial=nodes_initial, growth=2),
                    meta=dict(config="small", seed=seed, asymmetric=asymmetric))
