"""The hierarchy export that allocates nothing (nricp_lbvh_export_static).

It takes device buffers and keeps its intermediates in one static device
array shared by every call, so two calls in a row must each give exactly what
the allocating export (nricp_lbvh_export) gives for the same mesh -- the
second call must not see anything the first one left behind.  This file is
collected last so that it also runs after every other test in one process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from nricp_b200 import synthetic as S

pytestmark = pytest.mark.gpu

STATIC_FACE_LIMIT = 262144


def _host_export(points, faces):
    from nricp_b200._lib import check, load

    n = len(faces)
    out = dict(codes=np.zeros(n, np.uint32), order=np.zeros(n, np.uint32),
               left=np.zeros(max(1, n - 1), np.int32), right=np.zeros(max(1, n - 1), np.int32),
               bounds=np.zeros(6, np.float32))
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    check(load().nricp_lbvh_export(P(points, C.c_double), len(points), P(faces, C.c_int32), n,
                                   P(out["codes"], C.c_uint32), P(out["order"], C.c_uint32),
                                   P(out["left"], C.c_int32), P(out["right"], C.c_int32),
                                   P(out["bounds"], C.c_float)))
    out["left"], out["right"] = out["left"][: n - 1], out["right"][: n - 1]
    return out


def _device_buffers(points, faces):
    import torch

    n = len(faces)
    return dict(points=torch.from_numpy(points).cuda(), faces=torch.from_numpy(faces).cuda(),
                codes=torch.empty(n, dtype=torch.int32, device="cuda"),
                order=torch.empty(n, dtype=torch.int32, device="cuda"),
                left=torch.empty(max(1, n - 1), dtype=torch.int32, device="cuda"),
                right=torch.empty(max(1, n - 1), dtype=torch.int32, device="cuda"),
                bounds=torch.empty(6, dtype=torch.float32, device="cuda"))


def _static_call(buffers, vertex_count, face_count):
    import torch

    from nricp_b200._lib import load

    torch.cuda.synchronize()
    b = buffers
    return load().nricp_lbvh_export_static(
        b["points"].data_ptr(), vertex_count, b["faces"].data_ptr(), face_count,
        b["codes"].data_ptr(), b["order"].data_ptr(), b["left"].data_ptr(),
        b["right"].data_ptr(), b["bounds"].data_ptr(), torch.cuda.current_stream().cuda_stream)


def _read(buffers, n):
    return dict(codes=buffers["codes"].cpu().numpy().view(np.uint32),
                order=buffers["order"].cpu().numpy().view(np.uint32),
                left=buffers["left"].cpu().numpy()[: n - 1],
                right=buffers["right"].cpu().numpy()[: n - 1],
                bounds=buffers["bounds"].cpu().numpy())


def _mesh(subdivisions, seed):
    points, faces = S.icosphere(subdivisions)
    rng = np.random.default_rng(seed)
    points = points * rng.uniform(0.5, 2.0, size=3) + rng.normal(size=3)
    return np.ascontiguousarray(points, np.float64), np.ascontiguousarray(faces, np.int32)


def test_static_export_matches_the_allocating_export_on_two_calls(device):
    import torch

    from nricp_b200._abi import OK

    # a large mesh first, then a smaller one over the same static array
    meshes = [_mesh(5, 11), _mesh(3, 12)]
    for call, (points, faces) in enumerate(meshes):
        n = len(faces)
        buffers = _device_buffers(points, faces)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status = _static_call(buffers, len(points), n)
        free_after = torch.cuda.mem_get_info()[0]
        assert status == OK, f"call {call}: status {status}"
        if call == 1:
            # by the second call everything is loaded: no device memory moves
            assert free_after == free_before
        got = _read(buffers, n)
        want = _host_export(points, faces)
        for key in ("codes", "order", "left", "right", "bounds"):
            assert np.array_equal(got[key], want[key]), f"call {call}: {key}"


def test_static_export_rejects_meshes_beyond_its_limit(device):
    from nricp_b200._abi import ERR_CAPACITY
    from nricp_b200._lib import load

    points, faces = _mesh(1, 3)
    buffers = _device_buffers(points, faces)
    # the size check comes before any device work, so the small buffers are never read
    status = _static_call(buffers, len(points), STATIC_FACE_LIMIT + 1)
    assert status == ERR_CAPACITY
    message = load().nricp_last_error().decode()
    assert "262144" in message and "nricp_lbvh_export" in message


def _grid_at_the_limit(seed):
    """A wavy 513 x 257 vertex grid: 2 * 512 * 256 = 262,144 triangles, the
    static array's limit, so its largest layout (and the radix counts of every
    sort tile) is exercised."""
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(513), np.arange(257), indexing="ij")
    x, y = ii / 512.0, jj / 256.0 * 0.5
    z = 0.1 * np.sin(7.0 * x) * np.cos(11.0 * y) + rng.normal(scale=1e-3, size=x.shape)
    points = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    v = (ii[:-1, :-1] * 257 + jj[:-1, :-1]).reshape(-1)
    faces = np.concatenate([np.stack([v, v + 257, v + 1], 1), np.stack([v + 1, v + 257, v + 258], 1)])
    assert len(faces) == STATIC_FACE_LIMIT
    return np.ascontiguousarray(points, np.float64), np.ascontiguousarray(faces, np.int32)


def test_static_export_at_exactly_its_limit(device):
    from nricp_b200._abi import OK

    points, faces = _grid_at_the_limit(5)
    buffers = _device_buffers(points, faces)
    status = _static_call(buffers, len(points), len(faces))
    assert status == OK, f"status {status}"
    got = _read(buffers, len(faces))
    want = _host_export(points, faces)
    for key in ("codes", "order", "left", "right", "bounds"):
        assert np.array_equal(got[key], want[key]), key
