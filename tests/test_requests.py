"""Request preparation on the host (no device): the descriptor a batch
passes through the C ABI, built one by one or on threads, and the face-array
conversion, which follows the reference's forcecast to int64
(src/python/bindings.cpp:40-61) before narrowing to the ABI's int32."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from nricp_b200 import _abi
from nricp_b200 import synthetic as S
from nricp_b200.nricp_dp import _descs


def test_face_arrays_convert_like_a_forcecast():
    faces = np.array([[0, 1, 2], [2, 1, 3]])
    for dtype in (np.int32, np.int64, np.uint16, np.float64):
        out = _abi._faces(faces.astype(dtype), "faces")
        assert out.dtype == np.int32 and out.flags["C_CONTIGUOUS"]
        assert np.array_equal(out, faces)
    # floats truncate toward zero, as a cast to int64 does
    assert np.array_equal(_abi._faces(np.array([[0.9, 1.5, 2.99]]), "faces"), [[0, 1, 2]])
    # an int32 C-contiguous array is used as it is, without a copy
    same = faces.astype(np.int32)
    assert _abi._faces(same, "faces") is same
    # a non-contiguous int32 view becomes contiguous
    view = np.zeros((4, 6), np.int32)[:, ::2]
    assert _abi._faces(view, "faces").flags["C_CONTIGUOUS"]
    with pytest.raises(ValueError, match="must have shape"):
        _abi._faces(np.zeros((3, 4), np.int32), "faces")


def _fields(desc):
    d = desc.struct
    out = {}
    for name, ctype in d._fields_:
        value = getattr(d, name)
        if isinstance(value, (int, float)):
            out[name] = value
    arrays = {k: getattr(desc, k) for k in ("template_points", "template_faces", "target_points",
                                             "target_faces")}
    return out, arrays


def test_descriptors_built_on_threads_equal_the_serial_ones():
    cases = [S.small_case(seed=s, rings=8 + s, segments=10 + s) for s in range(10)]
    tuples = [(*c.args(), c.options) for c in cases]
    threaded = _descs(tuples, "route_b")
    serial = [_abi.Desc(*t[:5], route=_abi.ROUTE_B, **t[5]) for t in tuples]
    assert len(threaded) == len(serial) == 10
    for a, b in zip(threaded, serial):
        fa, aa = _fields(a)
        fb, ab = _fields(b)
        assert fa == fb
        for k in aa:
            assert aa[k].dtype == ab[k].dtype and np.array_equal(aa[k], ab[k]), k
        # the struct points into the descriptor's own arrays
        assert C.addressof(a.target_faces.ctypes.data_as(C.POINTER(C.c_int32)).contents) == \
            C.addressof(a.struct.target_faces.contents)


def test_mask_and_landmark_validation_follow_the_reference():
    from nricp_b200 import nricp_dp as dp

    assert dp.validate_mask([1, 0, 2, 0], 4) == 2
    assert dp.validate_mask([], 7) == 0
    with pytest.raises(ValueError, match="invalid mask: mask has 3 entries but the template has 4 vertices"):
        dp.validate_mask([1, 1, 1], 4)
    with pytest.raises(ValueError, match="mask excludes every vertex"):
        dp.validate_mask([0, 0], 2)
    dp.validate_landmarks([0, 3], [[0, 0, 0], [1, 1, 1]], 4)
    with pytest.raises(ValueError, match=r"invalid landmarks: landmark 1 points at template vertex 9 but the "
                                         r"template has 4 vertices; landmark 2 has a non-finite target; "
                                         r"landmark 3 marks template vertex 0 twice"):
        dp.validate_landmarks([0, 9, 1, 0], [[0, 0, 0], [1, 1, 1], [np.nan, 0, 0], [2, 2, 2]], 4)
    with pytest.raises(ValueError, match="landmark targets must have shape"):
        dp.validate_landmarks([0, 1], [[0, 0, 0]], 4)
