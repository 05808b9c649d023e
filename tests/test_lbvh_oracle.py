"""The LBVH restatement in the oracle, pinned without a GPU.

The reference builds its hierarchy on the device only (src/cuda/lbvh.cu), so
there is no CPU output of it to compare against.  This file states the
reference's build a second time, independently of the C restatement, in numpy
and plain Python, line by line from the reference, and checks that the two
agree bit for bit on small inputs:

* FP32 triangle centroids ``(a + b + c) / 3`` evaluated left to right (lbvh.cu:43-45);
* centroid bounds (lbvh.cu:91-124);
* 10-bit quantisation ``min(1023, max(0, (c - lo) * (1023 / (hi - lo))))``
  with a zero scale for an extent of at most 1e-10 (lbvh.cu:152-164);
* Morton interleave z<<2 | y<<1 | x with the expand-bits masks (lbvh.cu:131-143);
* a stable sort by code (the reference's radix sort keeps equal codes in index order);
* Karras' split search with index-XOR prefixes for equal codes (lbvh.cu:171-245).
"""

from __future__ import annotations

import numpy as np
import pytest

from nricp_b200 import synthetic as S


def expand_bits(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32) & np.uint32(0x000003FF)
    v = (v | (v << np.uint32(16))) & np.uint32(0x030000FF)
    v = (v | (v << np.uint32(8))) & np.uint32(0x0300F00F)
    v = (v | (v << np.uint32(4))) & np.uint32(0x030C30C3)
    v = (v | (v << np.uint32(2))) & np.uint32(0x09249249)
    return v


def morton_codes(points64, faces):
    p = np.asarray(points64, dtype=np.float32)
    a, b, c = p[faces[:, 0]], p[faces[:, 1]], p[faces[:, 2]]
    centroids = ((a + b) + c) / np.float32(3.0)
    lo, hi = centroids.min(0), centroids.max(0)
    extent = hi - lo
    scale = np.where(extent > np.float32(1e-10),
                     np.float32(1023.0) / np.where(extent > 0, extent, np.float32(1)),
                     np.float32(0)).astype(np.float32)
    q = np.minimum(np.float32(1023), np.maximum(np.float32(0), (centroids - lo) * scale))
    q = q.astype(np.uint32)  # truncation toward zero, as the float -> unsigned cast
    codes = (expand_bits(q[:, 2]) << np.uint32(2)) | (expand_bits(q[:, 1]) << np.uint32(1)) \
        | expand_bits(q[:, 0])
    return codes.astype(np.uint32), np.concatenate([lo, hi]).astype(np.float32)


def _clz(v: int) -> int:
    return 32 - int(v).bit_length() if v else 32


def karras(codes):
    codes = [int(c) for c in codes]
    n = len(codes)

    def lcp(i, j):
        if j < 0 or j >= n:
            return -1
        if codes[i] == codes[j]:
            return 32 + _clz(i ^ j)
        return _clz(codes[i] ^ codes[j])

    left, right = [], []
    for i in range(n - 1):
        pp, pn = lcp(i, i - 1), lcp(i, i + 1)
        d = 1 if pn > pp else -1
        pmin = min(pp, pn)
        span = 2
        while lcp(i, i + span * d) > pmin:
            span *= 2
        last, step = 0, span // 2
        while step >= 1:
            if lcp(i, i + (last + step) * d) > pmin:
                last += step
            step //= 2
        j = i + last * d
        lo, hi = min(i, j), max(i, j)
        node_prefix = lcp(lo, hi)
        offset, step = 0, hi - lo
        while True:
            step = (step + 1) // 2
            if lcp(lo, lo + offset + step) > node_prefix:
                offset += step
            if step <= 1:
                break
        split = lo + offset
        left.append(lo if lo == split else n + split)
        right.append(hi if split + 1 == hi else n + split + 1)
    return np.array(left, np.int32), np.array(right, np.int32)


def restated(points, faces):
    codes, bounds = morton_codes(points, faces)
    order = np.argsort(codes, kind="stable").astype(np.uint32)
    sorted_codes = codes[order]
    left, right = karras(sorted_codes)
    return dict(codes=sorted_codes, order=order, left=left, right=right, bounds=bounds)


def _meshes():
    rng = np.random.default_rng(0)
    p1, f1 = S.icosphere(3)
    p1 = p1 * rng.uniform(0.5, 2.0, size=3) + rng.normal(size=3)
    base = np.array([[0, 0, 0], [1e-9, 0, 0], [0, 1e-9, 0], [1, 1, 1]], dtype=np.float64)
    dup = np.array([[0, 1, 2]] * 37 + [[0, 1, 3], [1, 2, 3]], dtype=np.int32)
    flat = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], dtype=np.float64)
    flat_faces = np.array([[0, 1, 2], [1, 3, 2]], dtype=np.int32)
    p2, f2 = S.uv_sphere(rings=10, segments=12)
    return {
        "icosphere3": (p1, f1.astype(np.int32)),
        "duplicate_codes": (base, dup),
        "single_triangle": (base, dup[:1]),
        "flat_pair": (flat, flat_faces),      # zero z-extent: zero scale on that axis
        "uv_sphere_poles": (p2, f2.astype(np.int32)),  # coincident pole vertices
    }


@pytest.mark.parametrize("name", list(_meshes()))
def test_c_restatement_matches_the_line_by_line_restatement(oracle, name):
    points, faces = _meshes()[name]
    want = restated(points, faces)
    got = oracle.lbvh_build(points.astype(np.float32), faces)
    for key in ("bounds", "codes", "order", "left", "right"):
        assert np.array_equal(got[key], want[key]), key


def test_known_morton_codes():
    # corners of the unit cube of centroids: the lowest cell is code 0, the
    # highest 2^30 - 1, and x alone occupies the lowest bit of each triple
    assert expand_bits(np.array([1023]))[0] == 0x09249249
    tri = np.array([[0, 0, 0]] * 3 + [[3, 3, 3]] * 3 + [[3, 0, 0]] * 3, dtype=np.float64)
    faces = np.arange(9, dtype=np.int32).reshape(3, 3)
    codes, _ = morton_codes(tri, faces)
    assert list(codes) == [0, 0x3FFFFFFF, 0x09249249]


def test_hierarchy_is_a_binary_tree_over_sorted_leaves(oracle):
    points, faces = S.icosphere(5)
    got = oracle.lbvh_build(points.astype(np.float32), faces.astype(np.int32))
    n = len(faces)
    children = np.concatenate([got["left"], got["right"]])
    # every node but the root (internal node 0 = index n) is a child exactly once
    counts = np.bincount(children, minlength=2 * n - 1)
    assert counts[n] == 0 and np.all(np.delete(counts, n) == 1)
    assert np.all(np.diff(got["codes"].astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(got["order"]), np.arange(n, dtype=np.uint32))
