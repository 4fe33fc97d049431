"""The C++ binned-SAH builder / BVH2 layout / BLAS packing against the
Python restatement in oracle/bvh_ref.py (bit-exact), plus the structural
invariants of the reference's tests/unit/binnedSahBvh.test.ts:71-260 and
tests/unit/bvhAccel.test.ts:27-260."""
import ctypes as C
import math

import numpy as np
import pytest

from mutracer_b200 import abi
from oracle import bvh_ref


def cpp_build(aabbs, bins):
    aabbs = np.ascontiguousarray(aabbs, dtype=np.float32)
    n = aabbs.shape[0]
    cap = max(1, 2 * n - 1)
    bounds = np.zeros((cap, 6), np.float32)
    lf = np.zeros(cap, np.uint32)
    pc = np.zeros(cap, np.uint32)
    pi = np.zeros(max(1, n), np.uint32)
    nc = C.c_uint32()
    assert abi.lib().mtp_build_binned_sah(aabbs.ctypes.data if n else None, n, bins, C.byref(nc), bounds.ctypes.data,
                                          lf.ctypes.data, pc.ctypes.data, pi.ctypes.data) == abi.MT_OK
    m = nc.value
    return m, bounds[:m], lf[:m], pc[:m], pi[:n]


def random_boxes(rng, n, spread=10.0, size=1.0):
    c = rng.uniform(-spread, spread, size=(n, 3))
    h = rng.uniform(0.01, size, size=(n, 3))
    return np.concatenate([c - h, c + h], axis=1).astype(np.float32)


@pytest.mark.parametrize("n,bins,seed", [(1, 8, 0), (2, 8, 1), (7, 8, 2), (64, 8, 3), (257, 16, 4), (600, 8, 5),
                                         (300, 64, 6)])
def test_matches_restatement_bit_exact(n, bins, seed):
    boxes = random_boxes(np.random.default_rng(seed), n)
    got = cpp_build(boxes, bins)
    m, bounds, lf, pc, pi = bvh_ref.build_binned_sah(boxes, bins)
    assert got[0] == m
    assert np.array_equal(got[1].view(np.uint32), bounds[:m].view(np.uint32))
    assert np.array_equal(got[2], lf[:m]) and np.array_equal(got[3], pc[:m]) and np.array_equal(got[4], pi)


def _check_invariants(boxes, m, bounds, lf, pc, pi):
    seen = []
    stack = [0]
    while stack:
        node = stack.pop()
        if pc[node]:
            ids = pi[lf[node]: lf[node] + pc[node]]
            seen.extend(ids.tolist())
            lo, hi = bounds[node, :3], bounds[node, 3:]
            assert (boxes[ids, :3] >= lo).all() and (boxes[ids, 3:] <= hi).all()  # leaf bounds cover prims
            # tight: some primitive touches every face
            assert np.allclose(boxes[ids, :3].min(0), lo) and np.allclose(boxes[ids, 3:].max(0), hi)
        else:
            for ch in (lf[node], lf[node] + 1):
                assert (bounds[ch, :3] >= bounds[node, :3]).all() and (bounds[ch, 3:] <= bounds[node, 3:]).all()
                stack.append(int(ch))
    assert sorted(seen) == list(range(boxes.shape[0]))  # every primitive exactly once


def test_invariants_random():
    rng = np.random.default_rng(9)
    for n in (3, 50, 400):
        boxes = random_boxes(rng, n)
        _check_invariants(boxes, *cpp_build(boxes, 8))


def test_coincident_bounds_and_degenerate_inputs():
    same = np.tile(np.array([[0, 0, 0, 1, 1, 1]], np.float32), (20, 1))
    m, bounds, lf, pc, pi = cpp_build(same, 8)
    assert m == 1 and pc[0] == 20  # identical centroids cannot be split
    flat = np.tile(np.array([[0, 0, 0, 1, 1, 0]], np.float32), (5, 1))
    flat[:, [0, 3]] += np.arange(5, dtype=np.float32)[:, None]
    _check_invariants(flat, *cpp_build(flat, 8))
    m, *_ = cpp_build(np.zeros((0, 6), np.float32), 8)
    assert m == 0


def test_leaf_cost_stop():
    # Two far clusters split; a lone tight cluster of 2 stays a leaf (C_INT = C_TRAV = 1).
    boxes = np.array([[0, 0, 0, 1, 1, 1], [0.1, 0, 0, 1.1, 1, 1]], np.float32)
    m, bounds, lf, pc, pi = cpp_build(boxes, 8)
    assert m == 1
    far = np.concatenate([boxes, boxes + np.float32(100)])
    m, bounds, lf, pc, pi = cpp_build(far, 8)
    assert m >= 3 and pc[0] == 0


def test_blas_packing_matches_layout():
    rng = np.random.default_rng(3)
    nv, nt = 60, 80
    pos = rng.uniform(-1, 1, size=(nv, 3)).astype(np.float32)
    idx = rng.integers(0, nv, size=(nt, 3)).astype(np.uint32)
    vec4 = C.c_uint64()
    depth = C.c_uint32()
    L = abi.lib()
    assert L.mtp_build_blas(pos.ctypes.data, nv, idx.ctypes.data, nt, 8, None, 0, C.byref(vec4), C.byref(depth)) == 0
    buf = np.zeros(vec4.value * 4, np.float32)
    assert L.mtp_build_blas(pos.ctypes.data, nv, idx.ctypes.data, nt, 8, buf.ctypes.data, vec4.value, C.byref(vec4),
                            C.byref(depth)) == 0
    tri = pos[idx]
    boxes = np.concatenate([tri.min(1), tri.max(1)], axis=1)
    m, bounds, lf, pc, pi = bvh_ref.build_binned_sah(boxes, 8)
    order, offsets, vcount, max_depth = bvh_ref.layout_bvh2(m, lf, pc)
    assert vcount == vec4.value and max_depth == depth.value
    words = buf.view(np.int32).reshape(-1, 4)
    f = buf.reshape(-1, 4)
    for node in order:
        o = offsets[node]
        assert np.array_equal(f[o, :3], bounds[node, :3]) and np.array_equal(f[o + 1, :3], bounds[node, 3:])
        if pc[node]:
            assert words[o, 3] == -int(pc[node])  # negative count marks a leaf
            for i in range(int(pc[node])):
                t = int(pi[lf[node] + i])
                assert list(words[o + 2 + i, :3]) == list(idx[t].astype(np.int32)) and words[o + 2 + i, 3] == 0
        else:
            assert words[o, 3] == offsets[int(lf[node]) + 1]  # right child; left child follows at o + 2
            assert offsets[int(lf[node])] == o + 2


def test_instance_record_and_refit_host():
    from mutracer_b200 import scene
    host = scene.make_workload("instanced_spheres", width=16, height=16, params=(24, 3, 4, 64, 1))
    inp = host.refit_inputs()
    rec = host.instances.reshape(-1, 40)
    tl = host.bvh[: host.info.tlas_vec4 * 4].view(np.int32).reshape(-1, 4)
    # walk TLAS leaves: entry = (record slot, BLAS offset, source index, 0)
    stack, seen = [0], []
    while stack:
        node = stack.pop()
        w = tl[node, 3]
        if w >= 0:
            stack += [node + 2, int(w)]
            continue
        for i in range(-w):
            slot, boff, src, zero = tl[node + 2 + i]
            seen.append(src)
            assert zero == 0 and boff == inp["blas_offsets"][src]
            r = rec[slot]
            assert r[:1].view(np.int32)[0] == boff and r[1:2].view(np.int32)[0] == inp["vertex_offsets"][src]
            assert r[2:3].view(np.int32)[0] == inp["materials"][src]
            m = inp["transforms"][src].reshape(4, 4)
            assert np.array_equal(r[20:36], m.reshape(-1).astype(np.float32))
            inv = np.linalg.inv(m.T).T.reshape(-1)
            assert np.allclose(r[4:20], inv, rtol=1e-4, atol=1e-5)
    assert sorted(seen) == list(range(host.info.instances))
    before = host.bvh.copy()
    host.refit_host()  # unchanged transforms: refit reproduces the build exactly
    assert np.array_equal(host.bvh.view(np.uint32), before.view(np.uint32))


def test_js_min_max_rules():
    nz = -0.0
    assert math.copysign(1, bvh_ref.js_min(0.0, nz)) < 0 and math.copysign(1, bvh_ref.js_min(nz, 0.0)) < 0
    assert math.copysign(1, bvh_ref.js_max(0.0, nz)) > 0 and math.copysign(1, bvh_ref.js_max(nz, 0.0)) > 0
    assert math.isnan(bvh_ref.js_min(1.0, float("nan"))) and math.isnan(bvh_ref.js_max(float("nan"), 1.0))
    assert bvh_ref.js_min(2.0, 1.0) == 1.0 and bvh_ref.js_max(2.0, 1.0) == 2.0


def test_signed_zero_bounds_follow_math_min():
    """Bins merge with Math.min / Math.max (-0 below +0 in any order); the
    root box keeps the first strictly smaller value (`<`)."""
    nz = np.float32(-0.0)
    boxes = np.array([[0, 0, 0, 1, 1, 1], [nz, nz, 0, 1, 1, 1], [100, 0, 0, 101, 1, 1], [100, 0, 0, 101, 1, 1]],
                     np.float32)
    got = cpp_build(boxes, 8)
    m, bounds, lf, pc, pi = bvh_ref.build_binned_sah(boxes, 8)
    assert got[0] == m == 3
    assert np.array_equal(got[1].view(np.uint32), bounds[:m].view(np.uint32))
    assert np.array_equal(got[4], pi)
    left = int(lf[0])
    assert np.signbit(bounds[left, 0]) and np.signbit(bounds[left, 1])   # Math.min(+0, -0) = -0
    assert not np.signbit(bounds[0, 0]) and not np.signbit(bounds[0, 1])  # root: first of equal values


def test_blas_skips_nan_and_out_of_range_triangles():
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [np.nan, 0, 0], [5, 5, 5], [6, 5, 5], [5, 6, 5]], np.float32)
    idx = np.array([[0, 1, 2], [0, 3, 2], [4, 5, 6], [0, 1, 99]], np.uint32)
    L = abi.lib()
    vec4, depth = C.c_uint64(), C.c_uint32()
    assert L.mtp_build_blas(pos.ctypes.data, len(pos), idx.ctypes.data, len(idx), 8, None, 0, C.byref(vec4),
                            C.byref(depth)) == 0
    buf = np.zeros(vec4.value * 4, np.float32)
    assert L.mtp_build_blas(pos.ctypes.data, len(pos), idx.ctypes.data, len(idx), 8, buf.ctypes.data, vec4.value,
                            C.byref(vec4), C.byref(depth)) == 0
    words = buf.view(np.int32).reshape(-1, 4)
    leaves = []
    stack = [0]
    while stack:
        o = stack.pop()
        if words[o, 3] >= 0:
            stack += [o + 2, int(words[o, 3])]
        else:
            leaves += [tuple(words[o + 2 + i, :3]) for i in range(-words[o, 3])]
    assert sorted(leaves) == [(0, 1, 2), (4, 5, 6)]


def test_bin_edge_probe_stays_inside_its_ancestors():
    """binnedSahBvh.test.ts:106-131: a centroid on the boundary between two
    root bins is partitioned to the side whose bounds contain it."""
    f = lambda x: float(np.float32(x))
    lo, hi, c = -1000.0, f(1000.3), f(0.14999441802501678)
    boxes = [lo, 0, 0, lo + 0.01, 1, 1, hi - 0.01, 0, 0, hi, 1, 1, c, 0, 0, c, 1, 1]
    for b in range(8):
        x = lo + ((b + 0.5) * (hi - lo)) / 8
        boxes += [x - 0.01, 0, 0, x + 0.01, 1, 1]
    aabbs = np.array(boxes, np.float32).reshape(-1, 6)
    m, bounds, lf, pc, pi = cpp_build(aabbs, 8)
    ref = bvh_ref.build_binned_sah(aabbs, 8)
    assert m == ref[0] and np.array_equal(bounds.view(np.uint32), ref[1][:m].view(np.uint32))

    def contains(node):
        prims = list(pi[lf[node]: lf[node] + pc[node]]) if pc[node] else contains(lf[node]) + contains(lf[node] + 1)
        for p in prims:
            assert (aabbs[p, :3] >= bounds[node, :3]).all() and (aabbs[p, 3:] <= bounds[node, 3:]).all()
        return prims
    assert len(contains(0)) == len(aabbs)
