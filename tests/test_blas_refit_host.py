"""Host refitBLAS (mtp_refit_blas, the C++ restatement) against the Python
restatement in oracle/bvh_ref.py, and the properties of bvhAccel.ts:800-870:
an unchanged mesh refits to its build boxes, deformation moves every box
onto its leaves' vertices, non-finite and out-of-range vertices are skipped,
malformed buffers are rejected."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, blas
from oracle import bvh_ref


def host_refit(buf, pos):
    out = np.array(buf, np.float32)
    p = np.ascontiguousarray(pos, np.float32)
    area = C.c_double()
    st = abi.lib().mtp_refit_blas(out.ctypes.data, out.size // 4, p.ctypes.data if p.size else None, len(p),
                                  C.byref(area))
    return st, out, area.value


def mesh(seed, side=12):
    pos, idx = blas.terrain_mesh(side, side, seed=seed)
    pos += np.float32(0.25)                   # keep coordinates away from signed zeros
    return pos, idx


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_matches_python_restatement(seed):
    pos, idx = mesh(seed)
    buf, _ = blas.host_build(pos, idx)
    rng = np.random.default_rng(seed)
    moved = (pos + rng.normal(0, 0.2, pos.shape)).astype(np.float32)
    moved[rng.integers(0, len(moved), 5), 1] = np.nan
    st, got, area = host_refit(buf, moved)
    assert st == abi.MT_OK
    want, want_area = bvh_ref.refit_blas(buf, moved)
    assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
    assert area == want_area


def test_unchanged_mesh_keeps_build_boxes():
    pos, idx = mesh(4, side=30)
    buf, _ = blas.host_build(pos, idx)
    st, got, _ = host_refit(buf, pos)
    assert st == abi.MT_OK and got.tobytes() == buf.tobytes()


def test_boxes_follow_deformation():
    pos, idx = mesh(5, side=20)
    buf, _ = blas.host_build(pos, idx)
    moved = (pos * np.float32(3) + np.float32(7)).astype(np.float32)
    st, got, _ = host_refit(buf, moved)
    f = got.reshape(-1, 4)
    assert np.array_equal(f[0, :3], moved.min(0)) and np.array_equal(f[1, :3], moved.max(0))


def test_rejects_malformed_buffers():
    pos, idx = mesh(6)
    buf, _ = blas.host_build(pos, idx)
    bad = buf.copy().reshape(-1, 4)
    bad.view(np.int32)[0, 3] = len(bad) + 5     # right child past the end
    assert host_refit(bad.reshape(-1), pos)[0] == abi.MT_ERROR_INVALID_ARGUMENT
    bad = buf.copy().reshape(-1, 4)
    bad.view(np.int32)[0, 3] = 1                # right child before the left one
    assert host_refit(bad.reshape(-1), pos)[0] == abi.MT_ERROR_INVALID_ARGUMENT


def test_device_entry_points_validate_on_host():
    L = abi.lib()
    assert L.mtc_blas_refit_plan_bytes(0) == 0 and L.mtc_blas_refit_plan_bytes(100) > 0
    info = abi.BlasRefitPlanInfo()
    info.struct_size = 4
    assert L.mtc_blas_refit_prepare(C.c_void_p(256), 100, C.c_void_p(1 << 20), 1 << 30, C.byref(info), None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    info.struct_size = C.sizeof(info)
    assert L.mtc_blas_refit_prepare(C.c_void_p(256), 100, C.c_void_p(1 << 20), 16, C.byref(info), None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_refit_blas(C.c_void_p(256), 100, C.c_void_p(1 << 20), 0, None, 0, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_refit_blas(C.c_void_p(256), 100, C.c_void_p((1 << 20) + 8), 3, None, 0, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT


def test_refit_moves_parent_bounds():
    """bvhAccel.test.ts:181-197: moving one vertex to x = 8 moves the root's
    max x to 8."""
    pos = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 2, 0, 0, 3, 0, 0, 2, 1, 0], np.float32).reshape(-1, 3)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    buf, _ = blas.host_build(pos, idx)
    moved = pos.copy()
    moved[4, 0] = 8
    st, got, _ = host_refit(buf, moved)
    assert st == abi.MT_OK and got[4] == 8


def uv_sphere(width_segments, height_segments, radius=1.0):
    pos = []
    for y in range(height_segments + 1):
        v = y / height_segments
        for x in range(width_segments + 1):
            u = x / width_segments
            pos.append([-radius * np.cos(u * 2 * np.pi) * np.sin(v * np.pi), radius * np.cos(v * np.pi),
                        radius * np.sin(u * 2 * np.pi) * np.sin(v * np.pi)])
    idx = []
    w = width_segments + 1
    for y in range(height_segments):
        for x in range(width_segments):
            a, b, c, d = y * w + x + 1, y * w + x, (y + 1) * w + x, (y + 1) * w + x + 1
            if y != 0:
                idx.append([a, b, d])
            if y != height_segments - 1:
                idx.append([b, c, d])
    return np.array(pos, np.float32), np.array(idx, np.uint32)


def test_rebuild_hint_after_area_doubles():
    """binnedSahBvh.test.ts:196-207: refits at scale 0.99 and 1.3 keep the
    BLAS; at 1.6 the node area exceeds twice the build's (rebuild)."""
    pos, idx = uv_sphere(16, 8)
    buf, _ = blas.host_build(pos, idx)
    _, _, build_area = host_refit(buf, pos)
    for scale, keep in ((0.99, True), (1.3, True), (1.6, False)):
        st, got, area = host_refit(buf, (pos * np.float32(scale)).astype(np.float32))
        assert st == abi.MT_OK and (not (area > build_area * 2)) == keep
        f = got.reshape(-1, 4)
        assert np.allclose(f[0, :3], (pos * np.float32(scale)).min(0)) and \
            np.allclose(f[1, :3], (pos * np.float32(scale)).max(0))
