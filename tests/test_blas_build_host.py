"""Host side of the device BLAS build (no GPU): argument checks that return
before any CUDA call, the scratch and output size bounds, and the source
meshes a generated scene keeps for rebuilding its BLASes."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, scene


def _input(n=0, bins=8, positions=None, indices=None, vertices=0):
    inp = abi.BlasBuildInput()
    inp.struct_size = C.sizeof(inp)
    inp.bins, inp.triangle_count, inp.vertex_count = bins, n, vertices
    inp.positions, inp.indices = positions, indices
    return inp


def _result():
    res = abi.BlasBuildResult()
    res.struct_size = C.sizeof(res)
    return res


def test_sizes():
    L = abi.lib()
    assert L.mtc_blas_build_max_vec4(0) == 0
    assert L.mtc_blas_build_max_vec4(1) == 3 and L.mtc_blas_build_max_vec4(1000) == 4998
    a, b = L.mtc_blas_build_scratch_bytes(1000, 8), L.mtc_blas_build_scratch_bytes(100000, 8)
    assert 0 < a < b and b < 100000 * 400
    assert L.mtc_blas_build_scratch_bytes(1000, 0) == 0 and L.mtc_blas_build_scratch_bytes(1000, 65) == 0
    assert L.mtc_blas_build_scratch_bytes(1000, 64) > a


def test_validation_before_device_calls():
    L = abi.lib()
    res = _result()
    assert L.mtc_build_blas(C.byref(_input()), None, 0, None, 0, C.byref(res), None) == abi.MT_OK
    assert res.vec4_count == 0 and res.primitive_count == 0 and np.isinf(res.local_bounds[0])
    bad = _input()
    bad.struct_size = 4
    assert L.mtc_build_blas(C.byref(bad), None, 0, None, 0, C.byref(res), None) == abi.MT_ERROR_INVALID_ARGUMENT
    bad_res = _result()
    bad_res.struct_size = 8
    assert L.mtc_build_blas(C.byref(_input()), None, 0, None, 0, C.byref(bad_res), None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    for bins in (0, 65):
        assert L.mtc_build_blas(C.byref(_input(bins=bins)), None, 0, None, 0, C.byref(res), None) == \
            abi.MT_ERROR_INVALID_ARGUMENT
    # triangles but no index buffer / too little scratch / misaligned scratch
    assert L.mtc_build_blas(C.byref(_input(10, positions=16, vertices=3)), None, 0, None, 0, C.byref(res),
                            None) == abi.MT_ERROR_INVALID_ARGUMENT
    full = _input(10, positions=4096, indices=8192, vertices=3)
    need = L.mtc_blas_build_scratch_bytes(10, 8)
    assert L.mtc_build_blas(C.byref(full), C.c_void_p(1 << 20), need - 1, C.c_void_p(1 << 21), 64, C.byref(res),
                            None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_build_blas(C.byref(full), C.c_void_p((1 << 20) + 16), need, C.c_void_p(1 << 21), 64, C.byref(res),
                            None) == abi.MT_ERROR_INVALID_ARGUMENT


@pytest.mark.parametrize("kind,params", [("cornell", ()), ("instanced_spheres", (24, 3, 4, 64, 1))])
def test_scene_keeps_source_meshes(kind, params):
    """The kept meshes rebuild, on the host, exactly the BLAS regions of the
    scene's bvh buffer (the GPU test compares the device build with these)."""
    host = scene.SceneHost(kind, 16, 16, 1, params)
    assert host.info.blases >= 1
    for m in range(host.info.blases):
        pos, idx, offset, length, bins = host.mesh(m)
        assert bins in (8, 16) and pos.shape[1] == 3 and idx.shape[1] == 3
        buf = np.zeros(max(5 * len(idx), 1) * 4, np.float32)
        vec4, depth = C.c_uint64(), C.c_uint32()
        assert abi.lib().mtp_build_blas(pos.ctypes.data, len(pos), idx.ctypes.data, len(idx), bins, buf.ctypes.data,
                                        buf.size // 4, C.byref(vec4), C.byref(depth)) == abi.MT_OK
        assert vec4.value == length
        assert buf[: length * 4].tobytes() == host.bvh[offset * 4: (offset + length) * 4].tobytes()
    with pytest.raises(abi.MtError):
        host.mesh(host.info.blases)
