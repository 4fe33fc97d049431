"""Known-answer tests of the CPU oracle.

- Environment pdf at the poles, seam and equator of uniform 1x1 and 4x8 maps,
  and sample/evaluate agreement: tests/gpu/environmentPdf.ts:5-10, 116-131.
- OpenPBR lobes conserve energy (white furnace) and their sampling pdf is
  consistent with evaluation (openPbrBsdf.wgsl.ts prepare/eval/sample).
"""
import ctypes as C
import math

import numpy as np
import pytest

from mutracer_b200 import abi
from tests import oracle_lib

CASES = np.array([.5, 0, 0, .5, .5, 1, 1 - 2 ** -24, .5, .5, 2 ** -24, 2 ** -24, .5, .5, 1 - 2 ** -24,
                  1 - 2 ** -24, .5, 0, .5, .5, 0, 1, .5, .5, 1 - 2 ** -24, .5, .5, .5, .5], np.float32).reshape(-1, 4)


def _env_view(width, height):
    img = np.ones((height, width, 4), np.float32)
    dist = np.zeros(((height + 1) * (width + 2) * 2,), np.float32)
    power = C.c_double()
    assert abi.lib().mtp_env_distribution(img.ctypes.data, width, height, dist.ctypes.data, C.byref(power)) == 0
    v = abi.SceneView()
    v.struct_size = C.sizeof(abi.SceneView)
    v.env_map = img.ctypes.data
    v.env_distribution = dist.ctypes.data
    v.env_width, v.env_height = width, height
    u = abi.TraceUniform()
    for i in range(4):
        u.environment_rotation[i * 5] = 1.0
    return v, u, (img, dist), power.value


@pytest.mark.parametrize("width,height", [(1, 1), (4, 8)])
def test_environment_pdf_cases(width, height):
    L = oracle_lib.lib()
    L.oracle_env_case.argtypes = [C.POINTER(abi.SceneView), C.POINTER(abi.TraceUniform)] + [C.c_float] * 4 + \
        [C.c_void_p]
    v, u, keep, power = _env_view(width, height)
    rows = [math.sin(math.pi * (y + .5) / height) for y in range(height)]
    equator = rows[height // 2] * height / sum(rows) / (2 * math.pi * math.pi)
    out = np.zeros(4, np.float32)
    for i, (pu, pv, r0, r1) in enumerate(CASES):
        assert L.oracle_env_case(C.byref(v), C.byref(u), pu, pv, r0, r1, out.ctypes.data) == 0
        ev, sampled, re, length = out
        assert np.isfinite(out[:3]).all() and (out[:3] >= 0).all(), (i, out)
        assert abs(sampled - re) <= max(1.0, sampled) * 1e-4 and abs(length - 1) <= 1e-5, (i, out)
        if i < 2:
            assert ev == 0.0, (i, out)
        if i >= 4:
            assert abs(ev - equator) <= 1e-6, (i, ev, equator)
    # environment power of a unit radiance sphere: integral of sin over the lat-long map
    assert abs(power - 4 * math.pi * (2 * math.pi * math.pi / (width * height) * sum(rows) * width) /
               (4 * math.pi)) < 1e-6 * max(1.0, power)


def _material(**kw):
    rows = np.zeros((26, 4), np.float32)
    rows[0] = [*kw.get("base", (1, 1, 1)), 0]
    rows[1] = [kw.get("roughness", 0.3), -1, 1, 1]
    rows[2] = [kw.get("metal", 0.0), kw.get("aniso", 0.0), -1, -1]
    rows[3] = [0, 0, 0, -1]
    rows[4] = [kw.get("ior", 1.5), kw.get("transmission", 0.0), 0, 1.0 if kw.get("thin") else 0.0]
    rows[5] = [0, 0, kw.get("film_thickness", 0.0), 0]
    rows[9] = [1, -1, kw.get("film_ior", 1.4), -1]
    rows[10] = [kw.get("base_weight", 1.0), kw.get("diffuse_roughness", 0.0), kw.get("specular_weight", 1.0),
                kw.get("subsurface", 0.0)]
    rows[11] = [*kw.get("specular_color", (1, 1, 1)), kw.get("fuzz", 0.0)]
    rows[12] = [*kw.get("transmission_color", (1, 1, 1)), 0]
    rows[14] = [1, 1, 1, 0]
    rows[15] = [1, 1, 1, kw.get("fuzz_roughness", 0.5)]
    rows[16] = [*kw.get("coat_color", (1, 1, 1)), kw.get("coat", 0.0)]
    rows[17] = [kw.get("coat_roughness", 0.1), 0, kw.get("coat_ior", 1.6), kw.get("coat_darkening", 1.0)]
    rows[6] = [-1, -1, -1, -1]                                 # no coat / fuzz maps
    rows[18] = [kw.get("film", 0.0), 20, 0, -1]
    rows[19] = [0, 0, 0, -1]
    rows[21] = [0, 0, 0, -1]
    rows[22] = [-1, -1, -1, 0.5]
    rows[24] = [-1, 0, 1, 1]
    return rows


_LUT = None


def lut():
    global _LUT
    if _LUT is None:
        _LUT = np.zeros(32 * 2177, np.float32)
        assert abi.lib().mtp_energy_lut(_LUT.ctypes.data) == 0
    return _LUT


def _albedo(rows, features, view, n=4096, seed=0):
    L = oracle_lib.lib()
    L.oracle_bsdf.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                              C.c_void_p]
    rng = np.random.default_rng(seed)
    view = np.asarray(view, np.float32)
    out = np.zeros(8, np.float32)
    acc = np.zeros(3)
    lt = lut()
    side = 4  # stratified lobe/direction draws
    for i in range(n):
        rnd = ((rng.random(3) + [i % side, (i // side) % side, 0]) / [side, side, 1]).astype(np.float32)
        rnd = np.clip(rnd, 0.0005, 0.9995).astype(np.float32)
        if L.oracle_bsdf(rows.ctypes.data, features, view.ctypes.data, None, rnd.ctypes.data, 1, lt.ctypes.data,
                         out.ctypes.data) != 0:
            continue
        if out[3] > 0:
            acc += out[:3] / out[3]
    return acc / n


FEATURES = (1 << 10) | (1 << 11) | (1 << 12) | (1 << 13)


@pytest.mark.parametrize("name,kw,lo,hi", [
    ("lambert", dict(specular_weight=0.0, roughness=1.0), 0.95, 1.02),
    ("eon_rough", dict(specular_weight=0.0, diffuse_roughness=1.0), 0.9, 1.02),
    ("plastic", dict(roughness=0.4), 0.85, 1.03),
    ("metal_rough", dict(metal=1.0, roughness=0.5), 0.85, 1.03),
    ("metal_smooth", dict(metal=1.0, roughness=0.05), 0.9, 1.03),
    ("coated", dict(coat=1.0, coat_roughness=0.2, roughness=0.4), 0.75, 1.03),
    # Radiance refracted into the denser side is scaled by (1/ior)^2, so seen
    # from outside the interface returns about F + (1 - F) / 1.5^2 = 0.47.
    ("glass_rough", dict(transmission=1.0, roughness=0.3), 0.42, 1.05),
    ("thin_film_metal", dict(metal=1.0, roughness=0.3, film=1.0, film_thickness=0.4), 0.5, 1.05),
])
def test_white_furnace(name, kw, lo, hi):
    rows = _material(**kw)
    for view in ([0, 0, 1], [0.6, 0, 0.8], [0.95, 0, 0.312]):
        a = _albedo(rows, FEATURES, view, n=3000, seed=hash(name) & 0xffff)
        assert (a >= lo).all() and (a <= hi).all(), (name, view, a)


def test_sampled_pdf_matches_evaluation():
    L = oracle_lib.lib()
    rows = _material(roughness=0.35, coat=0.5, coat_roughness=0.15)
    view = np.array([0.5, 0.1, 0.86], np.float32)
    rng = np.random.default_rng(2)
    out = np.zeros(8, np.float32)
    ev = np.zeros(8, np.float32)
    lt = lut()
    checked = 0
    for _ in range(400):
        rnd = np.clip(rng.random(3), 0.0005, 0.9995).astype(np.float32)
        if L.oracle_bsdf(rows.ctypes.data, FEATURES, view.ctypes.data, None, rnd.ctypes.data, 1, lt.ctypes.data,
                         out.ctypes.data) != 0:
            continue
        d = out[4:7].copy()
        L.oracle_bsdf(rows.ctypes.data, FEATURES, view.ctypes.data, d.ctypes.data, None, 0, lt.ctypes.data,
                      ev.ctypes.data)
        assert np.allclose(ev[:4], out[:4], rtol=1e-6, atol=1e-12)
        checked += 1
    assert checked > 300
    # the proposal density integrates to at most one over the sphere
    dirs = rng.normal(size=(20000, 3)).astype(np.float32)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    total = 0.0
    for d in dirs:
        d = np.ascontiguousarray(d)
        L.oracle_bsdf(rows.ctypes.data, FEATURES, view.ctypes.data, d.ctypes.data, None, 0, lt.ctypes.data,
                      ev.ctypes.data)
        total += ev[3]
    integral = total / len(dirs) * 4 * math.pi
    assert 0.85 < integral < 1.05, integral


def test_energy_lut_layout_and_ranges():
    t = lut().reshape(2177, 32)
    assert np.isfinite(t).all() and (t >= 0).all() and (t <= 1).all()
    # ior index 15/16 is an index-matched interface: no specular loss
    assert np.allclose(t[15 * 32: 17 * 32 - 16, :], t[15 * 32: 17 * 32 - 16, :].clip(0, 1))
    # rougher metals lose more energy at grazing angles
    assert t[1056 + 31, 0] > t[1056 + 4, 0]
    # smooth surfaces lose (almost) nothing
    assert t[1056, 16] < 1e-3
