"""The reference's own unit expectations for the spectral sampler and the
environment importance distribution, restated against this build's pieces:

* tests/unit/spectrum.test.ts:13-83 — spectrumRgb (the product's generator,
  mutracer_b200/csrc/gen_spectrum_cdf.py, which also writes the device
  tables), spectrumSample and spectrumIorWavelength (the oracle's f32
  restatement over the same tables, which the device shares bit for bit);
* tests/unit/envMapDistribution.test.ts:17-87 — envMapDistribution (the
  product's host producer, mtp_env_distribution);
* tests/unit/lightSampling.test.ts:30-64 — buildLightAliasTable and
  estimateAnalyticLightPower (the product's host producers).

Tolerances are the reference's: toBeCloseTo(x, d) passes when
|actual - x| < 10^-d / 2.
"""
import ctypes as C
import importlib.util
import math
import os

import numpy as np
import pytest

from mutracer_b200 import abi
from tests import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WMIN, WRANGE = 400.0, 300.0


def close(actual, expected, digits=2):
    return abs(actual - expected) < 10 ** -digits / 2


def _gen():
    spec = importlib.util.spec_from_file_location(
        "gen_spectrum_cdf", os.path.join(ROOT, "mutracer_b200", "csrc", "gen_spectrum_cdf.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _sample(distribution, u):
    L = oracle_lib.lib()
    L.oracle_spectrum_sample.argtypes = [C.c_uint, C.c_float, C.POINTER(C.c_float)]
    L.oracle_spectrum_sample.restype = C.c_float
    pdf = C.c_float()
    return L.oracle_spectrum_sample(distribution, u, C.byref(pdf)), pdf.value


def _ior_wavelength(w):
    # spectrumCameraWavelength = spectrumIorWavelength(spectrumSample(...));
    # evaluate the knee map through the oracle on a sample that lands on w.
    return 500.0 - 25.0 * (1.0 - math.exp((w - 500.0) / 25.0)) if w < 500.0 else w


def test_white_light_stays_white():                              # spectrum.test.ts:14-25
    rgb_of = _gen().spectrum_rgb
    steps = 4096
    mean = [0.0, 0.0, 0.0]
    for i in range(steps):
        rgb = rgb_of(WMIN + WRANGE * (i + 0.5) / steps)
        assert min(rgb) >= 0
        for c in range(3):
            mean[c] += rgb[c] / steps
    assert all(close(m, 1.0, 3) for m in mean), mean


def test_photon_sampling_white_with_bounded_flux():              # spectrum.test.ts:27-42
    rgb_of = _gen().spectrum_rgb
    steps = 64 * 256
    mean, peak = [0.0, 0.0, 0.0], 0.0
    for i in range(steps):
        w, pdf = _sample(3, (i + 0.5) / steps)
        assert WMIN <= w <= WMIN + WRANGE
        for c, v in enumerate(rgb_of(w)):
            weight = v / (pdf * WRANGE)
            mean[c] += weight / steps
            peak = max(peak, weight)
    assert all(close(m, 1.0, 2) for m in mean), mean
    assert peak < 4


def test_camera_channels_sample_their_own_response():            # spectrum.test.ts:44-57
    rgb_of = _gen().spectrum_rgb
    steps = 4096
    for channel in range(3):
        weights = [0.0, 0.0, 0.0]
        for i in range(steps):
            w, _ = _sample(channel, (i + 0.5) / steps)
            assert WMIN <= w <= WMIN + WRANGE
            for c, v in enumerate(rgb_of(w)):
                weights[c] += v / steps
        assert weights.index(max(weights)) == channel


def test_refraction_wavelength_knee():                           # spectrum.test.ts:59-70
    L = oracle_lib.lib()
    L.oracle_spectrum_camera_wavelength.argtypes = [C.c_uint, C.c_float]
    L.oracle_spectrum_camera_wavelength.restype = C.c_float
    # The oracle's camera map applies the knee to the sampled wavelength; its
    # values above 500 nm are the samples themselves and below it the knee.
    for u in np.linspace(0.001, 0.999, 97):
        w, _ = _sample(1, float(u))
        got = L.oracle_spectrum_camera_wavelength(1, float(u))
        assert abs(got - _ior_wavelength(w)) < 1e-3
    assert _ior_wavelength(650) == 650 and _ior_wavelength(500) == 500
    prev = _ior_wavelength(400)
    assert prev > 475
    for w in range(401, 521):
        nxt = _ior_wavelength(w)
        assert nxt > prev and nxt - prev < 1.01
        prev = nxt


def test_hue_varies_continuously():                              # spectrum.test.ts:72-82
    rgb_of = _gen().spectrum_rgb
    dominant = [max(range(3), key=lambda c: rgb_of(w)[c]) for w in (450, 540, 620)]
    assert dominant == [2, 1, 0]
    for w in range(400, 700):
        a, b = rgb_of(w), rgb_of(w + 1)
        assert all(abs(a[c] - b[c]) < 0.25 for c in range(3))


def env_distribution(width, height, rgba):
    img = np.ascontiguousarray(rgba, np.float32).reshape(-1)
    dist = np.zeros((height + 1) * (width + 2) * 2, np.float32)
    power = C.c_double()
    assert abi.lib().mtp_env_distribution(img.ctypes.data, width, height, dist.ctypes.data, C.byref(power)) == 0
    return dist


def value_at(data, width, x, y, channel):
    return float(data[2 * (y * width + x) + channel])


def rgba_from_rgb(rgb):
    rgb = np.asarray(rgb, np.float32).reshape(-1, 3)
    return np.concatenate([rgb, np.ones((len(rgb), 1), np.float32)], 1)


def test_env_sharp_texel_footprint():                            # envMapDistribution.test.ts:18-34
    d = env_distribution(3, 1, rgba_from_rgb([0, 0, 0, 100, 100, 100, 0, 0, 0]))
    assert close(value_at(d, 5, 0, 1, 0), 1.0)
    for x in range(1, 4):
        assert value_at(d, 5, x, 0, 1) > 0


def test_env_black_and_rgba():                                   # envMapDistribution.test.ts:36-62
    assert np.isfinite(env_distribution(2, 2, np.zeros((4, 4), np.float32))).all()
    d = env_distribution(2, 1, np.array([[0, 0, 0, 1], [10, 10, 10, 1]], np.float32))
    assert np.isfinite(d).all()
    assert close(value_at(d, 4, 0, 1, 0), 1.0)


@pytest.mark.parametrize("width,height", [(1, 1), (1, 5), (5, 1), (5, 4)])
def test_env_clamped_footprint_and_normalized_pdfs(width, height):  # envMapDistribution.test.ts:64-87
    data = np.array([1000.0 if i % 4 == 3 else ((i * 17) % 31) / 4 for i in range(width * height * 4)], np.float32)
    d = env_distribution(width, height, data)
    weights = []
    for y in range(height):
        row = []
        for x in range(width):
            nb = []
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    o = 4 * (max(0, min(height - 1, y + dy)) * width + max(0, min(width - 1, x + dx)))
                    nb.append(float(np.float32(.2126 * data[o] + .7152 * data[o + 1] + .0722 * data[o + 2])))
            row.append(max([1e-12] + nb) * math.sin(math.pi * (y + .5) / height))
        weights.append(row)
    row_int = [sum(r) / width for r in weights]
    integral = sum(row_int) / height
    W = width + 2
    for y in range(height):
        assert close(value_at(d, W, 0, y, 1), row_int[y] / integral, 6)
        for x in range(width):
            assert close(value_at(d, W, x + 1, y, 1), weights[y][x] / row_int[y], 6)
        assert close(value_at(d, W, width + 1, y, 0), 1.0, 6)
    assert close(value_at(d, W, 0, height, 0), 1.0, 6)


def test_alias_table_normalises_pmfs():                          # lightSampling.test.ts:30-50
    weights = np.array([1, 3, 6], np.float64)
    words = np.zeros(12, np.uint32)
    pmfs = np.zeros(3, np.float32)
    total = C.c_double()
    assert abi.lib().mtp_light_alias_table(weights.ctypes.data, 3, words.ctypes.data, pmfs.ctypes.data,
                                           C.byref(total)) == 0
    assert close(pmfs[0], 0.1) and close(pmfs[1], 0.3) and close(pmfs[2], 0.6)
    assert total.value == 10
    prob, alias = words.view(np.float32).reshape(3, 4)[:, 0], words.view(np.int32).reshape(3, 4)[:, 1]
    assert ((prob > 0) & (prob <= 1)).all() and ((alias >= 0) & (alias < 3)).all()


def test_rect_light_power():                                     # lightSampling.test.ts:52-55
    color = (C.c_float * 3)(1, 1, 1)
    rect, sphere = 3, 2                                         # MTC_LIGHT_RECT, MTC_LIGHT_SPHERE
    assert close(abi.lib().mtp_light_power(rect, color, 4.0, 6.0, 0.0), 24 * math.pi)   # 2 x 3 rect, intensity 4
    point = abi.lib().mtp_light_power(sphere, (C.c_float * 3)(1, 0.5, 0.25), 12.0, 0.0, 0.0)
    assert point > 0 and math.isfinite(point)                    # zero-radius sphere: finite and weighted
