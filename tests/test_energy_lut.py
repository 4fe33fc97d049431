"""The OpenPBR energy-compensation table the BSDF samples, pinned to the
reference's own expectations (tests/unit/openPbrEnergyLut.test.ts of the
reference): the SHA-256 digests of the decoded table and of its two average
rows, the UNORM source anchors, and the physical contracts (ideal-metal and
ideal-dielectric directional losses complete the analytic single-scattering
GGX energy; the metal averages integrate the interpolated rows).

The table is Adobe's (adobe/openpbr-bsdf, Apache-2.0) as the reference decodes
it; mutracer_b200/csrc/gen_energy_lut.py wrote the committed file and the
build embeds it in the library, which returns it through mtp_energy_lut.
"""
import hashlib
import math
import os

import numpy as np
import pytest

from mutracer_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TABLE = os.path.join(ROOT, "mutracer_b200", "csrc", "openpbr_energy_lut.f32")
REFERENCE_LUT_SOURCE = "/root/reference/src/renderer/openPbrEnergyLut.ts"

AVERAGE_ROW = 1024
METAL_ROW = 1056
METAL_AVERAGE_ROW = 1088
DIELECTRIC_ROW = 1089
DIELECTRIC_AVERAGE_ROW = 2113
RATIO_ROW = 2145
HEIGHT = 2177


@pytest.fixture(scope="module")
def data():
    d = np.fromfile(TABLE, dtype="<f4")
    assert d.size == 32 * HEIGHT
    return d


def _sha(values):
    return hashlib.sha256(np.ascontiguousarray(values, dtype="<f4").tobytes()).hexdigest()


def test_library_serves_the_committed_table(data):
    got = np.zeros(32 * HEIGHT, np.float32)
    assert abi.lib().mtp_energy_lut(got.ctypes.data) == 0
    assert np.array_equal(got.view(np.uint32), data.view(np.uint32))


def test_decoded_table_digest(data):
    """openPbrEnergyLut.test.ts:15-33: rows up to the metal average, then each
    metal average repeated across a 32-wide row, as little-endian float32."""
    expanded = np.zeros(1120 * 32, np.float32)
    expanded[:METAL_AVERAGE_ROW * 32] = data[:METAL_AVERAGE_ROW * 32]
    for r in range(32):
        expanded[(1088 + r) * 32:(1089 + r) * 32] = data[METAL_AVERAGE_ROW * 32 + r]
    assert _sha(expanded) == "2030bf2adefb6fa94edcaf4ecdbd7d3b3b3f1b2d5b7babe450c57b9c05f43ebe"


@pytest.mark.parametrize("row,length,digest", [
    (METAL_AVERAGE_ROW, 32, "1c8094d267ebba1d1cbb422825e944585538160ff805630d16889cae1416e6c7"),
    (DIELECTRIC_AVERAGE_ROW, 1024, "26bb5452686e4a99d5c15c0bcf622a85bc6691d33b160bd340d4bb1124951cf3"),
])
def test_average_rows_digest(data, row, length, digest):
    """openPbrEnergyLut.test.ts:162-173."""
    assert _sha(data[row * 32:row * 32 + length]) == digest


def test_unorm_anchors_and_range(data):
    """openPbrEnergyLut.test.ts:41-56."""
    assert data.min() >= 0.0 and data.max() <= 1.0
    assert abs(data[29] - 50582 / 65535) <= 0.002
    assert abs(data[32 * 32 * 32 - 1] - 61816 / 65535) <= 0.002
    assert abs(data[AVERAGE_ROW * 32] - 8159 / 65535) <= 0.002
    assert abs(data[METAL_ROW * 32 - 1] - 60821 / 65535) <= 0.002


def _metal_loss(data, roughness, cosine):
    r, c = roughness * 31, np.asarray(cosine, np.float64) * 31
    r0 = math.floor(r)
    r1 = min(31, r0 + 1)
    c0 = np.floor(c).astype(np.int64)
    c1 = np.minimum(31, c0 + 1)
    d = data.astype(np.float64)

    def row(i):
        a, b = d[(METAL_ROW + i) * 32 + c0], d[(METAL_ROW + i) * 32 + c1]
        return a + (b - a) * (c - c0)
    a, b = row(r0), row(r1)
    return a + (b - a) * (r - r0)


def _ideal_metal_energy(roughness, view_cosine, steps=512):
    """Unit-Fresnel GGX reflectance integrated over the hemisphere
    (openPbrEnergyLut.test.ts:61-82)."""
    alpha = roughness * roughness
    view_x = math.sqrt(1 - view_cosine * view_cosine)

    def g1(mu):
        return 2 / (1 + np.sqrt(1 + alpha * alpha * (1 - mu * mu) / (mu * mu)))
    mu = ((np.arange(steps) + 0.5) / steps)[:, None]
    phi = ((np.arange(steps) + 0.5) * 2 * math.pi / steps)[None, :]
    radial = np.sqrt(1 - mu * mu)
    masking = g1(view_cosine) * g1(mu)
    dot_vl = view_x * radial * np.cos(phi) + view_cosine * mu
    half_z = (view_cosine + mu) / np.sqrt(2 + 2 * dot_vl)
    denom = 1 + half_z * half_z * (alpha * alpha - 1)
    ndf = alpha * alpha / (math.pi * denom * denom)
    return float((ndf * masking / (4 * view_cosine)).sum()) * 2 * math.pi / (steps * steps)


@pytest.mark.parametrize("roughness,cosine", [(.3, .9), (.6, .3), (.6, .9), (.9, .3)])
def test_metal_loss_completes_analytic_ggx(data, roughness, cosine):
    """openPbrEnergyLut.test.ts:95-98."""
    loss = float(_metal_loss(data, roughness, cosine))
    assert abs(_ideal_metal_energy(roughness, cosine) + loss - 1) < 0.0025


def test_metal_averages_integrate_the_interpolated_rows(data):
    """openPbrEnergyLut.test.ts:100-117."""
    n = 65536
    cosine = (np.arange(n) + 0.5) / n
    for alpha in (.01, .05, .1, .25, .5, 1):
        roughness = math.sqrt(alpha)
        average = float((2 * cosine * _metal_loss(data, roughness, cosine) / n).sum())
        index = roughness * 31
        i0 = math.floor(index)
        i1 = min(31, i0 + 1)
        a = float(data[METAL_AVERAGE_ROW * 32 + i0])
        b = float(data[METAL_AVERAGE_ROW * 32 + i1])
        stored = a + (b - a) * (index - i0)
        assert stored > 0
        assert abs(average / stored - 1) < 1e-6


def _dielectric_loss(data, eta, roughness, cosine):
    index = max(0.0, min(31.0, 15 - (1 / eta - 1) * 10 if eta < 1 else 16 + (eta - 1) * 10))
    r, c = roughness * 31, cosine * 31
    value = 0.0
    for i in range(2):
        for j in range(2):
            for k in range(2):
                row = DIELECTRIC_ROW + min(31, math.floor(index) + i) * 32 + min(31, math.floor(r) + j)
                value += (float(data[row * 32 + min(31, math.floor(c) + k)])
                          * (math.fmod(index, 1) if i else 1 - math.fmod(index, 1))
                          * (math.fmod(r, 1) if j else 1 - math.fmod(r, 1))
                          * (math.fmod(c, 1) if k else 1 - math.fmod(c, 1)))
    return value


def _ideal_dielectric_single_energy(eta, roughness, mu, n=256):
    """Visible-normal integral of GGX reflection plus refraction with Smith
    shadowing and the Fresnel split (openPbrEnergyLut.test.ts:137-163)."""
    alpha = roughness * roughness
    a2 = alpha * alpha
    vx = math.sqrt(1 - mu * mu)

    def g1(z):
        return 2 / (1 + np.sqrt(1 + a2 * (1 - z * z) / (z * z)))
    hz = ((np.arange(n) + 0.5) / n)[:, None]
    radial = np.sqrt(1 - hz * hz)
    denom = 1 + hz * hz * (a2 - 1)
    D = a2 / (math.pi * denom * denom)
    hx = radial * np.cos(((np.arange(n) + 0.5) * 2 * math.pi / n)[None, :])
    vh = vx * hx + mu * hz
    k = 1 - (1 - vh * vh) / (eta * eta)
    with np.errstate(invalid="ignore", divide="ignore"):
        ct = np.sqrt(np.maximum(k, 0))
        F = np.where(k > 0, 0.5 * (((vh - eta * ct) / (vh + eta * ct)) ** 2
                                   + ((eta * vh - ct) / (eta * vh + ct)) ** 2), 1.0)
        rz = 2 * vh * hz - mu
        weight = np.where(rz > 0, F * g1(rz), 0.0)
        tz = -mu / eta + (vh / eta - ct) * hz
        weight = weight + np.where((k > 0) & (tz < 0), (1 - F) * g1(tz), 0.0)
        term = np.where(vh > 0, D * g1(mu) * vh / mu * weight, 0.0)
    return float(term.sum()) * 2 * math.pi / (n * n)


@pytest.mark.parametrize("eta,roughness,cosine", [(1.5, .6, .3), (1.5, .6, .9), (2 / 3, .6, .3), (2 / 3, .6, .9)])
def test_dielectric_loss_completes_analytic_ggx(data, eta, roughness, cosine):
    """openPbrEnergyLut.test.ts:166-168."""
    total = _ideal_dielectric_single_energy(eta, roughness, cosine) + _dielectric_loss(data, eta, roughness, cosine)
    assert abs(total - 1) < 0.004


def test_dielectric_averages_are_u16_and_cosine_weighted(data):
    """openPbrEnergyLut.test.ts:170-184."""
    mu = (np.arange(1024) + 0.5) / 1024
    for ior_index in (0, 5, 10, 20, 25, 31):
        for roughness_index in (10, 19, 31):
            average = float(data[(DIELECTRIC_AVERAGE_ROW + ior_index) * 32 + roughness_index])
            assert abs(average * 65535 - round(average * 65535)) < 0.003
            eta = 1 / (1 + (15 - ior_index) / 10) if ior_index < 16 else 1 + (ior_index - 16) / 10
            integral = sum(2 * m * _dielectric_loss(data, eta, roughness_index / 31, m) / 1024 for m in mu)
            assert abs(integral - average) < 0.0025


def test_reflection_ratio_bounds(data):
    """openPbrEnergyLut.test.ts:186-193."""
    assert RATIO_ROW + 32 == HEIGHT
    ratios = data[RATIO_ROW * 32:]
    assert ratios.min() >= 0 and ratios.max() <= 1
    assert abs(float(ratios[16 * 32 + 31]) - 142 / 65535) < 5e-8


@pytest.mark.skipif(not os.path.exists(REFERENCE_LUT_SOURCE), reason="reference source tree not present")
def test_generator_reproduces_the_committed_table(data):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_energy_lut", os.path.join(ROOT, "mutracer_b200", "csrc", "gen_energy_lut.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    decoded = gen.decode(gen.read_strings(REFERENCE_LUT_SOURCE))
    assert np.array_equal(decoded.view(np.uint32), data.view(np.uint32))
