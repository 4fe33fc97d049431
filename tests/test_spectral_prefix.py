"""The shared-prefix spectral integrator (spectralPrefix.wgsl.ts and
rayTrace.compute.ts:1001-1041 of the reference) on the CPU oracle.

With three dispersion wavelengths the first wavelength path runs in RGB until
its first dispersive transmissive vertex and forks there; the other two resume
from that checkpoint (path, surface, guides and sampler state) instead of
retracing the prefix from the camera.  Every wavelength path restarts from the
same sampler state and RIS is channel-independent, so the prefix the later
paths skip is exactly the one they would have traced: the checkpoint changes
the work, never the result.  These tests pin both halves of that.
"""
import numpy as np

from mutracer_b200 import abi, scene
from tests import oracle_lib


def _render(flags_extra, spp=12, size=(40, 30), seed=3, params=(8,), wavelengths=3):
    host = scene.SceneHost("glass_spheres", size[0], size[1], seed, params)
    u = abi.TraceUniform.from_buffer_copy(host.uniform)
    u.dispersion_wavelengths = wavelengths
    host.set_uniform(u, None, host.flags | flags_extra)
    acc = oracle_lib.Accum(*size)
    traffic = oracle_lib.trace(host, acc, spp, traffic=True)
    return acc, traffic


def _bits_equal(a, b):
    return all(np.array_equal(getattr(a, k).view(np.uint32), getattr(b, k).view(np.uint32))
               for k in ("color", "normal", "albedo", "catcher"))


def test_shared_prefix_is_bit_identical_to_independent_wavelengths():
    shared, t_shared = _render(0)
    independent, t_indep = _render(abi.MTC_SCENE_SPECTRAL_INDEPENDENT)
    assert _bits_equal(shared, independent)
    # ...and traces fewer rays: the later wavelength paths skip the prefix.
    assert t_shared["paths"] == t_indep["paths"]
    assert t_shared["extension_rays"] < 0.9 * t_indep["extension_rays"]
    assert t_shared["shadow_rays"] < t_indep["shadow_rays"]


def test_shared_prefix_other_seed_and_deeper_paths():
    shared, _ = _render(0, spp=6, seed=7, params=(12,))
    independent, _ = _render(abi.MTC_SCENE_SPECTRAL_INDEPENDENT, spp=6, seed=7, params=(12,))
    assert _bits_equal(shared, independent)


def test_single_wavelength_ignores_the_flag():
    """dispersionWavelengths 1 is the hero-wavelength integrator, which never
    shares (spBegin's spEnabled is false)."""
    a, ta = _render(0, wavelengths=1, spp=6)
    b, tb = _render(abi.MTC_SCENE_SPECTRAL_INDEPENDENT, wavelengths=1, spp=6)
    assert _bits_equal(a, b)
    assert ta == tb
