"""The reference's own C hosts (native/examples/minimal-host.c, job-host.c,
scene-host.c, compiled unmodified by oracle/ref_hosts.py and linked to this
library) run on a B200.

* minimal-host builds a scene with the reference's header-only scene builder,
  commits, renders and reads pixels, and checks red > green.
* scene-host feeds malformed descriptors that must be rejected, then renders
  each accepted variant through mt_probe_render_scene; its HDR image meets the
  oracle bar (relMSE <= 1e-3, mean luminance within 0.5 %) against the CPU
  oracle on the same decoded scene, and equals a context render bit for bit.
* job-host drives two contexts created with the software backend through
  submit / poll / cancel / resume from another thread and compares their
  images with each other and with an expected image, which here is this
  library's blocking render of the same descriptor.
"""
import os
import subprocess

import numpy as np
import pytest

from mutracer_b200 import abi
from mutracer_b200 import descriptor as D
from mutracer_b200.context import Context
from tests import oracle_lib
from tests.test_gpu_parity import LUMA_BAR, REL_MSE_BAR, _image_metrics
from tests.test_reference_hosts import ACCEPTED, host, write_descriptor

pytestmark = pytest.mark.gpu


def test_minimal_host(cuda):
    r = subprocess.run([host("minimal-host"), "16"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert "mean red" in r.stdout


@pytest.mark.parametrize("variant", ACCEPTED)
def test_scene_host_probe_render_matches_oracle(cuda, variant, tmp_path):
    samples = 4
    data = write_descriptor(variant, tmp_path)
    out = tmp_path / "probe"
    r = subprocess.run([host("scene-host"), str(out), str(samples), variant], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, (variant, r.returncode, r.stderr)
    st, msg, scene = D.decode(data)
    assert st == abi.MT_OK, msg
    w, h = scene.width, scene.height
    probe = np.fromfile(out / "render.rgba32f", np.float32).reshape(h, w, 4)
    for name in ("normal.rgba32f", "albedo.rgba32f", "render.png", "result.json"):
        assert (out / name).exists(), name
    ctx = Context()
    try:
        ctx.commit_descriptor(data)
        ctx.render(samples)
        assert np.array_equal(ctx.read_pixels().reshape(h, w, 4), probe)
    finally:
        ctx.destroy()
    acc = oracle_lib.Accum(w, h)
    oracle_lib.trace(scene, acc, samples)
    rel_mse, luma = _image_metrics(probe, acc.resolved())
    assert np.isfinite(probe).all()
    assert rel_mse <= REL_MSE_BAR, (variant, rel_mse)
    assert luma <= LUMA_BAR, (variant, luma)


def test_job_host(cuda, tmp_path):
    samples = 16
    data = write_descriptor("emissive", tmp_path)
    desc = tmp_path / "emissive.bin"
    expected, out = tmp_path / "expected", tmp_path / "out"
    expected.mkdir()
    out.mkdir()
    ctx = Context()
    try:
        ctx.commit_descriptor(data)
        ctx.render(samples)
        for kind, name in ((abi.MT_IMAGE_HDR, "render"), (abi.MT_IMAGE_NORMAL, "normal"),
                           (abi.MT_IMAGE_ALBEDO, "albedo")):
            ctx.read_pixels(kind).astype(np.float32).tofile(expected / f"{name}.rgba32f")
    finally:
        ctx.destroy()
    r = subprocess.run([host("job-host"), str(desc), str(expected), str(out), str(samples)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert r.stdout.startswith("PASS"), r.stdout
