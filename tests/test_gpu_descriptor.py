"""mt_context_commit on a scene descriptor v8, on a B200: the image equals
the same decoded scene committed as a buffer bundle and traced through the
device-buffer entry point; image parity against the CPU oracle on a scene
using every analytic light type, an emissive mesh, instancing, generated
normals and an environment map with yaw; a rejected descriptor leaves the committed scene."""
import numpy as np
import pytest

from mutracer_b200 import abi, scene, trace
from mutracer_b200 import descriptor as D
from mutracer_b200.context import Context, default_settings
from tests import oracle_lib
from tests.test_blas_refit_host import uv_sphere
from tests.test_gpu_parity import LUMA_BAR, REL_MSE_BAR, _image_metrics, _render_pair

pytestmark = pytest.mark.gpu
F = np.float32


def room(width=96, height=72):
    d = D.Descriptor(width, height)
    quad = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F)
    floor = d.add_geometry(quad * F(3), [0, 2, 1, 0, 3, 2])
    wall = d.add_geometry(np.array([[-3, 0, -2], [3, 0, -2], [3, 3, -2], [-3, 3, -2]], F), [0, 1, 2, 0, 2, 3])
    spos, sidx = uv_sphere(24, 12, 0.6)
    sphere = d.add_geometry(spos, sidx)                              # normals generated
    cube = np.array([[x, y, z] for x in (-.2, .2) for y in (0, .4) for z in (-.2, .2)], F)
    cidx = [0, 2, 3, 0, 3, 1, 4, 5, 7, 4, 7, 6, 0, 1, 5, 0, 5, 4, 2, 6, 7, 2, 7, 3, 0, 4, 6, 0, 6, 2, 1, 3, 7, 1, 7, 5]
    box = d.add_geometry(cube, cidx)
    white = d.add_material(base_color=(0.75, 0.75, 0.72), roughness=0.8)
    red = d.add_material(base_color=(0.7, 0.15, 0.1), roughness=0.5)
    metal = d.add_material(base_color=(0.95, 0.8, 0.5), metalness=1.0, roughness=0.25)
    coated = d.add_material(base_color=(0.1, 0.3, 0.7), roughness=0.6, coat_weight=1.0, coat_roughness=0.05)
    glass = d.add_material(base_color=(1, 1, 1), transmission=1.0, roughness=0.0, ior=1.5)
    d.add_mesh(floor, white)
    d.add_mesh(wall, red)
    d.add_mesh(sphere, metal, transform=D.translate([-0.9, 0.6, 0]))
    d.add_mesh(sphere, glass, transform=D.translate([0.9, 0.6, 0.3], 0.8))
    transforms = np.array([D.translate([x, 0, 1.2]) for x in (-1.2, -0.4, 0.4, 1.2)], F)
    colors = np.array([[1, 1, 1], [1, .5, .5], [.5, 1, .5], [.5, .5, 1]], F)
    d.add_mesh(box, coated, batch=(transforms, colors))
    d.add_mesh(box, white, hidden=True)
    panel = d.add_geometry(np.array([[-.5, 0, -.3], [.5, 0, -.3], [.5, 0, .3], [-.5, 0, .3]], F), [0, 1, 2, 0, 2, 3])
    lamp = d.add_material(emission_color=(1.0, 0.85, 0.7), emission_luminance=3.0)
    d.add_mesh(panel, lamp, transform=[1, 0, 0, 0, 0, -1, 0, 0, 0, 0, -1, 0, -1.5, 2.6, -0.5, 1])  # facing down
    d.add_light(D.LIGHT_RECT, intensity=6, size=1.0, height_or_inner=0.6, transform=D.look_at([0, 2.8, 0.4], [0, 0, 0]))
    d.add_light(D.LIGHT_SPOT, color=(1, .8, .6), intensity=40, size=0.05, height_or_inner=15, spread_or_outer=35,
                transform=D.look_at([2, 2.5, 2], [0, 0, 0]))
    d.add_light(D.LIGHT_DISK, color=(.6, .8, 1), intensity=3, transform=D.look_at([-2, 2, 1], [0, 0.5, 0]), radius=0.3,
                normalize=False)
    d.add_light(D.LIGHT_CYLINDER, color=(1, .9, .7), intensity=2, transform=D.translate([0, 2.2, -1.5]), radius=0.05,
                length=1.5)
    d.add_light(D.LIGHT_SPHERE, color=(1, 1, 1), intensity=4, size=0.1, transform=D.translate([1.5, 1.5, 1.5]))
    d.add_light(D.LIGHT_DIRECTIONAL, color=(1, 1, .9), intensity=0.5, transform=D.look_at([1, 3, 2], [0, 0, 0]))
    sky = np.zeros((16, 32, 4), F)
    sky[..., :3] = np.linspace(0.2, 1.0, 16, dtype=F)[:, None, None] * np.array([0.5, 0.7, 1.0], F)
    sky[..., 3] = 1
    d.set_environment(d.add_texture_rgba32f(32, 16, sky), intensity=0.7, yaw=0.5)
    d.background = (0.05, 0.05, 0.08, 1.0)
    d.set_camera(fov=45, transform=D.look_at([0, 1.6, 4.2], [0, 0.7, 0]))
    return d


def test_context_commit_matches_bundle_and_device_path(cuda):
    import torch
    data = room(64, 48).to_bytes()
    st, msg, host = D.decode(data)
    assert st == abi.MT_OK, msg
    ctx = Context()
    try:
        ctx.commit_descriptor(data)
        ctx.render(4)
        via_descriptor = ctx.read_pixels()
        ctx.commit(host, default_settings())
        ctx.render(4)
        assert np.array_equal(ctx.read_pixels(), via_descriptor)
        # the decoded uniform carries the same defaults the commit applies
        dev = scene.DeviceScene(host, cuda)
        acc = trace.Accumulation(64, 48, cuda)
        trace.trace_samples(dev, acc, 4)
        torch.cuda.synchronize()
        want = (acc.color.cpu().numpy() / np.float32(4)).reshape(48, 64, 4)
        assert np.array_equal(via_descriptor, want)
        assert np.isfinite(via_descriptor).all() and via_descriptor[..., :3].mean() > 0.01
    finally:
        ctx.destroy()


def test_descriptor_scene_oracle_parity(cuda):
    st, msg, host = D.decode(room().to_bytes())
    assert st == abi.MT_OK, msg
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def test_rejected_descriptor_keeps_previous_scene(cuda):
    ctx = Context()
    try:
        ctx.commit_descriptor(room(32, 24).to_bytes())
        ctx.render(2)
        before = ctx.read_pixels().copy()
        bad = bytearray(room(32, 24).to_bytes())
        bad[0:4] = (9).to_bytes(4, "little")                        # version 9
        with pytest.raises(abi.MtError) as e:
            ctx.commit_descriptor(bytes(bad))
        assert e.value.status == abi.MT_ERROR_INVALID_ARGUMENT
        unsupported = room(32, 24)
        unsupported.add_material(extensions=[(52, 1)])                  # unlit
        with pytest.raises(abi.MtError) as e:
            ctx.commit_descriptor(unsupported.to_bytes())
        assert e.value.status == abi.MT_ERROR_UNAVAILABLE
        assert ctx.info().samples == 2
        assert np.array_equal(ctx.read_pixels(), before)
        ctx.render(2)
        assert ctx.info().samples == 4
    finally:
        ctx.destroy()
