"""Alpha coverage on a B200: the alpha-split integrator and the shadow rays'
coverage test.  A scene whose materials are all mask-mode at full coverage
renders bit-identical to the opaque scene (HAS_ALPHA code paths with nothing
transparent); a scene with blend opacity, a base-color alpha cutout, an
alpha-mapped mask fence and a half-transparent occluder meets the oracle
parity bar and is bit-identical through the batch entry point, the
wavefront engine and mt_context_commit."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, batch, scene, trace
from mutracer_b200 import descriptor as D
from mutracer_b200.context import Context
from tests.test_alpha import room
from tests.test_gpu_parity import LUMA_BAR, REL_MSE_BAR, _image_metrics, _render_pair
from tests.test_gpu_textures import uv_sphere

pytestmark = pytest.mark.gpu
F = np.float32
NONE = D.NO_TEXTURE
QUAD = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F)
QUAD_IDX = [0, 2, 1, 0, 3, 2]
QUAD_UV = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], F)


def decode(d):
    st, msg, host = D.decode(d.to_bytes())
    assert st == abi.MT_OK, msg
    return host


def render_device(cuda, host, spp):
    import torch
    dev = scene.DeviceScene(host, cuda)
    acc = trace.Accumulation(host.width, host.height, cuda)
    trace.trace_samples(dev, acc, spp)
    torch.cuda.synchronize()
    return dev, acc


def test_full_coverage_mask_scene_is_the_opaque_scene(cuda):
    import torch
    a = decode(room())
    b = decode(room("mask1"))
    assert b.bundle.flags & abi.MTC_SCENE_HAS_ALPHA
    _, acc_a = render_device(cuda, a, 16)
    dev_b, acc_b = render_device(cuda, b, 16)
    for x, y in ((acc_a.color, acc_b.color), (acc_a.normal, acc_b.normal), (acc_a.albedo, acc_b.albedo)):
        assert torch.equal(x, y)
    job = batch.RenderJob(dev_b, 16, device=cuda)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([job])
    sb.run()
    torch.cuda.synchronize()
    assert torch.equal(acc_a.color, job.acc.color)


def alpha_room(width=96, height=72):
    d = D.Descriptor(width, height)
    yy, xx = np.mgrid[0:16, 0:16]
    holes = np.full((16, 16, 4), 255, np.uint8)
    holes[..., 3] = np.where(((xx // 4) + (yy // 4)) % 2 == 0, 255, 0)     # base-color alpha cutout
    holes[..., :3] = [200, 120, 60]
    holes_tex = d.add_texture(16, 16, holes)
    fence = np.zeros((8, 8, 4), np.uint8)
    fence[..., 1] = np.where((xx[:8, :8] % 4 < 2) | (yy[:8, :8] % 4 < 2), 230, 20)  # alpha map: g
    fence_tex = d.add_texture(8, 8, fence, uv_scale=(2, 2))
    floor = d.add_geometry(QUAD * F(3), QUAD_IDX, uvs=QUAD_UV)
    wall = d.add_geometry(np.array([[-3, 0, -2], [3, 0, -2], [3, 3, -2], [-3, 3, -2]], F), [0, 1, 2, 0, 2, 3],
                          uvs=QUAD_UV)
    panel = d.add_geometry(np.array([[-.7, 0, 0], [.7, 0, 0], [.7, 1.4, 0], [-.7, 1.4, 0]], F), [0, 1, 2, 0, 2, 3],
                           uvs=QUAD_UV)
    spos, suv, sidx = uv_sphere(24, 12, 0.45)
    sphere = d.add_geometry(spos, sidx, uvs=suv)
    d.add_mesh(floor, d.add_material(base_color=(0.7, 0.7, 0.7), roughness=0.7))
    d.add_mesh(wall, d.add_material(base_color=(0.5, 0.6, 0.8), roughness=0.5))
    # blend: half-transparent glassy-green sheet
    d.add_mesh(panel, d.add_material(base_color=(0.2, 0.9, 0.3), roughness=0.3, opacity=0.5),
               transform=D.translate([-1.0, 0, 0.6]))
    # base-color alpha as opacity (auto -> blend, alpha 0 or 1 per texel)
    d.add_mesh(panel, d.add_material(base_color=(1, 1, 1), roughness=0.5, textures=(holes_tex, NONE, NONE, NONE),
                                     extensions=[(54, 1)]), transform=D.translate([0.9, 0, 0.4]))
    # mask: alpha-mapped fence with a cutoff
    d.add_mesh(panel, d.add_material(base_color=(0.9, 0.9, 0.9), roughness=0.6,
                                     extensions=[(40, fence_tex), (41, 2), (42, (0.5,))]),
               transform=D.translate([0, 0, -0.8]))
    # a partly covered sphere casting a partial shadow
    d.add_mesh(sphere, d.add_material(base_color=(0.9, 0.4, 0.4), roughness=0.2, opacity=0.35),
               transform=D.translate([0, 1.8, 0.3]))
    d.add_light(D.LIGHT_RECT, intensity=7, size=1.0, height_or_inner=0.8, transform=D.look_at([0, 2.9, 0.3], [0, 0, 0]))
    d.add_light(D.LIGHT_SPHERE, color=(1, 0.9, 0.8), intensity=3, size=0.1, transform=D.translate([1.5, 1.5, 1.8]))
    sky = np.zeros((8, 16, 4), F)
    sky[..., :3] = 0.3
    sky[..., 3] = 1
    d.set_environment(d.add_texture_rgba32f(16, 8, sky), intensity=0.5)
    d.set_camera(fov=45, transform=D.look_at([0, 1.5, 4.2], [0, 0.7, 0]))
    return d


def test_alpha_scene_oracle_parity(cuda):
    host = decode(alpha_room())
    assert host.bundle.flags & abi.MTC_SCENE_HAS_ALPHA
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def test_alpha_scene_identical_in_every_engine(cuda):
    import torch
    data = alpha_room(64, 48).to_bytes()
    host = decode(alpha_room(64, 48))
    dev, alone = render_device(cuda, host, 6)
    batched = trace.Accumulation(64, 48, cuda)
    jobs = (abi.JobDesc * 1)()
    jobs[0].scene, jobs[0].camera, jobs[0].uniform = dev.view, dev.camera, dev.uniform
    jobs[0].out, jobs[0].samples = batched.outputs, 6
    scratch = torch.zeros(abi.lib().mtc_batch_scratch_bytes(1), dtype=torch.uint8, device=cuda)
    abi.check(abi.lib().mtc_trace_batch(jobs, 1, None, C.c_void_p(scratch.data_ptr()), None, None,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    job = batch.RenderJob(dev, 6, device=cuda)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([job])
    sb.run()
    torch.cuda.synchronize()
    for other in (batched, job.acc):
        assert torch.equal(alone.color, other.color) and torch.equal(alone.normal, other.normal)
        assert torch.equal(alone.albedo, other.albedo)
    ctx = Context()
    try:
        ctx.commit_descriptor(data)
        ctx.render(6)
        want = (alone.color.cpu().numpy() / np.float32(6)).reshape(48, 64, 4)
        assert np.array_equal(ctx.read_pixels(), want)
    finally:
        ctx.destroy()
