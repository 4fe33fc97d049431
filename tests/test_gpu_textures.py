"""Material textures on a B200: mtc_sample_maps bit-identical to the CPU
restatement of sampleMap on the reference's lookup grid for every wrap mode,
byte and half-float storage; a textured scene (sRGB base-color checker,
normal maps with scaled UVs, a metallic-roughness map, base-color alpha as
transmission) with image parity against the oracle, and bit-identical through
the batch entry point, the wavefront engine and mt_context_commit; a scene
using every other supported slot (emissive map sampled by NEE, roughness,
metalness, specular, coat, fuzz, transmission, thin-film and alpha maps) with
image parity against the oracle."""
import ctypes as C
import math

import numpy as np
import pytest

from mutracer_b200 import abi, batch, scene, trace
from mutracer_b200 import descriptor as D
from mutracer_b200.context import Context
from tests import oracle_lib
from tests.test_gpu_parity import LUMA_BAR, REL_MSE_BAR, _image_metrics, _render_pair
from tests.test_textures import QUAD_UV, uv_grid

pytestmark = pytest.mark.gpu
F = np.float32
NONE = D.NO_TEXTURE
QUAD = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F)
QUAD_IDX = [0, 2, 1, 0, 3, 2]
WRAPS = [(0, 0), (1, 1), (2, 2), (0, 2), (1, 0)]


def uv_sphere(segments, rings, radius):
    """Latitude-longitude sphere with a UV seam (positions, uvs, indices)."""
    pos, uv, idx = [], [], []
    for r in range(rings + 1):
        v = r / rings
        th = math.pi * v
        for s in range(segments + 1):
            u = s / segments
            ph = 2 * math.pi * u
            pos.append([radius * math.sin(th) * math.cos(ph), radius * math.cos(th), radius * math.sin(th) * math.sin(ph)])
            uv.append([u, 1 - v])
    for r in range(rings):
        for s in range(segments):
            a, b = r * (segments + 1) + s, (r + 1) * (segments + 1) + s
            idx += [a, a + 1, b, a + 1, b + 1, b]
    return np.array(pos, F), np.array(uv, F), idx


def wrap_scene(float_storage):
    rng = np.random.default_rng(5)
    d = D.Descriptor(32, 32)
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    for k, (ws, wt) in enumerate(WRAPS):
        t = d.add_texture(5, 3, rng.integers(0, 256, (3, 5, 4), dtype=np.uint8), flip_y=bool(k % 2),
                          uv_scale=(1.25, -0.5 - k), uv_offset=(0.1 * k, -0.3), wrap_s=ws, wrap_t=wt)
        d.add_mesh(g, d.add_material(textures=(t, NONE, NONE, NONE)), transform=D.translate([0, 0.1 * k, 0]))
    if float_storage:
        t = d.add_texture_rgba32f(4, 4, rng.uniform(-2, 8, 64), wrap_s=2, wrap_t=0)
        d.add_mesh(g, d.add_material(textures=(NONE, NONE, t, NONE)))
    d.add_light(D.LIGHT_DIRECTIONAL, intensity=1, transform=D.look_at([0, 3, 1], [0, 0, 0]))
    d.set_camera(fov=40, transform=D.look_at([0, 2, 3], [0, 0, 0]))
    return d


@pytest.mark.parametrize("float_storage", [False, True])
def test_sample_maps_bit_identical_to_oracle(cuda, float_storage):
    import torch
    st, msg, host = D.decode(wrap_scene(float_storage).to_bytes())
    assert st == abi.MT_OK, msg
    maps = host.bundle.map_count
    grid = uv_grid()
    far = np.array([[1e6 + 0.25, -3e5 - 0.5], [-7.75, 12.5], [4096.125, -0.001], [1e-30, -1e-30]], F)
    uvs = np.concatenate([np.tile(grid, (maps + 2, 1)), np.tile(far, (maps, 1))])
    idx = np.concatenate([np.repeat(np.arange(-1, maps + 1), len(grid)), np.repeat(np.arange(maps), len(far))])
    idx = idx.astype(np.int32)
    dev = scene.DeviceScene(host, cuda)
    d_idx = torch.from_numpy(idx).to(cuda)
    d_uv = torch.from_numpy(uvs).to(cuda)
    d_out = torch.zeros((len(idx), 4), dtype=torch.float32, device=cuda)
    abi.check(abi.lib().mtc_sample_maps(C.byref(dev.view), C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_uv.data_ptr()),
                                        len(idx), C.c_void_p(d_out.data_ptr()),
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    got = d_out.cpu().numpy()
    want = oracle_lib.sample_maps(host, idx, uvs)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    outside = (idx < 0) | (idx >= maps)
    assert not got[outside].any() and got[~outside].any()


def textured_room(width=96, height=72):
    d = D.Descriptor(width, height)
    checker = np.zeros((8, 8, 4), np.uint8)
    yy, xx = np.mgrid[0:8, 0:8]
    on = (xx + yy) % 2 == 0
    checker[on] = [230, 200, 150, 255]
    checker[~on] = [40, 60, 120, 255]
    floor_tex = d.add_texture(8, 8, checker, uv_scale=(3, 3))
    # tangent-space bumps: n = normalize(sin, cos, 1) encoded as bytes
    ny, nx = np.mgrid[0:16, 0:16] / 16.0 * 2 * np.pi
    n = np.stack([0.6 * np.sin(nx), 0.6 * np.cos(ny), np.ones_like(nx)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    bumps = np.concatenate([np.round((n * 0.5 + 0.5) * 255), np.full((16, 16, 1), 255)], -1).astype(np.uint8)
    bump_tex = d.add_texture(16, 16, bumps, wrap_s=0, wrap_t=2)
    mr = np.zeros((8, 8, 4), np.uint8)
    mr[..., 1] = (np.arange(8) * 32 + 16)[None, :]            # roughness across u
    mr[..., 2] = np.where(np.arange(8) < 4, 255, 0)[:, None]  # metal in the top half
    mr_tex = d.add_texture(8, 8, mr, flip_y=True, wrap_s=1, wrap_t=1)
    alpha = np.full((4, 4, 4), 255, np.uint8)
    alpha[..., 3] = np.array([[0, 255, 0, 255], [255, 0, 255, 0]] * 2, np.uint8)
    alpha_tex = d.add_texture(4, 4, alpha)

    floor = d.add_geometry(QUAD * F(3), QUAD_IDX, uvs=QUAD_UV)
    wall = d.add_geometry(np.array([[-3, 0, -2], [3, 0, -2], [3, 3, -2], [-3, 3, -2]], F), [0, 1, 2, 0, 2, 3],
                          uvs=QUAD_UV)
    spos, suv, sidx = uv_sphere(32, 16, 0.6)
    sphere = d.add_geometry(spos, sidx, uvs=suv)
    panel = d.add_geometry(np.array([[-.6, 0, 0], [.6, 0, 0], [.6, 1.2, 0], [-.6, 1.2, 0]], F), [0, 1, 2, 0, 2, 3],
                           uvs=QUAD_UV)
    floor_mat = d.add_material(base_color=(1, 1, 1), roughness=0.6, textures=(floor_tex, NONE, NONE, NONE))
    wall_mat = d.add_material(base_color=(0.7, 0.7, 0.7), roughness=0.4, textures=(NONE, bump_tex, NONE, NONE),
                              extensions=[(45, (0.8, 0.8)), (56, (2.0, 2.0))])
    bumpy = d.add_material(base_color=(0.2, 0.5, 0.8), roughness=0.3, textures=(NONE, bump_tex, NONE, NONE))
    metal = d.add_material(base_color=(0.95, 0.75, 0.45), metalness=1.0, roughness=1.0,
                           textures=(NONE, NONE, mr_tex, NONE))
    glassy = d.add_material(base_color=(0.9, 1.0, 0.9), roughness=0.1, ior=1.5,
                            textures=(alpha_tex, NONE, NONE, NONE), extensions=[(54, 2), (37, 1)])
    d.add_mesh(floor, floor_mat)
    d.add_mesh(wall, wall_mat)
    d.add_mesh(sphere, bumpy, transform=D.translate([-0.9, 0.6, 0]))
    d.add_mesh(sphere, metal, transform=D.translate([0.9, 0.6, 0.2]))
    d.add_mesh(panel, glassy, transform=D.translate([0, 0, 1.0]))
    d.add_light(D.LIGHT_RECT, intensity=6, size=1.0, height_or_inner=0.6, transform=D.look_at([0, 2.8, 0.4], [0, 0, 0]))
    d.add_light(D.LIGHT_SPHERE, color=(1, 0.9, 0.8), intensity=4, size=0.1, transform=D.translate([1.5, 1.5, 1.5]))
    sky = np.zeros((8, 16, 4), F)
    sky[..., :3] = np.linspace(0.2, 1.0, 8, dtype=F)[:, None, None] * np.array([0.5, 0.7, 1.0], F)
    sky[..., 3] = 1
    d.set_environment(d.add_texture_rgba32f(16, 8, sky), intensity=0.5)
    d.set_camera(fov=45, transform=D.look_at([0, 1.6, 4.2], [0, 0.7, 0]))
    return d


def test_textured_scene_oracle_parity(cuda):
    st, msg, host = D.decode(textured_room().to_bytes())
    assert st == abi.MT_OK, msg
    assert host.bundle.map_count == 4 and host.bundle.vertex_layout.uv_offset == 4
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def test_textured_scene_identical_in_every_engine(cuda):
    import torch
    data = textured_room(64, 48).to_bytes()
    st, msg, host = D.decode(data)
    assert st == abi.MT_OK, msg
    dev = scene.DeviceScene(host, cuda)
    alone = trace.Accumulation(64, 48, cuda)
    trace.trace_samples(dev, alone, 6)
    # batch entry point
    batched = trace.Accumulation(64, 48, cuda)
    jobs = (abi.JobDesc * 1)()
    jobs[0].scene, jobs[0].camera, jobs[0].uniform = dev.view, dev.camera, dev.uniform
    jobs[0].out, jobs[0].samples = batched.outputs, 6
    scratch = torch.zeros(abi.lib().mtc_batch_scratch_bytes(1), dtype=torch.uint8, device=cuda)
    abi.check(abi.lib().mtc_trace_batch(jobs, 1, None, C.c_void_p(scratch.data_ptr()), None, None,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    # wavefront engine
    job = batch.RenderJob(dev, 6, device=cuda)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([job])
    sb.run()
    torch.cuda.synchronize()
    for other in (batched, job.acc):
        assert torch.equal(alone.color, other.color) and torch.equal(alone.normal, other.normal)
        assert torch.equal(alone.albedo, other.albedo)
    # the context entry point: same decoded scene, same image
    ctx = Context()
    try:
        ctx.commit_descriptor(data)
        ctx.render(6)
        want = (alone.color.cpu().numpy() / np.float32(6)).reshape(48, 64, 4)
        assert np.array_equal(ctx.read_pixels(), want)
    finally:
        ctx.destroy()
    assert alone.color[:, :3].mean().item() > 0.01


def slots_room(width=96, height=72):
    """Every supported texture slot on one scene: an emissive-mapped lamp
    (sampled by NEE at its UVs), roughness / metalness / specular maps,
    coat weight and coat roughness maps on an emitting coated sphere, fuzz
    maps, transmission and thin-film maps, an alpha map under the opaque
    alpha mode."""
    rng = np.random.default_rng(9)
    d = D.Descriptor(width, height)

    def noise(w, h):
        return d.add_texture(w, h, rng.integers(0, 256, (h, w, 4), dtype=np.uint8))
    yy, xx = np.mgrid[0:8, 0:8]
    glow = np.zeros((8, 8, 4), np.uint8)
    glow[(xx + yy) % 2 == 0] = [255, 200, 120, 255]
    glow[(xx + yy) % 2 == 1] = [60, 120, 255, 255]
    glow_tex = d.add_texture(8, 8, glow)
    floor = d.add_geometry(QUAD * F(3), QUAD_IDX, uvs=QUAD_UV)
    spos, suv, sidx = uv_sphere(24, 12, 0.45)
    sphere = d.add_geometry(spos, sidx, uvs=suv)
    panel = d.add_geometry(np.array([[-.5, 0, 0], [.5, 0, 0], [.5, 1.0, 0], [-.5, 1.0, 0]], F), [0, 1, 2, 0, 2, 3],
                           uvs=QUAD_UV)
    lamp_geo = d.add_geometry(np.array([[-.6, 0, -.4], [.6, 0, -.4], [.6, 0, .4], [-.6, 0, .4]], F),
                              [0, 2, 1, 0, 3, 2], uvs=QUAD_UV)
    floor_mat = d.add_material(base_color=(0.6, 0.6, 0.6), roughness=0.7, extensions=[(40, noise(4, 4)), (41, 1)])
    lamp = d.add_material(emission_color=(1, 1, 1), emission_luminance=5.0, textures=(NONE, NONE, NONE, glow_tex))
    spec = d.add_material(base_color=(0.8, 0.5, 0.3), roughness=0.8, metalness=1.0,
                          extensions=[(47, noise(8, 4)), (48, noise(4, 8)), (68, noise(4, 4)), (69, noise(4, 4))])
    coated = d.add_material(base_color=(0.3, 0.3, 0.3), roughness=0.5, coat_weight=1.0, coat_roughness=0.4,
                            emission_color=(1, 0.5, 0.2), emission_luminance=0.3,
                            extensions=[(26, (0.5, 0.8, 1.0)), (64, noise(8, 8)), (65, noise(8, 8))])
    fuzzy = d.add_material(base_color=(0.5, 0.2, 0.4), roughness=0.6,
                           extensions=[(22, (1.0,)), (66, noise(4, 4)), (67, noise(4, 4))])
    film = d.add_material(base_color=(1, 1, 1), roughness=0.05, transmission=1.0, ior=1.45, thin_walled=True,
                          extensions=[(31, (1.0,)), (32, (0.6,)), (49, noise(4, 4)), (50, noise(8, 8)),
                                      (62, (0.1,)), (63, 1)])
    d.add_mesh(floor, floor_mat)
    d.add_mesh(lamp_geo, lamp, transform=[1, 0, 0, 0, 0, -1, 0, 0, 0, 0, -1, 0, 0, 2.4, -0.3, 1])  # facing down
    d.add_mesh(sphere, spec, transform=D.translate([-1.1, 0.45, 0]))
    d.add_mesh(sphere, coated, transform=D.translate([0, 0.45, -0.4]))
    d.add_mesh(sphere, fuzzy, transform=D.translate([1.1, 0.45, 0]))
    d.add_mesh(panel, film, transform=D.translate([0, 0, 0.9]))
    d.add_light(D.LIGHT_SPHERE, color=(1, 0.95, 0.9), intensity=3, size=0.1, transform=D.translate([1.5, 2.0, 2.0]))
    d.set_camera(fov=45, transform=D.look_at([0, 1.4, 4.0], [0, 0.6, 0]))
    return d


def test_every_slot_scene_oracle_parity(cuda):
    st, msg, host = D.decode(slots_room().to_bytes())
    assert st == abi.MT_OK, msg
    assert host.bundle.map_count == 12 and host.uniform.light_choice_count >= 3
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def projection_room(width=96, height=72):
    """Spherical, cylindrical and triplanar projected checkers on spheres, and
    a triplanar-projected cutout (base-color alpha under mask mode) casting a
    patterned shadow: projected UVs at surface hits and in the shadow rays'
    coverage test."""
    d = D.Descriptor(width, height)
    yy, xx = np.mgrid[0:8, 0:8]
    checker = np.zeros((8, 8, 4), np.uint8)
    checker[(xx + yy) % 2 == 0] = [230, 210, 170, 255]
    checker[(xx + yy) % 2 == 1] = [40, 70, 140, 0]
    tex = d.add_texture(8, 8, checker)
    floor = d.add_geometry(QUAD * F(3), QUAD_IDX)
    spos, suv, sidx = uv_sphere(32, 16, 0.45)
    sphere = d.add_geometry(spos, sidx)                              # no UVs: projections only
    panel = d.add_geometry(np.array([[-.8, 0, -.6], [.8, 0, -.6], [.8, 0, .6], [-.8, 0, .6]], F), QUAD_IDX)
    d.add_mesh(floor, d.add_material(base_color=(0.7, 0.7, 0.7), roughness=0.8))
    for k, proj in enumerate((1, 2, 3)):
        m = d.add_material(base_color=(1, 1, 1), roughness=0.4, textures=(tex, NONE, NONE, NONE),
                           extensions=[(55, proj), (56, (2.0, 3.0))])
        d.add_mesh(sphere, m, transform=D.translate([-1.1 + 1.1 * k, 0.45, 0]))
    cutout = d.add_material(base_color=(1, 1, 1), roughness=0.5, textures=(tex, NONE, NONE, NONE),
                            extensions=[(55, 3), (56, (1.5, 1.5)), (54, 1), (41, 2), (42, (0.5,))])
    d.add_mesh(panel, cutout, transform=D.translate([0, 1.6, 0.2]))
    d.add_light(D.LIGHT_RECT, intensity=8, size=0.8, height_or_inner=0.8, transform=D.look_at([0, 2.8, 0.3], [0, 0, 0]))
    d.set_camera(fov=45, transform=D.look_at([0, 1.4, 3.8], [0, 0.5, 0]))
    return d


def test_projection_scene_oracle_parity(cuda):
    st, msg, host = D.decode(projection_room().to_bytes())
    assert st == abi.MT_OK, msg
    assert host.bundle.flags & abi.MTC_SCENE_HAS_ALPHA and host.bundle.vertex_layout.uv_offset == 0
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def uv1_room(width=96, height=72):
    """Maps on the secondary UV set: a floor whose base color reads UV1 and
    roughness reads UV0, and a lamp whose emissive map reads UV1 (also at its
    NEE light samples)."""
    d = D.Descriptor(width, height)
    yy, xx = np.mgrid[0:8, 0:8]
    checker = np.zeros((8, 8, 4), np.uint8)
    checker[(xx + yy) % 2 == 0] = [230, 200, 150, 255]
    checker[(xx + yy) % 2 == 1] = [40, 60, 120, 255]
    base_tex = d.add_texture(8, 8, checker, uv_channel=1)
    rough = np.zeros((8, 8, 4), np.uint8)
    rough[..., 1] = (np.arange(8) * 30 + 20)[None, :]
    rough_tex = d.add_texture(8, 8, rough)
    glow_tex = d.add_texture(8, 8, checker, uv_channel=1, wrap_s=2, wrap_t=2)
    uv1 = np.array([[0, 0], [4, 0], [4, 4], [0, 4]], F)
    floor = d.add_geometry(QUAD * F(3), QUAD_IDX, uvs=QUAD_UV, uv1s=uv1)
    lamp_geo = d.add_geometry(np.array([[-.6, 0, -.4], [.6, 0, -.4], [.6, 0, .4], [-.6, 0, .4]], F), QUAD_IDX,
                              uvs=QUAD_UV, uv1s=uv1 * F(0.5))
    d.add_mesh(floor, d.add_material(base_color=(1, 1, 1), roughness=0.9, textures=(base_tex, NONE, NONE, NONE),
                                     extensions=[(47, rough_tex)]))
    lamp = d.add_material(emission_color=(1, 1, 1), emission_luminance=4.0, textures=(NONE, NONE, NONE, glow_tex))
    d.add_mesh(lamp_geo, lamp, transform=[1, 0, 0, 0, 0, -1, 0, 0, 0, 0, -1, 0, 0, 2.2, 0, 1])
    d.set_camera(fov=50, transform=D.look_at([0, 1.6, 3.6], [0, 0.2, 0]))
    return d


def test_secondary_uv_scene_oracle_parity(cuda):
    st, msg, host = D.decode(uv1_room().to_bytes())
    assert st == abi.MT_OK, msg
    assert host.bundle.vertex_layout.uv1_offset == 6
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma
