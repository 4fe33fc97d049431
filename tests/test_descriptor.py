"""Scene descriptor v8 ingest on the host (mtp_descriptor_decode, the
decoding mt_context_commit runs): the decoded buffers against independent
NumPy restatements of the reference's conversions (camera-core.ts with the
vendored gl-matrix, packWgpuAnalyticLights + lightsData.ts, vertexNormals.ts,
scaleEnvironment / writeEnvironmentSettings), instancing and materials, and
the validator's rules of native/docs/scene-format.md (malformed descriptors
-> MT_ERROR_INVALID_ARGUMENT; valid ones using features this build does not
render -> MT_ERROR_UNAVAILABLE)."""
import math

import numpy as np
import pytest

from mutracer_b200 import abi
from mutracer_b200 import descriptor as D

F = np.float32
QUAD = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F)
QUAD_IDX = [0, 2, 1, 0, 3, 2]


def base(width=64, height=48):
    d = D.Descriptor(width, height)
    g = d.add_geometry(QUAD, QUAD_IDX)
    m = d.add_material(base_color=(0.7, 0.6, 0.5))
    d.add_mesh(g, m)
    d.add_light(D.LIGHT_RECT, intensity=5, size=0.5, height_or_inner=0.5, transform=D.look_at([0, 2, 0.001], [0, 0, 0]))
    d.set_camera(fov=40, transform=D.look_at([0, 1.5, 3], [0, 0, 0]))
    return d


def decoded(d):
    st, msg, host = D.decode(d.to_bytes())
    assert st == abi.MT_OK, msg
    return host


def rejected(d, status=abi.MT_ERROR_INVALID_ARGUMENT, data=None):
    st, msg, host = D.decode(d.to_bytes() if data is None else data)
    assert host is None and st == status, (st, msg)
    return msg


# ------------------------------------------------------------- restatements
def gl_invert(a):
    a = [float(x) for x in a]
    a00, a01, a02, a03, a10, a11, a12, a13, a20, a21, a22, a23, a30, a31, a32, a33 = a
    b00 = a00 * a11 - a01 * a10; b01 = a00 * a12 - a02 * a10; b02 = a00 * a13 - a03 * a10
    b03 = a01 * a12 - a02 * a11; b04 = a01 * a13 - a03 * a11; b05 = a02 * a13 - a03 * a12
    b06 = a20 * a31 - a21 * a30; b07 = a20 * a32 - a22 * a30; b08 = a20 * a33 - a23 * a30
    b09 = a21 * a32 - a22 * a31; b10 = a21 * a33 - a23 * a31; b11 = a22 * a33 - a23 * a32
    det = 1.0 / (b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06)
    return [(a11 * b11 - a12 * b10 + a13 * b09) * det, (a02 * b10 - a01 * b11 - a03 * b09) * det,
            (a31 * b05 - a32 * b04 + a33 * b03) * det, (a22 * b04 - a21 * b05 - a23 * b03) * det,
            (a12 * b08 - a10 * b11 - a13 * b07) * det, (a00 * b11 - a02 * b08 + a03 * b07) * det,
            (a32 * b02 - a30 * b05 - a33 * b01) * det, (a20 * b05 - a22 * b02 + a23 * b01) * det,
            (a10 * b10 - a11 * b08 + a13 * b06) * det, (a01 * b08 - a00 * b10 - a03 * b06) * det,
            (a30 * b04 - a31 * b02 + a33 * b00) * det, (a21 * b02 - a20 * b04 - a23 * b00) * det,
            (a11 * b07 - a10 * b09 - a12 * b06) * det, (a00 * b09 - a01 * b07 + a02 * b06) * det,
            (a31 * b01 - a30 * b03 - a32 * b00) * det, (a20 * b03 - a21 * b01 + a22 * b00) * det]


def gl_mul(a, b):
    out = [0.0] * 16
    for c in range(4):
        b0, b1, b2, b3 = b[c * 4: c * 4 + 4]
        for k in range(4):
            out[c * 4 + k] = b0 * a[k] + b1 * a[4 + k] + b2 * a[8 + k] + b3 * a[12 + k]
    return out


def f32(x):
    return float(F(x))


def camera_uniform(width, height, fov, near, far, zoom, f_stop, focus, sensor, mpu, world, ortho=None):
    world = [f32(v) for v in world]
    fov, near, far, zoom = f32(fov), f32(near), f32(far), f32(zoom)
    if ortho is None:
        eff = 2 * math.atan(math.tan(fov * math.pi / 180 / 2) / max(zoom, 2.220446049250313e-16))
        f = 1.0 / math.tan(eff / 2)
        nf = 1 / (near - far)
        proj = [f / (width / height), 0, 0, 0, 0, f, 0, 0, 0, 0, (far + near) * nf, -1, 0, 0, 2 * far * near * nf, 0]
    else:
        l, r, b, t = (f32(v) for v in ortho)
        left, right = (l + r) / 2 - (r - l) / (2 * zoom), (l + r) / 2 + (r - l) / (2 * zoom)
        bottom, top = (b + t) / 2 - (t - b) / (2 * zoom), (b + t) / 2 + (t - b) / (2 * zoom)
        lr, bt, nf = 1 / (left - right), 1 / (bottom - top), 1 / (near - far)
        proj = [-2 * lr, 0, 0, 0, 0, -2 * bt, 0, 0, 0, 0, 2 * nf, 0, (left + right) * lr, (top + bottom) * bt,
                (far + near) * nf, 1]
    vp = np.array(gl_mul(world, gl_invert(proj)), F)
    radius = 0.0
    f_stop, mpu, sensor = f32(f_stop), f32(mpu), f32(sensor)
    if f_stop > 0 and mpu > 0:
        focal = 0.5 * sensor * max(zoom, 2.220446049250313e-16) / math.tan(fov * math.pi / 360) if ortho is None else 0
        radius = focal / (2 * f_stop) / 1000 / mpu
        radius = radius if math.isfinite(radius) and radius > 0 else 0.0
    return vp, np.array(world, F), F(radius), F(focus)


def rigid_frame(m):
    def normalize(v, fb):
        n = math.hypot(*v)
        return [x / n for x in v] if n > 1e-12 else list(fb)
    z = normalize([m[8], m[9], m[10]], [0, 0, 1])
    p = m[0] * z[0] + m[1] * z[1] + m[2] * z[2]
    x = [m[0] - p * z[0], m[1] - p * z[1], m[2] - p * z[2]]
    if math.hypot(*x) <= 1e-12:
        x = [z[2], 0, -z[0]] if abs(z[1]) < .99 else [1, 0, 0]
    x = normalize(x, [1, 0, 0])
    y = [z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]]
    return x, y, [(-c) or 0.0 for c in z]


def light_rows(kind, color, intensity, size, hi, so, m, radius=0.0, length=0.0, normalize=False):
    """packWgpuAnalyticLights (wgpuSceneUniform.ts:70-152) for one light."""
    m = [f32(v) for v in m]
    color = [f32(c) for c in color]
    intensity, size, hi, so, radius, length = (f32(v) for v in (intensity, size, hi, so, radius, length))
    x, y, d = rigid_frame(m)
    r = np.zeros(24, F)
    r[0:3] = m[12:15]
    scale = intensity
    if kind == D.LIGHT_RECT:
        r[3], r[7] = 3, size * hi
        r[8:11] = [v * size for v in x]; r[11] = so; r[12:15] = [v * -hi for v in y]
    elif kind == D.LIGHT_SPHERE:
        r[3], r[7], r[11] = 2, 4 * math.pi * size ** 2, size
    elif kind == D.LIGHT_DIRECTIONAL:
        r[3] = 1; r[8:11] = d
    elif kind == D.LIGHT_SPOT:
        r[3], r[7], r[11] = 4, 4 * math.pi * size ** 2, size
        scale = intensity if size == 0 else intensity / (math.pi * size ** 2)
        r[8:11] = d
        r[12:14] = [math.cos(so * math.pi / 180), math.cos(min(hi, so) * math.pi / 180)]
    elif kind == D.LIGHT_DISK:
        area = math.pi * radius ** 2
        scale = intensity / max(area, 1e-8) if normalize else intensity
        r[3], r[7], r[11] = 5, area, radius
        r[8:11] = [v * radius for v in x]; r[12:15] = [v * -radius for v in y]
    else:
        area = 2 * math.pi * radius * length
        scale = intensity / max(area, 1e-8) if normalize else intensity
        r[3], r[7], r[11] = 6, area, radius
        r[8:11] = [v * length for v in x]; r[12:15] = [v * radius for v in y]
    r[4:7] = [c * scale for c in color]
    r[15] = -1
    r[20:23] = x
    return r


def vertex_normals(pos, idx):
    """accumulateVertexNormals (vertexNormals.ts:9-52) in f32 storage."""
    n = np.zeros(pos.shape, F)
    for t in range(0, len(idx), 3):
        i1, i2, i3 = idx[t:t + 3]
        p1, p2, p3 = pos[i1].astype(np.float64), pos[i2].astype(np.float64), pos[i3].astype(np.float64)
        v21, v32 = (p1 - p2).astype(F).astype(np.float64), (p2 - p3).astype(F).astype(np.float64)
        c = np.array([v21[1] * v32[2] - v21[2] * v32[1], v21[2] * v32[0] - v21[0] * v32[2],
                      v21[0] * v32[1] - v21[1] * v32[0]]).astype(F).astype(np.float64)
        for i in (i1, i2, i3):
            n[i] = (n[i].astype(np.float64) + c).astype(F)
    out = np.zeros_like(n)
    for i, v in enumerate(n.astype(np.float64)):
        ln = float(v @ v)
        if ln > 0:
            ln = 1 / math.sqrt(ln)
        out[i] = (v * ln).astype(F)
    return out


# ------------------------------------------------------------------ tests
@pytest.mark.parametrize("kw", [dict(fov=40), dict(fov=60, zoom=2.0, f_stop=2.8, focus_distance=3.0),
                                dict(fov=25, near=0.5, far=50, f_stop=1.4, sensor_height=36, meters_per_unit=0.01)])
def test_perspective_camera(kw):
    d = base(80, 50)
    world = D.look_at([1, 2, 4], [0, 0.5, 0])
    d.set_camera(transform=world, **kw)
    cam = decoded(d).bundle.camera
    full = dict(fov=45.0, near=0.1, far=1000.0, zoom=1.0, f_stop=0.0, focus_distance=10.0, sensor_height=24.0,
                meters_per_unit=1.0)
    full.update(kw)
    vp, view, radius, focus = camera_uniform(80, 50, full["fov"], full["near"], full["far"], full["zoom"],
                                             full["f_stop"], full["focus_distance"], full["sensor_height"],
                                             full["meters_per_unit"], world)
    assert np.array_equal(np.array(cam.view_projection_inv, F), vp)
    assert np.array_equal(np.array(cam.view_inv, F), view)
    assert F(cam.aperture_radius) == radius and F(cam.focus_distance) == focus


def test_orthographic_camera():
    d = base(64, 64)
    world = D.look_at([0, 5, 0.5], [0, 0, 0])
    d.set_camera(projection=1, left=-2, right=2, bottom=-1.5, top=1.5, near=0.1, far=20, zoom=1.25, f_stop=2.0,
                 transform=world)
    cam = decoded(d).bundle.camera
    vp, _, radius, _ = camera_uniform(64, 64, 45, 0.1, 20, 1.25, 2.0, 10, 24, 1, world, ortho=(-2, 2, -1.5, 1.5))
    assert np.array_equal(np.array(cam.view_projection_inv, F), vp)
    assert cam.aperture_radius == 0.0          # no lens for an orthographic camera


def test_light_rows_every_type():
    d = base()
    d.lights = []
    m1 = D.look_at([0.3, 2, 0.2], [0, 0, 0])
    m2 = [0.5, 0, 0, 0, 0, 2, 0, 0, 0, 0, 1, 0, 1, 2, 3, 1]            # scaled, not rigid
    specs = [(D.LIGHT_RECT, (1, .9, .8), 7, .5, .25, .6, m1, 0, 0, False),
             (D.LIGHT_SPHERE, (1, 1, 1), 3, .2, 0, 0, m2, 0, 0, False),
             (D.LIGHT_SPHERE, (.2, .4, .6), 12, 0, 0, 0, m1, 0, 0, False),
             (D.LIGHT_DIRECTIONAL, (1, 1, .5), 2, 0, 0, 0, m1, 0, 0, False),
             (D.LIGHT_SPOT, (1, .5, .25), 12, .1, 10, 30, m1, 0, 0, False),
             (D.LIGHT_SPOT, (1, .5, .25), 12, 0, 20, 20, m2, 0, 0, False),
             (D.LIGHT_DISK, (1, 1, 1), 4, 0, 0, 0, m1, .3, 0, True),
             (D.LIGHT_CYLINDER, (.5, 1, 1), 4, 0, 0, 0, m2, .1, 2.0, False)]
    for k, c, i, s, hi, so, m, r, ln, nz in specs:
        d.add_light(k, color=c, intensity=i, size=s, height_or_inner=hi, spread_or_outer=so, transform=m, radius=r,
                    length=ln, normalize=nz)
    h = decoded(d)                                   # keeps the host arrays alive
    rows = h.lights.reshape(-1, 24)
    for got, (k, c, i, s, hi, so, m, r, ln, nz) in zip(rows, specs):
        want = light_rows(k, c, i, s, hi, so, m, r, ln, nz)
        mask = np.ones(24, bool)
        mask[16] = False                                              # selection pmf: checked below
        assert np.array_equal(got[mask], want[mask]), (k, got, want)
    assert abs(rows[:, 16].sum() - 1) < 1e-6 and (rows[:, 16] > 0).all()


def test_generated_normals_equal_restatement():
    rng = np.random.default_rng(4)
    pos = rng.normal(size=(30, 3)).astype(F)
    idx = rng.integers(0, 30, size=60).astype(np.uint32)
    gen, given = D.Descriptor(16, 16), D.Descriptor(16, 16)
    for d, normals in ((gen, None), (given, vertex_normals(pos, idx))):
        g = d.add_geometry(pos, idx, normals=normals)
        d.add_mesh(g, d.add_material())
    a, b = decoded(gen), decoded(given)
    assert np.array_equal(a.attributes, b.attributes)
    assert np.array_equal(a.bvh.view(np.uint32), b.bvh.view(np.uint32))


def test_instancing_hidden_meshes_and_materials():
    d = D.Descriptor(32, 32)
    g = d.add_geometry(QUAD, QUAD_IDX)
    m0 = d.add_material(base_color=(1, 0, 0), roughness=0.6, metalness=0.25, ior=1.33)
    m1 = d.add_material(extensions=[(6, (0.5, 0.6, 0.7)), (29, (1.8,)), (22, (0.4,)), (23, (0.1, 0.2, 0.3)),
                                    (31, (0.5,)), (32, (0.7,)), (38, 1)])
    d.add_mesh(g, m0)
    d.add_mesh(g, m1, hidden=True)
    transforms = np.array([D.translate([k, 0, 0]) for k in range(3)], F)
    colors = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1]], F)
    d.add_mesh(g, m1, transform=D.translate([0, 1, 0], 2.0), batch=(transforms, colors))
    h = decoded(d)
    assert h.info.instances == 4 and h.info.blases == 1
    rec = h.instances.reshape(-1, 40)
    # instance records: material word, colors, local-to-world of batch members (mesh world outside local)
    mats = sorted(int(v) for v in rec[:, 2].view(np.int32))
    assert mats == [255, 255 + 256, 255 + 256, 255 + 256]
    got_colors = sorted(map(tuple, rec[:, 36:39].tolist()))
    assert got_colors == sorted([(1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1)])
    translations = sorted(map(tuple, rec[:, 32:35].tolist()))
    assert translations == sorted([(0, 0, 0), (0, 1, 0), (2, 1, 0), (4, 1, 0)])
    rows = h.materials.reshape(-1, 26, 4)
    assert np.allclose(rows[0, 0, :3], [1, 0, 0]) and np.isclose(rows[0, 1, 0], 0.6)
    assert np.isclose(rows[0, 2, 0], 0.25) and np.isclose(rows[0, 4, 0], 1.33)
    assert np.allclose(rows[1, 11, :3], [0.5, 0.6, 0.7]) and np.isclose(rows[1, 17, 2], 1.8)
    assert np.isclose(rows[1, 11, 3], 0.4) and np.allclose(rows[1, 15, :3], [0.1, 0.2, 0.3])
    assert np.isclose(rows[1, 18, 0], 0.5) and np.isclose(rows[1, 5, 2], 0.7) and rows[1, 23, 2] == 1


def test_environment_settings():
    d = base()
    px = np.random.default_rng(1).uniform(0, 2, size=(8, 16, 4)).astype(F)
    t = d.add_texture_rgba32f(16, 8, px)
    d.set_environment(t, intensity=2.5, yaw=0.7, background_intensity=0.5, background_yaw=1.1)
    d.background = (0.1, 0.2, 0.3, 1.0)
    h = decoded(d)
    want = px.reshape(-1, 4).copy()
    want[:, :3] = (want[:, :3].astype(np.float64) * 2.5).astype(F)
    assert np.array_equal(h.env_map.reshape(-1, 4), want)
    import ctypes as C
    dist = np.zeros(18 * 9 * 2, F)
    power = C.c_double()
    abi.lib().mtp_env_distribution(want.ctypes.data, 16, 8, dist.ctypes.data, C.byref(power))
    assert np.array_equal(h.env_distribution, dist)
    u = h.uniform
    c, s = math.cos(F(0.7)), math.sin(F(0.7))
    assert np.array_equal(np.array(u.environment_rotation, F),
                          np.array([c, 0, -s, 0, 0, 1, 0, 0, s, 0, c, 0, 0, 0, 0, 1], F))
    assert np.allclose(u.background_map_transform, [math.cos(F(1.1)), math.sin(F(1.1)), 0.5, 0])
    assert u.background_flags == 1 and np.allclose(u.background_color, [0.1, 0.2, 0.3, 1.0])
    assert u.scene_feature_flags & abi.MTC_FEATURE_USE_ENVMAP
    d.quality = D.QUALITY_HIDE_BACKGROUND | D.QUALITY_DISPERSION
    u = decoded(d).uniform
    assert u.background_flags == 0 and u.dispersion_wavelengths == 3


def _variant(mutate):
    d = base()
    data = np.frombuffer(d.to_bytes(), np.uint32).copy()
    mutate(d, data)
    return d, data


def _geom_word(data, k):
    return int(data[9]) + k


@pytest.mark.parametrize("name,mutate", [
    ("version", lambda d, w: w.__setitem__(0, 9)),
    ("total_words", lambda d, w: w.__setitem__(1, int(w[1]) + 1)),
    ("table outside", lambda d, w: w.__setitem__(12, int(w[1]) + 100)),
    ("table inside header", lambda d, w: w.__setitem__(11, 4)),
    ("no geometry", lambda d, w: w.__setitem__(4, 0)),
    ("size", lambda d, w: w.__setitem__(2, 9000)),
    ("quality bits", lambda d, w: w.__setitem__(22, 8)),
    ("reserved header", lambda d, w: w.__setitem__(15, 1)),
    ("reserved end", lambda d, w: w.__setitem__(30, 1)),
    ("nan background", lambda d, w: w.__setitem__(16, 0x7FC00000)),
    ("index past vertices", lambda d, w: w.__setitem__(int(w[_geom_word(w, 3)]), 99)),
    ("nan position", lambda d, w: w.__setitem__(int(w[_geom_word(w, 2)]) + 1, 0x7FC00000)),
    ("mesh geometry", lambda d, w: w.__setitem__(int(w[10]), 5)),
    ("mesh material", lambda d, w: w.__setitem__(int(w[10]) + 1, 3)),
    ("mesh flags", lambda d, w: w.__setitem__(int(w[10]) + 20, 2)),
    ("non-affine", lambda d, w: w.__setitem__(int(w[10]) + 4 + 3, np.array([0.5], F).view(np.uint32)[0])),
    ("singular", lambda d, w: w.__setitem__(int(w[10]) + 4, 0)),
    ("thin walled", lambda d, w: w.__setitem__(int(w[11]) + 14, 2)),
    ("camera projection", lambda d, w: w.__setitem__(int(w[14]), 2)),
    ("camera fov", lambda d, w: w.__setitem__(int(w[14]) + 1, np.array([0], F).view(np.uint32)[0])),
    ("camera reserved", lambda d, w: w.__setitem__(int(w[14]) + 13, 1)),
    ("light type", lambda d, w: w.__setitem__(int(w[12]), 6)),
    ("rect size", lambda d, w: w.__setitem__(int(w[12]) + 5, 0)),
    ("light reserved", lambda d, w: w.__setitem__(int(w[12]) + 11, 1)),
])
def test_malformed_descriptors_are_rejected(name, mutate):
    d, data = _variant(mutate)
    msg = rejected(d, data=data.tobytes())
    assert msg


def test_rejects_short_and_misaligned_buffers():
    assert D.decode(b"")[0] == abi.MT_ERROR_INVALID_ARGUMENT
    assert D.decode(base().to_bytes()[:-2])[0] == abi.MT_ERROR_INVALID_ARGUMENT
    assert D.decode(bytes(64))[0] == abi.MT_ERROR_INVALID_ARGUMENT


def test_spot_and_triangle_material_rules():
    d = base()
    d.add_light(D.LIGHT_SPOT, intensity=1, size=0, height_or_inner=40, spread_or_outer=30)
    assert "spot" in rejected(d)
    d = D.Descriptor(16, 16)
    g = d.add_geometry(QUAD, QUAD_IDX, material_indices=[0, 0, 1, 0])
    a, b = d.add_material(), d.add_material()
    d.add_mesh(g, a, material_table=[a, b])
    assert "same material" in rejected(d)


@pytest.mark.parametrize("name,build", [
    ("displacement map", lambda d: d.add_material(
        extensions=[(59, d.add_texture(1, 1, np.zeros((1, 1, 4), np.uint8)))])),
    ("alpha in a spectral scene", lambda d: d.add_mesh(0, d.add_material(opacity=0.5, extensions=[(15, (0.5,))]))),

    ("extension", lambda d: d.add_material(extensions=[(53, (0.1,))])),
    ("unlit", lambda d: d.add_material(extensions=[(52, 1)])),
    ("bevel", lambda d: setattr(d, "quality", D.QUALITY_BEVEL)),
])
def test_unsupported_features_are_named(name, build):
    d = base()
    build(d)
    msg = rejected(d, abi.MT_ERROR_UNAVAILABLE)
    assert "not supported" in msg


def test_multi_material_meshes_use_the_triangle_material_plane():
    """decodeMeshMaterials + packTriangleMaterials: the instance record
    carries the table's first material; every triangle record's plane word
    holds its vertices' table entry + 1; a geometry shared by meshes with
    different tables gets one BLAS per table."""
    d = D.Descriptor(16, 16)
    g = d.add_geometry(np.concatenate([QUAD, QUAD + F(3)]), QUAD_IDX + [i + 4 for i in QUAD_IDX],
                       material_indices=[0, 0, 0, 0, 1, 1, 1, 1])
    a, b, c = d.add_material(base_color=(1, 0, 0)), d.add_material(base_color=(0, 1, 0)), d.add_material()
    d.add_mesh(g, a, material_table=[a, b])
    d.add_mesh(g, a, material_table=[c, a], transform=D.translate([0, 5, 0]))
    d.add_mesh(g, a, material_table=[a, b], transform=D.translate([0, 9, 0]))   # shares the first BLAS
    h = decoded(d)
    ins = h.instances.reshape(-1, 40)
    assert sorted(int(x) for x in ins[:, 2].view(np.int32)) == [255 + (a << 8), 255 + (a << 8), 255 + (c << 8)]
    plane = h.triangle_materials
    assert plane is not None and plane.size == h.bundle.bvh_vec4_count
    info = h.info
    assert info.blases == 2
    # every triangle record (first word < 8 inside a BLAS) carries its table entry
    words = h.bvh.reshape(-1, 4).view(np.uint32)
    tl = h.uniform.blas_offset
    recs = [r for r in range(tl, len(words)) if plane[r]]
    assert set(int(plane[r]) for r in recs) == {a + 1, b + 1, c + 1}
    assert not plane[:tl].any()
    # uniform per-vertex indices: every triangle takes the table entry
    d = D.Descriptor(16, 16)
    g = d.add_geometry(QUAD, QUAD_IDX, material_indices=[1, 1, 1, 1])
    a, b = d.add_material(base_color=(1, 0, 0)), d.add_material(base_color=(0, 1, 0))
    d.add_mesh(g, a, material_table=[a, b])
    h = decoded(d)
    assert int(h.instances.reshape(-1, 40)[0, 2:3].view(np.int32)[0]) == 255 + (a << 8)
    assert set(int(x) for x in h.triangle_materials if x) == {b + 1}
    # no per-vertex materials: no plane
    assert decoded(base()).triangle_materials is None



def test_emissive_meshes_enter_the_light_table():
    """collectEmissiveTriangles / packEmissiveTriangles / prepareSceneLightSampling:
    world-space corners, areas, material index and selection pmf per triangle,
    then the choice table; weights are area x luminance(materialEmission)."""
    d = base()
    g = d.add_geometry(QUAD * F(0.5), QUAD_IDX)
    lamp = d.add_material(emission_color=(1.0, 0.8, 0.6), emission_luminance=4.0, coat_weight=0.5,
                          extensions=[(26, (0.25, 0.5, 1.0))])
    world = D.translate([0.5, 1.0, -0.25], 2.0)
    d.add_mesh(g, lamp, transform=world)
    h = decoded(d)
    u = h.uniform
    assert u.light_choice_texel_offset == 12 and u.light_choice_count == 1 + 2   # rect light + 2 triangles
    tex = h.light_sampling.reshape(-1, 4)
    pos = (QUAD * F(0.5)).astype(np.float64)
    wm = np.array(world, np.float64).reshape(4, 4).T
    wpos = ((wm[:3, :3] @ pos.T).T + wm[:3, 3]).astype(F)
    emission = np.array([1.0, 0.8, 0.6]) * 4.0
    emission *= 1 + 0.5 * (np.sqrt(np.array([0.25, 0.5, 1.0])) - 1)
    lum = max(float(emission @ [0.2126, 0.7152, 0.0722]), 0.0)
    pmfs = []
    for t in range(2):
        tri = wpos[QUAD_IDX[t * 3: t * 3 + 3]]
        rows = tex[t * 6: t * 6 + 6]
        assert np.array_equal(rows[0, :3], tri[0]) and np.array_equal(rows[1, :3], tri[1])
        assert np.array_equal(rows[2, :3], tri[2]) and rows[2, 3] == lamp
        e0, e1 = (tri[1] - tri[0]).astype(F), (tri[2] - tri[0]).astype(F)
        cr = np.cross(e0.astype(np.float64), e1.astype(np.float64)).astype(F).astype(np.float64)
        area = 0.5 * math.sqrt(float(cr @ cr))
        assert rows[1, 3] == F(area)
        pmfs.append(rows[0, 3])
    rect_power = 5 * math.pi * 0.25                      # intensity 5, 0.5 x 0.5 rect, white
    total = rect_power + 2 * area * lum
    assert abs(u.light_weight_total - total) < 1e-4 * total
    assert all(abs(p - area * lum / total) < 1e-6 for p in pmfs)
    mat_rows = h.materials.reshape(-1, 26, 4)
    assert np.allclose(mat_rows[lamp, 3, :3], emission.astype(F))


def test_vertex_colors_pack_like_compact_vertices():
    """compactVertices.ts:7-27, 79-88: RGBA8 words (Math.round(c * 255),
    alpha 255) when every component lies in [0, 1], f32x3 otherwise; meshes
    without colors are white."""
    d = base()
    cols = np.array([[0.0, 0.5, 1.0], [0.2, 0.4, 0.6], [1.0, 1.0, 1.0], [0.1, 0.9, 0.33]], F)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, colors=cols), 0, transform=D.translate([0, 1, 0]))
    h = decoded(d)
    lay = h.bundle.vertex_layout
    assert (lay.stride, lay.color_offset, lay.color_float) == (5, 4, 0)
    words = h.attributes.reshape(-1, 5)
    want = [int(np.floor(np.float64(r) * 255 + 0.5)) | int(np.floor(np.float64(g) * 255 + 0.5)) << 8 |
            int(np.floor(np.float64(b) * 255 + 0.5)) << 16 | 0xff000000 for r, g, b in cols]
    assert words[4:, 4].tolist() == want
    assert (words[:4, 4] == 0xffffffff).all()                      # the base quad: white
    d = base()
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, colors=cols * F(2)), 0)
    h = decoded(d)
    lay = h.bundle.vertex_layout
    assert (lay.stride, lay.color_offset, lay.color_float) == (7, 4, 1)
    words = h.attributes.reshape(-1, 7)
    assert np.array_equal(words[4:, 4:7].view(F), cols * F(2)) and np.array_equal(words[:4, 4:7].view(F), np.ones((4, 3), F))
