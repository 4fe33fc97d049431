"""Alpha coverage on the host: the descriptor's alpha modes resolved as
resolveMaterialAlphaMode does (MaterialState.ts:251-264) into the packed
rows and the scene's HAS_ALPHA flag, and the CPU oracle's alpha-split
integrator (rayTrace.compute.ts:815-890) with the shadow rays' coverage test
(intersectionAlpha.wgsl.ts): mask-mode materials at full coverage give the
opaque scene's image bit for bit, and a fully transparent blend occluder
leaves the image statistically unchanged."""
import numpy as np
import pytest

from mutracer_b200 import abi
from mutracer_b200 import descriptor as D
from tests import oracle_lib
from tests.test_descriptor import QUAD, QUAD_IDX, base, decoded

F = np.float32
NONE = D.NO_TEXTURE
QUAD_UV = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], F)


def rows(h):
    return h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)


@pytest.mark.parametrize("kw,mode", [
    ({}, 0),
    ({"opacity": 0.5}, 2),
    ({"extensions": [(42, (0.3,))]}, 1),
    ({"extensions": [(41, 2)]}, 1),
    ({"extensions": [(41, 3)]}, 2),
    ({"opacity": 0.5, "extensions": [(41, 1)]}, 0),
    ({"extensions": [(54, 1)]}, 2),
    ({"extensions": [(36, (0.25,))]}, 2),
])
def test_alpha_modes_resolve_like_the_reference(kw, mode):
    d = base()
    m = d.add_material(**kw)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX), m, transform=D.translate([0, 1, 0]))
    h = decoded(d)
    r = rows(h)[m]
    assert r[23, 3] == mode
    assert bool(h.bundle.flags & abi.MTC_SCENE_HAS_ALPHA) == (mode != 0)
    if "opacity" in kw:
        assert r[9, 0] == F(kw["opacity"])
    if kw.get("extensions") and kw["extensions"][0][0] == 42:
        assert r[22, 3] == F(0.3)


def test_alpha_map_under_auto_blends():
    d = base()
    t = d.add_texture(1, 1, np.full((1, 1, 4), 128, np.uint8))
    m = d.add_material(extensions=[(40, t)])
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), m)
    h = decoded(d)
    assert rows(h)[m, 23, 3] == 2 and rows(h)[m, 22, 2] == 0


def room(alpha_kind=None, occluder_opacity=None):
    """A floor under a rect light, a sphere-ish box and an occluding panel
    between light and floor.  alpha_kind "mask1": every material in mask mode
    at full coverage (the HAS_ALPHA code paths with nothing transparent)."""
    d = D.Descriptor(24, 18)
    ext = [(41, 2)] if alpha_kind == "mask1" else []
    floor = d.add_geometry(QUAD * F(2), QUAD_IDX)
    wall = d.add_geometry(np.array([[-2, 0, -1], [2, 0, -1], [2, 2, -1], [-2, 2, -1]], F), [0, 1, 2, 0, 2, 3])
    d.add_mesh(floor, d.add_material(base_color=(0.7, 0.7, 0.7), roughness=0.6, extensions=ext))
    d.add_mesh(wall, d.add_material(base_color=(0.6, 0.3, 0.2), roughness=0.4, extensions=ext))
    if occluder_opacity is not None:
        panel = d.add_geometry(QUAD * F(0.6), QUAD_IDX)
        d.add_mesh(panel, d.add_material(base_color=(0.2, 0.8, 0.2), opacity=occluder_opacity, extensions=[(41, 3)]),
                   transform=D.translate([0, 1.2, 0]))
    d.add_light(D.LIGHT_RECT, intensity=8, size=0.8, height_or_inner=0.8, transform=D.look_at([0, 2.2, 0.01], [0, 0, 0]))
    d.set_camera(fov=50, transform=D.look_at([0, 1.2, 3.0], [0, 0.4, 0]))
    return d


def render(d, spp):
    st, msg, h = D.decode(d.to_bytes())
    assert st == abi.MT_OK, msg
    acc = oracle_lib.Accum(h.width, h.height)
    oracle_lib.trace(h, acc, spp)
    return h, acc


def test_full_coverage_mask_scene_equals_opaque_scene_bit_for_bit():
    h0, a0 = render(room(), 8)
    h1, a1 = render(room("mask1"), 8)
    assert not h0.bundle.flags & abi.MTC_SCENE_HAS_ALPHA and h1.bundle.flags & abi.MTC_SCENE_HAS_ALPHA
    for x, y in ((a0.color, a1.color), (a0.normal, a1.normal), (a0.albedo, a1.albedo)):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_transparent_blend_occluder_changes_nothing_statistically():
    _, plain = render(room(), 256)
    h, clear = render(room(occluder_opacity=0.0), 256)
    assert h.bundle.flags & abi.MTC_SCENE_HAS_ALPHA
    _, solid = render(room(occluder_opacity=1.0), 256)
    lum = lambda a: float(a.resolved()[..., :3].mean())
    assert abs(lum(clear) - lum(plain)) <= 0.02 * lum(plain)
    assert lum(solid) < 0.97 * lum(plain)                 # the opaque panel does shadow the floor


def test_half_covered_occluder_lies_between():
    _, plain = render(room(), 128)
    _, half = render(room(occluder_opacity=0.5), 128)
    _, solid = render(room(occluder_opacity=1.0), 128)
    lum = lambda a: float(a.resolved()[..., :3].mean())
    assert lum(solid) < lum(half) < lum(plain)
