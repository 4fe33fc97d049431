"""Material textures on the host: descriptor texture records decoded into the
map table (scene-records.ts decodeTexture, MaterialData.ts, textureAtlas.ts,
textureAtlasPixels.ts, float16.ts), the texture rules of the reference's
validator, and the CPU restatement of sampleMap (materialBuffer.wgsl.ts
:316-378) against an independent float32 NumPy evaluation.

Pinned to the reference's own vectors in tests/unit/rawMaterialTextures.test.ts:
the half-float table (:93-97), HDR data kept in RGBA16F storage with one map
per texture (:35-47), and flip_y / byte sources in float storage (:49-66)."""
import numpy as np
import pytest

from mutracer_b200 import abi
from mutracer_b200 import descriptor as D
from tests import oracle_lib
from tests.test_descriptor import QUAD, QUAD_IDX, base, decoded, rejected

F = np.float32
NONE = D.NO_TEXTURE
QUAD_UV = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], F)


def half_bits(values):
    with np.errstate(over="ignore"):  # 65520 is stored as infinity
        return np.asarray(values, F).astype(np.float16).view(np.uint16)


def maps_of(host):
    rows = host.maps.reshape(-1, abi.MTC_MAP_VEC4_ROWS, 4)
    heads = rows[:, 0, :3].copy().view(np.uint32)
    return rows, heads


def texels_of(host, index):
    rows, heads = maps_of(host)
    w, h, first = (int(x) for x in heads[index])
    return host.map_texels.reshape(-1, 4)[first:first + w * h].reshape(h, w, 4).copy()


def textured(pixels, storage=0, slot=0, **kw):
    """base() with one textured material on a UV quad; `slot` 0 map, 1 normal,
    2 metallic-roughness."""
    d = base()
    h, w = np.asarray(pixels).shape[:2]
    t = d.add_texture(w, h, pixels, storage=storage, **kw)
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    slots = [NONE] * 4
    slots[slot] = t
    m = d.add_material(textures=tuple(slots))
    d.add_mesh(g, m, transform=D.translate([0, 0.5, 0]))
    return d, m


# ----------------------------------------------------------- storage
def test_half_float_table_matches_reference_vectors():
    # rawMaterialTextures.test.ts:93-97 (the finite entries)
    values = [0.0, -0.0, 1.0, -2.0, 65504.0, 65520.0, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -25, 2.0 ** -14,
              1 + 2.0 ** -11, 1 + 3 * 2.0 ** -11]
    bits = [0, 0x8000, 0x3c00, 0xc000, 0x7bff, 0x7c00, 1, 0, 2, 0x400, 0x3c00, 0x3c02]
    pixels = np.array(values, F).reshape(1, 3, 4)
    d, _ = textured(pixels, storage=1)
    h = decoded(d)  # keeps the decoded scene alive while its arrays are read
    got = texels_of(h, 0).reshape(-1)
    assert half_bits(got).tolist() == bits
    assert np.signbit(got[1])


def test_hdr_data_kept_in_half_float_and_one_map_per_texture():
    # rawMaterialTextures.test.ts:35-47: one texture in three slots is one map.
    d = base()
    t = d.add_texture_rgba32f(1, 1, [2, .5, .25, .75])
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    m = d.add_material(textures=(t, t, t, NONE))
    d.add_mesh(g, m)
    h = decoded(d)
    rows, heads = maps_of(h)
    assert len(rows) == 1 and rows[0, 2, 1] == 1.0                       # color linear
    assert half_bits(texels_of(h, 0).reshape(-1)).tolist() == [0x4000, 0x3800, 0x3400, 0x3a00]
    mat = h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)[m]
    assert mat[2, 2] == 0 and mat[1, 1] == 0 and mat[2, 3] == 0          # map, normal, metallic-roughness


def test_flip_y_and_byte_sources_in_float_storage():
    # rawMaterialTextures.test.ts:49-66: a byte texture beside a float one is
    # stored as half floats of byte / 255; flip_y reverses the rows.
    d = base()
    byte = d.add_texture(1, 2, np.array([[[255, 128, 0, 255]], [[0, 0, 0, 0]]], np.uint8))
    raw = d.add_texture_rgba32f(1, 2, [2, .5, 0, .75, 4, 1, 0, .25], flip_y=True, uv_channel=1)
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    d.add_mesh(g, d.add_material(textures=(byte, NONE, NONE, NONE)))
    d.add_mesh(g, d.add_material(textures=(raw, NONE, NONE, NONE)), transform=D.translate([0, 1, 0]))
    h = decoded(d)
    rows, _ = maps_of(h)
    assert rows[:, 2, 1].tolist() == [0, 1] and rows[:, 2, 0].tolist() == [0, 1]
    expect_byte = [0x3c00, int(half_bits([np.float64(128) / 255])[0]), 0, 0x3c00, 0, 0, 0, 0]
    assert half_bits(texels_of(h, 0).reshape(-1)).tolist() == expect_byte
    assert half_bits(texels_of(h, 1).reshape(-1)).tolist() == [0x4400, 0x3c00, 0, 0x3400, 0x4000, 0x3800, 0, 0x3a00]


def test_rgba8_texels_are_bytes_over_255_with_rows_flipped():
    rng = np.random.default_rng(3)
    pixels = rng.integers(0, 256, (3, 5, 4), dtype=np.uint8)
    d, m = textured(pixels, flip_y=True, uv_scale=(2, -1), uv_offset=(0.25, 0.5), wrap_s=2, wrap_t=1)
    h = decoded(d)
    want = pixels[::-1].astype(F) / F(255)
    assert np.array_equal(texels_of(h, 0), want)
    rows, heads = maps_of(h)
    assert heads[0].tolist() == [5, 3, 0]
    assert rows[0, 1].tolist() == [2, -1, 0.25, 0.5]
    assert rows[0, 2].tolist() == [0, 0, 2, 1]                            # uv set, sRGB, mirror, clamp


def test_material_rows_and_map_order():
    """MaterialData order: all base-color maps, then normal maps, then
    metallic-roughness maps; a shared pixel source is stored once."""
    d = base()
    px = np.full((2, 2, 4), 200, np.uint8)
    a = d.add_texture(2, 2, px)
    b = d.add_texture(2, 2, None, pixels_offset=d.texture_pixels_offset(a), wrap_s=1)  # same pixels
    n = d.add_texture(2, 2, np.full((2, 2, 4), 128, np.uint8))
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    m0 = d.add_material(textures=(NONE, n, b, NONE), extensions=[(45, (0.5, -2.0)), (56, (3.0, 4.0)), (54, 2)])
    m1 = d.add_material(textures=(a, NONE, NONE, NONE))
    d.add_mesh(g, m0)
    d.add_mesh(g, m1)
    h = decoded(d)
    rows, heads = maps_of(h)
    assert len(rows) == 3                                                # a (map), n (normal), b (mr)
    assert heads[0, 2] == heads[2, 2] and heads[1, 2] != heads[0, 2]     # b reuses a's texels
    assert rows[2, 2, 2] == 1 and rows[0, 2, 2] == 0
    mats = h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)
    assert mats[m0, 1, 1:].tolist() == [1, 0.5, -2.0]
    assert mats[m0, 2, 2:].tolist() == [-1, 2] and mats[m1, 2, 2:].tolist() == [0, -1]
    assert mats[m0, 5, 3] == 3 and mats[m1, 5, 3] == 0                  # transmission, opaque
    assert mats[m0, 7, 2:].tolist() == [3, 4] and mats[m1, 7, 2:].tolist() == [1, 1]


def test_vertex_layout_carries_uvs_only_when_maps_sample_them():
    d, _ = textured(np.zeros((1, 1, 4), np.uint8))
    h = decoded(d)
    lay = h.bundle.vertex_layout
    assert (lay.stride, lay.uv_offset) == (6, 4)
    words = h.attributes.reshape(-1, 6)
    assert np.array_equal(words[-4:, 4:6].view(F), QUAD_UV)             # the textured quad's vertices
    assert not words[:4, 4:6].any()                                      # base quad: no UVs -> zero
    d = base()
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), 0)
    lay = decoded(d).bundle.vertex_layout
    assert (lay.stride, lay.uv_offset) == (4, 0)


# ---------------------------------------------------------- validation
def _texture_word(d, k, value):
    def edit(words):
        o = int(words[13]) + k
        words[o] = value
    return edit


@pytest.mark.parametrize("k,value", [(0, 0), (1, 16385), (2, 2), (4, 2), (5, 2), (10, 3), (11, 3), (12, 2),
                                     (3, 0x7fffffff), (6, 0x7fc00000)])
def test_invalid_texture_records_are_rejected(k, value):
    d, _ = textured(np.zeros((1, 1, 4), np.uint8))
    w = np.frombuffer(d.to_bytes(), np.uint32).copy()
    _texture_word(d, k, value)(w)
    rejected(d, data=w.tobytes())


def test_texture_rejections_of_pixels_udim_and_references():
    d, _ = textured(np.array([[[1, 2, np.nan, 4]]], F), storage=1)
    assert "finite" in rejected(d)
    d, _ = textured(np.zeros((3, 15, 4), np.uint8), udim=1)               # udim needs multiples of ten
    rejected(d)
    d = base()
    d.add_material(textures=(3, NONE, NONE, NONE))
    assert "out of range" in rejected(d)
    d = base()
    d.add_material(extensions=[(44, 7)])
    assert "out of range" in rejected(d)
    d = base()
    d.add_material(extensions=[(54, 3)])
    rejected(d)
    d = base()
    d.add_material(extensions=[(45, (1.0, float("inf")))])
    rejected(d)


@pytest.mark.parametrize("name", ["displacement", "anisotropy map", "coat normal", "udim", "anisotropy"])
def test_unsupported_texture_features_are_named(name):
    px = np.zeros((10, 10, 4), np.uint8)
    d = base()
    t = d.add_texture(10, 10, px, udim=int(name == "udim"), uv_channel=int(name == "uv1"))
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV, **({"uv1s": QUAD_UV} if name == "uv1" else {}))
    slots, ext = [t, NONE, NONE, NONE], []
    if name == "displacement":
        ext = [(59, t)]
    elif name == "anisotropy map":
        ext = [(70, t)]
    elif name == "coat normal":
        ext = [(74, t)]
    elif name == "anisotropy":
        ext = [(9, (0.5,))]
    d.add_mesh(g, d.add_material(textures=tuple(slots), extensions=ext))
    assert "not supported" in rejected(d, abi.MT_ERROR_UNAVAILABLE)


def test_supported_neighbours_of_unsupported_cases():
    px = np.zeros((1, 1, 4), np.uint8)
    # base-color alpha as opacity under an opaque alpha mode stays opaque
    d = base()
    t = d.add_texture(1, 1, px)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV),
               d.add_material(textures=(t, NONE, NONE, NONE), extensions=[(54, 1), (41, 1)]))
    h = decoded(d)
    assert h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)[-1, 5, 3] == 2
    # uv channel 1 without any UV1 coordinates samples the primary set
    d = base()
    t = d.add_texture(1, 1, px, uv_channel=1)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), d.add_material(textures=(t, NONE, NONE, NONE)))
    decoded(d)
    # anisotropy without UVs or tangents anywhere
    d = base()
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX), d.add_material(extensions=[(9, (0.5,))]))
    decoded(d)
    # an alpha map under the opaque alpha mode changes nothing
    d = base()
    t = d.add_texture(1, 1, px)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV),
               d.add_material(extensions=[(40, t), (41, 1)]))
    decoded(d)


# ------------------------------------------------------------ sampling
def np_sample(texels, rec, idx_uv):
    """sampleMap in float32 NumPy, operation by operation (WGSL mix =
    a * (1 - t) + b * t)."""
    w, h = int(rec[0, :1].view(np.int32)[0]), int(rec[0, 1:2].view(np.int32)[0])
    sx, sy, ox, oy = (F(x) for x in rec[1])
    ms, mt = rec[2, 2], rec[2, 3]

    def wrap(v, mode):
        if mode < 0.5:
            return F(v - F(np.floor(v)))
        if mode < 1.5:
            return F(min(max(v, F(0)), F(1)))
        m = F(v - F(F(2) * F(np.floor(F(v * F(0.5))))))
        return F(F(1) - F(abs(F(F(1) - m))))

    out = []
    for u, v in idx_uv:
        tx = F(F(wrap(F(F(F(u) * sx) + ox), ms) * F(w)) - F(0.5))
        ty = F(F(wrap(F(F(F(v) * sy) + oy), mt) * F(h)) - F(0.5))
        fx, fy = F(np.floor(tx)), F(np.floor(ty))
        wx, wy = F(tx - fx), F(ty - fy)
        bx, by = int(fx), int(fy)

        def load(x, y):
            px = x % w if ms < 0.5 else min(max(x, 0), w - 1)
            py = y % h if mt < 0.5 else min(max(y, 0), h - 1)
            return texels[py, px].astype(F)

        def mix(p, q, k):
            return (p * (F(1) - k)).astype(F) + (q * k).astype(F)

        out.append(mix(mix(load(bx, by), load(bx + 1, by), wx), mix(load(bx, by + 1), load(bx + 1, by + 1), wx), wy))
    return np.array(out, F)


def uv_grid():
    # the lookup grid of the reference's filter check (tests/gpu/bindlessTextureSampling.ts:38-40)
    c = np.arange(257)
    return np.stack([(c % 17) / 8.0 - 0.5, (c // 17) / 7.0 - 0.5], 1).astype(F)


@pytest.mark.parametrize("wrap", [(0, 0), (1, 1), (2, 2), (0, 2), (1, 0)])
def test_oracle_sample_map_matches_numpy(wrap):
    rng = np.random.default_rng(11)
    pixels = rng.integers(0, 256, (3, 4, 4), dtype=np.uint8)
    d, _ = textured(pixels, wrap_s=wrap[0], wrap_t=wrap[1], uv_scale=(1.5, -0.75), uv_offset=(0.1, 0.3))
    h = decoded(d)
    rows, _ = maps_of(h)
    uvs = uv_grid()
    got = oracle_lib.sample_maps(h, np.zeros(len(uvs), np.int32), uvs)
    want = np_sample(texels_of(h, 0), rows[0], uvs)
    assert np.array_equal(got, want)


def test_oracle_sample_map_index_guards():
    d, _ = textured(np.full((1, 1, 4), 255, np.uint8))
    h = decoded(d)
    got = oracle_lib.sample_maps(h, np.array([-1, 1, 0], np.int32), np.zeros((3, 2), F))
    assert np.array_equal(got[:2], np.zeros((2, 4), F)) and np.array_equal(got[2], np.ones(4, F))


# ----------------------------------------------------------- all slots
SLOT_EXTENSIONS = {  # extension id -> (row, component) of the packed map index (materialLayoutSchema.ts)
    39: (2, 2), 40: (22, 2), 43: (3, 3), 44: (1, 1), 46: (2, 3), 47: (22, 0), 48: (22, 1), 49: (9, 3),
    50: (9, 1), 64: (6, 0), 65: (6, 1), 66: (6, 3), 67: (18, 3), 68: (19, 3), 69: (21, 3)}


def test_every_supported_slot_packs_its_map_index():
    """One texture per slot: the map list follows MATERIAL_TEXTURE_NAMES
    order (map, alphaMap, normalMap, emissiveMap, metallicRoughnessMap,
    roughnessMap, metalnessMap, transmissionMap, thinFilmMap, coatWeightMap,
    coatRoughnessMap, fuzzColorMap, fuzzRoughnessMap, specularWeightMap,
    specularColorMap), each index lands in its packed field."""
    order = [39, 40, 44, 43, 46, 47, 48, 49, 50, 64, 65, 66, 67, 68, 69]
    d = base()
    tex = {eid: d.add_texture(1, 1, np.full((1, 1, 4), 10 + k, np.uint8)) for k, eid in enumerate(order)}
    ext = [(eid, tex[eid]) for eid in sorted(tex)] + [(41, 1), (62, (-0.5,)), (63, 2)]
    m = d.add_material(extensions=ext, coat_weight=0.5)
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), m)
    h = decoded(d)
    rows = h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)[m]
    for position, eid in enumerate(order):
        r, c = SLOT_EXTENSIONS[eid]
        assert rows[r, c] == position, eid
    assert rows[25, 2:].tolist() == [0.0, 2.0]            # thin-film minimum clamped at 0, channel b
    assert rows[23, 3] == 0                                # opaque
    assert maps_of(h)[0].shape[0] == len(order)


def test_coat_weight_map_leaves_emission_raw():
    # materialEmission.ts:10-22: with a coat weight map the packed emission
    # carries no coat passage (the shader applies it per texel).
    d = base()
    t = d.add_texture(1, 1, np.full((1, 1, 4), 128, np.uint8))
    a = d.add_material(emission_color=(1, 1, 1), emission_luminance=2.0, coat_weight=1.0,
                       extensions=[(26, (0.25, 0.25, 0.25))])
    b = d.add_material(emission_color=(1, 1, 1), emission_luminance=2.0, coat_weight=1.0,
                       extensions=[(26, (0.25, 0.25, 0.25)), (64, t)])
    g = d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV)
    d.add_mesh(g, a)
    d.add_mesh(g, b, transform=D.translate([0, 1, 0]))
    rows = decoded(d).materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)
    assert np.allclose(rows[a, 3, :3], 1.0) and np.allclose(rows[b, 3, :3], 2.0)


def test_emissive_triangles_carry_corner_uvs():
    d = base()
    t = d.add_texture(2, 2, np.full((2, 2, 4), 200, np.uint8))
    uvs = np.array([[0.1, 0.2], [0.9, 0.2], [0.9, 0.8], [0.1, 0.8]], F)
    lamp = d.add_material(emission_color=(1, 1, 1), emission_luminance=3.0, textures=(NONE, NONE, NONE, t))
    d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=uvs), lamp, transform=D.translate([0, 1, 0]))
    h = decoded(d)
    tri = h.light_sampling.reshape(-1, 4)[:12].reshape(2, 6, 4)   # 2 triangles x 6 texels
    for k in range(2):
        corners = QUAD_IDX[k * 3:k * 3 + 3]
        want = uvs[corners].reshape(-1)
        assert np.array_equal(tri[k, 3:6].reshape(-1)[:6], want)
        assert np.array_equal(tri[k, 3:6].reshape(-1)[6:], want)      # secondary set repeats the primary
    assert h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)[lamp, 3, 3] == 0


@pytest.mark.parametrize("projection", [1, 2, 3])
def test_uv_projection_packs_and_renders(projection):
    """uvProjection (ext 55) lands in row 7.x with uvProjectionScale in 7.zw;
    the oracle renders a projected checker finitely and differently from
    plain UVs."""
    px = np.zeros((8, 8, 4), np.uint8)
    yy, xx = np.mgrid[0:8, 0:8]
    px[(xx + yy) % 2 == 0] = [255, 255, 255, 255]
    px[(xx + yy) % 2 == 1] = [20, 20, 20, 255]

    def scene(proj):
        d = base()
        t = d.add_texture(8, 8, px)
        ext = [(56, (2.0, 2.0))] + ([(55, proj)] if proj else [])
        m = d.add_material(textures=(t, NONE, NONE, NONE), extensions=ext)
        d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), m, transform=D.translate([0, 0.3, 0], 0.8))
        return d, m
    d, m = scene(projection)
    h = decoded(d)
    assert h.materials.reshape(-1, abi.MTC_MATERIAL_VEC4_ROWS, 4)[m, 7].tolist() == [projection, -1, 2, 2]
    acc = oracle_lib.Accum(h.width, h.height)
    oracle_lib.trace(h, acc, 4)
    h0 = decoded(scene(0)[0])
    acc0 = oracle_lib.Accum(h0.width, h0.height)
    oracle_lib.trace(h0, acc0, 4)
    assert np.isfinite(acc.color).all() and not np.array_equal(acc.color, acc0.color)


def test_secondary_uv_set_layout_and_sampling():
    """compactVertexLayout / packCompactVertices: UV1 words follow the UV
    pair when any geometry has them, geometries without UV1 repeat their
    primary UVs there (uv1 ?? uv); a map on uv_channel 1 samples them."""
    px = np.zeros((2, 2, 4), np.uint8)
    px[0, 0] = px[1, 1] = [255, 255, 255, 255]
    uv1 = np.array([[0.5, 0.5], [0.75, 0.5], [0.75, 0.75], [0.5, 0.75]], F)

    def scene(channel):
        d = base()
        t = d.add_texture(2, 2, px, uv_channel=channel)
        m = d.add_material(textures=(t, NONE, NONE, NONE))
        d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV, uv1s=uv1), m, transform=D.translate([0, 0.6, 0]))
        d.add_mesh(d.add_geometry(QUAD, QUAD_IDX, uvs=QUAD_UV), m, transform=D.translate([0, 0.3, 0]))
        return d
    h = decoded(scene(1))
    lay = h.bundle.vertex_layout
    assert (lay.stride, lay.uv_offset, lay.uv1_offset) == (8, 4, 6)
    words = h.attributes.reshape(-1, 8)
    assert np.array_equal(words[4:8, 6:8].view(F), uv1)              # the UV1 geometry
    assert np.array_equal(words[8:12, 6:8].view(F), QUAD_UV)         # uv1 ?? uv
    renders = []
    for channel in (0, 1):
        hh = decoded(scene(channel))
        acc = oracle_lib.Accum(hh.width, hh.height)
        oracle_lib.trace(hh, acc, 4)
        renders.append(acc.color.copy())
    assert np.isfinite(renders[1]).all() and not np.array_equal(renders[0], renders[1])
