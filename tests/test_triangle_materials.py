"""Per-triangle materials (the triangle material plane of the compact vertex
path: packTriangleMaterials, compactVertices.ts:93-102, read by
triangleMaterial, vertexAttributes.wgsl.ts:51-56).  On the CPU oracle a
mesh whose two halves select different table entries renders bit-identical
to the same halves as two meshes with one material each; the plane follows
the records when the BLASes are re-encoded in the BVH_GPU layout."""
import numpy as np

from mutracer_b200 import abi
from mutracer_b200 import descriptor as D
from tests import oracle_lib

F = np.float32
QUAD = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], F)
QUAD_IDX = [0, 2, 1, 0, 3, 2]


def halves(multi, width=32, height=24, emissive=False, colors=None):
    """colors: None, "rgba8" (vertex colors in [0, 1]) or "float" (some above 1)."""
    d = D.Descriptor(width, height)
    floor_colors = None
    if colors is not None:
        floor_colors = np.array([[1, 0.2, 0.2], [0.2, 1, 0.2], [0.2, 0.2, 1], [1, 1, 0.2]], F)
        if colors == "float":
            floor_colors = floor_colors * F(1.5)
    left, right = QUAD * F(0.5) + F([-0.6, 0, 0]), QUAD * F(0.5) + F([0.6, 0, 0])
    red = d.add_material(base_color=(0.8, 0.1, 0.1), roughness=0.5)
    green = d.add_material(base_color=(0.1, 0.8, 0.1), roughness=0.2, metalness=1.0,
                           emission_color=(1, 1, 1), emission_luminance=2.0 if emissive else 0.0)
    d.add_mesh(d.add_geometry(QUAD * F(3) + F([0, -0.01, 0]), QUAD_IDX, colors=floor_colors), d.add_material())
    if multi:
        g = d.add_geometry(np.concatenate([left, right]), QUAD_IDX + [i + 4 for i in QUAD_IDX],
                           material_indices=[0] * 4 + [1] * 4)
        d.add_mesh(g, red, material_table=[red, green], transform=D.translate([0, 0.5, 0]))
    else:
        d.add_mesh(d.add_geometry(left, QUAD_IDX), red, transform=D.translate([0, 0.5, 0]))
        d.add_mesh(d.add_geometry(right, QUAD_IDX), green, transform=D.translate([0, 0.5, 0]))
    d.add_light(D.LIGHT_RECT, intensity=6, size=1, height_or_inner=1, transform=D.look_at([0, 2, 0.01], [0, 0, 0]))
    d.set_camera(fov=50, transform=D.look_at([0, 1.5, 2.5], [0, 0.3, 0]))
    return d


def decode(d):
    st, msg, h = D.decode(d.to_bytes())
    assert st == abi.MT_OK, msg
    return h


def render(h, spp=16):
    acc = oracle_lib.Accum(h.width, h.height)
    oracle_lib.trace(h, acc, spp)
    return acc


def test_multi_material_mesh_equals_split_meshes_on_the_oracle():
    a, b = render(decode(halves(False))), render(decode(halves(True)))
    for x, y in ((a.color, b.color), (a.normal, b.normal), (a.albedo, b.albedo)):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_emissive_triangles_take_their_own_material():
    h = decode(halves(True, emissive=True))
    assert h.uniform.light_choice_count == 1 + 2            # the rect light and the green half's 2 triangles
    tri = h.light_sampling.reshape(-1, 4)[:12].reshape(2, 6, 4)
    assert (tri[:, 2, 3] == 1).all()                       # material index of the green material


def test_plane_follows_records_in_the_gpu_layout():
    h = decode(halves(True))
    plane0 = h.triangle_materials.copy()
    h.set_blas_layout(2)
    plane2 = h.triangle_materials
    words = h.bvh.reshape(-1, 4).view(np.uint32)
    assert plane2 is not None and plane2.size == words.shape[0]
    assert sorted(set(int(x) for x in plane0 if x)) == sorted(set(int(x) for x in plane2 if x)) == [1, 2]
    a, b = render(decode(halves(True))), render(h)
    assert np.array_equal(a.color.view(np.uint32), b.color.view(np.uint32))
