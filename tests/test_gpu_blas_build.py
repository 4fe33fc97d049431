"""Device BLAS build (mtc_build_blas) against the host producer (the C++
restatement of buildBLAS, itself checked bit for bit against the Python
restatement in oracle/bvh_ref.py): the BVH2 buffers must be identical byte for
byte, on meshes that take both the level-synchronous and the per-CTA paths,
the reference's edge cases (coincident and flat boxes, signed zeros, skipped
triangles) and several bin counts."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi

torch = pytest.importorskip("torch")


def host_blas(pos, idx, bins):
    from mutracer_b200 import blas
    return blas.host_build(pos, idx, bins)


def device_blas(pos, idx, bins):
    from mutracer_b200 import blas
    pos_t = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    idx_t = torch.from_numpy(np.ascontiguousarray(idx, np.uint32).view(np.int32)).cuda()
    builder = blas.BlasBuilder(max(idx.size // 3, 1), bins)
    buf, res = builder.build(pos_t, idx_t)
    torch.cuda.synchronize()
    return buf.cpu().numpy(), res


def grid_mesh(w, h, seed=0, amplitude=0.3):
    from mutracer_b200 import blas
    return blas.terrain_mesh(w, h, seed, amplitude)


def soup(n, seed=0, spread=10.0, size=0.3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    pos = (c + rng.uniform(-size, size, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    return pos, np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)


def check_same(pos, idx, bins=8):
    want, depth = host_blas(pos, idx, bins)
    got, res = device_blas(pos, idx, bins)
    assert res.vec4_count == want.size // 4
    assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
    assert res.max_depth == depth
    if want.size:
        assert np.array_equal(np.asarray(res.local_bounds, np.float32).view(np.uint32),
                              np.concatenate([want[0:3], want[4:7]]).view(np.uint32))
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (37, 3), (1000, 4), (1024, 5), (1025, 6), (5000, 7),
                                    (60000, 8)])
def test_soup_matches_host(n, seed):
    check_same(*soup(n, seed))


@pytest.mark.gpu
@pytest.mark.parametrize("bins", [1, 2, 8, 13, 16, 64])
def test_bins(bins):
    check_same(*soup(20000, 11), bins=bins)


@pytest.mark.gpu
def test_terrain_large_phase():
    res = check_same(*grid_mesh(400, 300, seed=3))          # 240k triangles
    assert res.primitive_count == 240000 and res.host_syncs > 5


@pytest.mark.gpu
def test_degenerate_boxes():
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    same = np.tile(tri, (3000, 1))                            # identical centroids: one big leaf
    check_same(same, np.arange(9000, dtype=np.uint32).reshape(-1, 3))
    line = np.zeros((6000, 3), np.float32)                    # boxes on the x axis: zero-area node
    line[:, 0] = np.repeat(np.arange(2000, dtype=np.float32), 3)
    check_same(line, np.arange(6000, dtype=np.uint32).reshape(-1, 3))
    pos, idx = grid_mesh(60, 60, seed=1, amplitude=0.0)        # flat: y extent zero
    check_same(pos, idx)
    # one far triangle beside a coincident cluster larger than a CTA subtree
    far = np.concatenate([np.tile(tri, (2500, 1)), tri + np.float32(100)])
    check_same(far, np.arange(far.shape[0], dtype=np.uint32).reshape(-1, 3))


@pytest.mark.gpu
def test_unbalanced_clusters():
    rng = np.random.default_rng(5)
    centres = (2.0 ** np.arange(24))[rng.integers(0, 24, 30000)]
    pos = (centres[:, None, None] * np.array([1, 0, 0]) + rng.uniform(-0.2, 0.2, (30000, 3, 3))).astype(np.float32)
    check_same(pos.reshape(-1, 3), np.arange(90000, dtype=np.uint32).reshape(-1, 3))


@pytest.mark.gpu
def test_signed_zero_and_skipped_triangles():
    pos, idx = soup(4000, 9, spread=1.0)
    pos[::7, 0] = np.float32(-0.0)
    pos[1::7, 0] = np.float32(0.0)
    pos[2::11, 1] = np.nan
    idx = idx.copy()
    idx[::13, 2] = 10 ** 9                                     # past the vertex array
    res = check_same(pos, idx)
    assert res.primitive_count < 4000


@pytest.mark.gpu
def test_empty_and_all_skipped():
    got, res = device_blas(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), 8)
    assert res.vec4_count == 0 and got.size == 0
    pos = np.full((3, 3), np.nan, np.float32)
    got, res = device_blas(pos, np.array([[0, 1, 2]], np.uint32), 8)
    assert res.vec4_count == 0 and res.primitive_count == 0


@pytest.mark.gpu
@pytest.mark.parametrize("kind,params", [("cornell", ()), ("instanced_spheres", (24, 3, 4, 64, 1)),
                                         ("glass_spheres", (8,))])
def test_scene_blases_rebuilt_on_device(kind, params):
    """Every BLAS region of a generated scene's bvh buffer equals the device
    build of that BLAS's source mesh."""
    from mutracer_b200 import scene
    host = scene.SceneHost(kind, 32, 32, 1, params)
    for m in range(host.info.blases):
        pos, idx, offset, length, bins = host.mesh(m)
        got, res = device_blas(pos, idx, bins)
        assert res.vec4_count == length
        want = host.bvh[offset * 4: (offset + length) * 4]
        assert got.view(np.uint32).tobytes() == want.view(np.uint32).tobytes()


@pytest.mark.gpu
def test_bin_edge_probe_as_triangles():
    """The bin-edge probe of binnedSahBvh.test.ts:106-131, each box given as
    a triangle spanning its corners (the triangle's box is the box)."""
    f = lambda x: float(np.float32(x))
    lo, hi, c = -1000.0, f(1000.3), f(0.14999441802501678)
    boxes = [[lo, 0, 0, lo + 0.01, 1, 1], [hi - 0.01, 0, 0, hi, 1, 1], [c, 0, 0, c, 1, 1]]
    for b in range(8):
        x = lo + ((b + 0.5) * (hi - lo)) / 8
        boxes.append([x - 0.01, 0, 0, x + 0.01, 1, 1])
    b = np.array(boxes, np.float32)
    pos = np.stack([b[:, :3], b[:, 3:], np.concatenate([b[:, :1], b[:, 4:5], b[:, 2:3]], 1)], 1).reshape(-1, 3)
    check_same(pos, np.arange(len(pos), dtype=np.uint32).reshape(-1, 3))
