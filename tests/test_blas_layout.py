"""BLAS layout code 2 (BVH_GPU: both child boxes in the parent node, the
layout intersect.wgsl.ts:453-497 traverses) against layout code 0 (BVH2).

A layout-2 scene here is the layout-0 scene re-encoded node for node, so a
ray visits the same nodes in the same order: the oracle's hits (instance, t,
barycentrics, triangle vertices) and renders are identical in both layouts.
Only the primitive record index (the hit's `record`) moves."""
import numpy as np

from mutracer_b200 import abi, scene
from tests import oracle_lib


def _pair(params=(24, 4, 8, 64, 2), w=40, h=30, seed=3):
    a = scene.SceneHost("instanced_spheres", w, h, seed, params)
    b = scene.SceneHost("instanced_spheres", w, h, seed, params)
    b.set_blas_layout(2)
    return a, b


def _tri_vertices(host, hits):
    words = host.bvh.view(np.int32).reshape(-1, 4)
    rec = hits[:, 2]
    out = np.full((len(hits), 3), -1, np.int64)
    ok = hits[:, 0] == 1
    out[ok] = words[rec[ok], :3]
    return out


def test_layout2_buffers_encode_the_same_trees():
    a, b = _pair()
    ia, ib = a.instances.view(np.uint32).reshape(-1, 40), b.instances.view(np.uint32).reshape(-1, 40)
    assert np.all(ia[:, 0] >> 30 == 0) and np.all(ib[:, 0] >> 30 == 2)
    assert np.array_equal(ia[:, 1:], ib[:, 1:])                  # all but the offset word
    tlas = a.info.tlas_vec4 * 4
    assert np.array_equal(a.bvh[:8], b.bvh[:8])                   # TLAS root box unchanged
    assert b.refit_inputs()["blas_layouts"].tolist() == [2] * a.info.instances
    assert b.bvh.size > tlas


def test_layout2_first_hits_match_layout0():
    a, b = _pair(params=(40, 6, 10, 64, 3))
    rays = oracle_lib.seeded_rays(a, 20000, seed=11)
    ha, hb = oracle_lib.first_hits(a, rays), oracle_lib.first_hits(b, rays)
    assert ha[:, 0].sum() > 5000
    for col in (0, 1, 3, 4, 5, 6):                                 # hit, instance, t, barycentrics
        assert np.array_equal(ha[:, col], hb[:, col]), col
    assert np.array_equal(_tri_vertices(a, ha), _tri_vertices(b, hb))


def test_layout2_renders_match_layout0():
    a, b = _pair(w=24, h=16)
    ra, rb = oracle_lib.Accum(24, 16), oracle_lib.Accum(24, 16)
    oracle_lib.trace(a, ra, 2)
    oracle_lib.trace(b, rb, 2)
    assert np.array_equal(ra.color, rb.color) and np.array_equal(ra.normal, rb.normal)


def test_layout2_survives_host_refit():
    a, b = _pair()
    b.refit_host()
    b.refresh()
    ib = b.instances.view(np.uint32).reshape(-1, 40)
    assert np.all(ib[:, 0] >> 30 == 2)
    assert abi.lib().mtp_scene_set_blas_layout(None, 2) == abi.MT_ERROR_INVALID_ARGUMENT
