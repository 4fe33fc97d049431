"""Device refitBLAS (mtc_blas_refit_prepare + mtc_refit_blas) against the
host restatement (mtp_refit_blas, itself checked against oracle/bvh_ref.py):
node boxes bit-identical after deformation, in standalone BLAS buffers and in
a BLAS region of a scene's bvh buffer, through a CUDA graph, and malformed
buffers rejected."""
import numpy as np
import pytest

from mutracer_b200 import abi, blas

torch = pytest.importorskip("torch")


def deformed(pos, seed, nan=3):
    rng = np.random.default_rng(seed)
    moved = (pos * np.float32(1.5) + rng.normal(0, 0.05, pos.shape)).astype(np.float32)
    if nan:
        moved[rng.integers(0, len(moved), nan), rng.integers(0, 3, nan)] = np.nan
    return moved


@pytest.mark.gpu
@pytest.mark.parametrize("side,seed", [(8, 0), (60, 1), (300, 2)])
def test_refit_matches_host(side, seed):
    pos, idx = blas.terrain_mesh(side, side, seed=seed)
    buf, _ = blas.host_build(pos, idx)
    dev = torch.from_numpy(buf.copy()).cuda()
    r = blas.BlasRefit(dev)
    moved = deformed(pos, seed)
    area = r.refit(torch.from_numpy(moved).cuda())
    want, want_area = blas.host_refit(buf, moved)
    assert dev.cpu().numpy().view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
    assert abs(area.item() - want_area) <= 1e-12 * abs(want_area)


@pytest.mark.gpu
def test_refit_scene_region_and_graph():
    from mutracer_b200 import scene
    host = scene.SceneHost("instanced_spheres", 16, 16, 1, (24, 3, 4, 64, 1))
    bvh = torch.from_numpy(host.bvh.copy()).cuda()
    pos, idx, offset, length, _ = host.mesh(1)
    region = bvh[offset * 4: (offset + length) * 4]
    r = blas.BlasRefit(region)
    moved_t = torch.from_numpy(deformed(pos, 7, nan=0)).cuda()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        r.refit(moved_t, stream)                    # warm-up outside the capture
    stream.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        r.refit(moved_t, torch.cuda.current_stream())
    for seed in (11, 12):
        moved = deformed(pos, seed, nan=1)
        moved_t.copy_(torch.from_numpy(moved))
        g.replay()
        torch.cuda.synchronize()
        want, _ = blas.host_refit(host.bvh[offset * 4: (offset + length) * 4], moved)
        assert region.cpu().numpy().view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
    # the rest of the scene buffer is untouched
    rest = np.concatenate([bvh[: offset * 4].cpu().numpy(), bvh[(offset + length) * 4:].cpu().numpy()])
    assert rest.tobytes() == np.concatenate([host.bvh[: offset * 4], host.bvh[(offset + length) * 4:]]).tobytes()


@pytest.mark.gpu
def test_refit_after_device_build_and_malformed():
    pos, idx = blas.terrain_mesh(200, 200, seed=9)
    b = blas.BlasBuilder(len(idx))
    buf, _ = b.build(torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    buf = buf.clone()
    r = blas.BlasRefit(buf)
    moved = deformed(pos, 3)
    r.refit(torch.from_numpy(moved).cuda())
    want, _ = blas.host_refit(blas.host_build(pos, idx)[0], moved)
    assert buf.cpu().numpy().view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
    bad = buf.clone()
    bad.view(torch.int32)[3] = bad.numel() // 4 + 10   # root's right child past the end
    with pytest.raises(abi.MtError):
        blas.BlasRefit(bad)


@pytest.mark.gpu
def test_device_rebuild_hint():
    """binnedSahBvh.test.ts:196-207 through the device refit's area."""
    from tests.test_blas_refit_host import uv_sphere
    pos, idx = uv_sphere(16, 8)
    buf, _ = blas.host_build(pos, idx)
    dev = torch.from_numpy(buf.copy()).cuda()
    r = blas.BlasRefit(dev)
    build_area = r.refit(torch.from_numpy(pos).cuda()).item()
    for scale, keep in ((0.99, True), (1.3, True), (1.6, False)):
        moved = (pos * np.float32(scale)).astype(np.float32)
        area = r.refit(torch.from_numpy(moved).cuda()).item()
        assert (not (area > build_area * 2)) == keep
        want, want_area = blas.host_refit(buf, moved)
        assert dev.cpu().numpy().view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
        assert abs(area - want_area) <= 1e-12 * want_area
