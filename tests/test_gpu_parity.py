"""GPU parity of the CUDA path against the CPU oracle, through the C ABI.

Bars: first-hit instance/record/t bit-exact (ties counted), image relMSE
<= 1e-3 and mean luminance within 0.5 % at the same seed, TLAS refit
bit-exact, batched jobs bit-identical to the same jobs alone.
"""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, scene, trace
from tests import oracle_lib

pytestmark = pytest.mark.gpu

REL_MSE_BAR = 1e-3
LUMA_BAR = 0.005


def _hits_equal(gpu, ref):
    g, r = gpu.view(np.int32), ref.view(np.int32)
    same = (g[:, 0] == r[:, 0]) & (g[:, 1] == r[:, 1]) & (g[:, 2] == r[:, 2]) & (g[:, 3] == r[:, 3])
    # A tie: both report a hit at the same t on different primitives.
    tie = (~same) & (g[:, 0] == 1) & (r[:, 0] == 1) & (g[:, 3] == r[:, 3])
    return same, tie


def _first_hit_case(cuda, host, n, seed):
    import torch
    dev = scene.DeviceScene(host, cuda)
    rays = oracle_lib.seeded_rays(host, n, seed=seed)
    ref = oracle_lib.first_hits(host, rays)
    gpu = trace.query_first_hit(dev, torch.from_numpy(rays).to(cuda)).cpu().numpy()
    torch.cuda.synchronize()
    same, tie = _hits_equal(gpu, ref)
    mismatches = int((~same).sum())
    ties = int(tie.sum())
    assert ref[:, 0].sum() > n // 4, "ray set should mostly hit the scene"
    assert mismatches == ties, f"{mismatches} hit mismatches, of which {ties} are ties"
    hit = ref[:, 0] == 1
    # barycentrics are bit-exact wherever the record matches
    both = same & hit
    assert np.array_equal(gpu[both, 4:7], ref[both, 4:7])
    return mismatches, ties


def test_first_hit_bitexact_cornell(cuda):
    host = scene.SceneHost("cornell", 64, 64, 1)
    _first_hit_case(cuda, host, 200_000, seed=3)


def test_first_hit_bitexact_large_1m(cuda):
    host = scene.make_workload("instanced_spheres", width=64, height=64)
    assert host.info.triangles > 4_000_000
    _first_hit_case(cuda, host, 1_000_000, seed=11)


def _render_pair(cuda, host, spp):
    import torch
    dev = scene.DeviceScene(host, cuda)
    acc = trace.Accumulation(host.width, host.height, cuda)
    trace.trace_samples(dev, acc, spp)
    torch.cuda.synchronize()
    gpu = acc.resolved().cpu().numpy()
    ref_acc = oracle_lib.Accum(host.width, host.height)
    oracle_lib.trace(host, ref_acc, spp)
    ref = ref_acc.resolved()
    return gpu, ref, acc, ref_acc


def _image_metrics(gpu, ref):
    a, b = gpu[..., :3].astype(np.float64), ref[..., :3].astype(np.float64)
    rel_mse = float(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))
    w = np.array([0.2126, 0.7152, 0.0722])
    la, lb = float((a @ w).mean()), float((b @ w).mean())
    return rel_mse, abs(la - lb) / max(lb, 1e-30)


def test_image_parity_cornell(cuda):
    host = scene.SceneHost("cornell", 128, 128, 1)
    gpu, ref, acc, ref_acc = _render_pair(cuda, host, 64)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma
    # per-pixel sample counts are exact
    assert np.array_equal(acc.normal[:, 3].cpu().numpy(), ref_acc.normal[:, 3])


def test_image_parity_cornell_full_config(cuda):
    """The small plain configuration at its full size: Cornell box 512x512,
    64 spp, 8 bounces, Sobol seed 0, 16 SAH bins."""
    host = scene.make_workload("cornell")
    assert (host.width, host.height, host.bundle.uniform.bounces, host.bundle.uniform.sequence_seed) == \
        (512, 512, 8, 0)
    gpu, ref, acc, ref_acc = _render_pair(cuda, host, 64)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma
    assert np.array_equal(acc.normal[:, 3].cpu().numpy(), ref_acc.normal[:, 3])


def test_image_parity_instanced(cuda):
    host = scene.make_workload("instanced_spheres", width=160, height=90)
    gpu, ref, _, _ = _render_pair(cuda, host, 8)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


def test_image_parity_zsobol_two_candidates(cuda):
    host = scene.SceneHost("cornell", 96, 96, 5)
    u = abi.TraceUniform.from_buffer_copy(host.uniform)
    u.direct_light_candidates = 3
    u.sequence_seed = 99
    host.set_uniform(u, None, (host.flags & ~abi.MTC_SCENE_PATTERN_MASK) | (1 << abi.MTC_SCENE_PATTERN_SHIFT))
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma


@pytest.mark.parametrize("wavelengths,independent", [(3, False), (3, True), (1, False)])
def test_image_parity_spectral_glass(cuda, wavelengths, independent):
    """Spectral integrator (rayTrace.compute.ts:947-1057): dispersive glass
    spheres with homogeneous interiors, three wavelength paths per sample
    sharing their RGB prefix (the default), three independent ones, or one
    hero wavelength."""
    host = scene.SceneHost("glass_spheres", 64, 48, 3, (8,))
    assert host.flags & abi.MTC_SCENE_SPECTRAL
    u = abi.TraceUniform.from_buffer_copy(host.uniform)
    u.dispersion_wavelengths = wavelengths
    host.set_uniform(u, None, host.flags | (abi.MTC_SCENE_SPECTRAL_INDEPENDENT if independent else 0))
    gpu, ref, acc, ref_acc = _render_pair(cuda, host, 16)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert np.isfinite(gpu).all()
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma
    assert np.array_equal(acc.normal[:, 3].cpu().numpy(), ref_acc.normal[:, 3])


def test_spectral_prefix_sharing_is_exact_on_the_device(cuda):
    """The shared prefix (spectralPrefix.wgsl.ts) only skips work: the device
    image is bit-identical to the independent-wavelength variant's, with
    fewer extension and shadow rays (device counters)."""
    import torch
    out = {}
    for independent in (False, True):
        host = scene.SceneHost("glass_spheres", 56, 40, 5, (10,))
        host.set_uniform(host.uniform, None,
                         host.flags | (abi.MTC_SCENE_SPECTRAL_INDEPENDENT if independent else 0))
        dev = scene.DeviceScene(host, cuda)
        acc = trace.Accumulation(56, 40, cuda)
        counters = trace.counters_tensor(cuda)
        trace.trace_samples(dev, acc, 8, counters=counters)
        torch.cuda.synchronize()
        out[independent] = (acc, counters.cpu().numpy())
    (a, ca), (b, cb) = out[False], out[True]
    for x, y in ((a.color, b.color), (a.normal, b.normal), (a.albedo, b.albedo), (a.catcher, b.catcher)):
        assert torch.equal(x, y)
    assert ca[0] == cb[0]                          # path samples
    assert ca[1] < 0.9 * cb[1] and ca[2] < cb[2]  # extension, shadow rays


def test_refit_device_matches_host(cuda):
    import torch
    host = scene.make_workload("instanced_spheres", width=32, height=32, params=(64, 4, 8, 256, 2))
    inputs = host.refit_inputs()
    rng = np.random.default_rng(5)
    t = inputs["transforms"].reshape(-1, 4, 4).copy()
    t[:, 3, :3] += rng.normal(scale=0.5, size=(t.shape[0], 3))  # move every instance
    t = t.reshape(-1, 16)
    host.set_transforms(t)
    inputs["transforms"] = t
    dev = scene.DeviceScene(host, cuda)          # uploads the pre-refit buffers
    host.refit_host()                            # reference refit on the host
    host.refresh()
    dinputs = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in inputs.items()}
    trace.refit_tlas(dev, dinputs)
    torch.cuda.synchronize()
    tlas_vec4 = host.info.tlas_vec4
    got_tlas = dev.bvh[: tlas_vec4 * 4].cpu().numpy()
    want_tlas = host.bvh[: tlas_vec4 * 4]
    assert np.array_equal(got_tlas.view(np.uint32), want_tlas.view(np.uint32))
    assert np.array_equal(dev.instances.cpu().numpy().view(np.uint32), host.instances.view(np.uint32))


def test_batch_matches_alone(cuda):
    import torch
    hosts = [scene.SceneHost("cornell", 64, 48, 1), scene.SceneHost("cornell", 40, 72, 2),
             scene.make_workload("instanced_spheres", width=48, height=32, params=(32, 4, 6, 256, 2))]
    spps = [5, 9, 3]
    devs = [scene.DeviceScene(h, cuda) for h in hosts]
    alone = []
    for d, s in zip(devs, spps):
        acc = trace.Accumulation(d.width, d.height, cuda)
        trace.trace_samples(d, acc, s)
        alone.append(acc)
    batched = [trace.Accumulation(d.width, d.height, cuda) for d in devs]
    jobs = (abi.JobDesc * len(devs))()
    for i, (d, s, acc) in enumerate(zip(devs, spps, batched)):
        jobs[i].scene = d.view
        jobs[i].camera = d.camera
        jobs[i].uniform = d.uniform
        jobs[i].out = acc.outputs
        jobs[i].samples = s
    scratch = torch.zeros(abi.lib().mtc_batch_scratch_bytes(len(devs)), dtype=torch.uint8, device=cuda)
    st = abi.lib().mtc_trace_batch(jobs, len(devs), None, C.c_void_p(scratch.data_ptr()), None, None,
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
    abi.check(st)
    torch.cuda.synchronize()
    for a, b in zip(alone, batched):
        for x, y in ((a.color, b.color), (a.normal, b.normal), (a.albedo, b.albedo), (a.catcher, b.catcher)):
            assert torch.equal(x, y)


def test_context_api_render_and_jobs(cuda):
    from mutracer_b200.context import Context
    host = scene.SceneHost("cornell", 48, 40, 1)
    ctx = Context()
    try:
        with pytest.raises(abi.MtError):
            ctx.render(1)                       # nothing committed yet
        ctx.commit(host)
        with pytest.raises(abi.MtError) as e:
            ctx.read_pixels()                   # no completed sample
        assert e.value.status == abi.MT_ERROR_INVALID_STATE
        ctx.render(4)
        img = ctx.read_pixels()
        assert img.shape == (40, 48, 4) and np.isfinite(img).all()
        # the same samples through the device-buffer entry point match exactly
        import torch
        dev = scene.DeviceScene(host, cuda)
        acc = trace.Accumulation(48, 40, cuda)
        trace.trace_samples(dev, acc, 4)
        torch.cuda.synchronize()
        ref = acc.resolved().cpu().numpy()
        assert np.array_equal(img, ref)
        job = ctx.submit(10)
        with pytest.raises(abi.MtError):
            ctx.render(1)                       # active job rejects blocking render
        import time
        deadline = time.monotonic() + 120.0
        while time.monotonic() < deadline:
            job.poll(3)
            if job.info().state == abi.MT_JOB_COMPLETE:
                break
            time.sleep(0.001)
        info = job.info()
        assert info.state == abi.MT_JOB_COMPLETE and info.completed_samples == 10 and info.base_samples == 4
        assert ctx.info().samples == 14
        # The job's batches (asynchronous wavefront launches) continue each
        # pixel's sample sequence: the image equals 14 samples traced at once.
        acc14 = trace.Accumulation(48, 40, cuda)
        trace.trace_samples(dev, acc14, 14)
        torch.cuda.synchronize()
        assert np.array_equal(ctx.read_pixels(), acc14.resolved().cpu().numpy())
        job2 = ctx.submit(8)
        job.__init__(job.handle)
        with pytest.raises(abi.MtError) as e:
            job.poll(1)                         # expired handle
        assert e.value.status == abi.MT_ERROR_INVALID_HANDLE
        job2.poll(2)
        job2.cancel()
        deadline = time.monotonic() + 120.0
        while time.monotonic() < deadline:
            job2.poll(0)
            if job2.info().state in (abi.MT_JOB_CANCELLED, abi.MT_JOB_COMPLETE):
                break
            time.sleep(0.001)
        assert job2.info().state == abi.MT_JOB_CANCELLED
        assert ctx.info().samples == 16
        # Recommits reuse (or grow) the context's device buffers: a larger
        # scene, then the first one again, each from zeroed accumulation.
        import torch
        for h, spp in ((scene.make_workload("instanced_spheres", width=64, height=48, params=(24, 4, 6, 64, 3)), 3),
                       (host, 2)):
            ctx.commit(h)
            assert ctx.info().samples == 0
            ctx.render(spp)
            d = scene.DeviceScene(h, cuda)
            a = trace.Accumulation(h.width, h.height, cuda)
            trace.trace_samples(d, a, spp)
            torch.cuda.synchronize()
            for kind, buf in ((abi.MT_IMAGE_HDR, a.color), (abi.MT_IMAGE_NORMAL, a.normal),
                              (abi.MT_IMAGE_ALBEDO, a.albedo)):
                # IEEE division by the sample count (torch divides by a
                # scalar through its reciprocal, so compute on the host)
                want = (buf.cpu().numpy() / np.float32(spp)).reshape(h.height, h.width, 4)
                assert np.array_equal(ctx.read_pixels(kind), want), kind
    finally:
        ctx.destroy()


def test_first_hits_layout2_bit_exact(cuda):
    """BVH_GPU BLASes (layout code 2) through the device traversal."""
    host = scene.make_workload("instanced_spheres", width=64, height=64, params=(128, 8, 16, 256, 2))
    host.set_blas_layout(2)
    _first_hit_case(cuda, host, 200_000, seed=13)


def test_layout2_images_equal_layout0_in_both_engines(cuda):
    import torch
    from mutracer_b200 import batch
    params = (48, 6, 10, 128, 3)
    a = scene.make_workload("instanced_spheres", width=72, height=40, params=params)
    b = scene.make_workload("instanced_spheres", width=72, height=40, params=params)
    b.set_blas_layout(2)
    da, db = scene.DeviceScene(a, cuda), scene.DeviceScene(b, cuda)
    ja, jb, jw = batch.RenderJob(da, 4, device=cuda), batch.RenderJob(db, 4, device=cuda), \
        batch.RenderJob(db, 4, device=cuda)
    ja.render_alone()
    jb.render_alone()
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([jw])
    sb.run()
    torch.cuda.synchronize()
    for x in (jb, jw):
        assert torch.equal(ja.acc.color, x.acc.color) and torch.equal(ja.acc.normal, x.acc.normal)


def test_context_jobs_on_a_spectral_scene_match_the_megakernel(cuda):
    """Job batches of the context API (asynchronous wavefront launches) on a
    dispersive glass scene, the shared-prefix spectral integrator with media,
    write the bits of the same samples traced by the plain megakernel."""
    import torch
    from mutracer_b200.context import Context
    host = scene.SceneHost("glass_spheres", 40, 32, 5, (6,))
    ctx = Context()
    try:
        import time
        ctx.commit(host)
        job = ctx.submit(7)
        deadline = time.monotonic() + 120.0
        while time.monotonic() < deadline:
            job.poll(2)
            if job.info().state == abi.MT_JOB_COMPLETE:
                break
            time.sleep(0.001)
        assert job.info().state == abi.MT_JOB_COMPLETE and ctx.info().samples == 7
        dev = scene.DeviceScene(host, cuda)
        acc = trace.Accumulation(40, 32, cuda)
        trace.trace_samples(dev, acc, 7)
        torch.cuda.synchronize()
        assert np.array_equal(ctx.read_pixels(), acc.resolved().cpu().numpy())
    finally:
        ctx.destroy()
