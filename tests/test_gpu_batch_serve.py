"""The batched form (graph-captured persistent launch, autotuned shapes) and
the served form (continuous batching over resident scenes) give every job
the bit-identical outputs of the same job rendered alone through
mtc_trace_samples."""
import pytest

from mutracer_b200 import abi, batch, scene, serve

pytestmark = pytest.mark.gpu


def _equal(a, b):
    import torch
    return all(torch.equal(x, y) for x, y in ((a.color, b.color), (a.normal, b.normal), (a.albedo, b.albedo),
                                              (a.catcher, b.catcher)))


def _small_jobs(cuda):
    specs = [batch.JobSpec(0, 40, 24, 3, 20_000, 2, 11), batch.JobSpec(1, 33, 47, 5, 60_000, 5, 12),
             batch.JobSpec(2, 64, 16, 2, 10_000, 1, 13), batch.JobSpec(3, 17, 9, 4, 120_000, 8, 14)]
    return batch.build_mixed(specs, cuda, env_width=64)


def test_graph_replay_matches_alone_and_picks_up_rewritten_table(cuda):
    import torch
    jobs = _small_jobs(cuda)
    alone = _small_jobs(cuda)
    b = batch.Batch(len(jobs), abi.BatchConfig.make(tile_width=4, items_per_fetch=2), cuda)
    b.set_jobs(jobs)
    b.capture()
    b.replay()
    torch.cuda.synchronize()
    for j in alone:
        j.render_alone()
    torch.cuda.synchronize()
    assert all(_equal(a.acc, j.acc) for a, j in zip(alone, jobs))
    # Rewrite the pinned table in place (other sample counts, fewer jobs) and
    # replay the same graph: the device reads the new header and entries.
    b.set_jobs(jobs[1:], [2, 1, 3])
    b.replay()
    torch.cuda.synchronize()
    for j, s in zip(alone[1:], [2, 1, 3]):
        j.render_alone(samples=s)
    torch.cuda.synchronize()
    assert all(_equal(a.acc, j.acc) for a, j in zip(alone, jobs))
    expected = sum(j.pixels * j.spp for j in jobs) + sum(j.pixels * s for j, s in zip(jobs[1:], [2, 1, 3]))
    assert int(b.counters[0].item()) == expected
    b.release()


def test_every_autotune_shape_gives_the_same_images(cuda):
    import torch
    ref = _small_jobs(cuda)
    for j in ref:
        j.render_alone(per_sample=True)
    torch.cuda.synchronize()
    best, timings = batch.autotune(_small_jobs(cuda), probe_samples=1, repeats=1, device=cuda)
    assert best is not None and len(timings) == len(batch.AUTOTUNE_SPACE)
    for shape in batch.AUTOTUNE_SPACE:
        jobs = _small_jobs(cuda)
        b = batch.Batch(len(jobs), abi.BatchConfig.make(*shape), cuda)
        b.set_jobs(jobs)
        b.launch()
        torch.cuda.synchronize()
        assert all(_equal(a.acc, j.acc) for a, j in zip(ref, jobs)), shape


def test_served_results_equal_alone(cuda):
    import torch
    pool = serve.ScenePool(cuda)
    for sid, (kind, params) in enumerate((("cornell", ()), ("instanced_spheres", (12, 3, 6, 64, 2)),
                                          ("instanced_spheres", (40, 4, 8, 64, 5)))):
        pool.add(sid, scene.SceneHost(kind, 32, 32, sid + 1, params))
    reqs = serve.poisson_requests(pool, 10, rate=400.0, seed=5, spp_range=(2, 9),
                                  resolutions=((24, 16), (40, 40), (13, 31)))
    srv = serve.Server(pool, job_bytes=3 * 40 * 40 * serve.ACCUMULATION_BYTES_PER_PIXEL, max_jobs=3,
                       quantum=2, device=cuda)
    stats = srv.run(reqs, keep_outputs=True)
    srv.release()
    assert stats["requests"] == 10 and stats["rounds"] >= 5
    assert stats["paths"] == sum(r.width * r.height * r.spp for r in reqs)
    assert all(r.completed >= r.admitted - 1e-3 and r.latency > 0 for r in reqs)
    for r in reqs:
        alone = batch.RenderJob(pool[r.scene_id], r.spp, r.width, r.height, camera=r.camera, device=cuda)
        alone.render_alone()
        torch.cuda.synchronize()
        assert _equal(alone.acc, r.job.acc), r.request_id


@pytest.mark.parametrize("engine", ["wavefront", "persistent"])
def test_served_results_equal_alone_both_engines(cuda, engine):
    import torch
    pool = serve.ScenePool(cuda)
    pool.add(0, scene.SceneHost("instanced_spheres", 32, 32, 4, (20, 4, 6, 64, 3)))
    pool.add(1, scene.SceneHost("glass_spheres", 32, 32, 2, (5,)))
    reqs = serve.poisson_requests(pool, 6, rate=300.0, seed=9, spp_range=(1, 7),
                                  resolutions=((20, 30), (33, 17)))
    srv = serve.Server(pool, job_bytes=1 << 30, max_jobs=4, quantum=3, engine=engine, device=cuda)
    srv.run(reqs, keep_outputs=True)
    srv.release()
    for r in reqs:
        alone = batch.RenderJob(pool[r.scene_id], r.spp, r.width, r.height, camera=r.camera, device=cuda)
        alone.render_alone(per_sample=True)
        torch.cuda.synchronize()
        assert _equal(alone.acc, r.job.acc), (engine, r.request_id)


def test_served_admission_respects_the_hbm_budget(cuda):
    pool = serve.ScenePool(cuda)
    pool.add(0, scene.SceneHost("cornell", 16, 16, 1))
    reqs = [serve.Request(i, 0, 64, 64, 3, 0.0) for i in range(6)]
    one = 64 * 64 * serve.ACCUMULATION_BYTES_PER_PIXEL
    srv = serve.Server(pool, job_bytes=2 * one, max_jobs=8, quantum=1, device=cuda)
    # The resident scene and the engine's state are charged against the budget.
    assert srv.fixed_bytes >= pool.device_bytes > 0 and srv.budget == srv.fixed_bytes + 2 * one
    stats = srv.run(reqs)
    srv.release()
    # At most two jobs fit at once, 3 samples each: 6 jobs need >= 9 rounds.
    assert stats["rounds"] >= 9
    with pytest.raises(RuntimeError):
        serve.Server(pool, job_bytes=one - 1, device=cuda).run([serve.Request(0, 0, 64, 64, 1, 0.0)])
    # A budget smaller than the resident scenes and engine state is refused.
    with pytest.raises(ValueError):
        serve.Server(pool, hbm_budget_bytes=pool.device_bytes, device=cuda)


@pytest.mark.parametrize("slots,refill,regroup,sort", [(1024, 1, 1, 0), (1 << 16, 8, 1, 1), (4096, 32, 3, 1),
                                                       (1 << 14, 16, abi.MTC_REGROUP_OFF, 0)])
def test_wavefront_matches_alone(cuda, slots, refill, regroup, sort):
    import torch
    jobs = _small_jobs(cuda)
    extra = batch.build_mixed([batch.JobSpec(9, 96, 80, 6, 40_000, 3, 21)], cuda, env_width=64)
    jobs += extra
    alone = _small_jobs(cuda) + batch.build_mixed([batch.JobSpec(9, 96, 80, 6, 40_000, 3, 21)], cuda, env_width=64)
    sb = batch.StreamBatch(len(jobs), abi.BatchConfig.make(tile_width=8),
                           abi.StreamConfig.make(slots=slots, iterations_per_check=3, refill_lanes=refill,
                                                 regroup_interval=regroup, sort_rays=sort), device=cuda)
    sb.set_jobs(jobs)
    sb.run()
    torch.cuda.synchronize()
    for j in alone:
        j.render_alone()
    torch.cuda.synchronize()
    for a, j in zip(alone, jobs):
        assert _equal(a.acc, j.acc), j.job_id
    c = sb.counters.cpu().tolist()
    assert c[0] == sum(j.pixels * j.spp for j in jobs)
    # A second run adds the same number of samples again, continuing each
    # pixel's sample sequence, like a second mtc_trace_samples call.
    sb.set_jobs(jobs, [2] * len(jobs))
    sb.run()
    for a in alone:
        a.render_alone(samples=2)
    torch.cuda.synchronize()
    for a, j in zip(alone, jobs):
        assert _equal(a.acc, j.acc), j.job_id


def test_wavefront_cornell_and_glass_scenes(cuda):
    """Analytic-light hits, media and transmission through the wavefront."""
    import torch
    for kind, params in (("cornell", ()), ("glass_spheres", (6,))):
        host = scene.SceneHost(kind, 48, 40, 3, params)
        dev = scene.DeviceScene(host, cuda)
        a = batch.RenderJob(dev, 5, device=cuda)
        b = batch.RenderJob(dev, 5, device=cuda)
        a.render_alone()
        sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=2048), device=cuda)
        sb.set_jobs([b])
        sb.run()
        torch.cuda.synchronize()
        assert _equal(a.acc, b.acc), kind


def test_edge_jobs_zero_samples_tiny_and_ragged_images(cuda):
    """Jobs with no samples, a 1x1 image and ragged image edges, through both
    batched engines, against the jobs alone."""
    import torch
    specs = [batch.JobSpec(0, 1, 1, 3, 10_000, 1, 31), batch.JobSpec(1, 7, 3, 0, 10_000, 2, 32),
             batch.JobSpec(2, 33, 17, 2, 20_000, 3, 33), batch.JobSpec(3, 5, 29, 1, 10_000, 1, 34)]

    def fresh():
        return batch.build_mixed(specs, cuda, env_width=64)

    alone = fresh()
    for j in alone:
        if j.spp:
            j.render_alone()
    for engine in ("persistent", "wavefront"):
        jobs = fresh()
        if engine == "persistent":
            b = batch.Batch(len(jobs), abi.BatchConfig.make(tile_width=32), cuda)
            b.set_jobs(jobs)
            b.launch()
        else:
            b = batch.StreamBatch(len(jobs), stream_config=abi.StreamConfig.make(slots=1024), device=cuda)
            b.set_jobs(jobs)
            b.run()
        torch.cuda.synchronize()
        for a, j in zip(alone, jobs):
            assert _equal(a.acc, j.acc), (engine, j.job_id)
        assert float(jobs[1].acc.normal[:, 3].sum()) == 0.0          # zero-sample job untouched
        assert int(b.counters[0].item()) == sum(j.pixels * j.spp for j in jobs)


def test_empty_batches_and_empty_scene(cuda):
    import torch
    sb = batch.StreamBatch(4, device=cuda)
    sb.set_jobs([])
    sb.run()                                             # nothing to do
    b = batch.Batch(4, None, cuda)
    b.set_jobs([])
    b.launch()
    torch.cuda.synchronize()
    assert int(sb.counters[0].item()) == 0 and int(b.counters[0].item()) == 0
    # A scene flagged empty (RayTraceUniform.isEmpty) only sees the background.
    host = scene.SceneHost("instanced_spheres", 24, 16, 2, (8, 2, 4, 64, 1))
    u = abi.TraceUniform.from_buffer_copy(host.uniform)
    u.is_empty = 1
    host.set_uniform(u)
    dev = scene.DeviceScene(host, cuda)
    a, w = batch.RenderJob(dev, 3, device=cuda), batch.RenderJob(dev, 3, device=cuda)
    a.render_alone()
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=1024), device=cuda)
    sb.set_jobs([w])
    sb.run()
    torch.cuda.synchronize()
    assert _equal(a.acc, w.acc)
    assert int(sb.counters[1].item()) == 0               # no extension ray traced


def test_stream_launch_is_asynchronous_and_reports_the_iteration_limit(cuda):
    """mtc_stream_launch enqueues the device-driven event loop and returns;
    mtc_stream_status reports the outcome.  An iteration limit below what the
    jobs need stops the run with MT_ERROR_TIMEOUT; a full run of the same
    state afterwards is complete and equals the jobs rendered alone."""
    import ctypes as C

    import torch
    L = abi.lib()
    alone = _small_jobs(cuda)
    for j in alone:
        j.render_alone()
    jobs = _small_jobs(cuda)
    sb = batch.StreamBatch(len(jobs), stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs(jobs)
    args = (C.c_void_p(sb.table.data_ptr()), sb.capacity)
    state = C.c_void_p(sb.state.data_ptr())

    for per_check in (0, 1, 8):                           # device-driven loop, host-driven loops
        limited = abi.StreamConfig.make(slots=4096, max_iterations=2, iterations_per_check=per_check)
        assert L.mtc_stream_run(*args, C.byref(limited), state, None, None) == abi.MT_ERROR_TIMEOUT
        assert L.mtc_stream_status(state, sb.capacity, C.byref(limited), None) == abi.MT_ERROR_TIMEOUT
    # The host-driven loop blocks, so it cannot be only enqueued.
    host = abi.StreamConfig.make(slots=4096, iterations_per_check=8)
    assert L.mtc_stream_launch(*args, C.byref(host), state, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    side = torch.cuda.Stream(device=cuda)
    for j in jobs:
        j.acc.zero_()
    torch.cuda.synchronize()
    stream = C.c_void_p(side.cuda_stream)
    assert L.mtc_stream_launch(*args, C.byref(sb.stream_config), state, C.c_void_p(sb.counters.data_ptr()),
                               stream) == abi.MT_OK
    assert L.mtc_stream_status(state, sb.capacity, C.byref(sb.stream_config), stream) == abi.MT_OK
    torch.cuda.synchronize()
    for a, j in zip(alone, jobs):
        assert _equal(a.acc, j.acc), j.job_id
    assert int(sb.counters[0].item()) == sum(j.pixels * j.spp for j in jobs)


def test_loop_graphs_of_many_shapes_and_states(cuda):
    """More launch shapes and state buffers than the per-device graph cache
    holds, interleaved: every run equals the jobs rendered alone."""
    import torch
    alone = _small_jobs(cuda)
    for j in alone:
        j.render_alone()
    batches = []
    for slots, regroup in ((1024, 1), (2048, 2), (4096, 1), (8192, abi.MTC_REGROUP_OFF), (1 << 14, 5), (3072, 1)):
        jobs = _small_jobs(cuda)
        sb = batch.StreamBatch(len(jobs), stream_config=abi.StreamConfig.make(slots=slots, regroup_interval=regroup),
                               device=cuda)
        batches.append((sb, jobs))
    for _ in range(2):
        for sb, jobs in batches:
            for j in jobs:
                j.acc.zero_()
            sb.set_jobs(jobs)
            sb.run()
            torch.cuda.synchronize()
            for a, j in zip(alone, jobs):
                assert _equal(a.acc, j.acc), (sb.stream_config.slots, j.job_id)


def test_queue_trace_adds_up_to_a_full_run(cuda):
    """bench.py's queue trace (runs stopped by their iteration limit after
    1, 2, ... iterations, from zeroed accumulation) gives per-iteration queue
    lengths that sum to the counters of one complete run."""
    import torch

    import bench
    host = scene.SceneHost("instanced_spheres", 48, 32, 2, (16, 4, 6, 64, 2))
    dev = scene.DeviceScene(host, cuda)
    job = batch.RenderJob(dev, 3, device=cuda)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([job])
    trace = bench.queue_trace(sb, sb.counters, 4096, 64)["queue_trace"]
    job.acc.zero_()
    sb.counters.zero_()
    sb.stream_config = abi.StreamConfig.make(slots=4096)
    sb.run()
    torch.cuda.synchronize()
    c = sb.counters.cpu().tolist()
    assert trace[-1]["extension"] == 0                 # the queue drained within the traced iterations
    assert sum(r["extension"] for r in trace) == c[1]
    assert sum(r["shadow"] for r in trace) == c[2]
    assert sum(r["finished"] for r in trace) == c[0] == 48 * 32 * 3
