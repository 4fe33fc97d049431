"""Batched form: many render jobs of uneven resolution, sample count and
scene size traced by one persistent launch.

The reference renders one job at a time, one compute dispatch per sample
(``dispatch_target``, native/host/src/lib.rs:1506-1560).  Here a set of jobs
becomes one job table (``mtc_batch_prepare``) that the persistent kernel
drains from a global work counter (``mtc_batch_launch``); the table lives in
pinned host memory, so the launch is captured once as a CUDA graph and
replayed after the table is rewritten in place.  ``autotune`` picks the
launch shape (block size, CTAs per SM, warp-tile shape, fetch grain) by
timing short probes of the actual batch.  No launch shape changes any job's
result: a pixel's samples always run in order on one lane.
"""
import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import abi, scene, trace

# Resolutions of the mixed-job workload (64 jobs per batch).
RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080))


@dataclass(frozen=True)
class JobSpec:
    """One job of a seeded mixed workload."""
    job_id: int
    width: int
    height: int
    spp: int
    triangles: int   # target instanced triangle count of its scene
    lights: int      # rect lights
    seed: int

    def scene_params(self, env_width=512, max_base_meshes=16):
        """instanced_spheres parameters (instances, base meshes, icosphere
        frequency, sky width, rect lights) giving about `triangles` instanced
        triangles: 20 * frequency^2 triangles per sphere, at most
        `max_base_meshes` distinct (BLAS) meshes."""
        instances = int(min(512, max(4, round(self.triangles / 2000))))
        freq = int(min(28, max(2, round(math.sqrt(self.triangles / (20.0 * instances))))))
        return (instances, min(max_base_meshes, instances), freq, env_width, self.lights)


def mixed_jobs(count=64, seed=0, spp_range=(4, 256), tri_range=(10_000, 2_000_000), light_range=(1, 8),
               spp_divisor=1):
    """Seeded mixed workload: resolution from RESOLUTIONS, spp log-uniform in
    spp_range (divided by spp_divisor, rounded up, for scaled-down runs),
    scene size log-uniform in tri_range, 1-8 lights, scene seed = job id."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for j in range(count):
        w, h = RESOLUTIONS[int(rng.integers(len(RESOLUTIONS)))]
        spp = int(round(math.exp(rng.uniform(math.log(spp_range[0]), math.log(spp_range[1])))))
        spp = max(1, -(-spp // spp_divisor))
        tris = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
        lights = int(rng.integers(light_range[0], light_range[1] + 1))
        out.append(JobSpec(j, w, h, spp, tris, lights, seed=j + 1))
    return out


class RenderJob:
    """A render job: a device-resident scene, a camera and uniform for one
    resolution, a target sample count and its own accumulation buffers
    (outColor / outNormal / outAlbedo / outShadowCatcher)."""

    def __init__(self, dev_scene, spp, width=None, height=None, camera=None, uniform=None, device="cuda",
                 job_id=0):
        self.scene = dev_scene
        self.job_id = job_id
        self.width = width or dev_scene.width
        self.height = height or dev_scene.height
        self.uniform = abi.TraceUniform.from_buffer_copy(uniform if uniform is not None else dev_scene.uniform)
        self.uniform.output_size[0] = float(self.width)
        self.uniform.output_size[1] = float(self.height)
        self.camera = abi.CameraUniform.from_buffer_copy(camera if camera is not None else dev_scene.camera)
        self.spp = int(spp)
        self.done = 0
        self.acc = trace.Accumulation(self.width, self.height, device)

    @property
    def pixels(self):
        return self.width * self.height

    def desc(self, samples):
        d = abi.JobDesc()
        d.scene = self.scene.view
        d.camera = self.camera
        d.uniform = self.uniform
        d.out = self.acc.outputs
        d.samples = int(samples)
        return d

    def render_alone(self, samples=None, per_sample=False, stream=None):
        """The job through the plain entry point: one mtc_trace_samples call
        for all samples, or (per_sample) one call per sample as the
        reference's host dispatches them."""
        n = self.spp if samples is None else samples
        if per_sample:
            for _ in range(n):
                trace.trace_samples(self.scene, self.acc, 1, uniform=self.uniform, camera=self.camera,
                                    stream=stream)
        else:
            trace.trace_samples(self.scene, self.acc, n, uniform=self.uniform, camera=self.camera, stream=stream)


def build_mixed(specs, device="cuda", env_width=512):
    """Host scenes, device scenes and RenderJobs for a list of JobSpecs."""
    jobs = []
    for sp in specs:
        host = scene.SceneHost("instanced_spheres", sp.width, sp.height, sp.seed, sp.scene_params(env_width))
        dev = scene.DeviceScene(host, device)
        jobs.append(RenderJob(dev, sp.spp, job_id=sp.job_id, device=device))
    return jobs


def _stream_ptr(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class _JobTable:
    """Pinned host job table for up to `capacity` jobs (mtc_batch_prepare)."""

    def __init__(self, capacity, config=None, device="cuda"):
        import torch
        self.capacity = int(capacity)
        self.device = torch.device(device)
        self.config = config if config is not None else abi.BatchConfig.make()
        self.table = torch.zeros(abi.lib().mtc_batch_table_bytes(self.capacity), dtype=torch.uint8).pin_memory()
        self.counters = trace.counters_tensor(self.device)
        self.jobs = []
        self.samples = []
        self.total_items = 0
        self.layout_mask = 0

    def set_jobs(self, jobs, samples=None):
        """Writes the table for `jobs` (RenderJob list), each adding
        samples[i] (default: its full spp) in the next launch."""
        if len(jobs) > self.capacity:
            raise ValueError(f"{len(jobs)} jobs exceed the batch capacity {self.capacity}")
        samples = samples if samples is not None else [j.spp for j in jobs]
        descs = (abi.JobDesc * max(1, len(jobs)))()
        for i, (j, s) in enumerate(zip(jobs, samples)):
            descs[i] = j.desc(s)
        total = C.c_uint32(0)
        abi.check(abi.lib().mtc_batch_prepare(descs, len(jobs), C.byref(self.config),
                                              C.c_void_p(self.table.data_ptr()), C.byref(total)))
        self.jobs = list(jobs)
        self.samples = list(samples)
        self.total_items = total.value
        # The kernel specialisation (BLAS layouts present) is chosen from the
        # table when a launch is issued or captured.
        mask = 0
        for j in jobs:
            mask |= j.scene.view.flags & abi.MTC_SCENE_BLAS_GPU_LAYOUT
        self.layout_mask = mask


class Batch(_JobTable):
    """Up to `capacity` jobs run by the persistent batched megakernel.

    ``set_jobs`` rewrites the pinned host table; ``launch`` enqueues the
    table copy, counter reset and kernel on a stream; ``capture`` records
    those three operations once as a CUDA graph that ``replay`` re-issues
    (it picks up whatever the table holds at replay time)."""

    def __init__(self, capacity, config=None, device="cuda"):
        import torch
        super().__init__(capacity, config, device)
        self.scratch = torch.zeros(abi.lib().mtc_batch_scratch_bytes(self.capacity), dtype=torch.uint8,
                                   device=self.device)
        self.graph = None
        self._graph_mask = None

    def launch(self, stream=None):
        abi.check(abi.lib().mtc_batch_launch(C.c_void_p(self.table.data_ptr()), self.capacity,
                                             C.byref(self.config), C.c_void_p(self.scratch.data_ptr()),
                                             C.c_void_p(self.counters.data_ptr()), _stream_ptr(stream)))

    def capture(self):
        import torch
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self.launch(side)
        torch.cuda.current_stream(self.device).wait_stream(side)
        self.graph = g
        self._graph_mask = self.layout_mask
        return g

    def replay(self):
        if self.graph is None or self._graph_mask != self.layout_mask:
            self.capture()
        self.graph.replay()

    @property
    def device_bytes(self):
        return self.scratch.numel()

    def release(self):
        self.graph = None


class StreamBatch(_JobTable):
    """Up to `capacity` jobs drained by the wavefront kernels
    (mtc_stream_run): extension traversal, shading, shadow traversal and
    accumulation over queues of `slots` in-flight path samples."""

    def __init__(self, capacity, config=None, stream_config=None, device="cuda"):
        import torch
        super().__init__(capacity, config, device)
        self.stream_config = stream_config if stream_config is not None else abi.StreamConfig.make()
        n = abi.lib().mtc_stream_state_bytes(self.capacity, C.byref(self.stream_config))
        if n == 0:
            raise abi.MtError(abi.MT_ERROR_INVALID_ARGUMENT, "stream config")
        self.state = torch.zeros(n, dtype=torch.uint8, device=self.device)

    def run(self, stream=None):
        abi.check(abi.lib().mtc_stream_run(C.c_void_p(self.table.data_ptr()), self.capacity,
                                           C.byref(self.stream_config), C.c_void_p(self.state.data_ptr()),
                                           C.c_void_p(self.counters.data_ptr()), _stream_ptr(stream)))

    @property
    def device_bytes(self):
        return self.state.numel()

    def release(self):
        pass


# Launch shapes the autotuner tries, in BatchConfig.make's order (block
# threads, warp tile width, CTAs per SM, items per fetch).  The kernel is
# compiled for 16 resident 128-thread CTAs per SM (32 registers), so 16 fills
# the SMs; larger grids only queue CTAs behind them.
AUTOTUNE_SPACE = (
    (128, 8, 16, 1), (128, 8, 16, 2), (128, 4, 16, 1), (128, 16, 16, 1),
    (128, 32, 16, 1), (64, 8, 32, 1), (128, 8, 8, 1), (128, 8, 12, 1),
)


def autotune(jobs, probe_samples=1, space=AUTOTUNE_SPACE, repeats=2, device="cuda"):
    """Times one probe batch per launch shape (every job at `probe_samples`
    samples) and returns (best BatchConfig, {shape: ms}).  The probes
    accumulate into the jobs' own buffers, which are cleared afterwards.
    Results never depend on the shape, so the choice affects only speed."""
    import torch
    timings = {}
    best, best_ms = None, float("inf")
    for shape in space:
        cfg = abi.BatchConfig.make(*shape)
        b = Batch(len(jobs), cfg, device)
        b.set_jobs(jobs, [probe_samples] * len(jobs))
        b.launch()
        torch.cuda.synchronize()
        ms = float("inf")
        for _ in range(repeats):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            b.launch()
            e.record()
            e.synchronize()
            ms = min(ms, s.elapsed_time(e))
        timings[shape] = ms
        if ms < best_ms:
            best, best_ms = cfg, ms
    for j in jobs:
        j.acc.zero_()
    torch.cuda.synchronize()
    return best, timings


# Wavefront knobs the autotuner walks one at a time (coordinate descent from
# the defaults): paths in flight ("queue depth"), idle lanes that trigger a
# ray refill in the traversal kernels, how often the shading queue is
# regrouped by material class (abi.MTC_REGROUP_OFF: never), whether the
# extension queue is ordered by (job, direction octant) before traversal, and
# how many traversal steps a lane takes between refill checks.
STREAM_SPACE = {
    "refill_lanes": (2, 4, 8),
    "regroup_interval": (1, 2, abi.MTC_REGROUP_OFF),
    "sort_rays": (0, 1),
    "steps_per_check": (4, 8, 16),
    "slots": (1 << 20, 1 << 21, 1 << 22),
}
STREAM_DEFAULT = {"slots": 1 << 21, "refill_lanes": 4, "regroup_interval": 1, "sort_rays": 0, "steps_per_check": 8}


def autotune_stream(jobs, probe_samples=1, space=STREAM_SPACE, device="cuda", batch_config=None):
    """Coordinate-descent tuning of the wavefront knobs on probe runs of the
    actual jobs (each at `probe_samples` samples).  Returns (best
    StreamConfig, {setting: ms}).  The probes accumulate into the jobs'
    buffers, which are cleared afterwards; no setting changes any result."""
    import torch
    best = dict(STREAM_DEFAULT)
    timings = {}
    cache = {}

    def probe(setting):
        key = tuple(sorted(setting.items()))
        if key in cache:
            return cache[key]
        sb = StreamBatch(len(jobs), batch_config, abi.StreamConfig.make(**setting), device)
        sb.set_jobs(jobs, [probe_samples] * len(jobs))
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        sb.run()
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e)
        del sb
        cache[key] = ms
        timings[",".join(f"{k}={v}" for k, v in key)] = ms
        return ms

    probe(best)  # warm-up of the code paths; timed again below
    cache.clear()
    timings.clear()
    for knob, values in space.items():
        results = {}
        for val in values:
            trial = dict(best)
            trial[knob] = val
            results[val] = probe(trial)
        best[knob] = min(results, key=results.get)
    for j in jobs:
        j.acc.zero_()
    torch.cuda.synchronize()
    return abi.StreamConfig.make(**best), timings


def total_paths(jobs, samples=None):
    samples = samples if samples is not None else [j.spp for j in jobs]
    return sum(j.pixels * s for j, s in zip(jobs, samples))


def run_plain(jobs, per_sample=True, stream=None):
    """The plain drop-in path over the jobs one after another, as the
    reference's host renders them (per_sample: one launch per sample)."""
    for j in jobs:
        j.render_alone(per_sample=per_sample, stream=stream)


def wall_ms(fn):
    import torch
    torch.cuda.synchronize()
    t = time.perf_counter()
    fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t) * 1e3
