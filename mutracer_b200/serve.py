"""Served form: a request loop over a pool of device-resident scenes.

Requests (scene, camera, resolution, target spp) arrive over time.  Each
round the loop admits waiting requests while the batch has a free slot and
their accumulation buffers fit the HBM budget, then runs every admitted job
for up to `quantum` more samples in one batched pass: a wavefront run
(mtc_stream_run, the default engine) or a replay of the captured persistent
megakernel launch (two job tables alternate, so the host prepares round k+1
while round k runs).  Jobs that reach their target spp complete and free
their slot and memory; requests that arrived meanwhile join the next round,
so new and running jobs share the device (continuous batching at sample
granularity, not a FIFO of whole renders).

A pixel's samples always run in order on one lane and each round resumes at
the pixel's accumulated sample count, so a job's outputs are bit-identical to
the same job rendered alone with mtc_trace_samples, whatever else shares its
rounds.  The reference has no serving layer; its per-job host loop
(native/host/src/lib.rs:1506-1560, one dispatch per sample) is the plain
baseline this form is measured against.
"""
import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi, batch, scene

ACCUMULATION_BYTES_PER_PIXEL = 96  # outColor + outNormal + outAlbedo (16 B each) + 3 x 16 B catcher


@dataclass
class Request:
    request_id: int
    scene_id: int
    width: int
    height: int
    spp: int
    arrival: float                      # seconds after the stream starts
    camera: object = None               # abi.CameraUniform (None: the scene's own)
    admitted: float = math.nan          # device seconds
    completed: float = math.nan         # device seconds
    job: object = field(default=None, repr=False)

    @property
    def latency(self):
        return self.completed - self.arrival


class ScenePool:
    """Device-resident scenes, keyed by id, with their HBM footprint."""

    def __init__(self, device="cuda"):
        self.device = device
        self.hosts, self.scenes = {}, {}

    def add(self, scene_id, host):
        self.hosts[scene_id] = host
        self.scenes[scene_id] = scene.DeviceScene(host, self.device)
        return self.scenes[scene_id]

    def __getitem__(self, scene_id):
        return self.scenes[scene_id]

    def __len__(self):
        return len(self.scenes)

    @property
    def device_bytes(self):
        return sum(s.device_bytes for s in self.scenes.values())


def build_pool(count, seed=7, device="cuda", tri_range=(10_000, 8_000_000), max_base_meshes=16,
               env_width=512):
    """`count` seeded instanced-sphere scenes (triangles log-uniform in
    tri_range, 1-8 rect lights), resident on the device."""
    pool = ScenePool(device)
    for sp in batch.mixed_jobs(count, seed=seed, tri_range=tri_range):
        host = scene.SceneHost("instanced_spheres", 256, 256, sp.seed, sp.scene_params(env_width, max_base_meshes))
        pool.add(sp.job_id, host)
    return pool


def orbit_camera(host, width, height, rng, fov_range=(30.0, 70.0)):
    """Camera at a random point of the scene's bounding sphere looking at its
    centre, vertical FOV uniform in fov_range."""
    b = np.array(host.info.world_bounds, dtype=np.float64)
    centre = 0.5 * (b[:3] + b[3:])
    radius = 0.5 * float(np.linalg.norm(b[3:] - b[:3]))
    while True:
        v = rng.normal(size=3)
        v[1] = abs(v[1])                 # above the ground plane
        if np.linalg.norm(v) > 1e-6:
            break
    eye = centre + radius * v / np.linalg.norm(v)
    cam = abi.CameraUniform()
    dbl3 = abi.C.c_double * 3
    fov = float(rng.uniform(*fov_range))
    abi.check(abi.lib().mtp_camera_look_at(width, height, dbl3(*eye), dbl3(*centre), dbl3(0.0, 1.0, 0.0), fov,
                                           abi.C.byref(cam)))
    return cam


def poisson_requests(pool, count, rate, seed=0, spp_range=(16, 128), resolutions=batch.RESOLUTIONS,
                     spp_divisor=1):
    """`count` requests with exponential inter-arrival times (rate per
    second) over the pool's scenes: uniform scene, resolution from
    `resolutions`, target spp uniform in spp_range (divided by spp_divisor,
    rounded up, for scaled-down runs), orbit camera."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ids = sorted(pool.scenes)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        sid = ids[int(rng.integers(len(ids)))]
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        spp = max(1, -(-int(rng.integers(spp_range[0], spp_range[1] + 1)) // spp_divisor))
        cam = orbit_camera(pool.hosts[sid], w, h, rng)
        out.append(Request(i, sid, w, h, spp, t, cam))
    return out


class Server:
    """Continuous-batching render server over a ScenePool.

    Admission is by HBM budget: the resident scenes and the engine's own
    state (job tables, path slots and queues) are charged first, and a
    request is admitted only while its accumulation buffers fit in what is
    left, so the device never holds more than `hbm_budget_bytes` for the
    pool, the engine and the admitted jobs together."""

    def __init__(self, pool, hbm_budget_bytes=None, max_jobs=64, quantum=8, config=None, use_graph=True,
                 engine="wavefront", stream_config=None, device="cuda", job_bytes=None):
        """engine "wavefront": each round is one mtc_stream_run over all
        admitted jobs; "persistent": each round replays the captured
        persistent-megakernel launch (two alternating tables, so the host
        prepares round k+1 while round k runs).  Give either the whole
        budget (hbm_budget_bytes) or what is left for admitted jobs beyond
        the resident scenes and engine state (job_bytes)."""
        if (hbm_budget_bytes is None) == (job_bytes is None):
            raise ValueError("give exactly one of hbm_budget_bytes and job_bytes")
        self.pool = pool
        self.max_jobs = int(max_jobs)
        self.quantum = int(quantum)
        self.device = device
        self.use_graph = use_graph
        self.engine = engine
        if engine == "wavefront":
            self.batches = [batch.StreamBatch(max_jobs, config, stream_config, device)]
        elif engine == "persistent":
            self.batches = [batch.Batch(max_jobs, config, device) for _ in range(2)]
        else:
            raise ValueError(f"engine {engine!r}")
        # Resident scenes and engine state, charged before any request.
        self.fixed_bytes = int(pool.device_bytes) + sum(int(b.device_bytes) for b in self.batches)
        self.budget = int(hbm_budget_bytes) if job_bytes is None else self.fixed_bytes + int(job_bytes)
        if self.fixed_bytes > self.budget:
            raise ValueError(f"the resident scenes and engine state ({self.fixed_bytes} B) exceed the HBM budget "
                             f"({self.budget} B)")

    def _bytes(self, req):
        return req.width * req.height * ACCUMULATION_BYTES_PER_PIXEL

    def run(self, requests, keep_outputs=False):
        """Serves `requests` (arrival times relative to the call) and returns
        a stats dict; each request gets admitted/completed device times."""
        import torch
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        active = []
        used = self.fixed_bytes
        start = torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream()
        torch.cuda.synchronize()
        start.record(stream)
        t0 = time.perf_counter()
        which = 0
        paths = 0
        n_rounds = 0
        in_flight = collections.deque()   # rounds launched and not yet retired

        def retire_one():
            nonlocal used
            ev, finished = in_flight.popleft()
            ev.synchronize()
            t = start.elapsed_time(ev) / 1e3
            for r in finished:
                r.completed = t
                used -= self._bytes(r)
                if not keep_outputs:
                    r.job = None

        while pending or waiting or active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while waiting and len(active) < self.max_jobs and used + self._bytes(waiting[0]) <= self.budget:
                r = waiting.popleft()
                r.job = batch.RenderJob(self.pool[r.scene_id], r.spp, r.width, r.height, camera=r.camera,
                                        device=self.device, job_id=r.request_id)
                r.admitted = time.perf_counter() - t0
                used += self._bytes(r)
                active.append(r)
            if not active:
                if in_flight:
                    retire_one()
                    continue
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.05)))
                    continue
                if waiting:
                    raise RuntimeError("a request does not fit the HBM budget on its own")
                break
            # The table about to be rewritten was last used len(batches)
            # rounds ago; make sure that round has run.
            while len(in_flight) >= len(self.batches):
                retire_one()
            b = self.batches[which % len(self.batches)]
            samples = [min(self.quantum, r.spp - r.job.done) for r in active]
            b.set_jobs([r.job for r in active], samples)
            if self.engine == "wavefront":
                b.run(stream)
            elif self.use_graph:
                b.replay()
            else:
                b.launch(stream)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            finished = []
            for r, s in zip(active, samples):
                r.job.done += s
                paths += r.job.pixels * s
                if r.job.done >= r.spp:
                    finished.append(r)
            active = [r for r in active if r.job.done < r.spp]
            in_flight.append((ev, finished))
            which += 1
            n_rounds += 1
        while in_flight:
            retire_one()
        end = max(r.completed for r in requests)
        lat = np.array([r.latency for r in requests])
        return {
            "requests": len(requests), "rounds": n_rounds, "paths": paths,
            "device_seconds": end, "mpaths_per_s": paths / end / 1e6,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "resident_bytes": self.fixed_bytes,
        }

    def release(self):
        for b in self.batches:
            b.release()


def main(argv=None):
    """Rate sweep of the served form: one JSON line per arrival rate."""
    import argparse
    import json
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--scenes", type=int, default=32)
    p.add_argument("--base-meshes", type=int, default=64, help="distinct meshes per scene at most")
    p.add_argument("--requests", type=int, default=64)
    p.add_argument("--rates", default="5,10,20,50,100,200")
    p.add_argument("--spp-divisor", type=int, default=16)
    p.add_argument("--quantum", type=int, default=4)
    p.add_argument("--budget-gb", type=float, default=24.0)
    p.add_argument("--max-jobs", type=int, default=64)
    a = p.parse_args(argv)
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    pool = build_pool(a.scenes, device=dev, max_base_meshes=a.base_meshes)
    build_s = time.perf_counter() - t0
    srv = Server(pool, hbm_budget_bytes=int(a.budget_gb * 1024 ** 3), max_jobs=a.max_jobs, quantum=a.quantum,
                 device=dev)
    srv.run(poisson_requests(pool, 4, 1000.0, seed=3, spp_divisor=a.spp_divisor))
    for rate in (float(r) for r in a.rates.split(",")):
        reqs = poisson_requests(pool, a.requests, rate, seed=11, spp_divisor=a.spp_divisor)
        stats = srv.run(reqs)
        stats.update(rate_per_s=rate, scenes=len(pool), pool_gb=round(pool.device_bytes / 1e9, 3),
                     pool_build_s=round(build_s, 1), spp_divisor=a.spp_divisor, quantum=a.quantum,
                     budget_gb=a.budget_gb, offered_s=round(reqs[-1].arrival, 3))
        print(json.dumps({k: (round(v, 4) if isinstance(v, float) else v) for k, v in stats.items()}), flush=True)
    srv.release()


if __name__ == "__main__":
    main()
