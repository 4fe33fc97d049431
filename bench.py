"""Benchmark: converged Mpaths/s of the B200 path tracer on one GPU.

Headline workload (the large plain-method configuration): 256 seeded affine
instances of 16 displaced icospheres (15,680 triangles each, 4,014,080
instanced triangles), 2048x1024 analytic sky plus 4 rect lights, 1920x1080,
16 spp, 6 bounces, OpenPBR diffuse / F82 metal / coat.  One step renders the
whole job from zeroed accumulation buffers through the wavefront engine
(mtc_stream_run; `--form megakernel` times the plain drop-in megakernel
mtc_trace_samples instead).  The other engine renders the same job beside it
and must produce the same bits.

Also reported on the same line: the batched form (the mixed 64-job workload:
plain megakernel job by job, one sample per launch as the reference's host
dispatches, vs. the persistent and wavefront batched forms), the served form
(Poisson requests over resident scenes: sustained Mpaths/s, p50/p99),
end-to-end throughput through the public context API with host buffers, the
HBM roofline and the CPU oracle baseline.

`--impl reference` times the reference algorithm's CPU implementation (the
C++ oracle restating the WGSL megakernel; the reference itself only runs
under a graphics API) on the box's host cores.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged Mpaths/s on 1 B200, batched+served vs plain; p50/p99 job latency"
WORKLOAD = "instanced_spheres"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default=WORKLOAD, choices=["instanced_spheres", "cornell", "glass_spheres"])
    p.add_argument("--width", type=int, default=None)
    p.add_argument("--height", type=int, default=None)
    p.add_argument("--spp", type=int, default=None)
    p.add_argument("--form", default="wavefront", choices=["megakernel", "wavefront"],
                   help="engine of the headline step: the wavefront kernels (mtc_stream_run, the default, also "
                        "what mt_context_render runs) or the plain drop-in megakernel (mtc_trace_samples)")
    p.add_argument("--slots", type=int, default=1 << 21, help="wavefront paths in flight")
    p.add_argument("--refill-lanes", type=int, default=0, help="wavefront traversal refill threshold (0: default)")
    p.add_argument("--steps-per-check", type=int, default=0,
                   help="wavefront traversal steps between refill checks (0: default)")
    p.add_argument("--host-loop", type=int, default=0,
                   help="wavefront form: drive the event loop from the host, checking the queue every N iterations "
                        "(every kernel a separate launch, so that ncu sees each; default 0: the device-driven "
                        "loop, one graph launch per run)")
    p.add_argument("--queue-trace", type=int, default=0,
                   help="wavefront form: print the extension, shadow and finished-path counts of each of the first "
                        "N event iterations of one run (runs stopped after 1..N iterations) and exit")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--mixed-jobs", type=int, default=64)
    p.add_argument("--mixed-spp-divisor", type=int, default=4,
                   help="scale the mixed jobs' spp (log-uniform 4-256) down by this factor")
    p.add_argument("--batch-all", action="store_true",
                   help="also time the plain per-job launches and the persistent megakernel on the mixed jobs")
    p.add_argument("--deep-jobs", type=int, default=16)
    p.add_argument("--deep-spp-divisor", type=int, default=64,
                   help="scale the deep-transport jobs' 256 spp down by this factor")
    p.add_argument("--serve-requests", type=int, default=48)
    p.add_argument("--serve-rates", default="5,50,200", help="Poisson arrival rates (requests/s), one run each")
    p.add_argument("--serve-scenes", type=int, default=32)
    p.add_argument("--serve-quantum", type=int, default=4, help="samples per job per served round")
    p.add_argument("--serve-spp-divisor", type=int, default=4,
                   help="scale the requests' target spp (uniform 16-128) down by this factor")
    p.add_argument("--serve-budget-gb", type=float, default=24.0,
                   help="HBM budget of the server: resident scenes + engine state + admitted accumulation")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def oracle_traffic(host, rows=8, spp=2):
    """Algorithmic bytes per path sample from the instrumented CPU oracle on a
    row sample of the same workload."""
    from tests import oracle_lib
    acc = oracle_lib.Accum(host.width, host.height)
    total = None
    for r in np.linspace(0, host.height - 1, rows).astype(int):
        t = oracle_lib.trace(host, acc, spp, rows=(int(r), int(r) + 1), traffic=True)
        total = t if total is None else {k: total[k] + t[k] for k in t}
    return oracle_lib.algorithmic_bytes(total), total


# DRAM bytes (read + write) measured by ncu, per unit of work: the plain
# megakernel per path sample, the wavefront kernels per queued ray or
# finished path (small-case captures; the wavefront's normalised by exact
# queue lengths), scaled by the units this step processed.
MEGAKERNEL_TRAFFIC = ("k_trace_instanced_spheres_960x540_4spp.md", "dram_bytes_per_path:")
WAVEFRONT_TRAFFIC = ("wavefront_dram_per_kernel_instanced_spheres_960x540_4spp.md",
                     ("dram_bytes_per_extension_ray:", "dram_bytes_per_shaded_ray:", "dram_bytes_per_shadow_ray:",
                      "dram_bytes_per_finished_path:"))


def _profile_values(name, keys):
    values = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            for k in keys:
                if line.startswith(k):
                    values[k] = float(line.split(":")[1])
    except OSError:
        pass
    return values


def measured_traffic(form, args, host, spp, units=None):
    """DRAM bytes (read + write) of one step of this workload from the
    committed ncu summaries; (None, None) where none applies.  `units`
    (extension rays, shadow rays, paths of one step) scales the wavefront's
    per-unit figures."""
    if args.workload != WORKLOAD:
        return None, None
    if form == "megakernel":
        name, key = MEGAKERNEL_TRAFFIC
        v = _profile_values(name, (key,))
        if key not in v:
            return None, None
        return int(v[key] * host.width * host.height * spp), "profiles/" + name + " (per path x this step's paths)"
    name, keys = WAVEFRONT_TRAFFIC
    v = _profile_values(name, keys)
    if units is None or len(v) != len(keys):
        return None, None
    ext, shadow, paths = units
    total = (v[keys[0]] + v[keys[1]]) * ext + v[keys[2]] * shadow + v[keys[3]] * paths
    return int(total), "profiles/" + name + " (per-unit figures x this step's rays and paths)"


def cpu_baseline(host, spp, seconds, keep=None):
    """The CPU oracle on all host cores over a bounded row sample (full spp).
    With `keep` (a dict), the oracle accumulation and the rows it rendered are
    left there for the parity check."""
    from tests import oracle_lib
    acc = oracle_lib.Accum(host.width, host.height)
    # Rows in a strided order (0, 37, 74, ...) so the sample covers the whole
    # image rather than its cheapest band.
    stride = 37
    order = [r for k in range(stride) for r in range(k, host.height, stride)]
    rows, done_paths, elapsed = 0, 0, 0.0
    t0 = time.perf_counter()
    while elapsed < seconds and rows < len(order):
        r = order[rows]
        oracle_lib.trace(host, acc, spp, rows=(r, r + 1))
        done_paths += host.width * spp
        rows += 1
        elapsed = time.perf_counter() - t0
    mp = done_paths / elapsed / 1e6
    if keep is not None:
        keep["acc"], keep["rows"] = acc, order[:rows]
    return {"value": round(mp, 4), "unit": "Mpaths/s", "cores": oracle_lib.threads(), "kind": "port",
            "sample": f"{rows} rows (stride {stride}) of {host.width}x{host.height} at {spp} spp "
                      f"({done_paths} path samples, {elapsed:.1f} s)"}


def row_parity(gpu_color, gpu_normal, oracle_acc, rows, width, height):
    """Image parity of the timed GPU image against the CPU oracle on the rows
    the oracle rendered (same seed, same spp): relative MSE of the resolved
    HDR rows and relative mean-luminance difference, against the bars
    relMSE <= 1e-3 and luminance within 0.5 %."""
    rows = np.asarray(sorted(rows), dtype=np.int64)
    g = gpu_color.reshape(height, width, 4)[rows, :, :3].astype(np.float64)
    gn = np.maximum(gpu_normal.reshape(height, width, 4)[rows, :, 3:4], 1.0)
    o = oracle_acc.color.reshape(height, width, 4)[rows, :, :3].astype(np.float64)
    on = np.maximum(oracle_acc.normal.reshape(height, width, 4)[rows, :, 3:4], 1.0)
    a, b = g / gn, o / on
    rel = float(((a - b) ** 2).sum() / max(float((b ** 2).sum()), 1e-30))
    w = np.array([0.2126, 0.7152, 0.0722])
    la, lb = float((a @ w).mean()), float((b @ w).mean())
    luma = abs(la - lb) / max(lb, 1e-30)
    counts = bool(np.array_equal(gpu_normal.reshape(height, width, 4)[rows, :, 3],
                                 oracle_acc.normal.reshape(height, width, 4)[rows, :, 3]))
    return {"rows": int(len(rows)), "pixels": int(len(rows) * width), "rel_mse": float(f"{rel:.3e}"),
            "luma_rel": float(f"{luma:.3e}"), "sample_counts_equal": counts,
            "pass": bool(rel <= 1e-3 and luma <= 0.005 and counts),
            "bars": "relMSE <= 1e-3, mean luminance within 0.5 %, same per-pixel sample counts"}


def workload_desc(name, host, spp):
    b = host.bundle
    env = f"{b.env_width}x{b.env_height} sky" if b.env_width else "no env map"
    return (f"{name} {host.width}x{host.height} {spp} spp, bounces {b.uniform.bounces}, "
            f"{host.info.triangles} instanced tris ({host.info.unique_triangles} unique), {env} + "
            f"{b.lights_count} analytic lights")


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from mutracer_b200 import scene
    host = scene.make_workload(args.workload, width=args.width, height=args.height)
    spp = args.spp
    per_step = max(1.0, args.cpu_seconds / max(1, args.steps))
    for _ in range(args.warmup):
        cpu_baseline(host, spp, 0.5)
    vals = []
    samples = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        b = cpu_baseline(host, spp, per_step)
        vals.append(b["value"])
        samples.append(b["sample"])
    wall = time.perf_counter() - t0
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpaths/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1000 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": workload_desc(args.workload, host, spp), "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": samples[-1]},
            "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def flush_l2(buf):
    buf.add_(1.0)


def queue_trace(sb, counters, slots, iterations):
    """Queue sizes of each event iteration of one wavefront run: the run is
    repeated from zeroed accumulation (a pixel's sample index is its
    accumulated count), stopped by its iteration limit after 1, 2, ...
    `iterations` iterations, and the counter totals are differenced.  For an RGB
    scene every queued extension ray is traced and every finished slot ends a
    path, so the three counts are the queue lengths k_wf_extend (and
    k_wf_shade), k_wf_shadow and k_wf_finish see in that iteration; they
    normalise single-launch profiler captures to bytes per ray."""
    import torch
    from mutracer_b200 import abi
    rows, last = [], [0, 0, 0]
    for k in range(1, iterations + 1):
        sb.stream_config = abi.StreamConfig.make(slots=slots, max_iterations=k,
                                                 iterations_per_check=sb.stream_config.iterations_per_check)
        counters.zero_()
        for j in sb.jobs:                 # every run starts from sample 0 of every pixel
            j.acc.zero_()
        try:
            sb.run()
        except abi.MtError as err:
            if err.status != abi.MT_ERROR_TIMEOUT:
                raise
        torch.cuda.synchronize()
        c = [int(x) for x in counters.cpu().tolist()[:3]]
        rows.append({"iteration": k - 1, "extension": c[1] - last[1], "shadow": c[2] - last[2],
                     "finished": c[0] - last[0]})
        last = c
    return {"queue_trace": rows, "slots": slots}


def run_b200(args):
    import torch
    from mutracer_b200 import abi, scene, trace
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev_id = torch.device("cuda", local)
    host = scene.make_workload(args.workload, width=args.width, height=args.height)
    dev = scene.DeviceScene(host, dev_id)
    acc = trace.Accumulation(host.width, host.height, dev_id)
    spp = args.spp
    stream = torch.cuda.current_stream()
    counters = trace.counters_tensor(dev_id)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev_id)  # 256 MB > 126 MB L2
    paths_per_step = host.width * host.height * spp

    if args.form == "wavefront":
        from mutracer_b200 import batch
        job = batch.RenderJob(dev, spp, device=dev_id)
        acc = job.acc
        sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=args.slots, refill_lanes=args.refill_lanes,
                                                                      iterations_per_check=args.host_loop,
                                                                      steps_per_check=args.steps_per_check),
                               device=dev_id)
        sb.counters = counters
        sb.set_jobs([job])
        if args.queue_trace:
            print(json.dumps(queue_trace(sb, counters, args.slots, args.queue_trace)), flush=True)
            return

        def step():
            acc.zero_()
            sb.run()
    else:
        def step():
            acc.zero_()
            trace.trace_samples(dev, acc, spp, counters=counters)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    counters.zero_()
    times = []
    with ClockSampler(local) as clocks:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush_l2(flush)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step()
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device=dev_id)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    mpaths = paths_per_step * args.steps * world / (total_ms / 1000.0) / 1e6
    cnt = counters.cpu().numpy()
    rays_per_step = float(cnt[1] + cnt[2]) / args.steps
    result = {"metric": METRIC, "value": round(mpaths, 3), "unit": "Mpaths/s", "n_gpus": world,
              "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
              "data": "synthetic (seeded generator, random-init scene)",
              "config": {"workload": workload_desc(args.workload, host, spp),
                         "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                         "l2": "flushed between steps (256 MB write)",
                         "form": "plain megakernel (mtc_trace_samples)" if args.form == "megakernel"
                         else f"wavefront (mtc_stream_run, {args.slots} slots, "
                              + (f"host-driven loop, check every {args.host_loop} iterations)" if args.host_loop
                                 else "device-driven loop)")},
              "mrays_per_s": round(rays_per_step / (ms_per_step / 1000.0) / 1e6, 2),
              "mrays_per_s_extension": round(float(cnt[1]) / args.steps / (ms_per_step / 1000.0) / 1e6, 2),
              "mrays_per_s_shadow": round(float(cnt[2]) / args.steps / (ms_per_step / 1000.0) / 1e6, 2),
              "gpu_launches": int(cnt[3]),
              "clocks": clocks.summary()}
    # End to end through the context API on every rank (its own replica); the
    # slowest rank sets the step time of the whole job.
    e2e = None
    if not args.no_e2e:
        if world > 1:
            torch.distributed.barrier()
        e2e = e2e_context(host, spp, max(1, min(args.steps, 3)))
        if world > 1:
            t = torch.tensor([e2e["ms_per_step"]], device=dev_id)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e["ms_per_step"] = round(float(t.item()), 2)
            e2e["value"] = round(world * paths_per_step / (float(t.item()) / 1000.0) / 1e6, 3)
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    # Roofline (HBM-bound path; L2-level traffic proxy per path sample).
    peak, peak_kind = load_peaks()
    try:
        bpp, traffic = oracle_traffic(host)
        achieved = bpp * paths_per_step / (ms_per_step / 1000.0) / 1e9
        dram, source = measured_traffic(args.form, args, host, spp,
                                        units=(float(cnt[1]) / args.steps, float(cnt[2]) / args.steps,
                                               float(paths_per_step)))
        result["roofline"] = {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                              "frac": round(achieved / peak, 4), "traffic": dram,
                              "peak_source": peak_kind,
                              "bytes_per_path": round(bpp, 1),
                              "kernel": "k_trace (one launch per step)" if args.form == "megakernel" else
                              "all wavefront kernels of the step (k_wf_extend the largest, ~44 %)",
                              "traffic_source": source}
    except Exception as exc:  # the oracle library may be absent on a box
        result["roofline"] = {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                              "traffic": None, "error": str(exc)[:200]}
    if e2e is not None:
        result["e2e"] = e2e
    # The CPU baseline and the single-GPU batched and served forms run at N=1.
    if world == 1:
        try:
            keep = {}
            result["cpu_baseline"] = cpu_baseline(host, spp, args.cpu_seconds, keep)
            # The oracle rows double as the parity check of the timed image
            # (the last timed step's accumulation, same seed and spp).
            result["parity"] = row_parity(acc.color.cpu().numpy(), acc.normal.cpu().numpy(), keep["acc"],
                                          keep["rows"], host.width, host.height)
        except Exception as exc:
            result["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    if not args.no_batch and world == 1:
        if args.form == "megakernel":
            result["wavefront_same_job"] = same_job_wavefront(dev, acc, spp, paths_per_step, dev_id, flush)
        else:
            result["megakernel_same_job"] = same_job_megakernel(args, host, dev, acc, spp, paths_per_step, dev_id,
                                                                flush)
        del dev, acc, flush
        torch.cuda.empty_cache()
        result["batched"] = mixed_batch(args, dev_id)
        result["served"] = served_stream(args, dev_id)
        result["deep_transport"] = deep_transport(args, dev_id)
        result["blas_build"] = blas_build(args, dev_id)
    print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def e2e_context(host, spp, steps):
    """The same job through the public context API with host buffers: commit
    (host-to-device copy of the bundle), render (which runs the wavefront
    engine), read_pixels (device-to-host)."""
    from mutracer_b200.context import Context
    ctx = Context()
    b = host.bundle
    h2d = (b.bvh_vec4_count * 16 + b.instance_count * 160 + b.attribute_words * 4 + b.material_count * 416
           + b.env_width * b.env_height * 16 + (b.env_width + 2) * (b.env_height + 1) * 8
           + b.light_sampling_texels * 16 + 32 * 2177 * 4 + b.lights_count * 96)
    d2h = host.width * host.height * 16  # read_pixels: one averaged f32 RGBA image
    out = np.empty((host.height, host.width, 4), np.float32)
    ctx.commit(host)
    ctx.render(1)
    ctx.read_pixels(out=out)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.commit(host)
        ctx.render(spp)
        ctx.read_pixels(out=out)
    dt = (time.perf_counter() - t0) / steps
    ctx.destroy()
    return {"value": round(host.width * host.height * spp / dt / 1e6, 3), "unit": "Mpaths/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(dt * 1000, 2),
            "path": "mt_context_commit_bundle + mt_context_render (wavefront) + mt_context_read_pixels"}


def _timed(fn, stream):
    import torch
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    fn()
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e)


def same_job_megakernel(args, host, dev, acc, spp, paths, dev_id, flush):
    """The headline job through the plain drop-in megakernel
    (mtc_trace_samples), timed like the headline steps, with its own
    roofline, and checked bit-identical to the wavefront image."""
    import torch
    from mutracer_b200 import trace
    wave = acc.color.clone()
    mega = trace.Accumulation(host.width, host.height, dev_id)
    counters = trace.counters_tensor(dev_id)
    stream = torch.cuda.current_stream()
    times = []
    for it in range(4):                   # one warm-up, three timed
        mega.zero_()
        flush_l2(flush)
        ms = _timed(lambda: trace.trace_samples(dev, mega, spp, counters=counters), stream)
        if it:
            times.append(ms)
    ms = sum(times) / len(times)
    out = {"ms_per_step": round(ms, 2), "mpaths_per_s": round(paths / ms / 1e3, 3),
           "bit_identical_to_wavefront": bool(torch.equal(mega.color, wave)),
           "gpu_launches_per_step": 1}
    peak, kind = load_peaks()
    try:
        bpp, _ = oracle_traffic(host)
        achieved = bpp * paths / (ms / 1000.0) / 1e9
        dram, source = measured_traffic("megakernel", args, host, spp)
        out["roofline"] = {"bound": "hbm", "kernel": "k_trace", "achieved": round(achieved, 2), "peak": peak,
                           "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": dram,
                           "traffic_source": source, "peak_source": kind}
    except Exception as exc:
        out["roofline"] = {"error": str(exc)[:200]}
    del mega
    return out


def same_job_wavefront(dev, acc, spp, paths, dev_id, flush):
    """The headline job through mtc_stream_run (default knobs), timed like the
    plain steps (L2 flushed, CUDA events), and checked bit-identical to the
    plain megakernel's image of the last timed step."""
    import torch
    from mutracer_b200 import abi, batch
    plain = acc.color.clone()
    job = batch.RenderJob(dev, spp, device=dev_id)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(), device=dev_id)
    sb.set_jobs([job])
    stream = torch.cuda.current_stream()
    times = []
    for it in range(4):                   # one warm-up, three timed
        job.acc.zero_()
        flush_l2(flush)
        ms = _timed(sb.run, stream)
        if it:
            times.append(ms)
    ms = sum(times) / len(times)
    out = {"ms_per_step": round(ms, 2), "mpaths_per_s": round(paths / ms / 1e3, 3),
           "bit_identical_to_plain": bool(torch.equal(job.acc.color, plain)),
           "config": "defaults: 2M slots, refill at 4 idle lanes, 8 steps per refill check, regroup every "
                     "iteration"}
    del sb, job
    return out


def mixed_batch(args, dev_id):
    """The mixed 64-job workload four ways, each job from zeroed buffers:
    plain per-sample (one mtc_trace_samples launch per sample per job, the
    reference host's dispatch pattern), plain per-job (one launch per job with
    all its samples), persistent (all jobs in one persistent-megakernel
    launch replayed from a captured CUDA graph) and wavefront (all jobs in
    one mtc_stream_run, knobs from the autotuner).  Every job's image is
    bit-identical across the four (checked here on every job)."""
    import torch
    from mutracer_b200 import batch
    stream = torch.cuda.current_stream()
    specs = batch.mixed_jobs(args.mixed_jobs, seed=0, spp_divisor=args.mixed_spp_divisor)
    t0 = time.perf_counter()
    jobs = batch.build_mixed(specs, dev_id)
    build_s = time.perf_counter() - t0
    paths = batch.total_paths(jobs)

    def zero():
        for j in jobs:
            j.acc.zero_()

    t0 = time.perf_counter()
    scfg, timings = batch.autotune_stream(jobs, probe_samples=1, device=dev_id)
    tune_s = time.perf_counter() - t0
    pb = batch.Batch(len(jobs), None, dev_id)
    pb.set_jobs(jobs)
    pb.capture()
    sb = batch.StreamBatch(len(jobs), None, scfg, dev_id)
    sb.set_jobs(jobs)
    res = {}
    ref = None
    methods = [("plain_per_sample", lambda: batch.run_plain(jobs, per_sample=True), 1)]
    if args.batch_all:
        methods += [("plain_per_job", lambda: batch.run_plain(jobs, per_sample=False), 1),
                    ("persistent_graph", pb.replay, 2)]
    methods.append(("wavefront", sb.run, 2))
    for name, fn, runs in methods:
        ms = []
        for it in range(runs):            # graph capture / first-run work in an untimed run; the last is timed
            zero()
            ms.append(_timed(fn, stream))
        res[name] = {"ms": round(ms[-1], 2), "mpaths_per_s": round(paths / ms[-1] / 1e3, 3)}
        imgs = [j.acc.color.clone() for j in jobs]
        if ref is None:
            ref = imgs
        res[name]["bit_identical_to_plain"] = all(torch.equal(a, b) for a, b in zip(imgs, ref))
        del imgs
    pb.release()
    del sb
    res.update({
        "workload": f"{len(jobs)} jobs, resolution from {{256^2, 512^2, 1280x720, 1920x1080}}, spp log-uniform "
                    f"[4,256] / {args.mixed_spp_divisor} (rounded up), instanced-sphere scenes 10k-2M tris, "
                    f"1-8 rect lights + 512x256 sky, depth 6, seed 0",
        "paths": int(paths), "scene_build_s": round(build_s, 1), "autotune_s": round(tune_s, 1),
        "wavefront_config": {"slots": scfg.slots, "refill_lanes": scfg.refill_lanes,
                             "regroup_interval": scfg.regroup_interval, "sort_rays": scfg.sort_rays,
                             "steps_per_check": scfg.steps_per_check,
                             "traversal_ctas_per_sm": scfg.traversal_ctas_per_sm},
        "autotune_probe_ms": {k: round(v, 2) for k, v in timings.items()},
        "speedup_vs_plain_per_sample": round(res["plain_per_sample"]["ms"] / res["wavefront"]["ms"], 3),
    })
    if args.batch_all:
        res["speedup_vs_plain_per_job"] = round(res["plain_per_job"]["ms"] / res["wavefront"]["ms"], 3)
    del jobs
    torch.cuda.empty_cache()
    return res


def deep_transport(args, dev_id):
    """Deep transport: concurrent spectral glass-sphere jobs (32 dispersive
    spheres with scattering interiors, IOR 1.5, Abbe 40, 1 sphere light,
    bounces 32 -> the reference's 20-event cap, 1280x720), plain per-sample
    megakernel vs one wavefront pass; images bit-identical."""
    import torch
    from mutracer_b200 import batch, scene
    stream = torch.cuda.current_stream()
    spp = max(1, 256 // args.deep_spp_divisor)
    jobs = []
    for j in range(args.deep_jobs):
        host = scene.SceneHost("glass_spheres", 1280, 720, j + 1, (32,))
        jobs.append(batch.RenderJob(scene.DeviceScene(host, dev_id), spp, device=dev_id, job_id=j))
    paths = batch.total_paths(jobs)
    sb = batch.StreamBatch(len(jobs), None, None, dev_id)
    sb.set_jobs(jobs)
    res = {}
    ref = None
    for name, fn in (("plain_per_sample", lambda: batch.run_plain(jobs, per_sample=True)), ("wavefront", sb.run)):
        ms = []
        for it in range(2):               # one warm-up, one timed
            for j in jobs:
                j.acc.zero_()
            ms.append(_timed(fn, stream))
        res[name] = {"ms": round(ms[-1], 2), "mpaths_per_s": round(paths / ms[-1] / 1e3, 3)}
        imgs = [j.acc.color.clone() for j in jobs]
        if ref is None:
            ref = imgs
        res[name]["bit_identical_to_plain"] = all(torch.equal(a, b) for a, b in zip(imgs, ref))
    res.update({
        "workload": f"{len(jobs)} spectral glass jobs (32 dispersive spheres with homogeneous interiors, seeds "
                    f"1-{len(jobs)}), 1280x720, {spp} spp (256 / {args.deep_spp_divisor}), bounces 32 (20-event cap)",
        "paths": int(paths),
        "speedup_vs_plain_per_sample": round(res["plain_per_sample"]["ms"] / res["wavefront"]["ms"], 3),
    })
    del sb, jobs
    torch.cuda.empty_cache()
    return res


def blas_build(args, dev_id):
    """BLAS build and refit on the device (mtc_build_blas, mtc_refit_blas)
    against the host producer (the C++ restatements of buildBLAS and
    refitBLAS, one core) on the same seeded terrain meshes; the buffers must
    be byte-identical.  The host build runs on the smaller mesh only (about
    7 s); the device build on both."""
    import torch
    from mutracer_b200 import blas
    res = {}
    for side in (1000, 2000):
        pos, idx = blas.terrain_mesh(side, side, seed=3)
        n = len(idx)
        pos_t = torch.from_numpy(pos).to(dev_id)
        idx_t = torch.from_numpy(idx.view(np.int32)).to(dev_id)
        builder = blas.BlasBuilder(n, 8, dev_id)
        out = torch.empty(blas.max_vec4(n) * 4, dtype=torch.float32, device=dev_id)
        builder.build(pos_t, idx_t, out)
        ms = []
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            buf, info = builder.build(pos_t, idx_t, out)   # returns once the buffer is complete
            ms.append((time.perf_counter() - t0) * 1e3)
        entry = {"triangles": n, "device_ms": round(float(np.median(ms)), 2), "nodes": int(info.node_count),
                 "max_depth": int(info.max_depth), "host_syncs": int(info.host_syncs),
                 "mtris_per_s": round(n / float(np.median(ms)) / 1e3, 1)}
        # refitBLAS after a deformation (x1.5): plan once, then one launch per depth.
        bvh = buf.clone()
        t0 = time.perf_counter()
        refit = blas.BlasRefit(bvh)
        entry["refit_plan_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
        moved_t = pos_t * 1.5
        refit.refit(moved_t)
        rms = []
        for _ in range(5):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            refit.refit(moved_t, area=False)
            ev[1].record()
            torch.cuda.synchronize()
            rms.append(ev[0].elapsed_time(ev[1]))
        entry["refit_device_ms"] = round(float(np.median(rms)), 3)
        if side == 1000:
            t0 = time.perf_counter()
            want, _ = blas.host_build(pos, idx, 8)
            entry["host_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
            entry["speedup_vs_host"] = round(entry["host_ms"] / entry["device_ms"], 1)
            entry["byte_identical"] = buf.cpu().numpy().view(np.uint32).tobytes() == want.view(np.uint32).tobytes()
            moved = moved_t.cpu().numpy()
            t0 = time.perf_counter()
            want_refit, _ = blas.host_refit(want, moved)
            entry["refit_host_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
            entry["refit_byte_identical"] = \
                bvh.cpu().numpy().view(np.uint32).tobytes() == want_refit.view(np.uint32).tobytes()
        res[f"terrain_{n}"] = entry
        del builder, out, buf, pos_t, idx_t, bvh, refit
        torch.cuda.empty_cache()
    res["workload"] = ("seeded terrain meshes (1000^2 and 2000^2 cells, 2 triangles each, shuffled), bins 8; host "
                       "producer = C++ restatement of buildBLAS / refitBLAS on one core; refit after scaling the "
                       "positions by 1.5")
    return res


def served_stream(args, dev_id):
    """Poisson request stream over a pool of resident scenes, served by
    continuous batching; p50/p99 time-to-target-spp and sustained Mpaths/s."""
    import torch
    from mutracer_b200 import batch, scene, serve
    t0 = time.perf_counter()
    pool = serve.build_pool(args.serve_scenes, seed=7, device=dev_id)
    build_s = time.perf_counter() - t0
    budget = int(args.serve_budget_gb * 1024 ** 3)
    srv = serve.Server(pool, hbm_budget_bytes=budget, max_jobs=64, quantum=args.serve_quantum, device=dev_id)
    warm = serve.poisson_requests(pool, 4, 1000.0, seed=12, spp_divisor=args.serve_spp_divisor)
    srv.run(warm)
    rates = {}
    for rate in (float(r) for r in args.serve_rates.split(",")):
        reqs = serve.poisson_requests(pool, args.serve_requests, rate, seed=11, spp_divisor=args.serve_spp_divisor)
        stats = srv.run(reqs)
        stats["offered_s"] = reqs[-1].arrival
        rates[f"{rate:g}"] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in stats.items()
                              if k != "resident_bytes"}
    resident = srv.fixed_bytes
    srv.release()
    return {
        "rates_per_s": rates,
        "workload": f"{args.serve_requests} requests per rate, Poisson arrivals, {len(pool)} resident scenes "
                    f"({pool.device_bytes / 1e9:.2f} GB, 10k-8M instanced tris), orbit cameras FOV 30-70, "
                    f"resolution from {{256^2, 512^2, 1280x720, 1920x1080}}, target spp U[16,128] / "
                    f"{args.serve_spp_divisor}",
        "hbm_budget_gb": args.serve_budget_gb, "resident_gb": round(resident / 1e9, 3),
        "pool_build_s": round(build_s, 1), "quantum_spp": args.serve_quantum, "max_jobs": 64,
        "engine": "wavefront (mtc_stream_run per round)",
    }


def main():
    args = parse()
    from mutracer_b200 import scene
    w = scene.WORKLOADS[args.workload]
    args.width = args.width or w["width"]
    args.height = args.height or w["height"]
    args.spp = args.spp or w["spp"]
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
