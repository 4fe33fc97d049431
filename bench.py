"""Benchmark: converged Mpaths/s of the path-tracing megakernel on one B200.

Workload (the large plain-method configuration): 256 seeded affine instances
of 16 displaced icospheres (15,680 triangles each, 4,014,080 instanced
triangles), 2048x1024 analytic sky plus 4 rect lights, 1920x1080, 16 spp,
6 bounces, OpenPBR diffuse / F82 metal / coat.  One step renders the whole
job (16 spp over 1080p) from zeroed accumulation buffers.

Also reported on the same line: the batched form (mixed 64-job workload in one
persistent launch vs. the plain kernel job by job), end-to-end throughput
through the public context API with host buffers, the HBM roofline of the
megakernel and the CPU oracle baseline.

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
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--spp", type=int, default=16)
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
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


def cpu_baseline(host, spp, seconds):
    """The CPU oracle on all host cores over a bounded row sample (full spp)."""
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
    return {"value": round(mp, 4), "unit": "Mpaths/s", "cores": oracle_lib.threads(), "kind": "port",
            "sample": f"{rows} rows (stride {stride}) of {host.width}x{host.height} at {spp} spp "
                      f"({done_paths} path samples, {elapsed:.1f} s)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from mutracer_b200 import scene
    host = scene.make_workload(WORKLOAD, width=args.width, height=args.height)
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
            "config": {"workload": f"{WORKLOAD} {args.width}x{args.height} {spp} spp depth 6, 4,014,080 instanced tris",
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": samples[-1]},
            "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def flush_l2(buf):
    buf.add_(1.0)


def run_b200(args):
    import torch
    from mutracer_b200 import abi, scene, trace
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev_id = torch.device("cuda", local)
    host = scene.make_workload(WORKLOAD, width=args.width, height=args.height)
    dev = scene.DeviceScene(host, dev_id)
    acc = trace.Accumulation(host.width, host.height, dev_id)
    spp = args.spp
    stream = torch.cuda.current_stream()
    counters = trace.counters_tensor(dev_id)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev_id)  # 256 MB > 126 MB L2
    paths_per_step = host.width * host.height * spp

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
              "config": {"workload": f"{WORKLOAD} {host.width}x{host.height} {spp} spp depth 6, "
                                     f"{host.info.triangles} instanced tris ({host.info.unique_triangles} unique), "
                                     f"2048x1024 sky + 4 rect lights",
                         "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                         "l2": "flushed between steps (256 MB write)", "form": "plain megakernel"},
              "mrays_per_s": round(rays_per_step / (ms_per_step / 1000.0) / 1e6, 2),
              "gpu_launches": args.steps,
              "clocks": clocks.summary()}
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    # Roofline (HBM-bound path; L2-level traffic proxy per path sample).
    peak, peak_kind = load_peaks()
    try:
        bpp, traffic = oracle_traffic(host)
        achieved = bpp * paths_per_step / (ms_per_step / 1000.0) / 1e9
        result["roofline"] = {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                              "frac": round(achieved / peak, 4), "traffic": None,
                              "peak_source": peak_kind,
                              "bytes_per_path": round(bpp, 1)}
    except Exception as exc:  # the oracle library may be absent on a box
        result["roofline"] = {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                              "traffic": None, "error": str(exc)[:200]}
    try:
        result["cpu_baseline"] = cpu_baseline(host, spp, args.cpu_seconds)
    except Exception as exc:
        result["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    if not args.no_e2e:
        result["e2e"] = e2e_context(host, spp, max(1, min(args.steps, 3)))
    print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def e2e_context(host, spp, steps):
    """The same job through the public context API with host buffers: commit
    (host-to-device copy of the bundle), render, read_pixels (device-to-host)."""
    from mutracer_b200.context import Context
    ctx = Context()
    b = host.bundle
    h2d = (b.bvh_vec4_count * 16 + b.instance_count * 160 + b.attribute_words * 4 + b.material_count * 416
           + b.env_width * b.env_height * 16 + (b.env_width + 2) * (b.env_height + 1) * 8
           + b.light_sampling_texels * 16 + 32 * 2177 * 4 + b.lights_count * 96)
    d2h = host.width * host.height * 16 * 2
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
            "ms_per_step": round(dt * 1000, 2), "path": "mt_context_commit_bundle + render + read_pixels"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
