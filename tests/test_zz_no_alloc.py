"""The allocation-free batched entry point (mtc_trace_batch_noalloc), called
through the C ABI, against the existing batched entry point.

mtc_trace_batch_noalloc serves callers that cannot let the library allocate
device memory (a host that owns the whole device budget, a plugin inside such
a host, a serving loop that cannot afford a synchronising cudaMalloc): its
job table and queue counter live in one fixed array inside the library.  Two
calls in a row must each reproduce mtc_trace_batch exactly (the shared array
is rewritten and its counter cleared by every call).  This file is collected
last so that a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, scene, trace
from tests import oracle_lib

pytestmark = pytest.mark.gpu


def _jobs(devs, accs, spps):
    jobs = (abi.JobDesc * len(devs))()
    for i, (d, a, s) in enumerate(zip(devs, accs, spps)):
        jobs[i].scene = d.view
        jobs[i].camera = d.camera
        jobs[i].uniform = d.uniform
        jobs[i].out = a.outputs
        jobs[i].samples = s
    return jobs


def test_noalloc_batch_matches_allocating_batch(cuda):
    import torch
    L = abi.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    hosts = [scene.SceneHost("cornell", 56, 40, 3), scene.SceneHost("cornell", 33, 47, 4),
             scene.make_workload("instanced_spheres", width=40, height=24, params=(16, 2, 5, 128, 1))]
    spps = [6, 3, 4]
    devs = [scene.DeviceScene(h, cuda) for h in hosts]

    ref = [trace.Accumulation(d.width, d.height, cuda) for d in devs]
    scratch = torch.zeros(L.mtc_batch_scratch_bytes(len(devs)), dtype=torch.uint8, device=cuda)
    abi.check(L.mtc_trace_batch(_jobs(devs, ref, spps), len(devs), None, C.c_void_p(scratch.data_ptr()), None, None,
                                stream))
    torch.cuda.synchronize()

    for call in range(2):  # two calls in a row reuse the one shared scratch array
        got = [trace.Accumulation(d.width, d.height, cuda) for d in devs]
        status = torch.full((1,), 7, dtype=torch.int32, device=cuda)
        counters = trace.counters_tensor(cuda)
        abi.check(L.mtc_trace_batch_noalloc(_jobs(devs, got, spps), len(devs), None,
                                            C.c_void_p(status.data_ptr()), C.c_void_p(counters.data_ptr()), stream))
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        assert int(counters[0].item()) == sum(d.width * d.height * s for d, s in zip(devs, spps))
        for a, b in zip(ref, got):
            for x, y in ((a.color, b.color), (a.normal, b.normal), (a.albedo, b.albedo), (a.catcher, b.catcher)):
                assert torch.equal(x, y), f"call {call}"

    # The first job's image also meets the oracle bar (relMSE <= 1e-3, mean
    # luminance within 0.5 %) on its own, independent of mtc_trace_batch.
    oracle = oracle_lib.Accum(hosts[0].width, hosts[0].height)
    oracle_lib.trace(hosts[0], oracle, spps[0])
    a = got[0].resolved().cpu().numpy()[..., :3].astype(np.float64)
    b = oracle.resolved()[..., :3].astype(np.float64)
    rel = float(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-30))
    w = np.array([0.2126, 0.7152, 0.0722])
    luma = abs(float((a @ w).mean()) - float((b @ w).mean())) / max(float((b @ w).mean()), 1e-30)
    assert rel <= 1e-3 and luma <= 0.005, (rel, luma)


def test_noalloc_batch_applies_the_batch_config(cuda):
    """Tile width, block size, CTAs per SM and fetch grain change the schedule,
    never the result."""
    import torch
    L = abi.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    host = scene.SceneHost("cornell", 37, 29, 2)
    dev = scene.DeviceScene(host, cuda)
    ref = trace.Accumulation(37, 29, cuda)
    abi.check(L.mtc_trace_batch_noalloc(_jobs([dev], [ref], [3]), 1, None, None, None, stream))
    cfg = abi.BatchConfig(struct_size=C.sizeof(abi.BatchConfig), block_threads=64, tile_width=4, ctas_per_sm=3,
                          items_per_fetch=5)
    got = trace.Accumulation(37, 29, cuda)
    abi.check(L.mtc_trace_batch_noalloc(_jobs([dev], [got], [3]), 1, C.byref(cfg), None, None, stream))
    torch.cuda.synchronize()
    assert torch.equal(ref.color, got.color) and torch.equal(ref.normal, got.normal)


def test_noalloc_batch_rejects_what_the_allocating_batch_rejects(cuda):
    """One validator serves both batched entry points: a vertex layout whose
    normal words lie past the vertex record, and launch shapes out of range,
    are refused by both before anything runs."""
    import torch
    L = abi.lib()
    host = scene.SceneHost("cornell", 8, 8, 1)
    dev = scene.DeviceScene(host, cuda)
    acc = trace.Accumulation(8, 8, cuda)
    scratch = torch.zeros(L.mtc_batch_scratch_bytes(1), dtype=torch.uint8, device=cuda)
    jobs = _jobs([dev], [acc], [1])
    stride = jobs[0].scene.vertex_layout.stride
    jobs[0].scene.vertex_layout.normal_offset = stride  # one word past the record
    assert L.mtc_trace_batch(jobs, 1, None, C.c_void_p(scratch.data_ptr()), None, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_trace_batch_noalloc(jobs, 1, None, None, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    jobs = _jobs([dev], [acc], [1])
    for bad in (dict(ctas_per_sm=33), dict(block_threads=96 + 1), dict(tile_width=3), dict(items_per_fetch=17)):
        cfg = abi.BatchConfig(struct_size=C.sizeof(abi.BatchConfig), **bad)
        assert L.mtc_trace_batch(jobs, 1, C.byref(cfg), C.c_void_p(scratch.data_ptr()), None, None, None) == \
            abi.MT_ERROR_INVALID_ARGUMENT, bad
        assert L.mtc_trace_batch_noalloc(jobs, 1, C.byref(cfg), None, None, None) == \
            abi.MT_ERROR_INVALID_ARGUMENT, bad
    torch.cuda.synchronize()
    assert float(acc.normal[..., 3].sum()) == 0.0  # nothing ran


def test_noalloc_batch_rejects_more_jobs_than_its_fixed_scratch(cuda):
    L = abi.lib()
    host = scene.SceneHost("cornell", 8, 8, 1)
    dev = scene.DeviceScene(host, cuda)
    n = abi.MTC_BATCH_NOALLOC_MAX_JOBS + 1
    accs = [trace.Accumulation(8, 8, cuda) for _ in range(n)]
    jobs = _jobs([dev] * n, accs, [1] * n)
    assert L.mtc_trace_batch_noalloc(jobs, n, None, None, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_trace_batch_noalloc(None, 1, None, None, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
