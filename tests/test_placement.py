"""Multi-GPU path on CPU: job placement across ranks and the host-side
metadata exchange, with two gloo ranks.  Jobs are rendered by the CPU oracle
here (no GPU); on GPUs each rank runs the same placement through its own
device.  The per-job results must not depend on where a job runs."""
import hashlib
import os
import socket

import numpy as np
import pytest

from mutracer_b200 import batch, placement, scene


def _jobs():
    specs = [batch.JobSpec(i, w, h, s, t, 2, i + 1) for i, (w, h, s, t) in
             enumerate(((24, 16, 2, 10_000), (8, 8, 5, 40_000), (32, 8, 1, 10_000), (16, 16, 3, 80_000),
                        (12, 20, 2, 20_000)))]
    return specs


def _render(spec):
    from tests import oracle_lib
    host = scene.SceneHost("instanced_spheres", spec.width, spec.height, spec.seed, spec.scene_params(64))
    acc = oracle_lib.Accum(host.width, host.height)
    oracle_lib.trace(host, acc, spec.spp)
    return hashlib.sha256(np.ascontiguousarray(acc.color).tobytes()).hexdigest()


def test_place_is_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    costs = list(rng.lognormal(10, 1.5, size=64))
    for n in (1, 2, 4, 8):
        a, b = placement.place(costs, n), placement.place(list(costs), n)
        assert a == b
        assert set(a) <= set(range(n))
        assert sorted(sum((placement.rank_jobs(costs, r, n) for r in range(n)), [])) == list(range(64))
        # LPT bound: no rank exceeds 4/3 of the mean load or the largest job
        mean = sum(costs) / n
        assert placement.imbalance(costs, n) * mean <= max(4.0 / 3.0 * mean, max(costs)) * (1 + 1e-12)
    even = list(np.random.default_rng(4).uniform(1.0, 2.0, size=64))
    assert placement.imbalance(even, 8) < 1.05
    with pytest.raises(ValueError):
        placement.place(costs, 0)


def test_job_cost_orders_by_work():
    assert placement.job_cost(1920, 1080, 16, 4_000_000) > placement.job_cost(1920, 1080, 16, 10_000)
    assert placement.job_cost(512, 512, 64) == 4 * placement.job_cost(256, 256, 64)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        specs = _jobs()
        costs = [placement.job_cost(s.width, s.height, s.spp, s.triangles) for s in specs]
        mine = placement.rank_jobs(costs, rank, world)
        results = {i: _render(specs[i]) for i in mine}
        every = placement.gather({"rank": rank, "placement": placement.place(costs, world), "results": results})
        if rank == 0:
            out.put(every)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_render_their_share_identically():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    every = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert every[0]["placement"] == every[1]["placement"]          # one placement on every rank
    merged = {}
    for e in every:
        assert not (set(merged) & set(e["results"]))                 # no job runs twice
        merged.update(e["results"])
    specs = _jobs()
    assert sorted(merged) == list(range(len(specs)))
    for i, spec in enumerate(specs):                                 # placement does not change results
        assert merged[i] == _render(spec)
