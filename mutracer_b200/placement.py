"""Job placement across GPUs for the batched and served forms.

Render jobs are independent and scenes are read-only, so N GPUs share a job
list with no data-path collective: every rank computes the same placement,
renders the jobs placed on it with its own device and scene replicas, and
only per-job metadata (timings, path counts, image checksums) crosses ranks,
through torch.distributed host-side collectives (gloo on CPU, NCCL on GPUs).
The reference has no multi-device path; its per-job work is one dispatch loop
on one adapter (native/host/src/lib.rs:1506-1560).
"""
import math


def job_cost(width, height, spp, triangles=1):
    """Estimated device time of a job: path samples, weighted by the depth of
    its scene's BVH (log2 of the triangle count)."""
    return float(width) * float(height) * float(spp) * (1.0 + 0.1 * math.log2(max(int(triangles), 1)))


def place(costs, world_size):
    """Longest-processing-time-first placement: jobs in decreasing cost, each
    on the least-loaded rank (lowest rank on ties).  Deterministic, so every
    rank derives the same assignment from the same list.  Returns the rank of
    each job."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return owner


def rank_jobs(costs, rank, world_size):
    """Indices of the jobs placed on `rank`, in their original order."""
    owner = place(costs, world_size)
    return [i for i, r in enumerate(owner) if r == rank]


def imbalance(costs, world_size):
    """Max rank load over the mean rank load (1.0 = perfect balance)."""
    owner = place(costs, world_size)
    load = [0.0] * world_size
    for c, r in zip(costs, owner):
        load[r] += c
    mean = sum(load) / world_size
    return max(load) / mean if mean > 0 else 1.0


def gather(obj):
    """All ranks' `obj` (a picklable host object) on every rank; the list of
    one object without an initialised process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
