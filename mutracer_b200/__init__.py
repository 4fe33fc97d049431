"""mutracer_b200: B200-native (sm_100a) progressive path-tracing megakernel
behind MuTracer's flattened-buffer contract and C ABI.

Layers:
  abi      ctypes mirror of include/mutracer_b200.h; loads _lib/libmutracer_b200.so
  scene    seeded synthetic scenes in the reference's buffer formats (host + device)
  trace    kernel-level entry points (progressive pass, first-hit query, TLAS refit)
  context  mt_context_* / mt_job_* persistent API
  batch    batched persistent multi-job form and its autotuner
  serve    served form: resident scene pool, HBM-budget admission, continuous batching
"""
from . import abi  # noqa: F401

__all__ = ["abi", "scene", "trace", "context", "batch", "serve", "build_library"]


def build_library(force=False):
    from .build import build
    return build(force=force)
