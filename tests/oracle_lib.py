"""Test-side access to the CPU oracle (oracle/_build/liboracle.so).

Only tests, __graft_entry__.smoke() and bench.py's CPU baseline use this; the
product never calls the oracle.
"""
import ctypes as C
import os

import numpy as np

from mutracer_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None


def lib():
    global _lib
    if _lib is None:
        from oracle import build
        path = build.build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.oracle_query_first_hit.argtypes = [C.POINTER(abi.SceneView), C.POINTER(abi.TraceUniform), P, C.c_uint32,
                                             P, C.c_int]
        L.oracle_trace_samples.argtypes = [C.POINTER(abi.SceneView), C.POINTER(abi.CameraUniform),
                                           C.POINTER(abi.TraceUniform), P, P, P, P, C.c_uint32, C.c_uint32,
                                           C.c_uint32, C.c_int, P]
        for name in ("oracle_sample_hash", "oracle_owen", "oracle_sobol_d1", "oracle_reverse_bits"):
            getattr(L, name).restype = C.c_uint32
        L.oracle_sample_hash.argtypes = [C.c_uint32]
        L.oracle_sample_seed.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_sample_seed.restype = C.c_uint32
        L.oracle_owen.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_sobol_d1.argtypes = [C.c_uint32]
        L.oracle_reverse_bits.argtypes = [C.c_uint32]
        L.oracle_zsobol_index.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_zsobol_index.restype = C.c_uint32
        L.oracle_morton2.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_morton2.restype = C.c_uint32
        L.oracle_structured_sample.argtypes = [C.c_uint32] * 6 + [C.c_int, C.c_uint32, P]
        L.oracle_sample_maps.argtypes = [C.POINTER(abi.SceneView), P, P, C.c_uint32, P]
        _lib = L
    return _lib


def threads():
    return max(1, os.cpu_count() or 1)


def first_hits(host_scene, rays):
    """querySceneSoftware on the CPU for an (n, 8) float32 ray array."""
    rays = np.ascontiguousarray(rays, dtype=np.float32)
    hits = np.zeros((rays.shape[0], 8), dtype=np.int32)
    v = host_scene.host_view()
    lib().oracle_query_first_hit(C.byref(v), C.byref(host_scene.uniform), rays.ctypes.data, rays.shape[0],
                                 hits.ctypes.data, threads())
    return hits


def sample_maps(host_scene, indices, uvs):
    """sampleMap on the CPU: (n, 4) float32 texels for map `indices` (n,) at
    `uvs` (n, 2)."""
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    uvs = np.ascontiguousarray(uvs, dtype=np.float32)
    out = np.zeros((indices.shape[0], 4), np.float32)
    v = host_scene.host_view()
    lib().oracle_sample_maps(C.byref(v), indices.ctypes.data, uvs.ctypes.data, indices.shape[0], out.ctypes.data)
    return out


class Accum:
    def __init__(self, width, height):
        n = width * height
        self.width, self.height = width, height
        self.color = np.zeros((n, 4), np.float32)
        self.normal = np.zeros((n, 4), np.float32)
        self.albedo = np.zeros((n, 4), np.float32)
        self.catcher = np.zeros((n * 3, 4), np.float32)

    def resolved(self):
        return (self.color / np.maximum(self.normal[:, 3:4], 1.0)).reshape(self.height, self.width, 4)


def trace(host_scene, acc, samples, rows=None, uniform=None, camera=None, traffic=False):
    """`samples` progressive passes of the CPU oracle into `acc` (host arrays)."""
    v = host_scene.host_view()
    u = uniform if uniform is not None else host_scene.uniform
    cam = camera if camera is not None else host_scene.camera
    tr = (C.c_uint64 * 8)() if traffic else None
    r0, r1 = rows if rows is not None else (0, 0)
    lib().oracle_trace_samples(C.byref(v), C.byref(cam), C.byref(u), acc.color.ctypes.data, acc.normal.ctypes.data,
                               acc.albedo.ctypes.data, acc.catcher.ctypes.data, samples, r0, r1, threads(),
                               tr)
    if traffic:
        keys = ("box_tests", "prim_records", "tri_tests", "instance_visits", "material_fetches", "paths",
                "extension_rays", "shadow_rays")
        return dict(zip(keys, list(tr)))
    return None


def algorithmic_bytes(t):
    """Per-path L2-level traffic proxy: 32 B per node box, 16 B per leaf
    primitive record, 48 B per triangle (three vertex positions), 160 B per
    instance visit, 416 B per material fetch, 128 B of accumulation."""
    paths = max(1, t["paths"])
    total = (32 * t["box_tests"] + 16 * t["prim_records"] + 48 * t["tri_tests"] + 160 * t["instance_visits"]
             + 416 * t["material_fetches"] + 128 * paths)
    return total / paths


def seeded_rays(host_scene, n, seed=7, miss_fraction=0.1):
    """Rays from a sphere around the scene toward points inside its bounds."""
    rng = np.random.default_rng(seed)
    b = np.array(host_scene.info.world_bounds, dtype=np.float64)
    lo, hi = b[:3], b[3:]
    center = (lo + hi) / 2
    radius = np.linalg.norm(hi - lo) * 0.75 + 1e-3
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    origin = center + u * radius
    target = lo + rng.random((n, 3)) * (hi - lo)
    d = target - origin
    miss = rng.random(n) < miss_fraction
    d[miss] = rng.normal(size=(int(miss.sum()), 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = origin
    rays[:, 4:7] = d
    return rays
