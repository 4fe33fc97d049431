"""BLAS build on the device (mtc_build_blas): the reference's buildBLAS
(src/renderer/bvhAccel.ts:200-286) for a triangle mesh already in device
memory, producing the same BVH2 buffer as the host producer."""
import ctypes as C

import numpy as np

from . import abi


def scratch_bytes(triangles, bins=8):
    return int(abi.lib().mtc_blas_build_scratch_bytes(int(triangles), int(bins)))


def max_vec4(triangles):
    return int(abi.lib().mtc_blas_build_max_vec4(int(triangles)))


class BlasBuilder:
    """Reusable scratch for device BLAS builds of up to `max_triangles`."""

    def __init__(self, max_triangles, bins=8, device="cuda"):
        import torch
        self.device = torch.device(device)
        self.bins = int(bins)
        self.max_triangles = int(max_triangles)
        need = scratch_bytes(self.max_triangles, self.bins)
        if not need:
            raise ValueError("unsupported triangle count or bin count")
        self.scratch = torch.empty(need, dtype=torch.uint8, device=self.device)

    def build(self, positions, indices, out=None, stream=None):
        """positions: (V, 3) float32, indices: (T, 3) int32/uint32 (both on
        the device).  Returns (buffer, result): buffer is a float32 tensor of
        result.vec4_count * 4 values (a view of `out` when given)."""
        import torch
        positions = positions.contiguous()
        indices = indices.contiguous()
        if positions.dtype != torch.float32 or indices.dtype not in (torch.int32,):
            raise TypeError("positions must be float32 and indices int32 (u32 bit patterns)")
        tris = indices.numel() // 3
        if tris > self.max_triangles:
            raise ValueError(f"{tris} triangles exceed this builder's {self.max_triangles}")
        inp = abi.BlasBuildInput()
        inp.struct_size = C.sizeof(inp)
        inp.bins = self.bins
        inp.positions = positions.data_ptr() if positions.numel() else None
        inp.indices = indices.data_ptr() if indices.numel() else None
        inp.vertex_count = positions.numel() // 3
        inp.triangle_count = tris
        cap = max_vec4(tris)
        if out is None:
            out = torch.empty(max(cap, 1) * 4, dtype=torch.float32, device=self.device)
        res = abi.BlasBuildResult()
        res.struct_size = C.sizeof(res)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        abi.check(abi.lib().mtc_build_blas(C.byref(inp), C.c_void_p(self.scratch.data_ptr()), self.scratch.numel(),
                                           C.c_void_p(out.data_ptr()), out.numel() // 4, C.byref(res),
                                           C.c_void_p(st.cuda_stream)))
        return out[: res.vec4_count * 4], res


class BlasRefit:
    """refitBLAS on the device for one layout-0 BLAS (a device tensor view of
    its vec4 words): the plan is made once (mtc_blas_refit_prepare); refit()
    rewrites every node box from new positions (mtc_refit_blas,
    asynchronous, capturable)."""

    def __init__(self, bvh, stream=None):
        import torch
        self.bvh = bvh
        self.vec4 = bvh.numel() // 4
        self.plan = torch.empty(int(abi.lib().mtc_blas_refit_plan_bytes(self.vec4)), dtype=torch.uint8,
                                device=bvh.device)
        self.area = torch.zeros(1, dtype=torch.float64, device=bvh.device)
        info = abi.BlasRefitPlanInfo()
        info.struct_size = C.sizeof(info)
        st = stream if stream is not None else torch.cuda.current_stream(bvh.device)
        abi.check(abi.lib().mtc_blas_refit_prepare(C.c_void_p(bvh.data_ptr()), self.vec4,
                                                   C.c_void_p(self.plan.data_ptr()), self.plan.numel(),
                                                   C.byref(info), C.c_void_p(st.cuda_stream)))
        self.levels, self.nodes = info.levels, info.node_count

    def refit(self, positions, stream=None, area=True):
        """positions: (V, 3) float32 on the device.  Returns the device
        float64 tensor receiving the summed surface area (when area)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(self.bvh.device)
        abi.check(abi.lib().mtc_refit_blas(C.c_void_p(self.bvh.data_ptr()), self.vec4,
                                           C.c_void_p(self.plan.data_ptr()), self.levels,
                                           C.c_void_p(positions.data_ptr()) if positions.numel() else None,
                                           positions.numel() // 3,
                                           C.c_void_p(self.area.data_ptr()) if area else None,
                                           C.c_void_p(st.cuda_stream)))
        return self.area


def host_refit(buffer, positions):
    """The host refitBLAS (C++ restatement) on a copy: (buffer f32, area)."""
    out = np.array(buffer, np.float32)
    pos = np.ascontiguousarray(positions, np.float32)
    area = C.c_double()
    abi.check(abi.lib().mtp_refit_blas(out.ctypes.data, out.size // 4, pos.ctypes.data if pos.size else None,
                                       len(pos), C.byref(area)))
    return out, area.value


def terrain_mesh(w, h, seed=0, amplitude=0.3):
    """Seeded height-field mesh over the unit square: (w+1) x (h+1) vertices,
    2 w h triangles in a shuffled order (positions f32 (V, 3), indices u32
    (T, 3))."""
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:h + 1, 0:w + 1].astype(np.float32)
    z = amplitude * rng.standard_normal(xs.shape).astype(np.float32)
    pos = np.stack([xs / w, z, ys / h], -1).reshape(-1, 3)
    v = (np.arange(h)[:, None] * (w + 1) + np.arange(w)[None, :]).reshape(-1)
    a, b, c, d = v, v + 1, v + w + 1, v + w + 2
    idx = np.concatenate([np.stack([a, b, d], 1), np.stack([a, d, c], 1)]).astype(np.uint32)
    return pos, idx[rng.permutation(len(idx))]


def host_build(positions, indices, bins=8):
    """The host producer (the C++ restatement of buildBLAS): (buffer f32,
    max depth)."""
    pos = np.ascontiguousarray(positions, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    nt = idx.size // 3
    buf = np.zeros(max(5 * nt, 1) * 4, np.float32)
    vec4, depth = C.c_uint64(), C.c_uint32()
    abi.check(abi.lib().mtp_build_blas(pos.ctypes.data, pos.size // 3, idx.ctypes.data, nt, int(bins),
                                       buf.ctypes.data, buf.size // 4, C.byref(vec4), C.byref(depth)))
    return buf[: vec4.value * 4], depth.value


def main(argv=None):
    """Builds a seeded terrain mesh on the device (one warm-up build, then
    timed builds) and prints one JSON line per timed build."""
    import argparse
    import json
    import time

    import torch
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--side", type=int, default=2000, help="cells per side (2 side^2 triangles)")
    p.add_argument("--bins", type=int, default=8)
    p.add_argument("--repeat", type=int, default=1)
    p.add_argument("--refit", action="store_true", help="also time the refit plan and device refits")
    a = p.parse_args(argv)
    pos, idx = terrain_mesh(a.side, a.side, seed=3)
    pos_t, idx_t = torch.from_numpy(pos).cuda(), torch.from_numpy(idx.view(np.int32)).cuda()
    builder = BlasBuilder(len(idx), a.bins)
    out = torch.empty(max_vec4(len(idx)) * 4, dtype=torch.float32, device="cuda")
    builder.build(pos_t, idx_t, out)
    for _ in range(a.repeat):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, res = builder.build(pos_t, idx_t, out)
        ms = (time.perf_counter() - t0) * 1e3
        print(json.dumps({"triangles": len(idx), "ms": round(ms, 3), "nodes": res.node_count,
                          "max_depth": res.max_depth, "host_syncs": res.host_syncs}), flush=True)
    if a.refit:
        bvh = out[: res.vec4_count * 4]
        t0 = time.perf_counter()
        r = BlasRefit(bvh)
        plan_ms = (time.perf_counter() - t0) * 1e3
        moved = pos_t * 1.5
        r.refit(moved)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for _ in range(a.repeat):
            ev[0].record()
            r.refit(moved, area=False)
            ev[1].record()
            torch.cuda.synchronize()
            print(json.dumps({"refit_triangles": len(idx), "plan_ms": round(plan_ms, 3), "levels": r.levels,
                              "refit_ms": round(ev[0].elapsed_time(ev[1]), 3)}), flush=True)


if __name__ == "__main__":
    main()
