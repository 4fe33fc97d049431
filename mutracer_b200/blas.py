"""BLAS build on the device (mtc_build_blas): the reference's buildBLAS
(src/renderer/bvhAccel.ts:200-286) for a triangle mesh already in device
memory, producing the same BVH2 buffer as the host producer."""
import ctypes as C

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
