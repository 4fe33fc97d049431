"""Python mirror of the reference's dispatch for this path.

``trace_samples`` is the per-sample progressive pass of the WGSL megakernel
(rayTrace.compute.ts:1157-1263, dispatched by native/host/src/lib.rs:1506-1560)
on device buffers; ``query_first_hit`` is querySceneSoftware
(intersect.wgsl.ts:660-684); ``refit_tlas`` is refitTLAS
(bvhAccel.ts:579-740).  All of them call the CUDA library through the C ABI.
"""
import ctypes as C

from . import abi


def _stream_ptr(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class Accumulation:
    """The four G3 accumulation buffers (outColor, outNormal, outAlbedo,
    outShadowCatcher), zero-initialised, on the device."""

    def __init__(self, width, height, device="cuda"):
        import torch
        n = width * height
        self.width, self.height = width, height
        self.color = torch.zeros((n, 4), dtype=torch.float32, device=device)
        self.normal = torch.zeros((n, 4), dtype=torch.float32, device=device)
        self.albedo = torch.zeros((n, 4), dtype=torch.float32, device=device)
        self.catcher = torch.zeros((n * 3, 4), dtype=torch.float32, device=device)
        self.outputs = abi.Outputs(self.color.data_ptr(), self.normal.data_ptr(), self.albedo.data_ptr(),
                                   self.catcher.data_ptr())

    def zero_(self):
        for t in (self.color, self.normal, self.albedo, self.catcher):
            t.zero_()

    def resolved(self):
        """HDR image divided by the per-pixel completed count (as read_pixels)."""
        cnt = self.normal[:, 3:4].clamp_min(1.0)
        return (self.color / cnt).reshape(self.height, self.width, 4)


def trace_samples(scene, acc, samples, uniform=None, camera=None, counters=None, stream=None):
    view = scene.view
    u = uniform if uniform is not None else scene.uniform
    cam = camera if camera is not None else scene.camera
    cnt = C.c_void_p(counters.data_ptr()) if counters is not None else None
    st = abi.lib().mtc_trace_samples(C.byref(view), C.byref(cam), C.byref(u), C.byref(acc.outputs), samples, cnt,
                                     _stream_ptr(stream))
    abi.check(st)


def query_first_hit(scene, rays, stream=None):
    """rays: (n, 8) float32 device tensor (o.xyz, pad, d.xyz, pad).
    Returns an (n, 8) int32/float32 record tensor in mtc_hit layout."""
    import torch
    n = rays.shape[0]
    hits = torch.empty((n, 8), dtype=torch.int32, device=rays.device)
    st = abi.lib().mtc_query_first_hit(C.byref(scene.view), C.c_void_p(rays.data_ptr()), n,
                                       C.c_void_p(hits.data_ptr()), _stream_ptr(stream))
    abi.check(st)
    return hits


def refit_tlas(scene, inputs, stream=None):
    """Full device refit of the scene's TLAS and instance records from the
    per-source-instance inputs (dict of device tensors)."""
    tlas_vec4 = scene.host.info.tlas_vec4
    st = abi.lib().mtc_refit_tlas(
        C.c_void_p(scene.bvh.data_ptr()), tlas_vec4, C.c_void_p(scene.instances.data_ptr()),
        scene.host.bundle.instance_count,
        *[C.c_void_p(inputs[k].data_ptr()) for k in ("transforms", "local_bounds", "blas_offsets", "blas_layouts",
                                                      "vertex_offsets", "materials", "colors")],
        _stream_ptr(stream))
    abi.check(st)


def counters_tensor(device="cuda"):
    import torch
    return torch.zeros(4, dtype=torch.int64, device=device)
