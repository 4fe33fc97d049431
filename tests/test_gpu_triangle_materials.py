"""Per-triangle materials and vertex colors on a B200: the device image of a
mesh whose halves select different table entries is bit-identical to the
split meshes' image, in the BVH2 and BVH_GPU layouts and through the batch
entry point, the wavefront engine and mt_context_commit; image parity against
the oracle, with RGBA8 and float vertex colors on the floor."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, batch, scene, trace
from mutracer_b200.context import Context
from tests.test_gpu_parity import LUMA_BAR, REL_MSE_BAR, _image_metrics, _render_pair
from tests.test_triangle_materials import decode, halves

pytestmark = pytest.mark.gpu


def device_render(cuda, host, spp):
    import torch
    dev = scene.DeviceScene(host, cuda)
    acc = trace.Accumulation(host.width, host.height, cuda)
    trace.trace_samples(dev, acc, spp)
    torch.cuda.synchronize()
    return dev, acc


def test_multi_material_mesh_equals_split_meshes(cuda):
    import torch
    _, split = device_render(cuda, decode(halves(False, 64, 48, emissive=True)), 8)
    multi_host = decode(halves(True, 64, 48, emissive=True))
    dev, multi = device_render(cuda, multi_host, 8)
    assert torch.equal(split.color, multi.color) and torch.equal(split.albedo, multi.albedo)
    gpu_layout = decode(halves(True, 64, 48, emissive=True))
    gpu_layout.set_blas_layout(2)
    _, multi2 = device_render(cuda, gpu_layout, 8)
    assert torch.equal(multi.color, multi2.color)
    # batch entry point and wavefront engine
    batched = trace.Accumulation(64, 48, cuda)
    jobs = (abi.JobDesc * 1)()
    jobs[0].scene, jobs[0].camera, jobs[0].uniform = dev.view, dev.camera, dev.uniform
    jobs[0].out, jobs[0].samples = batched.outputs, 8
    scratch = torch.zeros(abi.lib().mtc_batch_scratch_bytes(1), dtype=torch.uint8, device=cuda)
    abi.check(abi.lib().mtc_trace_batch(jobs, 1, None, C.c_void_p(scratch.data_ptr()), None, None,
                                        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    job = batch.RenderJob(dev, 8, device=cuda)
    sb = batch.StreamBatch(1, stream_config=abi.StreamConfig.make(slots=4096), device=cuda)
    sb.set_jobs([job])
    sb.run()
    torch.cuda.synchronize()
    assert torch.equal(multi.color, batched.color) and torch.equal(multi.color, job.acc.color)
    ctx = Context()
    try:
        ctx.commit_descriptor(halves(True, 64, 48, emissive=True).to_bytes())
        ctx.render(8)
        want = (multi.color.cpu().numpy() / np.float32(8)).reshape(48, 64, 4)
        assert np.array_equal(ctx.read_pixels(), want)
    finally:
        ctx.destroy()


@pytest.mark.parametrize("colors", [None, "rgba8", "float"])
def test_multi_material_oracle_parity(cuda, colors):
    host = decode(halves(True, 96, 72, emissive=True, colors=colors))
    if colors:
        assert host.bundle.vertex_layout.color_offset and host.bundle.vertex_layout.color_float == (colors == "float")
    gpu, ref, _, _ = _render_pair(cuda, host, 32)
    rel_mse, luma = _image_metrics(gpu, ref)
    assert rel_mse <= REL_MSE_BAR, rel_mse
    assert luma <= LUMA_BAR, luma
