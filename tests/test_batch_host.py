"""Host-side logic of the batched and served forms (no GPU): the job table
written by mtc_batch_prepare, launch-shape validation, the seeded mixed-job
and Poisson request generators, and the look-at camera helper."""
import ctypes as C

import numpy as np
import pytest

from mutracer_b200 import abi, batch, scene, serve


def _desc(host, samples, out_base=0x10000):
    d = abi.JobDesc()
    d.scene = host.host_view()
    d.camera = host.camera
    d.uniform = host.uniform
    # prepare never dereferences the outputs; any non-null device address will do
    d.out = abi.Outputs(out_base, out_base + 0x100, out_base + 0x200, out_base + 0x300)
    d.samples = samples
    return d


def _prepare(descs, cfg):
    L = abi.lib()
    table = np.zeros(L.mtc_batch_table_bytes(len(descs)), np.uint8)
    arr = (abi.JobDesc * len(descs))(*descs)
    total = C.c_uint32()
    st = L.mtc_batch_prepare(arr, len(descs), C.byref(cfg) if cfg is not None else None,
                             C.c_void_p(table.ctypes.data), C.byref(total))
    return st, table, total.value


@pytest.mark.parametrize("tile_width", [1, 4, 8, 16, 32])
def test_prepare_header_counts_warp_tiles(tile_width):
    hosts = [scene.SceneHost("cornell", 37, 23, 1), scene.SceneHost("cornell", 64, 64, 2),
             scene.SceneHost("cornell", 5, 90, 3)]
    samples = [3, 0, 7]
    cfg = abi.BatchConfig.make(tile_width=tile_width)
    st, table, total = _prepare([_desc(h, s) for h, s in zip(hosts, samples)], cfg)
    assert st == abi.MT_OK
    th = 32 // tile_width
    want = sum(-(-h.width // tile_width) * -(-h.height // th) for h, s in zip(hosts, samples) if s)
    assert total == want
    header = table[:256].view(np.uint32)
    assert (header[0], header[1], header[2]) == (3, want, tile_width)
    assert abi.lib().mtc_batch_table_bytes(3) == 256 + 3 * (len(table) - 256) // 3


def test_prepare_and_launch_reject_bad_shapes():
    host = scene.SceneHost("cornell", 16, 16, 1)
    for kw in (dict(tile_width=3), dict(tile_width=64), dict(block_threads=96 + 64), dict(block_threads=48),
               dict(items_per_fetch=17), dict(ctas_per_sm=33)):
        st, _, _ = _prepare([_desc(host, 1)], abi.BatchConfig.make(**kw))
        assert st == abi.MT_ERROR_INVALID_ARGUMENT, kw
    bad = abi.BatchConfig.make()
    bad.struct_size = 8
    assert _prepare([_desc(host, 1)], bad)[0] == abi.MT_ERROR_INVALID_ARGUMENT
    d = _desc(host, 1)
    d.out.color = None
    assert _prepare([d], None)[0] == abi.MT_ERROR_INVALID_ARGUMENT
    L = abi.lib()
    table = np.zeros(L.mtc_batch_table_bytes(1), np.uint8)
    assert L.mtc_batch_launch(None, 1, None, C.c_void_p(16), None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_batch_launch(C.c_void_p(table.ctypes.data), 1, C.byref(abi.BatchConfig.make(tile_width=3)),
                              C.c_void_p(16), None, None) == abi.MT_ERROR_INVALID_ARGUMENT


def test_mixed_jobs_are_seeded_and_in_range():
    a, b = batch.mixed_jobs(64, seed=3), batch.mixed_jobs(64, seed=3)
    assert a == b
    assert a != batch.mixed_jobs(64, seed=4)
    assert {(j.width, j.height) for j in a} <= set(batch.RESOLUTIONS)
    assert all(4 <= j.spp <= 256 for j in a)
    assert all(10_000 <= j.triangles <= 2_000_000 for j in a)
    assert all(1 <= j.lights <= 8 for j in a)
    spp = np.log([j.spp for j in batch.mixed_jobs(2000, seed=1)])
    assert abs(spp.mean() - 0.5 * (np.log(4) + np.log(256))) < 0.15    # log-uniform
    scaled = batch.mixed_jobs(64, seed=3, spp_divisor=8)
    assert [s.spp for s in scaled] == [max(1, -(-j.spp // 8)) for j in a]


@pytest.mark.parametrize("tris", [10_000, 150_000, 2_000_000, 8_000_000])
def test_scene_params_hit_the_triangle_target(tris):
    sp = batch.JobSpec(0, 256, 256, 4, tris, 3, 1)
    inst, bases, freq, env, lights = sp.scene_params()
    got = inst * 20 * freq * freq
    assert 0.7 * tris <= got <= 1.4 * tris
    assert bases <= 16 and lights == 3 and env == 512


def test_look_at_matches_generator_camera():
    host = scene.SceneHost("cornell", 96, 64, 1)
    cam = abi.CameraUniform()
    d3 = C.c_double * 3
    assert abi.lib().mtp_camera_look_at(96, 64, d3(0, 1, 3.4), d3(0, 1, 0), d3(0, 1, 0), 40.0,
                                        C.byref(cam)) == abi.MT_OK
    assert bytes(cam) == bytes(host.camera)
    assert abi.lib().mtp_camera_look_at(96, 64, d3(0, 1, 3.4), d3(0, 1, 0), d3(0, 1, 0), 0.0,
                                        C.byref(cam)) == abi.MT_ERROR_INVALID_ARGUMENT


class _FakePool:
    def __init__(self, hosts):
        self.hosts = dict(enumerate(hosts))
        self.scenes = dict(self.hosts)


def test_poisson_requests_rate_and_ranges():
    pool = _FakePool([scene.SceneHost("cornell", 8, 8, 1), scene.SceneHost("cornell", 8, 8, 2)])
    reqs = serve.poisson_requests(pool, 400, rate=50.0, seed=2)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert abs(np.diff(arr).mean() - 1 / 50.0) < 0.25 / 50.0
    assert all(16 <= r.spp <= 128 for r in reqs)
    assert {r.scene_id for r in reqs} == {0, 1}
    assert {(r.width, r.height) for r in reqs} <= set(batch.RESOLUTIONS)
    again = serve.poisson_requests(pool, 400, rate=50.0, seed=2)
    assert [bytes(r.camera) for r in again] == [bytes(r.camera) for r in reqs]


def test_plain_entry_points_validate_before_touching_the_device():
    """Argument checks of the C ABI run on the host: rejected calls and
    zero-sample calls return without a CUDA call (this runs without a GPU)."""
    L = abi.lib()
    host = scene.SceneHost("cornell", 16, 16, 1)
    view, cam, uni = host.host_view(), host.camera, host.uniform
    out = abi.Outputs(0x1000, 0x2000, 0x3000, 0x4000)
    assert L.mtc_trace_samples(C.byref(view), C.byref(cam), C.byref(uni), C.byref(out), 0, None, None) == abi.MT_OK
    assert L.mtc_trace_samples(None, C.byref(cam), C.byref(uni), C.byref(out), 1, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    bad = abi.Outputs(0x1000, 0, 0x3000, 0x4000)
    assert L.mtc_trace_samples(C.byref(view), C.byref(cam), C.byref(uni), C.byref(bad), 1, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    v2 = abi.SceneView.from_buffer_copy(view)
    v2.struct_size = 4
    assert L.mtc_trace_samples(C.byref(v2), C.byref(cam), C.byref(uni), C.byref(out), 1, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_query_first_hit(None, None, 0, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_average_output(None, 4, 1, None, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_average_output(C.c_void_p(16), 4, 0, C.c_void_p(16), C.c_void_p(16), None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    cfg = abi.StreamConfig.make(slots=100)                # below the 1024-slot minimum
    assert L.mtc_stream_state_bytes(4, C.byref(cfg)) == 0
    assert L.mtc_stream_run(None, 4, None, C.c_void_p(16), None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_stream_launch(None, 4, None, C.c_void_p(16), None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_stream_launch(C.c_void_p(16), 0, None, C.c_void_p(16), None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_stream_status(None, 4, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_stream_status(C.c_void_p(16), 4, C.byref(cfg), None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert L.mtc_stream_state_bytes(4, None) > (1 << 20) * 400


def test_every_autotune_shape_is_a_valid_batch_config():
    """The autotuner's launch shapes (BatchConfig.make order) all pass the
    batched entry points' validation (batchShape)."""
    from mutracer_b200 import batch
    L = abi.lib()
    table = (C.c_uint8 * L.mtc_batch_table_bytes(1))()
    for shape in batch.AUTOTUNE_SPACE:
        cfg = abi.BatchConfig.make(*shape)
        assert L.mtc_batch_prepare(None, 0, C.byref(cfg), table, None) == abi.MT_OK, shape
    bad = abi.BatchConfig.make(128, 12, 16, 1)           # a warp tile width that does not divide 32
    assert L.mtc_batch_prepare(None, 0, C.byref(bad), table, None) == abi.MT_ERROR_INVALID_ARGUMENT
