"""The C-ABI library loads, exports every symbol include/*.h declares, and
its struct layouts match the Python mirror.  No compute call needs a GPU here."""
import ctypes as C
import os
import re

import pytest

from mutracer_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b((?:mt|mtc)_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_symbols_exported():
    lib = abi.lib()
    names = declared_functions()
    assert {"mtc_trace_samples", "mtc_query_first_hit", "mtc_refit_tlas", "mtc_trace_batch",
            "mt_context_commit_bundle", "mt_job_poll"} <= names
    for name in sorted(names):
        assert hasattr(lib, name), name


def test_struct_layouts():
    lib = abi.lib()
    sizes = (C.c_uint32 * 32)()
    n = lib.mtc_struct_sizes(sizes, 32)
    assert n == len(abi.STRUCT_ORDER)
    for i, cls in enumerate(abi.STRUCT_ORDER):
        assert C.sizeof(cls) == sizes[i], cls.__name__
    assert C.sizeof(abi.TraceUniform) == 320          # RayTraceUniform, wgpuSceneUniform.ts:13-55
    assert abi.TraceUniform.blas_offset.offset == 88
    assert abi.TraceUniform.sequence_seed.offset == 156
    assert abi.TraceUniform.environment_rotation.offset == 176
    assert abi.TraceUniform.background_map_rotation.offset == 256
    assert C.sizeof(abi.RenderSettings) == 64          # mutracer-context.h:125-129
    assert lib.mtc_abi_version() == 1


def test_settings_defaults_match_reference():
    s = abi.RenderSettings()
    assert abi.lib().mt_render_settings_default(C.byref(s)) == abi.MT_OK
    assert (s.sampling_pattern, s.seed, s.max_samples, s.bounces, s.direct_light_candidates, s.bevel_samples) == \
        (abi.MT_SAMPLING_SOBOL, 12345, 64, 6, 2, 8)
    assert s.clamping == 0.0 and s.transmissive_output_alpha_min == 1.0
    assert abi.lib().mt_render_settings_default(None) == abi.MT_ERROR_INVALID_ARGUMENT


def test_entry_points_reject_invalid_arguments_without_launching():
    lib = abi.lib()
    assert lib.mtc_trace_samples(None, None, None, None, 1, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    v = abi.SceneView()
    v.struct_size = 7  # wrong struct_size
    assert lib.mtc_query_first_hit(C.byref(v), None, 0, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert lib.mtc_trace_batch(None, 1, None, None, None, None, None) == abi.MT_ERROR_INVALID_ARGUMENT
    assert lib.mtc_refit_tlas(None, 0, None, 0, None, None, None, None, None, None, None, None) == \
        abi.MT_ERROR_INVALID_ARGUMENT
    assert lib.mtc_batch_scratch_bytes(4) >= 4 * 256


def test_handles_and_status_codes_without_gpu():
    import torch
    lib = abi.lib()
    err = C.create_string_buffer(128)
    h = C.c_uint64()
    st = lib.mt_context_create(C.byref(h), err, 128)
    if torch.cuda.is_available():
        pytest.skip("covered by the GPU context test")
    assert st == abi.MT_ERROR_UNAVAILABLE
    assert b"CUDA" in err.value
    assert lib.mt_context_render(12345, 1, err, 128) == abi.MT_ERROR_INVALID_HANDLE
    assert lib.mt_job_poll(999, 1, err, 128) == abi.MT_ERROR_INVALID_HANDLE
    # truncated, NUL-terminated error message
    small = C.create_string_buffer(5)
    assert lib.mt_context_destroy(4242, small, 5) == abi.MT_ERROR_INVALID_HANDLE
    assert len(small.value) == 4
