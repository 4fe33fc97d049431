"""The reference's own C hosts against this library, without a GPU.

oracle/ref_hosts.py compiles native/examples/{minimal,job,scene}-host.c of
the reference, unmodified, against the reference's public headers and links
them to libmutracer_b200.so: every entry point they call resolves in this
library.  scene-host.c writes its descriptor variants without touching the
library (samples 0); here each variant is decoded the way mt_context_commit
decodes it: the variants that use only what this build renders are accepted,
the others are refused by name with MT_ERROR_UNAVAILABLE.  The GPU half
(tests/test_gpu_reference_hosts.py) renders them.
"""
import ctypes as C
import os
import subprocess

import pytest

from mutracer_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

# Variants of scene-host.c make_scene and what this build does with them.
ACCEPTED = ("baseline", "textures", "transforms", "orthographic", "emissive", "missing-normals", "float-textures",
            "sphere-light", "directional-light", "spot-light", "disk-light", "cylinder-light", "lights-1024", "alpha",
            "v2-alpha")
REFUSED = {  # variant -> the feature named in the refusal
    "v2-environment": "material extension 71", "v2-environment-only": "material extension 71",
    "v2-background": "a background map", "v2-hidden-background": "material extension 71",
    "v2-film": "material extension 71", "v2-medium": "material extension 71", "v2-bevel": "bevel",
    "v2-vertices": "material extension 71", "v2-multimaterial": "material extension 71",
    "v2-instances": "material extension 71", "v2-empty-batch": "material extension 71",
    "v3-displacement-uv": "material extension 60", "v3-ies": "material extension 71",
    "v3-rect-texture": "material extension 71",
}


def host(name):
    path = os.path.join(REF, name)
    if not os.path.exists(path):
        pytest.skip("reference hosts not built (oracle/ref_hosts.py needs the reference tree)")
    return path


def write_descriptor(variant, directory):
    path = os.path.join(str(directory), variant + ".bin")
    r = subprocess.run([host("scene-host"), path, "0", variant], capture_output=True, timeout=60)
    assert r.returncode == 0, (variant, r.returncode, r.stderr)
    return open(path, "rb").read()


def decode(data):
    L = abi.lib()
    st = C.c_int32(0)
    err = C.create_string_buffer(512)
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    handle = L.mtp_descriptor_decode(buf, len(data), C.byref(st), err, 512)
    if handle:
        L.mtp_scene_free(handle)
    return st.value, err.value.decode()


def test_hosts_link_against_this_library():
    for name in ("minimal-host", "job-host", "scene-host"):
        out = subprocess.run(["ldd", host(name)], capture_output=True, text=True).stdout
        assert "libmutracer_b200.so" in out and "not found" not in out, out


@pytest.mark.parametrize("variant", ACCEPTED)
def test_scene_host_descriptor_accepted(variant, tmp_path):
    st, msg = decode(write_descriptor(variant, tmp_path))
    assert st == abi.MT_OK, (variant, msg)


@pytest.mark.parametrize("variant", sorted(REFUSED))
def test_scene_host_descriptor_refused_by_name(variant, tmp_path):
    st, msg = decode(write_descriptor(variant, tmp_path))
    assert st == abi.MT_ERROR_UNAVAILABLE, (variant, st, msg)
    assert REFUSED[variant] in msg
