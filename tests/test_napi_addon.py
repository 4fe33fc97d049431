"""The Node-API addon (native/napi/mutracer_b200_napi.c) compiles against
this repository's header and the Node-API declarations it uses (node is not
installed here, so tests/napi_stub/node_api.h stands in for node's header),
and wraps every context and job entry point of the library."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "native", "napi", "mutracer_b200_napi.c")


def test_addon_compiles_without_warnings(tmp_path):
    out = tmp_path / "addon.o"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-fPIC", "-c", SRC, "-o", str(out),
                        "-I", os.path.join(ROOT, "tests", "napi_stub"), "-I", os.path.join(ROOT, "include")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    symbols = subprocess.run(["nm", "-u", str(out)], capture_output=True, text=True).stdout
    for name in ("mt_context_create", "mt_context_create_with_backend", "mt_context_backend", "mt_context_destroy",
                 "mt_context_commit", "mt_context_commit_with_settings", "mt_context_cancel_commit",
                 "mt_context_render", "mt_context_reset", "mt_context_wait", "mt_context_info",
                 "mt_context_read_pixels", "mt_context_submit", "mt_job_poll", "mt_job_info", "mt_job_cancel",
                 "mt_render_settings_default"):
        assert re.search(r"\bU " + name + r"\b", symbols), name


def test_addon_exports():
    text = open(SRC).read()
    names = set(re.findall(r'\{"(\w+)", [A-Z]\w+\}', text))
    assert {"create", "createWithBackend", "backend", "destroy", "commit", "cancelCommit", "render", "reset",
            "wait", "info", "readPixels", "submit", "jobPoll", "jobInfo", "jobCancel"} <= names
