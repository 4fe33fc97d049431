"""Build recipe for the CPU oracle (test infrastructure only).

Compiles the C++ restatement of the reference megakernel into
``oracle/_build/liboracle.so`` with ``-O2 -ffp-contract=off`` so every f32
product and sum is rounded separately, as the WGSL source states it.  The
reference itself (WGSL + TypeScript + Rust/wgpu) cannot be compiled here, so
there is no ``oracle/_ref`` build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["oracle_trace.cpp", "oracle_bsdf.cpp", "oracle_shade.cpp", "oracle_api.cpp"]
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    headers = [os.path.join(HERE, h) for h in ("om.h", "oracle_core.h", "oracle_bsdf.h")]
    headers.append(os.path.join(HERE, "..", "include", "mutracer_b200.h"))
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(p) for p in srcs + headers)
        if os.path.getmtime(LIB) >= newest:
            return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-fPIC", "-shared",
           "-pthread", "-o", LIB + ".tmp"] + srcs
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
