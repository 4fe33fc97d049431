"""In-tree build of libmutracer_b200.so for sm_100a.

nvcc compiles the device code (-gencode arch=compute_100a,code=sm_100a) and
the host C++ (scene producers, C ABI, context API); the CUDA runtime is linked
statically so the library only needs the driver on the GPU machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libmutracer_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU = ["megakernel.cu", "batch_noalloc.cu", "wavefront.cu", "bvh_build.cu", "blas_refit.cu"]
CPP = ["scene_prep.cpp", "host_api.cpp", "context.cpp", "sizes.cpp", "descriptor.cpp"]


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(HERE, "..", "include", "mutracer_b200.h"))
    return files


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB):
        if os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in _deps()):
            return LIB
    os.makedirs(OUT, exist_ok=True)
    objs = []
    procs = []
    for src in CU:
        obj = os.path.join(OUT, src + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for src in CPP:
        obj = os.path.join(OUT, src + ".o")
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-pthread", "-I/usr/local/cuda/include", "-c",
               os.path.join(CSRC, src), "-o", obj]
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("compilation failed")
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs,
                           "-Xcompiler", "-pthread"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
