"""Build recipe for the reference's own C host programs (test drivers of the
drop-in boundary, not part of the product).

Compiles, unmodified and from where they lie in the reference tree,
native/examples/minimal-host.c, job-host.c and scene-host.c against the
reference's public headers (native/include) and links them to this
repository's libmutracer_b200.so, the library that replaces the reference's
native host.  The binaries go to oracle/_ref/ (ignored by git; they travel
with the working tree to a GPU machine, where the reference tree is absent,
and find the library through an rpath relative to themselves).

Run: python oracle/ref_hosts.py            (needs the reference tree)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REFERENCE = os.environ.get("MUTRACER_REFERENCE", "/root/reference")
EXAMPLES = os.path.join(REFERENCE, "native", "examples")
INCLUDE = os.path.join(REFERENCE, "native", "include")
OUT = os.path.join(HERE, "_ref")
LIB_DIR = os.path.join(ROOT, "mutracer_b200", "_lib")
HOSTS = ("minimal-host", "job-host", "scene-host")


def available():
    return all(os.path.exists(os.path.join(EXAMPLES, h + ".c")) for h in HOSTS)


def binary(name):
    return os.path.join(OUT, name)


def build(force=False):
    """Compiles the hosts when the reference tree is present; returns the
    list of binaries (empty when it is not)."""
    if not available():
        return []
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from mutracer_b200 import build as product
    lib = product.build()
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name in HOSTS:
        src = os.path.join(EXAMPLES, name + ".c")
        out = binary(name)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src),
                                                                               os.path.getmtime(lib)):
            built.append(out)
            continue
        cmd = ["gcc", "-std=gnu11", "-O2", "-I", INCLUDE, "-I", EXAMPLES, src, "-o", out + ".tmp",
               "-L", LIB_DIR, "-l:libmutracer_b200.so", "-Wl,-rpath,$ORIGIN/../../mutracer_b200/_lib",
               "-lm", "-pthread"]
        subprocess.check_call(cmd)
        os.replace(out + ".tmp", out)
        built.append(out)
    return built


if __name__ == "__main__":
    print("\n".join(build(force="--force" in sys.argv)) or "reference tree not present: nothing built")
