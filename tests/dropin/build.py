"""Build recipe of the drop-in test models (test infrastructure): compiles the
reference-style models of tests/dropin/ (PHOLD over the device queue functions, PHOLD
through the reference's host queue names, an A* agent model) against include/gpq/queue.cuh
and include/gpq/legacy.h into tests/dropin/_build/libdropin.so, linked with
gpupq_b200/lib/libgpq.so."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libdropin.so")
SRCS = [os.path.join(HERE, f) for f in ("phold_model.cu", "phold_legacy.cu", "astar_model.cu")]


def build(force=False):
    libdir = os.path.join(ROOT, "gpupq_b200", "lib")
    deps = SRCS + [__file__, os.path.join(HERE, "phold_handler.cuh"), os.path.join(ROOT, "include", "gpq.h")]
    deps += [os.path.join(ROOT, "include", "gpq", f) for f in ("queue.cuh", "legacy.h", "astar.h", "model.h")]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["nvcc", "-shared", "-o", OUT, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", HERE] + SRCS + [
           "-L", libdir, "-lgpq", "-Xlinker", "-rpath," + libdir]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
