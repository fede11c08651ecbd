"""Build recipe of the drop-in test model (test infrastructure): compiles
tests/dropin/phold_model.cu against include/gpq/queue.cuh into
tests/dropin/_build/libdropin.so, linked with gpupq_b200/lib/libgpq.so."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libdropin.so")
SRC = os.path.join(HERE, "phold_model.cu")


def build(force=False):
    libdir = os.path.join(ROOT, "gpupq_b200", "lib")
    deps = [SRC, __file__, os.path.join(ROOT, "include", "gpq", "queue.cuh"), os.path.join(ROOT, "include", "gpq.h")]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["nvcc", "-shared", "-o", OUT, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lgpq", "-Xlinker", "-rpath," + libdir]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
