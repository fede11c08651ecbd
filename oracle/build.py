"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/phold_oracle.cpp (and the two A* oracles) into oracle/_build/libgpq_oracle.so
with g++.  FP contraction is disabled so that float32 results are bit-identical to the
GPU build.  Called by __graft_entry__.build() and by the tests when the library is missing.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libgpq_oracle.so")
SOURCES = ["phold_oracle.cpp", "astar_oracle.cpp", "astar_ref_oracle.cpp"]


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB):
        lib_mtime = os.path.getmtime(LIB)
        if all(os.path.getmtime(s) <= lib_mtime for s in srcs + [__file__]):
            return LIB
    cmd = ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-pthread", "-o", LIB] + srcs
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
