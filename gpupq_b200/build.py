"""Build recipe for libgpq.so (sm_100a).

All CUDA sources under gpupq_b200/csrc are compiled by one nvcc call into
gpupq_b200/lib/libgpq.so (in-tree, so the built library travels with the repository
snapshot).  The CUDA runtime is linked statically; host code is compiled with
-ffp-contract=off so that host-side float math matches the device bit for bit.
"""
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libgpq.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _inputs():
    files = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    files += glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "gpq", "*"))
    return files + [os.path.abspath(__file__)]


def _digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for f in sorted(_inputs()):
        h.update(os.path.relpath(f, ROOT).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def up_to_date() -> bool:
    """True when libgpq.so exists and was built from the current sources (content hash,
    so copying the tree elsewhere does not force a rebuild)."""
    stamp = LIB + ".sha256"
    if not (os.path.exists(LIB) and os.path.exists(stamp)):
        return False
    with open(stamp) as fh:
        return fh.read().strip() == _digest()


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = ["nvcc", "-shared", "-o", tmp, "-I", INCLUDE, "-I", CSRC] + NVCC_FLAGS + list(extra or []) + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    with open(LIB + ".sha256", "w") as fh:
        fh.write(_digest() + "\n")
    return LIB


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None
    print(build(force=True, verbose=True, extra=extra))
