"""Build recipe for libgpq.so (sm_100a).

All CUDA sources under gpupq_b200/csrc are compiled (one nvcc per file, in parallel)
and linked into gpupq_b200/lib/libgpq.so (in-tree, so the built library travels with the
repository snapshot).  The CUDA runtime is linked statically; host code is compiled with
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


def _object_digest(src: str, headers_digest: str, flags) -> str:
    import hashlib
    h = hashlib.sha256(headers_digest.encode())
    h.update(" ".join(flags).encode())
    with open(src, "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()


def _headers_digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for f in sorted(set(_inputs()) - set(sources())):
        h.update(os.path.relpath(f, ROOT).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compiles every .cu under csrc to an object (in parallel, one nvcc per file; an
    object whose source, headers and flags are unchanged is reused) and links them."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(LIB_DIR, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    flags = NVCC_FLAGS + list(extra or [])
    hd = _headers_digest()

    def compile_one(src):
        name = os.path.splitext(os.path.basename(src))[0]
        obj = os.path.join(obj_dir, name + ".o")
        dg = _object_digest(src, hd, flags)
        stamp = obj + ".sha256"
        if not force and os.path.exists(obj) and os.path.exists(stamp):
            with open(stamp) as fh:
                if fh.read().strip() == dg:
                    return obj
        cmd = ["nvcc", "-c", "-o", obj + ".tmp", "-I", INCLUDE, "-I", CSRC] + flags + [src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(obj + ".tmp", obj)
        with open(stamp, "w") as fh:
            fh.write(dg + "\n")
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 4))) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    cmd = ["nvcc", "-shared", "-o", tmp] + [f for f in flags if f != "-lineinfo"] + objs
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
