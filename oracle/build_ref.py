"""Build recipe for oracle/_ref: the reference's own per-LP queues and DES loop, run by the
adapter model (test infrastructure only).

For each variant (queue x workload) this script
  1. copies the reference's source files it needs, unmodified, from /root/reference/src
     into a scratch directory under /tmp (never into this repository);
  2. writes a config.h of its own into that directory -- the reference configures every
     size at compile time through src/config.h (NUM_LPS, queue kind, DEVICE_MEMORY_MB,
     LOOKAHEAD, MAX_TS, ...), so each workload needs its own;
  3. compiles them with nvcc for sm_100a (-rdc=true: the reference's window minimum
     launches CUB's DeviceReduce from a kernel, src/local_array_queue.cu:132-146) together
     with oracle/ref_adapter/*.cu, writing the binary to oracle/_ref/ref_phold_<variant>.

Flags follow src/Makefile:15-24 except that the vendored CUB 1.4.1 is not on the include
path (it trips the toolkit Thrust's version check); the toolkit's CUB is used instead.
No reference file is patched.  Two settings of the generated config.h make the reference's
integer keys carry this project's float32 semantics:
  * LOOKAHEAD expands, in device code, to gpq_ref_window_offset(global_min), so the queues'
    own window tests `key < global_min + LOOKAHEAD` (src/local_array_queue.cu:750,766,
    src/local_heap_queue.cu:436, src/local_splay_queue.cu:350) become
    `bits(ts) < bits(fl(m + lookahead))` for keys packed as (bits(ts) << 32) | id;
  * MAX_TS is bits(end_time) << 32, so des_run's `current_ts < MAX_TS`
    (src/des.cu:179-187) stops once the minimum timestamp reaches the end time.
MAX_WCT and MAX_EVENTS are 0: runs end by simulated time only.

The binaries run on the GPU box (tests/test_reference_queues_gpu.py); /root/reference is
only read here, at build time.

    python oracle/build_ref.py [--only VARIANT] [--force]
"""
import argparse
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_SRC = "/root/reference/src"
OUT_DIR = os.path.join(HERE, "_ref")
ADAPTER = os.path.join(HERE, "ref_adapter")

# the reference's files each queue needs (all unmodified)
COMMON = ["des.cu", "des.h", "model.h", "queue.h", "queue.cuh", "queue_item.h", "util.cuh", "sort.cuh",
          "cuda_bitset.cuh", "local_array_queue.cuh", "local_heap_queue.cuh", "local_splay_queue.cuh",
          "heap_queue.cuh", "global_array_queue.cuh"]
QUEUES = {
    "laq": ("_LOCAL_ARRAY_QUEUE", ["local_array_queue.cu", "sort.cu"]),
    "lhq": ("_LOCAL_HEAP_QUEUE", ["local_heap_queue.cu"]),
    "lsq": ("_LOCAL_SPLAY_QUEUE", ["local_splay_queue.cu"]),
}
# workloads: the 1,024-LP workload and the 65,536-LP ring workload cut to end time 3
WORKLOADS = {
    "c1": dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0,
               ring_width=0, ring_threshold=0, memory_mb=2000),
    "c2r": dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=3.0, seed=7, dest_mode=1,
                ring_width=16, ring_threshold=int(0.9 * 4294967296.0), memory_mb=2000),
}
VARIANTS = {f"{q}_{w}": (q, w) for q in QUEUES for w in WORKLOADS}

CONFIG_TEMPLATE = """// Generated by oracle/build_ref.py for the reference-queue variant {name}.
#pragma once
#include <stdint.h>
#include <limits.h>

#define {queue_macro}
#define _PHOLD

#define VERBOSE 0
#define PRINT_STATUS_INTERVAL 2
#define VERBOSE_DEBUG 0
#define _TIMER

#define MAX_EVENTS 0
#define MAX_WCT 0
// stop once the minimum timestamp reaches the end time (keys are bits(ts) << 32 | id)
#define MAX_TS ((long)((unsigned long long){end_bits}u << 32))

#define DEVICE_MEMORY_MB {memory_mb}
#define ENQUEUE_MAX 4

#define NUM_LPS {num_lps}
#define NUM_NODES_PER_LP 1
#define NUM_NODES (NUM_LPS * NUM_NODES_PER_LP)
#define SEED 0
#define PHOLD_LAMBDA 1.0
#define PHOLD_POPULATION {events_per_lp}

#define A_STAR_GRID_X 256
#define A_STAR_GRID_Y 256
#define HQ_NUM_QUEUES 1
#define HQ_NODE_SIZE (256 * 1024)
#define QUEUE_SIZE 8

#define _LAQ_INSERTION_SORT
#define LOCAL_ARRAY_QUEUE_BACKED_BY_HEAP_ITEMS_MAX 1
#define LOCAL_ARRAY_QUEUE_BACKED_BY_HEAP_ITEM_DIST_THRESHOLD 1000
#define QUICKSORT_STACK_SIZE (FEL_SIZE / 100 > 0 ? FEL_SIZE / 100 : 1)
#define LOCAL_ARRAY_QUEUE_PARALLEL_INSERT_NUM_THREADS 64

#define MAX_THREADS__PHOLD 256
#define MAX_THREADS__LOCAL_ARRAY_QUEUE 256
#define MAX_THREADS__HEAP_QUEUE 256
#define MAX_THREADS__GLOBAL_ARRAY_QUEUE 256
#define LOCAL_ARRAY_QUEUE_SINGLE_PASS_MAX_ENQUEUE 8
#define LOCAL_ARRAY_QUEUE_BACKWARD
#define CUDA_DEVICE 0

#define NUM_AGENTS 1
#define NUM_CONCURRENT_AGENTS NUM_LPS

// the workload of the adapter model
#define GPQ_REF_SEED {seed}ull
#define GPQ_REF_EVENTS_PER_LP {events_per_lp}u
#define GPQ_REF_LOOKAHEAD {lookahead!r}f
#define GPQ_REF_END_TIME {end_time!r}f
#define GPQ_REF_DEST_MODE {dest_mode}u
#define GPQ_REF_RING_WIDTH {ring_width}u
#define GPQ_REF_RING_THRESHOLD {ring_threshold}u
#define GPQ_REF_MAX_CALLS 200000ull

// The queues test `key < global_min + LOOKAHEAD`.  With key = bits(ts) << 32 | id and
// global_min the smallest key, global_min + gpq_ref_window_offset(global_min) equals
// bits(fl(m + lookahead)) << 32, m = ts(global_min), so the test is ts < m + lookahead in
// float32.  An empty minimum (LONG_MAX, no event queued) keeps its value.
static __host__ __device__ __forceinline__ long gpq_ref_window_offset(long g) {{
#if defined(__CUDA_ARCH__)
  const unsigned int tb = (unsigned int)((unsigned long long)g >> 32);
  if (tb >= 0x7f800000u) return 0;
  const float b = __fadd_rn(__uint_as_float(tb), GPQ_REF_LOOKAHEAD);
  return (long)((unsigned long long)__float_as_uint(b) << 32) - g;
#else
  (void)g;
  return 0;
#endif
}}
#if defined(__CUDA_ARCH__)
#define LOOKAHEAD (gpq_ref_window_offset(global_min))
#else
#define LOOKAHEAD 0L
#endif
"""

NVCC_FLAGS = ["-std=c++17", "-O3", "-arch=sm_100a", "-rdc=true", "--expt-extended-lambda", "-Xptxas", "-dlcm=ca",
              "-w"]


def _f32_bits(x):
    import struct
    return struct.unpack("<I", struct.pack("<f", x))[0]


def binary_path(variant):
    return os.path.join(OUT_DIR, f"ref_phold_{variant}")


def config_text(variant):
    q, w = VARIANTS[variant]
    wl = WORKLOADS[w]
    import numpy as np
    return CONFIG_TEMPLATE.format(name=variant, queue_macro=QUEUES[q][0], end_bits=_f32_bits(wl["end_time"]),
                                  **{k: (float(np.float32(v)) if isinstance(v, float) else v) for k, v in wl.items()})


def _digest(variant):
    h = hashlib.sha256(config_text(variant).encode())
    for f in sorted(os.listdir(ADAPTER)):
        with open(os.path.join(ADAPTER, f), "rb") as fh:
            h.update(fh.read())
    h.update(" ".join(NVCC_FLAGS).encode())
    with open(os.path.join(ROOT, "include", "gpq", "model.h"), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()


def up_to_date(variant):
    b = binary_path(variant)
    stamp = b + ".sha256"
    if not (os.path.exists(b) and os.path.exists(stamp)):
        return False
    with open(stamp) as fh:
        return fh.read().strip() == _digest(variant)


def build_variant(variant, force=False, verbose=False):
    if not force and up_to_date(variant):
        return binary_path(variant)
    if not os.path.isdir(REF_SRC):
        raise FileNotFoundError("the reference sources are not present; oracle/_ref cannot be built here")
    q, _ = VARIANTS[variant]
    os.makedirs(OUT_DIR, exist_ok=True)
    scratch = tempfile.mkdtemp(prefix=f"gpq_refbuild_{variant}_")
    try:
        for f in COMMON + QUEUES[q][1]:
            shutil.copy2(os.path.join(REF_SRC, f), os.path.join(scratch, f))
        with open(os.path.join(scratch, "config.h"), "w") as fh:
            fh.write(config_text(variant))
        srcs = [os.path.join(scratch, f) for f in QUEUES[q][1] + ["des.cu"]]
        srcs += [os.path.join(ADAPTER, "phold_adapter.cu"), os.path.join(ADAPTER, "ref_main.cu")]
        out = binary_path(variant)
        cmd = ["nvcc"] + NVCC_FLAGS + ["-I", scratch, "-I", os.path.join(ROOT, "include"), "-I", ADAPTER,
                                       "-o", out + ".tmp"] + srcs + ["-lcudadevrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(out + ".tmp", out)
        with open(out + ".sha256", "w") as fh:
            fh.write(_digest(variant) + "\n")
        return out
    finally:
        shutil.rmtree(scratch, ignore_errors=True)


def build(force=False, verbose=False, only=None):
    """Builds every variant when the reference sources are present (in this container);
    elsewhere keeps the prebuilt binaries.  Returns {variant: path}."""
    from concurrent.futures import ThreadPoolExecutor
    names = [only] if only else list(VARIANTS)
    if not os.path.isdir(REF_SRC):
        return {v: binary_path(v) for v in names if os.path.exists(binary_path(v))}
    with ThreadPoolExecutor(max_workers=min(len(names), os.cpu_count() or 4)) as ex:
        paths = list(ex.map(lambda v: build_variant(v, force, verbose), names))
    return dict(zip(names, paths))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None, choices=list(VARIANTS))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for v, p in build(force=a.force, verbose=True, only=a.only).items():
        print(v, p)
