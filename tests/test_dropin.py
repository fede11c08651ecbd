"""The device-side drop-in header (include/gpq/queue.cuh): a PHOLD model written like the
reference's (a handler kernel calling queue_peek / queue_set_done / queue_insert, a host
loop of get-min / window / handler / post steps) builds against the header and, on the
GPU, commits exactly the oracle's per-LP sequences through a gpupq_b200 local array
queue and through a local heap queue."""
import ctypes
import os
import shutil

import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _lib():
    import importlib.util
    spec = importlib.util.spec_from_file_location("dropin_build", os.path.join(HERE, "dropin", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    path = m.build()
    lib = ctypes.CDLL(path)
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
    lib.dropin_phold_run.argtypes = [ctypes.POINTER(G.PholdConfig), u32p, u64p, u64p,
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib.dropin_phold_run.restype = ctypes.c_int
    return lib


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_dropin_model_builds():
    G.lib()  # libgpq.so present (built by the package)
    assert _lib() is not None


@pytest.mark.gpu
@pytest.mark.parametrize("queue", ["laq", "lhq"])
@pytest.mark.parametrize("dest", ["uniform", "ring"])
def test_dropin_model_matches_oracle(gpu_lib, dest, queue):
    ring = dest == "ring"
    cfgd = dict(num_lps=700, events_per_lp=8, lookahead=0.5, end_time=15.0, seed=31,
                dest_mode=1 if ring else 0)
    cfg = G.make_phold_config(**cfgd, ring_width=16, queue=queue, capacity=256, insert_capacity=64)
    L = cfgd["num_lps"]
    count = np.zeros(L, np.uint32)
    csum = np.zeros(L, np.uint64)
    ohash = np.zeros(L, np.uint64)
    steps, committed = ctypes.c_uint64(), ctypes.c_uint64()
    st = _lib().dropin_phold_run(ctypes.byref(cfg), count, csum, ohash, ctypes.byref(steps), ctypes.byref(committed))
    assert st == 0, G.last_error()
    o = O.phold(O.make_cfg(**cfgd, ring_width=16, ring_frac=0.9), 0)
    assert np.array_equal(count, o["count"])
    assert np.array_equal(csum, o["csum"])
    assert np.array_equal(ohash, o["ohash"])
    assert committed.value == o["committed"]
    assert steps.value >= o["steps"]  # one event per LP per step, as in the reference


@pytest.mark.gpu
def test_dropin_insert_overflow_is_reported(gpu_lib):
    cfg = G.make_phold_config(64, 16, 0.5, 10.0, 5, queue="laq", capacity=256, insert_capacity=1)
    z = np.zeros(64, np.uint32), np.zeros(64, np.uint64), np.zeros(64, np.uint64)
    st = _lib().dropin_phold_run(ctypes.byref(cfg), *z, ctypes.byref(ctypes.c_uint64()), ctypes.byref(ctypes.c_uint64()))
    assert st == 4  # GPQ_ERR_INSERT_FULL from the post after the overflowing handler
