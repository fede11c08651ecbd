"""The device-side drop-in headers (include/gpq/queue.cuh, include/gpq/legacy.h).

* A PHOLD model written like the reference's (a handler kernel calling queue_peek /
  queue_set_done / queue_insert, a host loop of get-min / window / handler / post steps)
  builds against the header and, on the GPU, commits exactly the oracle's per-LP
  sequences through every queue kind, in exactly the window count of the reference's
  one-event-per-LP schedule.
* The same model driven through the reference's host queue names (queue_init,
  queue_post_init, queue_get_min_ts, queue_pre, queue_post, get_dequeue_count,
  queue_finish) gives the same results.
* An A* agent model (one open list per agent: queue_insert_or_update, queue_is_empty,
  queue_clear) finds the oracle's optimal cost on every grid."""
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
    lib.dropin_phold_run_legacy.argtypes = lib.dropin_phold_run.argtypes
    lib.dropin_phold_run_legacy.restype = ctypes.c_int
    lib.dropin_astar_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, u32p,
                                     ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib.dropin_astar_run.restype = ctypes.c_int
    return lib


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_dropin_model_builds():
    G.lib()  # libgpq.so present (built by the package)
    assert _lib() is not None


@pytest.mark.gpu
@pytest.mark.parametrize("queue", ["laq", "lhq", "lsq", "gaq", "hq"])
@pytest.mark.parametrize("dest", ["uniform", "ring"])
@pytest.mark.parametrize("host_api", ["gpq", "legacy"])
def test_dropin_model_matches_oracle(gpu_lib, dest, queue, host_api):
    if host_api == "legacy" and dest == "ring" and queue in ("lsq", "hq"):
        pytest.skip("covered by the uniform case (the host path is the same)")
    ring = dest == "ring"
    cfgd = dict(num_lps=700, events_per_lp=8, lookahead=0.5, end_time=15.0, seed=31,
                dest_mode=1 if ring else 0)
    cfg = G.make_phold_config(**cfgd, ring_width=16, queue=queue, capacity=256, insert_capacity=64)
    L = cfgd["num_lps"]
    count = np.zeros(L, np.uint32)
    csum = np.zeros(L, np.uint64)
    ohash = np.zeros(L, np.uint64)
    steps, committed = ctypes.c_uint64(), ctypes.c_uint64()
    run = _lib().dropin_phold_run if host_api == "gpq" else _lib().dropin_phold_run_legacy
    st = run(ctypes.byref(cfg), count, csum, ohash, ctypes.byref(steps), ctypes.byref(committed))
    assert st == 0, G.last_error()
    o = O.phold(O.make_cfg(**cfgd, ring_width=16, ring_frac=0.9), 0)
    assert np.array_equal(count, o["count"])
    assert np.array_equal(csum, o["csum"])
    assert np.array_equal(ohash, o["ohash"])
    assert committed.value == o["committed"]
    # one event per LP per window, as in the reference: the oracle's one-per-LP schedule
    # gives the exact window count
    o1 = O.phold(O.make_cfg(**cfgd, ring_width=16, ring_frac=0.9), one_per_lp=True)
    assert np.array_equal(count, o1["count"]) and np.array_equal(ohash, o1["ohash"])
    if queue == "hq":
        # the heap queue hands out only its root's safe items (as the reference's,
        # src/heap_queue.cu:1588-1592): an LP whose next safe item is below the root
        # takes it a window later, so the schedule may need more windows
        assert steps.value >= o1["steps"]
    else:
        assert steps.value == o1["steps"]
    assert o1["steps"] > o["steps"]


@pytest.mark.gpu
def test_dropin_insert_overflow_is_reported(gpu_lib):
    cfg = G.make_phold_config(64, 16, 0.5, 10.0, 5, queue="laq", capacity=256, insert_capacity=1)
    z = np.zeros(64, np.uint32), np.zeros(64, np.uint64), np.zeros(64, np.uint64)
    st = _lib().dropin_phold_run(ctypes.byref(cfg), *z, ctypes.byref(ctypes.c_uint64()), ctypes.byref(ctypes.c_uint64()))
    assert st == 4  # GPQ_ERR_INSERT_FULL from the post after the overflowing handler


@pytest.mark.gpu
@pytest.mark.parametrize("queue", ["laq", "lhq"])
def test_dropin_astar_agents_find_optimal_cost(gpu_lib, queue):
    grids = np.concatenate([G.astar_grid(w, h, d, seed, conn=4, start=0, goal=w * h - 1)
                            for seed, (w, h, d) in enumerate([(64, 64, 0.2), (48, 64, 0.25), (64, 40, 0.1),
                                                              (33, 57, 0.3), (64, 64, 0.35), (16, 16, 0.0)] * 6)])
    n = len(grids)
    cost = np.zeros(n, np.uint32)
    pops, rounds = ctypes.c_uint64(), ctypes.c_uint64()
    st = _lib().dropin_astar_run(ctypes.c_void_p(grids.ctypes.data), n, G.QUEUE_NAMES[queue], cost,
                                 ctypes.byref(pops), ctypes.byref(rounds))
    assert st == 0, G.last_error()
    for i in range(n):
        want = O.astar({k: int(grids[i][k]) for k in O.ASTAR_FIELDS})
        assert int(cost[i]) == want["cost"], (i, int(cost[i]), want["cost"])
    assert pops.value > 0 and rounds.value > 100
