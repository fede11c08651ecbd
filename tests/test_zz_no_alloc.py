"""The allocation-free PHOLD entry point (gpq_phold_run_static) against the allocating one.

gpq_phold_run_static exists for callers that cannot allocate device memory while they
run -- e.g. an application whose device memory belongs to another allocator or a fixed
plan, or a latency-bound loop that cannot pay for cudaMalloc/cudaFree.  It keeps all
queue state in one fixed 16 MiB device array, so its results must equal the normal
create/populate/run path exactly.  Its file name sorts it after the other test files so
that a run stopping at the first failure has executed them first; no test depends on that
order (each test here creates its own handles and static runs).
"""
import ctypes

import numpy as np
import pytest

import gpupq_b200 as G

CFG_A = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0)
CFG_B = dict(num_lps=500, events_per_lp=8, lookahead=0.1, end_time=30.0, seed=5, dest_mode=1, ring_width=16)


def _reference_path(cfgd):
    cfg = G.make_phold_config(**cfgd, loop="persistent")
    with G.Phold(cfg) as h:
        h.populate()
        h.run()
        r = h.result()
        s = h.lp_stats()
    return r, s


def _static_path(cfgd, initial=None):
    import torch
    L = cfgd["num_lps"]
    cfg = G.make_phold_config(**cfgd, loop="persistent")
    count = torch.full((L,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    csum = torch.full((L,), 123, dtype=torch.int64, device="cuda")
    ohash = torch.full((L,), -7, dtype=torch.int64, device="cuda")
    d_init = None
    keep = None
    if initial is not None:
        keep = torch.from_numpy(initial.view(np.uint8).copy()).cuda()
        d_init = ctypes.c_void_p(keep.data_ptr())
    torch.cuda.synchronize()
    res = G.PholdResult()
    st = G.lib().gpq_phold_run_static(ctypes.byref(cfg), d_init, ctypes.c_void_p(count.data_ptr()),
                                      ctypes.c_void_p(csum.data_ptr()), ctypes.c_void_p(ohash.data_ptr()),
                                      ctypes.byref(res), None)
    torch.cuda.synchronize()
    G.check(st, "gpq_phold_run_static")
    s = {"count": count.cpu().numpy().view(np.uint32), "csum": csum.cpu().numpy().view(np.uint64),
         "ohash": ohash.cpu().numpy().view(np.uint64)}
    return res.as_dict(), s


def _same(a, b):
    (ra, sa), (rb, sb) = a, b
    for k in ("committed", "steps", "pending", "pending_csum", "digest"):
        assert ra[k] == rb[k], k
    for k in ("count", "csum", "ohash"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.gpu
def test_static_entry_point_matches_allocating_path(gpu_lib):
    want_a = _reference_path(CFG_A)
    want_b = _reference_path(CFG_B)
    # consecutive calls share the fixed array; each must start from a clean state
    _same(_static_path(CFG_A), want_a)
    _same(_static_path(CFG_B), want_b)
    _same(_static_path(CFG_A), want_a)
    # caller-provided initial events (device array) give the same run
    init = G.initial_events(G.make_phold_config(**CFG_B))
    _same(_static_path(CFG_B, init), want_b)
    assert want_a[0]["committed"] == 820705


@pytest.mark.gpu
def test_static_entry_point_and_handles_interleaved(gpu_lib):
    """Handles created before and after a static call keep working, and so does the static
    call: the shared-memory limits of the kernels they share are only ever raised."""
    want_a = _reference_path(CFG_A)
    # a handle with a large window (insert capacity 128) exists across a static call
    big = dict(CFG_A, insert_capacity=128)
    with G.Phold(G.make_phold_config(**big, loop="persistent")) as h:
        h.populate()
        _same(_static_path(CFG_A), want_a)
        h.run()
        r, s = h.result(), h.lp_stats()
    _same((r, s), want_a)
    # a handle with a small window and few events per LP, then the static call again
    small = dict(CFG_B, insert_capacity=8, events_per_lp=2)
    with G.Phold(G.make_phold_config(**small, loop="persistent")) as h:
        h.populate()
        h.run()
        assert h.result()["status_code"] == 0
    _same(_static_path(CFG_A), want_a)


def test_static_entry_point_rejects_other_queue_forms():
    for mode in (1, 2):
        cfg = G.make_phold_config(**CFG_A, laq_mode=mode)
        res = G.PholdResult()
        st = G.lib().gpq_phold_run_static(ctypes.byref(cfg), None, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                          ctypes.c_void_p(16), ctypes.byref(res), None)
        assert st == 7  # GPQ_ERR_UNSUPPORTED, before any device work
        assert "laq_mode" in G.last_error()


def test_static_entry_point_rejects_oversized_config():
    cfg = G.make_phold_config(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=10.0, seed=7)
    res = G.PholdResult()
    st = G.lib().gpq_phold_run_static(ctypes.byref(cfg), None, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                      ctypes.c_void_p(16), ctypes.byref(res), None)
    assert st == 1  # GPQ_ERR_INVALID, before any device work
    msg = G.last_error()
    assert "needs" in msg and "16777216" in msg
