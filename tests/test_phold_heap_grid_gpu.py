"""GPU parity of the parallel heap queue's grid form (node sizes above 1,024 items, the
whole GPU working each node merge in one cooperative launch) against the CPU oracle and
the committed full-size results, bit for bit."""
import json
import os

import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
C1 = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0)
REF_NODE_SIZE = 256 * 1024  # HQ_NODE_SIZE, src/config.h:88


def _oracle(cfgd, threads=0):
    return O.phold(O.make_cfg(**cfgd), threads)


def _run(cfgd, node_size, steps=None, initial=None):
    cap = 1 << max(6, (cfgd["events_per_lp"] - 1).bit_length())  # the population check's per-LP bound
    cfg = G.make_phold_config(**cfgd, queue="hq", node_size=node_size, capacity=cap)
    with G.Phold(cfg) as h:
        h.populate(initial)
        if steps is None:
            h.run()
            calls = 1
        else:
            calls, done = 0, False
            while not done:
                done = h.step(steps)
                calls += 1
        r = h.result()
        s = h.lp_stats()
        grid = h.launch_info()["grid"]
    return r, s, grid, calls


def _assert_same(r, s, o):
    assert r["status_code"] == 0, r
    assert np.array_equal(s["count"], o["count"])
    assert np.array_equal(s["csum"], o["csum"])
    assert np.array_equal(s["ohash"], o["ohash"])
    for k in ("committed", "pending", "pending_csum", "steps"):
        assert r[k] == o[k], k


@pytest.mark.parametrize("node_size", [2048, 16384, REF_NODE_SIZE])
def test_plain_workload(gpu_lib, node_size):
    """1,024 LPs x 16 events to end time 100: eight nodes of 2,048, one full root of
    16,384, and a root of the reference's default size holding the whole population."""
    o = _oracle(C1)
    r, s, grid, _ = _run(C1, node_size)
    _assert_same(r, s, o)
    assert r["committed"] == 820705
    assert grid > 1  # the grid form, not the one-CTA kernel


@pytest.mark.parametrize("node_size", [2048, 4096])
def test_deep_heap(gpu_lib, node_size):
    """3,000 LPs x 20 events (60,000 items): 30 or 15 nodes, so insert-update pieces walk
    paths of up to four full ancestors and delete-update walks to the leaves."""
    cfgd = dict(num_lps=3000, events_per_lp=20, lookahead=0.2, end_time=12.0, seed=31, dest_mode=1, ring_width=7)
    o = _oracle(cfgd)
    r, s, _, _ = _run(cfgd, node_size)
    _assert_same(r, s, o)


def test_large_workload_reduced(gpu_lib):
    """65,536 LPs x 64 events (4,194,304 items) to end time 3: sixteen nodes of 256 K and a
    single full root of 4 M items, against the committed oracle results."""
    with open(os.path.join(HERE, "golden", "phold_golden.json")) as fh:
        g = json.load(fh)["phold_large_65536lp_x64_ring16_T3"]
    cfgd = g["config"]
    for node_size in (REF_NODE_SIZE, 1 << 22):
        r, s, _, _ = _run(cfgd, node_size)
        assert r["status_code"] == 0, r
        assert r["committed"] == g["committed"]
        assert r["steps"] == g["windows"]
        assert r["pending"] == g["pending"]
        assert str(r["pending_csum"]) == g["pending_csum"]
        assert str(r["digest"]) == g["digest"]
        assert O.lp_sha256(s["count"], s["csum"], s["ohash"]) == g["lp_sha256"]


def test_step_api_resumes(gpu_lib):
    """Seven windows per call: the heap and its last node carry over between launches."""
    o = _oracle(C1)
    r, s, _, calls = _run(C1, 2048, steps=7)
    _assert_same(r, s, o)
    assert calls > 10


@pytest.mark.parametrize("cfgd", [
    dict(num_lps=1, events_per_lp=1, lookahead=0.5, end_time=30.0, seed=1, dest_mode=0),
    dict(num_lps=7, events_per_lp=5, lookahead=0.25, end_time=40.0, seed=9, dest_mode=0),
    dict(num_lps=64, events_per_lp=4, lookahead=1.0, end_time=0.0, seed=2, dest_mode=0),
    # lookahead far above the spread: the whole population is safe in most windows
    dict(num_lps=3000, events_per_lp=6, lookahead=20.0, end_time=60.0, seed=17, dest_mode=1, ring_width=4),
    # many events of one LP in one batch (two LPs, long queues)
    dict(num_lps=2, events_per_lp=3000, lookahead=0.5, end_time=3.0, seed=5, dest_mode=0),
    # two LPs, batches of nearly the whole population (16,384): in windows where one LP's
    # share passes 8,192 its LP-range bucket outgrows a key tile, and the one-phase batch
    # gives way to the general path
    dict(num_lps=2, events_per_lp=8192, lookahead=50.0, end_time=400.0, seed=5, dest_mode=0),
])
def test_edge_shapes(gpu_lib, cfgd):
    o = _oracle(cfgd)
    r, s, _, _ = _run(cfgd, 2048)
    _assert_same(r, s, o)


def test_host_initial_events(gpu_lib):
    """Host-provided initial events with late starts for half the LPs."""
    cfgd = dict(num_lps=500, events_per_lp=8, lookahead=0.3, end_time=20.0, seed=8, dest_mode=1, ring_width=3)
    ev = G.initial_events(G.make_phold_config(**cfgd))
    ev["ts"][ev["lp"] >= 250] += np.float32(5.0)
    cfg_one = G.make_phold_config(**cfgd, queue="hq", node_size=256)
    with G.Phold(cfg_one) as h:
        h.populate(ev)
        h.run()
        r0, s0 = h.result(), h.lp_stats()
    r, s, _, _ = _run(cfgd, 4096, initial=ev)
    assert r["status_code"] == 0 and r0["status_code"] == 0
    for k in ("committed", "pending", "pending_csum", "digest", "steps"):
        assert r[k] == r0[k], k
    for k in ("count", "csum", "ohash"):
        assert np.array_equal(s[k], s0[k]), k


def test_bucket_overflow_falls_back(gpu_lib):
    """Half the population 1,000 time units ahead: the root's quantiles (the one-phase
    insert's splitters) all lie far beyond the children, so every child lands in one bucket,
    which overflows shared memory; the general path takes over, window after window.  The
    20,000 near events also make batches too large for the one-phase ranks."""
    cfgd = dict(num_lps=40, events_per_lp=1000, lookahead=1.0, end_time=30.0, seed=12, dest_mode=0)
    ev = G.initial_events(G.make_phold_config(**cfgd))
    ev["ts"][ev["id"] % 2 == 1] += np.float32(1000.0)
    cfg_one = G.make_phold_config(**cfgd, queue="hq", node_size=1024, capacity=1024)
    with G.Phold(cfg_one) as h:
        h.populate(ev)
        h.run()
        r0, s0 = h.result(), h.lp_stats()
    r, s, _, _ = _run(cfgd, REF_NODE_SIZE, initial=ev)
    assert r["status_code"] == 0 and r0["status_code"] == 0
    for k in ("committed", "pending", "pending_csum", "digest", "steps"):
        assert r[k] == r0[k], k
    for k in ("count", "csum", "ohash"):
        assert np.array_equal(s[k], s0[k]), k
