"""GPU parity of the PHOLD engine against the CPU oracle (bit-exact: integer counts,
64-bit checksums and float32 timestamps compared as bits)."""
import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C1 = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0)


def _oracle(cfgd, threads=0):
    keys = ("num_lps", "events_per_lp", "lookahead", "end_time", "seed", "dest_mode", "ring_width")
    return O.phold(O.make_cfg(**{k: v for k, v in cfgd.items() if k in keys}), threads)


_ORACLE_CACHE = {}


def _oracle_cached(cfgd):
    key = tuple(sorted(cfgd.items()))
    if key not in _ORACLE_CACHE:
        _ORACLE_CACHE[key] = _oracle(cfgd, threads=8)
    return _ORACLE_CACHE[key]


def _run(cfgd, **kw):
    if kw.get("queue") == "laqs":  # the local array queue's selection form
        kw = dict(kw, queue="laq", laq_mode=1)
    if kw.get("queue") == "laqb":  # the local array queue's bucketed form
        kw = dict(kw, queue="laq", laq_mode=2)
    if kw.get("queue") == "gaqg":  # the global array queue's graph-replayed kernel sequence
        kw = dict(kw, queue="gaq", gaq_engine=1)
    cfg = G.make_phold_config(**cfgd, **kw)
    with G.Phold(cfg) as h:
        h.populate()
        h.run()
        r = h.result()
        s = h.lp_stats()
    return r, s


def _assert_same(r, s, o, check_steps=True):
    """Bit-exact outputs, window count included."""
    assert r["status_code"] == 0, r
    assert np.array_equal(s["count"], o["count"])
    assert np.array_equal(s["csum"], o["csum"])
    assert np.array_equal(s["ohash"], o["ohash"])
    assert r["committed"] == o["committed"]
    assert r["pending"] == o["pending"]
    assert r["pending_csum"] == o["pending_csum"]
    if check_steps:
        assert r["steps"] == o["steps"]


def test_children_match_oracle(gpu_lib):
    cfgd = dict(num_lps=5000, events_per_lp=3, lookahead=0.1, end_time=10.0, seed=7, dest_mode=1, ring_width=16)
    cfg = G.make_phold_config(**cfgd)
    ev = G.initial_events(cfg)
    rng = np.random.default_rng(0)
    ev["ts"] = (rng.random(len(ev)) * 1000).astype(np.float32)
    ch = G.children(cfg, ev)
    ots, olp = O.child(O.make_cfg(**cfgd), ev["ts"], ev["lp"], ev["id"])
    assert np.array_equal(ch["ts"].view(np.uint32), ots.view(np.uint32))
    assert np.array_equal(ch["lp"], olp)
    assert np.array_equal(ch["id"], ev["id"])


QUEUE_SHAPES = [("laq", 4), ("laq", 8), ("laq", 16), ("laq", 32), ("laqs", 4), ("laqs", 8), ("laqs", 32), ("laqb", 4),
                ("laqb", 8), ("laqb", 16), ("laqb", 32), ("lhq", 1),
                ("lhq", 8), ("lhq", 32), ("lsq", 1), ("gaq", 8), ("gaqg", 8), ("hq", 8)]


@pytest.mark.parametrize("loop", ["plain", "persistent"])
@pytest.mark.parametrize("queue,lanes", QUEUE_SHAPES)
def test_phold_plain_workload_bit_exact(gpu_lib, loop, queue, lanes):
    """1024 LPs x 16 events, lookahead 1.0, end 100, uniform destinations, seed 42."""
    o = _oracle(C1)
    r, s = _run(C1, loop=loop, queue=queue, lanes_per_lp=lanes)
    _assert_same(r, s, o)
    assert r["committed"] == 820705


@pytest.mark.parametrize("node_size", [2, 16, 256, 1024])
def test_phold_heap_queue_node_sizes(gpu_lib, node_size):
    """The parallel heap with nodes from 2 to 1024 items (deep and shallow heaps)."""
    cfgd = dict(num_lps=300, events_per_lp=7, lookahead=0.3, end_time=25.0, seed=21, dest_mode=1, ring_width=5)
    o = _oracle(cfgd)
    r, s = _run(cfgd, queue="hq", node_size=node_size)
    _assert_same(r, s, o)


@pytest.mark.parametrize("queue,loop,lanes,block", [
    ("laq", "plain", 8, 256), ("laq", "persistent", 4, 128), ("laq", "persistent", 8, 256),
    ("laq", "persistent", 16, 512), ("laq", "persistent", 32, 256), ("laqs", "persistent", 8, 128),
    ("laqs", "plain", 16, 256), ("laqb", "persistent", 4, 128), ("laqb", "persistent", 8, 128),
    ("laqb", "persistent", 16, 256), ("laqb", "plain", 8, 256), ("lhq", "persistent", 8, 128), ("lhq", "plain", 4, 256), ("lsq", "persistent", 1, 128), ("lsq", "plain", 1, 256),
    ("gaq", "plain", 8, 256), ("gaqg", "plain", 8, 256), ("hq", "persistent", 8, 256)])
def test_phold_large_reduced_bit_exact(gpu_lib, queue, loop, lanes, block):
    """The 65,536-LP ring workload cut to end time 3 (checked by the threaded oracle)."""
    cfgd = dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=3.0, seed=7, dest_mode=1, ring_width=16)
    o = _oracle_cached(cfgd)
    r, s = _run(cfgd, queue=queue, loop=loop, capacity=256, insert_capacity=64, lanes_per_lp=lanes,
                block_threads=block)
    _assert_same(r, s, o)


@pytest.mark.parametrize("cfgd,kw", [
    (dict(num_lps=1, events_per_lp=1, lookahead=0.5, end_time=30.0, seed=1, dest_mode=0), {}),
    (dict(num_lps=7, events_per_lp=5, lookahead=0.25, end_time=40.0, seed=9, dest_mode=0), dict(block_threads=32)),
    (dict(num_lps=100, events_per_lp=33, lookahead=0.05, end_time=8.0, seed=11, dest_mode=1, ring_width=2),
     dict(capacity=128, insert_capacity=128)),
    (dict(num_lps=333, events_per_lp=200, lookahead=0.02, end_time=2.0, seed=13, dest_mode=1, ring_width=1),
     dict(capacity=512, insert_capacity=256)),
    (dict(num_lps=64, events_per_lp=4, lookahead=1.0, end_time=0.0, seed=2, dest_mode=0), {}),
    # lookahead far above the spread: nearly every queued event is safe in every window,
    # which overflows the per-warp staging area and exercises the in-group fallback
    (dict(num_lps=3000, events_per_lp=60, lookahead=20.0, end_time=60.0, seed=17, dest_mode=1, ring_width=4),
     dict(capacity=256, insert_capacity=256)),
])
@pytest.mark.parametrize("queue,loop,lanes", [("laq", "plain", 32), ("laq", "persistent", 4), ("laq", "persistent", 8),
                                              ("laq", "persistent", 32), ("laqs", "persistent", 8), ("laqs", "plain", 32),
                                              ("laqs", "persistent", 4), ("laqb", "persistent", 4),
                                              ("laqb", "persistent", 8), ("laqb", "plain", 32), ("laqb", "persistent", 32),
                                              ("lhq", "persistent", 8), ("lhq", "plain", 1),
                                              ("lsq", "persistent", 1), ("lsq", "plain", 1), ("gaq", "plain", 8),
                                              ("gaqg", "plain", 8),
                                              ("hq", "persistent", 8)])
def test_phold_edge_shapes(gpu_lib, cfgd, kw, queue, loop, lanes):
    o = _oracle(cfgd)
    r, s = _run(cfgd, queue=queue, loop=loop, lanes_per_lp=lanes, **kw)
    _assert_same(r, s, o)


@pytest.mark.parametrize("laq_mode", [0, 2])
def test_host_initial_events_path(gpu_lib, laq_mode):
    cfg = G.make_phold_config(**C1, laq_mode=laq_mode)
    ev = G.initial_events(cfg)
    with G.Phold(cfg) as h:
        h.populate(ev)
        h.run()
        r1 = h.result()
        h.populate()
        h.run()
        r2 = h.result()
    assert r1["digest"] == r2["digest"] and r1["committed"] == r2["committed"] == 820705


@pytest.mark.parametrize("laq_mode", [0, 2])
def test_step_api_resumes(gpu_lib, laq_mode):
    cfg = G.make_phold_config(**C1, loop="plain", laq_mode=laq_mode)
    o = _oracle(C1)
    with G.Phold(cfg) as h:
        h.populate()
        done = False
        n = 0
        while not done:
            done = h.step(7)
            n += 1
        r = h.result()
        s = h.lp_stats()
    _assert_same(r, s, o)
    assert n > 10


@pytest.mark.parametrize("queue", ["laq", "laqs", "lhq", "lsq"])
def test_queue_overflow_reported(gpu_lib, queue):
    # per-LP capacity 32 with 32 initial events: the first child overflows the queue
    cfgd = dict(num_lps=16, events_per_lp=32, lookahead=0.01, end_time=50.0, seed=3, dest_mode=0)
    r, _ = _run(cfgd, queue=queue, capacity=32, insert_capacity=64)
    assert r["status_code"] in (3, 4)


@pytest.mark.parametrize("shift", ["all", "half", "far"])
def test_bucketed_form_matches_sorted_form_on_shifted_starts(gpu_lib, shift):
    """Host-provided initial events with a late start (the minimum jumps over every bucket
    before window 0), half the LPs starting late, or some events beyond the bucket horizon
    (they wait in the spill lists): the bucketed form equals the sorted form bit for bit."""
    cfgd = dict(num_lps=64, events_per_lp=16, lookahead=0.25, end_time=80.0, seed=5, dest_mode=1, ring_width=3)
    ev = G.initial_events(G.make_phold_config(**cfgd))
    if shift == "all":
        ev["ts"] += np.float32(30.0)
    elif shift == "half":
        ev["ts"][ev["lp"] >= 32] += np.float32(30.0)
    else:
        ev["ts"][ev["id"] % 5 == 0] += np.float32(45.0)
    out = []
    for mode, loop in ((0, "persistent"), (2, "persistent"), (2, "plain")):
        with G.Phold(G.make_phold_config(**cfgd, laq_mode=mode, loop=loop)) as h:
            h.populate(ev)
            h.run()
            r = h.result()
            s = h.lp_stats()
        assert r["status_code"] == 0, (mode, loop, r)
        out.append((r, s))
    (r0, s0) = out[0]
    for r, s in out[1:]:
        for k in ("committed", "pending", "pending_csum", "digest", "steps"):
            assert r[k] == r0[k], k
        for k in ("count", "csum", "ohash"):
            assert np.array_equal(s[k], s0[k]), k
