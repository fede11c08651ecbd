"""Full-size PHOLD runs against the committed oracle results (tests/golden/phold_golden.json,
made by tests/golden/make_phold_golden.py): the 65,536-LP ring workload to end time 1000
(3.8 G committed events, 10,001 windows) through the bucketed and the sorted local array
queue and the global array queue, and the 1,024-LP workload through all five queue kinds.
Every output is compared bit for bit: committed, windows, pending, pending checksum, the
digest over the per-LP outputs and a sha256 of the per-LP arrays."""
import json
import os

import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "phold_golden.json")) as fh:
    GOLDEN = json.load(fh)


def _check(name, queue="laq", laq_mode=0, loop="persistent", **kw):
    g = GOLDEN[name]
    cfgd = dict(g["config"])
    cfg = G.make_phold_config(**cfgd, queue=queue, laq_mode=laq_mode, loop=loop, **kw)
    with G.Phold(cfg) as h:
        h.populate()
        h.run()
        r = h.result()
        s = h.lp_stats()
    assert r["status_code"] == 0, r
    assert r["committed"] == g["committed"]
    assert r["steps"] == g["windows"]
    assert r["pending"] == g["pending"]
    assert r["pending_csum"] == int(g["pending_csum"])
    assert r["digest"] == int(g["digest"])
    assert O.digest(s["count"], s["csum"], s["ohash"]) == int(g["digest"])
    assert O.lp_sha256(s["count"], s["csum"], s["ohash"]) == g["lp_sha256"]
    return r


@pytest.mark.gpu
@pytest.mark.slow
@pytest.mark.parametrize("queue,laq_mode,gaq_engine", [("laq", 2, 0), ("laq", 0, 0), ("gaq", 0, 0), ("gaq", 0, 1)])
def test_large_workload_full_end_time(gpu_lib, queue, laq_mode, gaq_engine):
    """65,536 LPs x 64, ring +-16, lookahead 0.1, end time 1000, seed 7 (the global array
    queue as one sorted array in one launch, and as the graph-replayed kernel sequence)."""
    r = _check("phold_large_65536lp_x64_ring16_T1000", queue=queue, laq_mode=laq_mode, capacity=256,
               gaq_engine=gaq_engine)
    assert r["committed"] > 3_800_000_000


@pytest.mark.gpu
@pytest.mark.parametrize("queue,gaq_engine", [("laq", 0), ("lhq", 0), ("lsq", 0), ("gaq", 0), ("gaq", 1), ("hq", 0)])
def test_plain_workload_every_kind(gpu_lib, queue, gaq_engine):
    _check("phold_plain_1024lp_x16_T100", queue=queue, gaq_engine=gaq_engine)


def test_golden_one_per_lp_entries_agree_with_full_drain():
    """The reference's schedule (one event per LP per window) commits the same per-LP
    sequences in more windows."""
    for a, b in (("phold_plain_1024lp_x16_T100", "phold_plain_1024lp_x16_T100_one_per_lp"),
                 ("phold_large_65536lp_x64_ring16_T3", "phold_large_65536lp_x64_ring16_T3_one_per_lp")):
        ga, gb = GOLDEN[a], GOLDEN[b]
        for k in ("committed", "pending", "pending_csum", "digest", "lp_sha256"):
            assert ga[k] == gb[k], (a, k)
        assert gb["windows"] > ga["windows"]
