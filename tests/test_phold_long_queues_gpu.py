"""Long per-LP queues (the case the reference's local array queue backed by a heap is
for, src/local_array_queue.cu:517-561,603-681): 4,096 LPs with 4,096 pending events each
and lookahead 0.01 (about 40 safe events per LP per window), against the committed oracle
results.  The bucketed local array queue keeps such queues without per-insert ordering
(near events in time buckets, the rest in the per-LP spill lists); the sorted form and
the per-LP heap run the same workload beside it."""
import json
import os

import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NAME = "phold_long_4096lp_x4096_ring16_T2"


@pytest.mark.parametrize("queue,kw", [("laq", dict(laq_mode=2, capacity=8192)),
                                      ("laq", dict(laq_mode=0, capacity=8192, insert_capacity=128)),
                                      ("lhq", dict(capacity=8192, insert_capacity=128))])
def test_long_queues_exact(gpu_lib, queue, kw):
    with open(os.path.join(HERE, "golden", "phold_golden.json")) as fh:
        g = json.load(fh)[NAME]
    cfg = G.make_phold_config(**g["config"], queue=queue, loop="persistent", **kw)
    with G.Phold(cfg) as h:
        h.populate()
        h.run()
        r = h.result()
        s = h.lp_stats()
    assert r["status_code"] == 0, r
    assert (r["committed"], r["steps"], r["pending"]) == (g["committed"], g["windows"], g["pending"])
    assert r["pending_csum"] == int(g["pending_csum"]) and r["digest"] == int(g["digest"])
    assert O.lp_sha256(s["count"], s["csum"], s["ohash"]) == g["lp_sha256"]
    print(f"{queue} {kw}: {r['elapsed_ms']:.1f} ms, {r['committed'] / r['elapsed_ms'] / 1e6:.2f} G events/s")
