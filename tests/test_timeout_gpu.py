"""Bounded device waits run out and report GPQ_ERR_TIMEOUT, and the context stays usable.

Every grid barrier of the persistent kernels polls at most gpq_set_spin_limit times and
then sets GPQ_ERR_TIMEOUT and returns; a block that passes a barrier alone meets the next
one with the same bound, so every block of the launch ends.  With a limit of one poll the
first barrier of a launch over hundreds of CTAs runs out (the CTAs do not all arrive
within one poll).  Nothing faults and nothing waits without a bound.  After the limit is
restored, the same handle runs the workload exactly again.
"""
import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEFAULT_SPIN = 1 << 24
CFG = dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=2.0, seed=7, dest_mode=1, ring_width=16)


@pytest.fixture
def spin_one_poll(gpu_lib):
    G.check(G.lib().gpq_set_spin_limit(1), "gpq_set_spin_limit")
    try:
        yield
    finally:
        G.check(G.lib().gpq_set_spin_limit(DEFAULT_SPIN), "gpq_set_spin_limit")


@pytest.mark.parametrize("laq_mode", [2, 0])
def test_phold_barrier_timeout_then_exact(spin_one_poll, laq_mode):
    cfg = G.make_phold_config(**CFG, laq_mode=laq_mode, capacity=256, loop="persistent")
    with G.Phold(cfg) as h:
        h.populate()
        st = G.lib().gpq_phold_run(h._h, None)
        r = h.result()
        assert 5 in (st, r["status_code"]), (st, r)
        assert h.launch_info()["grid"] > 100
        G.check(G.lib().gpq_set_spin_limit(DEFAULT_SPIN), "gpq_set_spin_limit")
        h.populate()
        h.run()
        r = h.result()
        s = h.lp_stats()
    o = O.phold(O.make_cfg(**CFG), 8)
    assert r["status_code"] == 0
    assert r["committed"] == o["committed"] and r["steps"] == o["steps"]
    assert np.array_equal(s["ohash"], o["ohash"]) and np.array_equal(s["count"], o["count"])


def test_astar_barrier_timeout_then_exact(spin_one_poll):
    q = G.astar_queries(11, 64, 8, 64, 512, 0.1, 0.3)
    with G.AStar(tile=32) as a:
        with pytest.raises(G.GpqError) as e:
            a.solve(q)
        assert e.value.status == 5
        G.check(G.lib().gpq_set_spin_limit(DEFAULT_SPIN), "gpq_set_spin_limit")
        res = a.solve(q)
    for i in range(len(q)):
        want = O.astar({k: int(q[i][k]) for k in O.ASTAR_FIELDS})
        assert res[i]["status"] == 0
        for k in ("cost", "expanded", "gsum", "path_len", "path_hash"):
            assert int(res[i][k]) == want[k], (i, k)
