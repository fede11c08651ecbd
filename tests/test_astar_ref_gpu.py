"""Reference-semantics A* on the GPU against its CPU oracle, every agent bit for bit
(found, the goal's half-precision f, pops, rounds), with any number of concurrent slots:
agents are independent, so the slot schedule changes nothing."""
import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _check(m, agents, slots, open_capacity=0):
    with G.AStarRef(m.shape[1], m.shape[0], slots=slots, open_capacity=open_capacity) as a:
        got = a.solve(m, agents)
    _, want = O.astar_ref(m, agents, threads=8)
    assert (got["status"] == 0).all()
    for k in ("found", "pops", "rounds"):
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got["cost"].view(np.uint32), want["cost"].view(np.uint32))
    return got


@pytest.mark.parametrize("w,h,frac,slots", [(64, 64, 0.2, 64), (128, 96, 0.25, 7), (256, 256, 0.2, 2048),
                                            (256, 256, 0.2, 1), (37, 211, 0.1, 300)])
def test_agents_match_oracle(gpu_lib, w, h, frac, slots):
    m = G.astar_ref_map(w, h, frac, 1.0, seed=w + h)
    n = 64 if slots == 1 else 600
    agents = G.astar_ref_agents(m, n, seed=7)
    r = _check(m, agents, slots)
    assert r["found"].sum() > n // 2


def test_edge_agents(gpu_lib):
    m = np.zeros((16, 16), np.uint8)
    m[:, 8] = 1
    agents = np.array([(5 * 16 + 2, 5 * 16 + 2), (0, 255), (0, 15 * 16 + 7)], G.ASTAR_REF_AGENT_DTYPE)
    r = _check(m, agents, slots=2)
    assert list(r["found"]) == [1, 0, 1]


def test_open_list_overflow_is_reported(gpu_lib):
    m = np.zeros((64, 64), np.uint8)
    agents = np.array([(0, 64 * 64 - 1)], G.ASTAR_REF_AGENT_DTYPE)
    with G.AStarRef(64, 64, slots=1, open_capacity=16) as a:
        r = a.solve(m, agents)
    assert r[0]["status"] == 3  # GPQ_ERR_QUEUE_FULL
