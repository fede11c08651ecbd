"""CPU checks of the reference-semantics A* oracle (oracle/astar_ref_oracle.cpp)."""
import numpy as np

import gpupq_b200 as G
from oracle import oracle as O


def test_half_conversion_is_ieee_round_to_nearest_even():
    """Pinned to numpy's binary16 conversion (IEEE 754 round to nearest even)."""
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.uniform(0, 70000, 4000), rng.uniform(0, 2e-4, 1000), rng.uniform(0, 300, 4000),
                           np.array([0.0, 65504.0, 65519.99, 65520.0, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26, 1.0005])])
    for v in vals.astype(np.float32):
        want = np.float32(np.float16(v)) if v < 65520 else np.float32(np.inf)
        got = O.lib().oracle_to_half(float(v))
        assert got == want or (np.isinf(got) and np.isinf(want)), (float(v), got, want)
        bits = int(np.array([want], np.float16).view(np.uint16)[0])
        assert O.lib().oracle_half_bits(float(v)) == bits


def test_octile_h_in_double_rounded_to_float():
    for (x0, y0, x1, y1) in [(0, 0, 3, 7), (10, 200, 255, 0), (5, 5, 5, 5), (0, 0, 255, 255), (17, 3, 1, 250)]:
        dx, dy = abs(x0 - x1), abs(y0 - y1)
        want = np.float32(2 ** 0.5 * min(dx, dy) + max(dx, dy) - min(dx, dy))
        assert O.lib().oracle_astar_ref_h(x0, y0, x1, y1) == want


def test_agent_edge_cases():
    m = np.zeros((16, 16), np.uint8)
    m[:, 8] = 1  # a wall splits the map
    agents = np.zeros(3, G.ASTAR_REF_AGENT_DTYPE)
    agents[0] = (5 * 16 + 2, 5 * 16 + 2)    # start == goal: found at once with f = 0
    agents[1] = (0, 15 * 16 + 15)           # across the wall: no path
    agents[2] = (0, 15 * 16 + 7)            # same side
    _, r = O.astar_ref(m, agents)
    assert (r[0]["found"], r[0]["cost"], r[0]["pops"], r[0]["rounds"]) == (1, 0.0, 1, 1)
    assert r[1]["found"] == 0 and r[1]["pops"] >= 8 * 16 and r[2]["found"] == 1  # every reachable cell popped
    assert r[2]["cost"] >= 15.0  # at least the straight-line octile distance of 15 rows


def test_map_and_agents_are_deterministic():
    m1 = G.astar_ref_map(64, 48, 0.2, 1.0, seed=3)
    m2 = G.astar_ref_map(64, 48, 0.2, 1.0, seed=3)
    assert np.array_equal(m1, m2) and 0.1 < m1.mean() < 0.5
    a = G.astar_ref_agents(m1, 50, seed=4)
    assert np.array_equal(a, G.astar_ref_agents(m1, 50, seed=4))
    flat = m1.reshape(-1)
    assert not flat[a["start"]].any() and not flat[a["goal"]].any()
