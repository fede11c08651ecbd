"""CPU tests of the A* oracle and of the host-side query generator.

The reference has no A* test and no golden vector (src/ holds no test of a_star.cu), so
the oracle is pinned here against an independent restatement: a pure-Python Dijkstra
from the start gives g*, and under a consistent heuristic the expanded set of the
pinned semantics is exactly {c : g*(c) + h(c) <= C*}; the canonical path is re-walked
from g*.
"""
import heapq

import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

MIX_M1 = 0xBF58476D1CE4E5B9
MIX_M2 = 0x94D049BB133111EB
PHI = 0x9E3779B97F4A7C15
M64 = (1 << 64) - 1


def mix(z):
    z = ((z ^ (z >> 30)) * MIX_M1) & M64
    z = ((z ^ (z >> 27)) * MIX_M2) & M64
    return z ^ (z >> 31)


def draw(seed, i, tsb, k):
    return mix(mix(seed ^ ((i * PHI) & M64)) ^ ((tsb << 8) | (k & 0xFF)))


def blocked_grid(g):
    w, h = g["width"], g["height"]
    b = np.zeros(w * h, bool)
    for c in range(w * h):
        b[c] = (draw(g["seed"], c, 0x41535452, 0) >> 40) < g["block_thr"]
    b[g["start"]] = False
    b[g["goal"]] = False
    return b


def moves(g, blk, c):
    w, h = g["width"], g["height"]
    x, y = c % w, c // w
    dirs = [(1, 0), (-1, 0), (0, 1), (0, -1)]
    if g["conn"] == 8:
        dirs += [(1, 1), (-1, 1), (1, -1), (-1, -1)]
    for k, (dx, dy) in enumerate(dirs):
        nx, ny = x + dx, y + dy
        if not (0 <= nx < w and 0 <= ny < h):
            continue
        n = ny * w + nx
        if blk[n]:
            continue
        if k >= 4 and (blk[y * w + nx] or blk[ny * w + x]):
            continue
        yield n, (1 if g["conn"] == 4 else (10 if k < 4 else 14))


def heur(g, c):
    w = g["width"]
    dx = abs(c % w - g["goal"] % w)
    dy = abs(c // w - g["goal"] // w)
    return dx + dy if g["conn"] == 4 else 10 * max(dx, dy) + 4 * min(dx, dy)


def dijkstra_reference(g):
    blk = blocked_grid(g)
    inf = 0xFFFFFFFF
    dist = np.full(g["width"] * g["height"], inf, np.int64)
    dist[g["start"]] = 0
    pq = [(0, g["start"])]
    while pq:
        d, c = heapq.heappop(pq)
        if d > dist[c]:
            continue
        for n, cost in moves(g, blk, c):
            if d + cost < dist[n]:
                dist[n] = d + cost
                heapq.heappush(pq, (d + cost, n))
    cs = int(dist[g["goal"]])
    exp, gsum = 0, 0
    for c in range(len(dist)):
        if dist[c] == inf or (cs != inf and dist[c] + heur(g, c) > cs):
            continue
        exp += 1
        gsum = (gsum + mix((c << 32) | int(dist[c]))) & M64
    path_hash, plen = 0, 0
    if cs != inf:
        cur, i = g["goal"], 0
        while True:
            path_hash = (path_hash + mix((((i << 32) | cur) + PHI) & M64)) & M64
            i += 1
            if cur == g["start"]:
                break
            cand = [p for p, cost in moves(g, blk, cur)
                    if dist[p] != inf and dist[p] + cost == dist[cur] and dist[p] + heur(g, p) <= cs]
            cur = min(cand)
        plen = i
    return {"cost": cs, "expanded": exp, "gsum": gsum, "path_len": plen, "path_hash": path_hash}


def _grid(w, h, dens, seed, conn, start, goal):
    return {"seed": seed, "width": w, "height": h, "block_thr": int(dens * 16777216.0), "conn": conn,
            "start": start, "goal": goal}


CASES = [
    _grid(24, 24, 0.2, 3, 4, 0, 24 * 24 - 1),
    _grid(40, 17, 0.3, 5, 4, 3, 40 * 17 - 2),
    _grid(32, 32, 0.25, 9, 8, 0, 32 * 32 - 1),
    _grid(33, 29, 0.1, 1, 8, 500, 7),
    _grid(16, 16, 0.6, 2, 4, 0, 255),     # dense: goal likely unreachable
    _grid(1, 50, 0.0, 4, 4, 0, 49),       # a corridor
    _grid(20, 20, 0.2, 8, 8, 37, 37),     # start == goal
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_matches_dijkstra(case):
    g = CASES[case]
    want = dijkstra_reference(g)
    got = O.astar(g)
    for k in ("cost", "expanded", "gsum", "path_len", "path_hash"):
        assert got[k] == want[k], (k, got[k], want[k])
    assert got["pops"] == got["expanded"]  # the oracle closes exactly the pinned set


def test_oracle_plain_grid_known_answer():
    """2048 x 2048, Bernoulli(0.2) from seed 3, (0,0) -> (2047,2047), 4-connected: the
    cost equals the Manhattan distance and half the grid lies on the f = C* layer."""
    g = _grid(2048, 2048, 0.2, 3, 4, 0, 2048 * 2048 - 1)
    r = O.astar(g)
    assert r["cost"] == 4094
    assert r["path_len"] == 4095
    assert r["expanded"] == 1993051


@pytest.mark.parametrize("conn,lo,hi,dlo,dhi,seed", [(8, 64, 1024, 0.1, 0.3, 11), (4, 128, 4096, 0.2, 0.2, 99)])
def test_query_generator_matches_oracle(conn, lo, hi, dlo, dhi, seed):
    prod = G.astar_queries(seed, 40, conn, lo, hi, dlo, dhi)
    for i in range(40):
        want = O.astar_query(seed, i, conn, lo, hi, dlo, dhi)
        for k in O.ASTAR_FIELDS:
            assert int(prod[i][k]) == want[k], (i, k)
        assert lo <= want["width"] <= hi and want["start"] != want["goal"]


def test_query_sides_are_log_uniform():
    q = G.astar_queries(11, 400, 8, 64, 1024, 0.1, 0.3)
    ls = np.log2(q["width"].astype(float))
    assert 6.0 <= ls.min() and ls.max() <= 10.0
    assert abs(ls.mean() - 8.0) < 0.25  # log-uniform on [6, 10]
