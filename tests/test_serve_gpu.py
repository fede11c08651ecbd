"""GPU tests of serving (gpq_serve_run): every request of a mixed stream of A* queries
and PHOLD runs gets the same result in the continuous-batching mix as alone (the plain
one-request-per-launch path), with admissions throttled by the memory budget."""
import ctypes
import random

import numpy as np
import pytest

import gpupq_b200 as G

pytestmark = pytest.mark.gpu

A_KEYS = ("cost", "path_len", "expanded", "gsum", "path_hash")
P_KEYS = ("committed", "steps", "pending", "pending_csum", "digest", "final_min")


def _mixed(n, seed, rate=400.0):
    rng = random.Random(seed)
    reqs = (G.ServeRequest * n)()
    t = 0.0
    for i in range(n):
        t += rng.expovariate(rate)
        q = reqs[i]
        q.arrival = t
        if rng.random() < 0.7:
            q.kind = G.REQ_ASTAR
            g = G.astar_queries(seed, 1, rng.choice([4, 8]), 64, 700, 0.1, 0.3, first=i)[0]
            for k in ("seed", "width", "height", "block_thr", "conn", "start", "goal"):
                setattr(q.astar, k, int(g[k]))
        else:
            q.kind = G.REQ_PHOLD
            L = rng.choice([1, 5, 256, 1000, 5000])
            q.phold = G.make_phold_config(L, rng.choice([1, 8, 32]), rng.choice([0.5, 1.0]),
                                          rng.choice([0.0, 10.0, 40.0]), seed * 1000 + i)
    return reqs


def _compare(batched, plain, reqs, n):
    for i in range(n):
        assert batched[i].status == 0 and plain[i].status == 0, (i, batched[i].status, plain[i].status)
        if reqs[i].kind == G.REQ_ASTAR:
            for k in A_KEYS:
                assert getattr(batched[i].astar, k) == getattr(plain[i].astar, k), (i, k)
        else:
            for k in P_KEYS:
                assert getattr(batched[i].phold, k) == getattr(plain[i].phold, k), (i, k)


@pytest.mark.parametrize("phold_form", [0, 1])
@pytest.mark.parametrize("realtime", [False, True])
def test_mix_equals_alone(gpu_lib, realtime, phold_form):
    """PHOLD runs kept in sorted rings (form 0) or time buckets (form 1) while served."""
    n = 60
    reqs = _mixed(n, 5)
    plain, ps = G.serve(reqs, n, mode=G.SERVE_PLAIN, realtime=realtime, tile=32)
    batched, bs = G.serve(reqs, n, mode=G.SERVE_BATCHED, realtime=realtime, budget=4 << 30, astar_rounds=8,
                          phold_windows=8, tile=32, phold_form=phold_form)
    _compare(batched, plain, reqs, n)
    assert bs["max_resident"] > 1
    for s in (ps, bs):
        assert s["p50"] <= s["p99"] <= s["p999"] <= s["makespan"] + 1e-9
    for i in range(n):
        assert batched[i].admitted <= batched[i].finished
        if realtime:
            assert batched[i].admitted >= reqs[i].arrival - 1e-6


def test_tight_budget_waits_and_refuses(gpu_lib):
    """A budget that holds only a few requests: later ones wait for memory, results stay
    exact; a request larger than the whole budget is refused with GPQ_ERR_NOMEM."""
    n = 24
    reqs = _mixed(n, 7)
    big = n - 1
    reqs[big].kind = G.REQ_ASTAR
    reqs[big].astar.seed, reqs[big].astar.conn = 3, 4
    reqs[big].astar.block_thr = G.density_threshold(0.2)
    reqs[big].astar.width = reqs[big].astar.height = 8000
    reqs[big].astar.start, reqs[big].astar.goal = 0, 8000 * 8000 - 1
    plain, _ = G.serve(reqs, n - 1, mode=G.SERVE_PLAIN, realtime=False, tile=32)
    batched, bs = G.serve(reqs, n, mode=G.SERVE_BATCHED, realtime=False, budget=128 << 20, astar_share=0.1,
                          astar_rounds=4, phold_windows=4, tile=32)
    assert batched[big].status == 6
    _compare(batched, plain, reqs, n - 1)
    assert bs["max_resident"] < n - 1
    first_done = min(batched[i].finished for i in range(n - 1))
    assert any(batched[i].admitted >= first_done for i in range(n - 1))  # some request waited for memory


def test_stream_generator_shape(gpu_lib):
    reqs, n = G.serve_stream(99, 2000.0, 2.0)
    assert 3600 < n < 4400  # Poisson(4000)
    kinds = np.array([reqs[i].kind for i in range(n)])
    assert 0.75 < (kinds == G.REQ_ASTAR).mean() < 0.85
    arr = np.array([reqs[i].arrival for i in range(n)])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 2.0
    sides = np.array([reqs[i].astar.width for i in range(n) if reqs[i].kind == G.REQ_ASTAR])
    assert sides.min() >= 128 and sides.max() <= 4096
    lps = np.array([reqs[i].phold.num_lps for i in range(n) if reqs[i].kind == G.REQ_PHOLD])
    assert lps.min() >= 256 and lps.max() <= 65536
