"""Host logic of the autotuners (gpupq_b200.autotune) on CPU, with fake engines in place of
the GPU handles: the fastest agreeing candidate wins, candidates that fail or overflow are
skipped, a candidate whose results differ from the others is an error, and the cache
answers the next call without timing anything."""
import json

import numpy as np
import pytest

import gpupq_b200 as G
from gpupq_b200 import autotune as T


class FakeAStar:
    """Times and results by configuration; tile 128 fails like an oversized shared-memory
    request; `bad` (tile, window, ctas_per_sm) gives a different expanded count."""
    calls = 0
    bad = None

    def __init__(self, tile=64, window=0, ctas_per_sm=0):
        FakeAStar.calls += 1
        if tile == 128:
            raise G.GpqError(1, "gpq_astar_create", "tile too large")
        self.kw = (tile, window, ctas_per_sm)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def solve(self, grids):
        r = np.zeros(len(grids), G.ASTAR_RESULT_DTYPE)
        r["cost"] = 7
        r["expanded"] = 100 + (1 if self.kw == FakeAStar.bad else 0)
        return r

    def stats(self):
        tile, window, ctas = self.kw
        return {"total_ms": 10.0 + abs(tile - 64) / 8 + abs(window - 40) / 10 + abs(ctas - 1)}


def _grids():
    return np.concatenate([G.astar_grid(100, 80, 0.2, 1, conn=8), G.astar_grid(64, 64, 0.3, 2, conn=8)])


def test_astar_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "AStar", FakeAStar)
    monkeypatch.setattr(T, "SHIPPED", str(tmp_path / "none.json"))
    cache = str(tmp_path / "cache.json")
    FakeAStar.calls, FakeAStar.bad = 0, None
    best = T.tune_astar(_grids(), space={"tile": [32, 64, 128]}, cache=cache)
    assert best == {"tile": 64, "window": 40, "ctas_per_sm": 1}  # window in move costs x 10 (8-connected)
    assert FakeAStar.calls == 3 * 3 * 4
    entry = json.load(open(cache))[T.astar_workload_key(_grids())]
    assert entry["best"] == best and len(entry["all"]) == 2 * 3 * 4  # tile 128 was rejected
    FakeAStar.calls = 0
    assert T.tune_astar(_grids(), cache=cache) == best and FakeAStar.calls == 0


def test_astar_window_unit_for_4_connected(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "AStar", FakeAStar)
    monkeypatch.setattr(T, "SHIPPED", str(tmp_path / "none.json"))
    grids = G.astar_grid(50, 50, 0.2, 3, conn=4)
    best = T.tune_astar(grids, space={"window": [2, 4, 10], "tile": [64], "ctas_per_sm": [1]},
                        cache=str(tmp_path / "c.json"))
    assert best["window"] == 10  # 4-connected: move cost 1, so 10 is the closest to 40


def test_astar_disagreement_is_an_error(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "AStar", FakeAStar)
    monkeypatch.setattr(T, "SHIPPED", str(tmp_path / "none.json"))
    FakeAStar.bad = (64, 100, 2)
    try:
        with pytest.raises(RuntimeError, match="disagrees"):
            T.tune_astar(_grids(), cache=str(tmp_path / "c.json"))
    finally:
        FakeAStar.bad = None


def test_astar_key_separates_workload_classes():
    a = T.astar_workload_key(_grids())
    b = T.astar_workload_key(_grids()[:1])
    c = T.astar_workload_key(G.astar_grid(100, 80, 0.2, 1, conn=4))
    assert len({a, b, c}) == 3 and "|astar|" in a


class FakePhold:
    """PHOLD handle: per-window time by shape; lanes 32 overflows (status 4); committed
    count and digest equal for every shape unless `bad` names one."""
    bad = None

    def __init__(self, cfg):
        self.cfg = cfg

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def populate(self):
        pass

    def run(self):
        pass

    def result(self):
        c = self.cfg
        shape = (c["lanes_per_lp"], c["block_threads"], c["insert_capacity"], c.get("laq_mode", 0))
        t = 1.0 + c["block_threads"] / 1024 + c["lanes_per_lp"] / 64 + (0 if c.get("laq_mode") == 2 else 0.5)
        return {"status_code": 4 if c["lanes_per_lp"] == 32 and c.get("laq_mode") != 2 else 0,
                "committed": 1000, "digest": 5 + (shape == FakePhold.bad), "steps": 10, "elapsed_ms": 10 * t}


def test_phold_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "Phold", FakePhold)
    monkeypatch.setattr(T, "make_phold_config", lambda **kw: kw)
    monkeypatch.setattr(T, "SHIPPED", str(tmp_path / "none.json"))
    cache = str(tmp_path / "cache.json")
    cfgd = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=1, dest_mode=0, capacity=256)
    best = T.tune_phold(cfgd, queue="laq", windows=10, cache=cache)
    assert best["laq_mode"] == 2 and best["block_threads"] == 64
    entry = json.load(open(cache))[T.workload_key(cfgd, "laq", "persistent")]
    # the bucketed form varies only its CTA size: 4 sizes, duplicates removed
    assert sum(1 for e in entry["all"] if e["shape"]["laq_mode"] == 2) == 4
    assert all(e["shape"]["lanes_per_lp"] != 32 for e in entry["all"] if e["shape"]["laq_mode"] == 0)
    monkeypatch.setattr(T, "Phold", None)  # a cached answer touches no engine
    assert T.tune_phold(cfgd, queue="laq", windows=10, cache=cache) == best


def test_phold_disagreement_is_an_error(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "Phold", FakePhold)
    monkeypatch.setattr(T, "make_phold_config", lambda **kw: kw)
    monkeypatch.setattr(T, "SHIPPED", str(tmp_path / "none.json"))
    FakePhold.bad = (16, 128, 64, 0)
    try:
        cfgd = dict(num_lps=64, events_per_lp=4, lookahead=1.0, end_time=10.0, seed=2, dest_mode=0, capacity=64)
        with pytest.raises(RuntimeError, match="disagrees"):
            T.tune_phold(cfgd, queue="laq", windows=5, cache=str(tmp_path / "c.json"))
    finally:
        FakePhold.bad = None
