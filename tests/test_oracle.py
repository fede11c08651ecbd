"""CPU tests of the oracle: pinned against the reference's own known-answer tests, and
the sequential and window-synchronous drivers checked against each other."""
import json
import math
import os
import random
import struct

import numpy as np
import pytest

from oracle import oracle as O
from oracle.queue_model import QueueModel

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")


@pytest.fixture(scope="module")
def kats():
    with open(GOLDEN) as f:
        return json.load(f)


def _ring(cap, slots):
    r = np.full(cap, -999, np.int64)
    for k, v in slots.items():
        r[int(k)] = v
    return r


def test_kat_quicksort(kats):
    k = kats["ring_helpers"]["quicksort"]
    a = np.array(k["input"], np.int64)
    O.lib().oracle_ring_quicksort(a, len(a), k["left"], k["right"])
    assert a.tolist() == k["expect"]


def test_kat_search_ringbuffer(kats):
    k = kats["ring_helpers"]["search_ringbuffer"]
    r = _ring(k["cap"], k["slots"])
    for item, pos in k["queries"]:
        assert O.lib().oracle_ring_search(r, k["cap"], k["read"], k["write"], item) == pos


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_kat_insert_sorted(kats, idx):
    k = kats["ring_helpers"]["insert_sorted"][idx]
    r = _ring(k["cap"], k["slots"])
    O.lib().oracle_ring_insert_sorted(r, k["cap"], k["read"], k["write"], k["item"])
    for slot, v in k["expect_slots"].items():
        assert r[int(slot)] == v, (slot, r.tolist())


def test_quicksort_wrapping_ranges():
    rng = random.Random(5)
    for _ in range(200):
        cap = rng.randint(2, 40)
        n = rng.randint(1, cap)
        left = rng.randrange(cap)
        right = (left + n - 1) % cap
        ring = np.array([rng.randint(0, 50) for _ in range(cap)], np.int64)
        idx = [(left + i) % cap for i in range(n)]
        want = sorted(ring[idx].tolist())
        O.lib().oracle_ring_quicksort(ring, cap, left, right)
        assert ring[idx].tolist() == want


def _apply_queue_kat(k):
    m = QueueModel(k["num_lps"], root_size=k.get("node_size", 0) if k.get("kind") == "hq" else 0)
    nid = 0
    batches = k.get("insert_batches") or [k["inserts"]]
    for b in batches:
        for lp, ts in b:
            m.insert(float(ts), lp, nid)
            nid += 1
        m.post()
    if "inserts_2" in k:
        for lp, ts in k["inserts_2"]:
            m.insert(float(ts), lp, nid)
            nid += 1
        m.post()
    return m


def test_kats_queue_level(kats):
    for name, k in kats["queue_level"].items():
        m = _apply_queue_kat(k)
        if "expect_lp" in k:
            for lp, want in k["expect_lp"].items():
                assert [it[0] for it in m.lp_items(int(lp))] == want, name
        if "expect_min" in k:
            assert m.get_min() == k["expect_min"], name
        if "expect_global" in k:
            assert [it[0] for it in m.global_items()] == k["expect_global"], name
        if "expect_dequeued" in k:
            bound = m.get_min() + k["lookahead"]
            got = m.dequeue(bound, k.get("max_per_lp", 0))
            assert [[it[1], it[0]] for it in got] == k["expect_dequeued"], name
            if "expect_remaining" in k:
                assert [it[0] for it in m.global_items()] == k["expect_remaining"], name


def test_logf_close_to_libm():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.random(2000).astype(np.float32) + np.float32(1e-7),
                         np.float32([1.0, 0.5, 2 ** -24, 0.70710677, 0.7071068])])
    for x in xs:
        got = O.logf(float(x))
        want = math.log(float(x))
        assert abs(got - want) <= 4e-7 * max(1.0, abs(want)), (x, got, want)
    assert struct.pack("<f", O.logf(1.0)) == struct.pack("<f", 0.0)


C1 = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0)


@pytest.mark.parametrize("cfg,threads", [
    (dict(num_lps=64, events_per_lp=4, lookahead=0.5, end_time=20.0, seed=1, dest_mode=0), 1),
    (dict(num_lps=64, events_per_lp=4, lookahead=0.5, end_time=20.0, seed=1, dest_mode=0), 3),
    (dict(num_lps=257, events_per_lp=9, lookahead=0.1, end_time=5.0, seed=7, dest_mode=1, ring_width=16), 4),
    (dict(num_lps=40, events_per_lp=2, lookahead=2.0, end_time=50.0, seed=3, dest_mode=1, ring_width=3), 8),
    (C1, 4),
])
def test_seq_equals_window(cfg, threads):
    c = O.make_cfg(**cfg)
    a = O.phold(c, 0)
    b = O.phold(c, threads)
    for k in ("count", "csum", "ohash"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("committed", "steps", "pending", "pending_csum"):
        assert a[k] == b[k], k
    assert a["committed"] == int(a["count"].sum())
    assert a["pending"] == cfg["num_lps"] * cfg["events_per_lp"]  # population is conserved


def test_c1_known_values():
    """Regression pin of the oracle on the 1024-LP workload (values produced by this
    oracle; the GPU must reproduce them)."""
    a = O.phold(O.make_cfg(**C1), 0)
    assert a["committed"] == 820705
    assert a["steps"] == 100


def test_zero_end_time_commits_nothing():
    a = O.phold(O.make_cfg(num_lps=8, events_per_lp=2, lookahead=1.0, end_time=0.0, seed=1), 0)
    assert a["committed"] == 0 and a["steps"] == 0 and a["pending"] == 16
