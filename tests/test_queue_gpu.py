"""GPU tests of the queue objects (gpq_queue_*) against the reference's known-answer
vectors and against the queue-level model, operation by operation."""
import json
import os
import random

import numpy as np
import pytest

import gpupq_b200 as G
from oracle.queue_model import QueueModel

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")
KINDS = ["laq", "lhq", "lsq", "gaq", "hq"]


def _items(pairs, id0=0):
    a = np.zeros(len(pairs), G.ITEM_DTYPE)
    for i, (lp, ts) in enumerate(pairs):
        a[i] = (float(ts), lp, id0 + i, lp)
    return a


def _global(q):
    allit = np.concatenate([q.dump(lp) for lp in range(q.num_lps)])
    order = np.lexsort((allit["id"], allit["lp"], allit["ts"].view(np.uint32)))
    return allit[order]


@pytest.mark.parametrize("kind", KINDS)
def test_reference_queue_kats(gpu_lib, kind):
    kats = json.load(open(GOLDEN))["queue_level"]
    for name, k in kats.items():
        with G.Queue(kind, k["num_lps"], capacity=64, insert_capacity=32, node_size=k.get("node_size", 0)) as q:
            nid = 0
            for batch in k.get("insert_batches") or [k["inserts"]]:
                q.insert(_items(batch, nid))
                nid += len(batch)
                q.post()
            if "inserts_2" in k:
                q.insert(_items(k["inserts_2"], nid))
                q.post()
            if "expect_lp" in k:
                for lp, want in k["expect_lp"].items():
                    assert q.dump(int(lp))["ts"].tolist() == want, name
            if "expect_min" in k:
                assert q.get_min() == k["expect_min"], name
            if "expect_global" in k:
                assert _global(q)["ts"].tolist() == k["expect_global"], name
            if "expect_dequeued" in k:
                bound = np.float32(q.get_min()) + np.float32(k["lookahead"])
                got = q.dequeue(float(bound), k.get("max_per_lp", 0))
                assert [[int(r["lp"]), float(r["ts"])] for r in got] == k["expect_dequeued"], name
                if "expect_remaining" in k:
                    assert _global(q)["ts"].tolist() == k["expect_remaining"], name


@pytest.mark.parametrize("kind", ["laq"])
def test_ring_wraparound_like_reference(gpu_lib, kind):
    """src/test_laq.cu:189-236: a sorted run that wraps the end of an 8-slot ring takes a
    new item in the middle and at the front."""
    for item, want in [(5, [2, 4, 5, 6, 8, 10]), (1, [1, 2, 4, 6, 8, 10])]:
        with G.Queue(kind, 1, capacity=8, insert_capacity=8) as q:
            q.insert(_items([(0, 100 + i) for i in range(5)]))
            q.post()
            assert len(q.dequeue(1e9)) == 5  # read pointer now at slot 5
            q.insert(_items([(0, t) for t in (2, 4, 6, 8, 10)], 10))
            q.post()
            q.insert(_items([(0, item)], 20))
            q.post()
            assert q.dump(0)["ts"].tolist() == want


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_ops_match_model(gpu_lib, kind, seed):
    rng = random.Random(seed)
    L = rng.choice([1, 3, 37, 300])
    cap = 128
    m = QueueModel(L, root_size=16 if kind == "hq" else 0)
    nid = 0
    with G.Queue(kind, L, capacity=cap, insert_capacity=64, node_size=16) as q:
        for step in range(40):
            n = rng.randint(0, 60)
            pairs = []
            for _ in range(n):
                lp = rng.randrange(L)
                if m.length(lp) + sum(1 for p in pairs if p[0] == lp) >= cap - 1:
                    continue
                if sum(1 for p in pairs if p[0] == lp) >= 64:
                    continue
                ts = rng.choice([rng.random() * 100, float(rng.randint(0, 20))])
                pairs.append((lp, np.float32(ts)))
            arr = _items(pairs, nid)
            for r in arr:
                m.insert(float(r["ts"]), int(r["lp"]), int(r["id"]))
            nid += len(pairs)
            q.insert(arr)
            q.post()
            m.post()
            mn = q.get_min()
            assert mn == np.float32(m.get_min())
            if rng.random() < 0.6 and np.isfinite(mn):
                bound = float(np.float32(mn) + np.float32(rng.choice([0.5, 5.0, 30.0])))
                mpl = rng.choice([0, 1, 2])
                got = q.dequeue(bound, mpl)
                want = m.dequeue(bound, mpl)
                assert [(float(r["ts"]), int(r["lp"]), int(r["id"])) for r in got] == want
            if rng.random() < 0.1:
                lp = rng.randrange(L)
                q.clear(lp)
                m.clear(lp)
            for lp in rng.sample(range(L), min(L, 5)):
                assert q.length(lp) == m.length(lp)
                d = q.dump(lp)
                assert [(float(r["ts"]), int(r["lp"]), int(r["id"])) for r in d] == m.lp_items(lp)
        enq, deq = q.counts()
        assert enq == m.enqueued and deq == m.dequeued


@pytest.mark.parametrize("kind", KINDS)
def test_insert_overflow_is_an_error(gpu_lib, kind):
    """More inserts between two posts than the buffers hold (per LP for the local queues,
    insert_capacity * num_lps in total for the global array) is reported, never dropped
    silently."""
    with G.Queue(kind, 2, capacity=16, insert_capacity=4) as q:
        with pytest.raises(G.GpqError) as e:
            q.insert(_items([(0, i) for i in range(6)] + [(1, i) for i in range(3)]))
            q.post()
        assert e.value.status in (3, 4)
