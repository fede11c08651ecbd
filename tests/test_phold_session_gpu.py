"""GPU tests of resident PHOLD runs (gpq_phold_session_*): every run of a batch or of a
stream with admissions between steps commits exactly what it commits alone on the
single-run engine (committed count, windows, digest over the per-LP outputs, pending
events, final minimum)."""
import random

import pytest

import gpupq_b200 as G

pytestmark = pytest.mark.gpu

KEYS = ("committed", "steps", "pending", "pending_csum", "digest", "final_min")


def _alone(cfg):
    c = G.make_phold_config(cfg.num_lps, cfg.events_per_lp, cfg.lookahead, cfg.end_time, cfg.seed,
                            dest_mode=cfg.dest_mode, ring_width=cfg.ring_width or 16, queue="laq",
                            capacity=256, insert_capacity=64, loop="persistent")
    c.ring_threshold = cfg.ring_threshold
    with G.Phold(c) as h:
        h.populate()
        h.run()
        return h.result()


def _runs(seed, n):
    rng = random.Random(seed)
    out = []
    for i in range(n):
        L = rng.choice([1, 3, 40, 256, 700, 3000])
        ring = L > 40 and rng.random() < 0.5
        out.append(G.make_phold_config(L, rng.choice([1, 4, 16, 32]), rng.choice([0.1, 0.5, 1.0]),
                                       rng.choice([0.0, 5.0, 20.0, 60.0]), 1000 + i,
                                       dest_mode=G.DEST_RING if ring else G.DEST_UNIFORM, ring_width=16))
    return out


def _d(r):
    return r if isinstance(r, dict) else r.as_dict()


def _same(a, b):
    a, b = _d(a), _d(b)
    for k in KEYS:
        assert a[k] == b[k], (k, a[k], b[k])
    assert a["status"] == 0 and b["status"] == 0


@pytest.mark.parametrize("bucketed", [False, True])
def test_batch_equals_alone(gpu_lib, bucketed):
    runs = _runs(1, 24)
    with G.PholdSession(max_lps=sum(c.num_lps for c in runs), max_instances=64, bucketed=bucketed) as s:
        slot_of = {s.admit(c): i for i, c in enumerate(runs)}
        s.step(0)
        got = {slot_of[sl]: r for sl, r in s.collect()}
        assert s.usage() == (0, 0)
    assert len(got) == len(runs)
    for i, c in enumerate(runs):
        _same(got[i], _alone(c))


@pytest.mark.parametrize("bucketed", [False, True])
@pytest.mark.parametrize("windows", [1, 5, 40])
def test_stream_equals_alone(gpu_lib, windows, bucketed):
    """Runs admitted while others are mid-run, into an LP space that holds only some of
    them at a time (LPs and slots of finished runs are reused)."""
    runs = _runs(2, 20)
    want = [_alone(c) for c in runs]
    got, slot_of, pending, refused = {}, {}, list(range(len(runs))), 0
    with G.PholdSession(max_lps=4000, max_instances=8, bucketed=bucketed) as s:
        for _ in range(100000):
            while pending:
                sl = s.admit(runs[pending[0]])
                if sl is None:
                    refused += 1
                    break
                slot_of[sl] = pending.pop(0)
            s.step(windows)
            for sl, r in s.collect():
                got[slot_of.pop(sl)] = r
            if not pending and not slot_of:
                break
    assert refused > 0 and len(got) == len(runs)
    for i in range(len(runs)):
        _same(got[i], want[i])
