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


def _drive(s, runs, slot_of, pending, windows, got):
    """Admit, step and collect until every run has finished; returns the results by run."""
    for _ in range(100000):
        while pending:
            sl = s.admit(runs[pending[0]])
            if sl is None:
                break
            slot_of[sl] = pending.pop(0)
        s.step(windows)
        for sl, r in s.collect():
            got[slot_of.pop(sl)] = _d(r)
        if not pending and not slot_of:
            return got
    raise AssertionError("runs did not finish")


@pytest.mark.parametrize("bucketed", [False, True])
def test_session_snapshot_resumes_exactly(gpu_lib, bucketed):
    """Snapshot a session mid-stream (some runs mid-run, one admitted but not started,
    LP ranges reused), finish it; restore the snapshot into a fresh session and into one
    that already holds other runs, finish those: every run ends the same three times and
    as it ends alone."""
    runs = _runs(3, 14)
    kw = dict(max_lps=4000, max_instances=8, bucketed=bucketed)
    with G.PholdSession(**kw) as s:
        slot_of, pending, got = {}, list(range(len(runs))), {}
        for _ in range(3):  # a few steps, with collections that free slots and LPs
            while pending:
                sl = s.admit(runs[pending[0]])
                if sl is None:
                    break
                slot_of[sl] = pending.pop(0)
            s.step(4)
            for sl, r in s.collect():
                got[slot_of.pop(sl)] = _d(r)
        if pending:  # one run admitted but not started when the snapshot is taken
            sl = s.admit(runs[pending[0]])
            if sl is not None:
                slot_of[sl] = pending.pop(0)
        snap = s.snapshot()
        state = (dict(slot_of), list(pending), dict(got))
        first = _drive(s, runs, slot_of, pending, 4, got)
    for target_busy in (False, True):
        with G.PholdSession(**kw) as t:
            if target_busy:
                for c in _runs(9, 3):
                    t.admit(c)
                t.step(2)
            t.restore(snap)
            slot_of, pending, got = dict(state[0]), list(state[1]), dict(state[2])
            again = _drive(t, runs, slot_of, pending, 4, got)
            assert t.usage() == (0, 0)
        assert sorted(again) == sorted(first) == list(range(len(runs)))
        for i in range(len(runs)):
            _same(again[i], first[i])
    for i, c in enumerate(runs):
        _same(first[i], _alone(c))


def test_session_snapshot_rejects_other_parameters(gpu_lib):
    with G.PholdSession(max_lps=1000, max_instances=4) as s:
        s.admit(_runs(4, 1)[0])
        snap = s.snapshot()
    with G.PholdSession(max_lps=2000, max_instances=4) as t:
        with pytest.raises(G.GpqError):
            t.restore(snap)
    with G.PholdSession(max_lps=1000, max_instances=4, bucketed=True) as t:
        with pytest.raises(G.GpqError):
            t.restore(snap)
    with G.PholdSession(max_lps=1000, max_instances=4) as t:
        with pytest.raises(G.GpqError):
            t.restore(snap[:-5])
