"""GPU tests of PHOLD snapshots (gpq_phold_snapshot / gpq_phold_restore): a run stopped
after some windows, saved to the host and restored into a fresh handle (or back into its
own handle after it went on) ends exactly where the uninterrupted run ends, for every
queue kind; snapshots of another configuration or cut short are refused."""
import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C1 = dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0)
KINDS = [("laq", 0), ("laq", 1), ("laq", 2), ("lhq", 0), ("lsq", 0), ("gaq", 0), ("gaqg", 0), ("hq", 0)]


def _cfg(queue, mode, loop="plain", **over):
    if queue == "gaqg":  # the global array queue's graph-replayed kernel sequence
        return G.make_phold_config(**dict(C1, **over), queue="gaq", gaq_engine=1, loop=loop)
    return G.make_phold_config(**dict(C1, **over), queue=queue, laq_mode=mode, loop=loop)


def _finish(h):
    while not h.step(50):
        pass
    return h.result(), h.lp_stats()


def _same(a, b):
    (ra, sa), (rb, sb) = a, b
    for k in ("committed", "steps", "pending", "pending_csum", "digest", "status_code"):
        assert ra[k] == rb[k], (k, ra[k], rb[k])
    for k in ("count", "csum", "ohash"):
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.parametrize("queue,mode", KINDS)
def test_resume_equals_uninterrupted(gpu_lib, queue, mode):
    with G.Phold(_cfg(queue, mode)) as h:
        h.populate()
        assert not h.step(37)
        snap = h.snapshot()
        full = _finish(h)
        o = O.phold(O.make_cfg(**C1))
        assert full[0]["committed"] == o["committed"] and np.array_equal(full[1]["ohash"], o["ohash"])
        with G.Phold(_cfg(queue, mode)) as h2:  # a fresh handle of the same configuration
            h2.restore(snap)
            _same(_finish(h2), full)
        h.restore(snap)  # back into the handle that went on
        _same(_finish(h), full)


@pytest.mark.parametrize("queue,mode", [("laq", 0), ("laq", 2)])
def test_resume_in_the_persistent_loop(gpu_lib, queue, mode):
    with G.Phold(_cfg(queue, mode)) as h:
        h.populate()
        h.step(20)
        snap = h.snapshot()
        full = _finish(h)
    with G.Phold(_cfg(queue, mode, loop="persistent")) as h2:
        with pytest.raises(G.GpqError):  # another configuration (loop mode differs)
            h2.restore(snap)
    with G.Phold(_cfg(queue, mode)) as h3:
        h3.restore(snap)
        h3.run()
        _same((h3.result(), h3.lp_stats()), full)


def test_bad_snapshots_are_refused(gpu_lib):
    with G.Phold(_cfg("laq", 2)) as h:
        h.populate()
        h.step(5)
        snap = h.snapshot()
        with pytest.raises(G.GpqError):
            h.restore(snap[: len(snap) // 2])
        bad = snap.copy()
        bad[0] ^= 1
        with pytest.raises(G.GpqError):
            h.restore(bad)
        with G.Phold(_cfg("laq", 2, seed=43)) as other:
            with pytest.raises(G.GpqError):
                other.restore(snap)
