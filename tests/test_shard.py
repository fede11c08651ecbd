"""Sharded PHOLD (gpupq_b200.shard, gpq_phold_shard_*).

CPU: the exchange protocol (window minimum by MIN all-reduce, children handed over by a
variable-size all-to-all, injected before the next window) over gloo with 2 and 3 ranks,
each rank's shard an oracle-backed stand-in for the device shard (same methods, per-LP
heaps, the oracle's event function); the per-LP outputs, pending events and window count
must equal the unsharded oracle run exactly.  GPU: real device shards, several in one
process on one GPU (run_local) and two gloo ranks sharing the GPU (run_distributed; their
kernels never wait on each other, the host exchanges between windows), against the
single-run engine."""
import heapq
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

MASK = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15


def _mix(z):
    z &= MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def _bits(t):
    return int(np.float32(t).view(np.uint32))


class OracleShard:
    """LPs [b, e) of the run on the host: per-LP heaps keyed (ts bits, id), a window takes
    every event below min(m + lookahead, end time) in key order (include/gpq/model.h), the
    children come from the oracle's event function."""

    def __init__(self, ocfg, rank, world):
        L = ocfg.num_lps
        self.P = -(-L // world)
        self.b, self.e = min(L, rank * self.P), min(L, rank * self.P + self.P)
        self.cfg, self.rank, self.world = ocfg, rank, world
        self.q = {lp: [] for lp in range(self.b, self.e)}
        self.count = {lp: 0 for lp in self.q}
        self.csum = {lp: 0 for lp in self.q}
        self.ohash = {lp: 0 for lp in self.q}
        self.steps = 0
        self._out = None

    def _push(self, ts, lp, eid):
        heapq.heappush(self.q[lp], (_bits(ts), int(eid), np.float32(ts)))

    def _min(self):
        heads = [h[0][2] for h in self.q.values() if h]
        return float(min(heads)) if heads else float("inf")

    def populate(self):
        ts, lp, ids = O.initial(self.cfg)
        for t, l, i in zip(ts, lp, ids):
            if self.b <= l < self.e:
                self._push(t, int(l), i)
        return self._min()

    def window(self, m):
        bound = np.float32(np.float32(m) + np.float32(self.cfg.lookahead))
        end = np.float32(self.cfg.end_time)
        evs = []
        for lp in range(self.b, self.e):
            h = self.q[lp]
            while h and h[0][2] < bound and h[0][2] < end:
                tb, eid, t = heapq.heappop(h)
                hs = _mix((eid << 32) | tb)
                seq = self.count[lp]
                self.count[lp] = seq + 1
                self.csum[lp] = (self.csum[lp] + hs) & MASK
                self.ohash[lp] = (self.ohash[lp] + _mix(hs + seq * GOLDEN)) & MASK
                evs.append((t, lp, eid))
        out = [[] for _ in range(self.world)]
        lm = float("inf")
        if evs:
            cts, clps = O.child(self.cfg, [e[0] for e in evs], [e[1] for e in evs], [e[2] for e in evs])
            for (t, lp, eid), ct, cl in zip(evs, cts, clps):
                lm = min(lm, float(ct))
                dest = int(cl) // self.P
                if dest == self.rank:
                    self._push(ct, int(cl), eid)
                else:
                    out[dest].append((_bits(ct), int(cl), eid, lp))
        self.steps += 1
        self._out = out
        return min(lm, self._min()), np.array([len(o) for o in out], np.uint32)

    def outbox(self, counts, device):
        return [torch.tensor(np.array(o, np.uint32).reshape(-1, 4).view(np.int32), dtype=torch.int32)
                for o in self._out]

    def inject(self, items):
        for row in items.cpu().numpy().view(np.uint32).reshape(-1, 4):
            assert self.b <= row[1] < self.e
            self._push(np.uint32(row[0]).view(np.float32), int(row[1]), int(row[2]))

    def per_lp(self):
        return {lp: (self.count[lp], self.csum[lp], self.ohash[lp]) for lp in self.q}

    def result(self):
        pend = [(t, eid) for h in self.q.values() for (_, eid, t) in h]
        dig = 0
        for lp in self.q:
            lph = (_mix(_mix((lp << 32) | self.count[lp]) ^ self.csum[lp]) + self.ohash[lp]) & MASK
            dig = (dig + _mix(lph)) & MASK
        return {"committed": sum(self.count.values()), "pending": len(pend),
                "pending_csum": sum(_mix((eid << 32) | _bits(t)) for t, eid in pend) & MASK, "digest": dig,
                "final_min": self._min(), "steps": self.steps, "status": 0}


CASES = [dict(num_lps=64, events_per_lp=4, lookahead=0.5, end_time=20.0, seed=11, dest_mode=0),
         dict(num_lps=50, events_per_lp=2, lookahead=1.0, end_time=30.0, seed=12, dest_mode=1, ring_width=8)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_worker(rank, world, port, case, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from gpupq_b200 import shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sh = OracleShard(O.make_cfg(**case), rank, world)
        res = S.run_distributed(sh, case["end_time"])
        lps = [None] * world
        dist.all_gather_object(lps, sh.per_lp())
        if rank == 0:
            merged = {}
            for d in lps:
                merged.update(d)
            q.put((res, merged))
    finally:
        dist.destroy_process_group()


def _check_vs_oracle(case, res, per_lp):
    want = O.phold(O.make_cfg(**case), threads=1)
    L = case["num_lps"]
    assert sorted(per_lp) == list(range(L))
    assert [per_lp[lp][0] for lp in range(L)] == want["count"].tolist()
    assert [per_lp[lp][1] for lp in range(L)] == want["csum"].tolist()
    assert [per_lp[lp][2] for lp in range(L)] == want["ohash"].tolist()
    assert res["committed"] == want["committed"] and res["pending"] == want["pending"]
    assert res["pending_csum"] == want["pending_csum"] and res["steps"] == want["steps"]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_gloo_ranks_match_the_unsharded_oracle(world, case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_worker, args=(r, world, port, CASES[case], q)) for r in range(world)]
    for p in procs:
        p.start()
    res, per_lp = q.get(timeout=180)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    _check_vs_oracle(CASES[case], res, per_lp)


@pytest.mark.parametrize("world", [1, 4])
def test_local_driver_matches_the_unsharded_oracle(world):
    from gpupq_b200 import shard as S
    case = CASES[0]
    shards = [OracleShard(O.make_cfg(**case), r, world) for r in range(world)]
    res = S.run_local(shards, case["end_time"])
    per_lp = {}
    for s in shards:
        per_lp.update(s.per_lp())
    _check_vs_oracle(case, res, per_lp)


def test_combine_checks_window_counts():
    from gpupq_b200 import shard as S
    a = dict(committed=1, pending=2, pending_csum=(1 << 64) - 1, digest=5, final_min=3.0, steps=7, status=0)
    b = dict(committed=4, pending=1, pending_csum=2, digest=6, final_min=2.5, steps=7, status=0)
    c = S.combine([a, b])
    assert c["committed"] == 5 and c["pending_csum"] == 1 and c["final_min"] == 2.5 and c["steps"] == 7
    with pytest.raises(RuntimeError):
        S.combine([a, dict(b, steps=8)])


# ---- device shards ----

GPU_CASES = [dict(num_lps=3000, events_per_lp=8, lookahead=0.5, end_time=40.0, seed=21, dest_mode=0),
             dict(num_lps=4096, events_per_lp=16, lookahead=0.1, end_time=10.0, seed=22, dest_mode=1),
             dict(num_lps=1000, events_per_lp=4, lookahead=1.0, end_time=60.0, seed=23, dest_mode=1, ring_width=4)]


def _gpu_cfg(case, queue):
    import gpupq_b200 as G
    laq_mode = 0
    if queue == "laqb":  # the local array queue's bucketed form
        queue, laq_mode = "laq", 2
    return G.make_phold_config(case["num_lps"], case["events_per_lp"], case["lookahead"], case["end_time"],
                               case["seed"], dest_mode=case["dest_mode"], ring_width=case.get("ring_width", 16),
                               queue=queue, capacity=256, insert_capacity=64, loop="plain", laq_mode=laq_mode)


def _alone(case, queue):
    import gpupq_b200 as G
    with G.Phold(_gpu_cfg(case, queue)) as h:
        h.populate()
        h.run()
        return h.result()


KEYS = ("committed", "steps", "pending", "pending_csum", "digest", "final_min")
ORACLE_KEYS = ("committed", "steps", "pending", "pending_csum", "digest")
_ORACLE_RUNS = {}


def _oracle_run(case):
    """The unsharded CPU oracle of a GPU case (the checker for the sharded device runs)."""
    key = tuple(sorted(case.items()))
    if key not in _ORACLE_RUNS:
        _ORACLE_RUNS[key] = O.phold(O.make_cfg(**case), threads=4)
    return _ORACLE_RUNS[key]


def _assert_oracle(res, case):
    want = _oracle_run(case)
    for k in ORACLE_KEYS:
        assert res[k] == want[k], (k, res[k], want[k])


@pytest.mark.gpu
@pytest.mark.parametrize("queue", ["laq", "laqb", "lhq", "lsq"])
@pytest.mark.parametrize("world", [1, 2, 3])
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_device_shards_in_one_process(gpu_lib, case, world, queue):
    from gpupq_b200 import shard as S
    c = GPU_CASES[case]
    shards = [S.PholdShard(_gpu_cfg(c, queue), r, world) for r in range(world)]
    try:
        res = S.run_local(shards, c["end_time"])
    finally:
        for s in shards:
            s.close()
    want = _alone(c, queue)
    for k in KEYS:
        assert res[k] == want[k], (k, res[k], want[k])
    assert res["status"] == 0
    _assert_oracle(res, c)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_device_shards_direct_hand_over(gpu_lib, case, world):
    """Bucketed shards connected for direct hand-over: children are filed straight into the
    destination shard's buckets by the window that makes them; no exchange between windows."""
    from gpupq_b200 import shard as S
    c = GPU_CASES[case]
    shards = [S.PholdShard(_gpu_cfg(c, "laqb"), r, world) for r in range(world)]
    try:
        S.connect(shards)
        res = S.run_local_direct(shards, c["end_time"])
    finally:
        for s in shards:
            s.close()
    want = _alone(c, "laqb")
    for k in KEYS:
        assert res[k] == want[k], (k, res[k], want[k])
    assert res["status"] == 0
    _assert_oracle(res, c)


@pytest.mark.gpu
def test_direct_hand_over_refuses_other_forms(gpu_lib):
    import ctypes
    import gpupq_b200 as G
    from gpupq_b200 import shard as S
    shards = [S.PholdShard(_gpu_cfg(GPU_CASES[0], "laq"), r, 2) for r in range(2)]
    try:
        arr = (ctypes.c_void_p * 2)(*[s._h.value for s in shards])
        assert G.lib().gpq_phold_shard_connect(shards[0]._h, ctypes.cast(arr, ctypes.c_void_p), 2) == 1
    finally:
        for s in shards:
            s.close()


def _device_worker(rank, world, port, case, q, queue="laq"):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from gpupq_b200 import shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        with S.PholdShard(_gpu_cfg(case, queue), rank, world) as sh:
            res = S.run_distributed(sh, case["end_time"])
        if rank == 0:
            q.put(res)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("queue", ["laq", "laqb"])
def test_device_shards_over_gloo(gpu_lib, queue):
    c = GPU_CASES[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_device_worker, args=(r, 2, port, c, q, queue)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    want = _alone(c, queue)
    for k in KEYS:
        assert res[k] == want[k], (k, res[k], want[k])
    _assert_oracle(res, c)


@pytest.mark.gpu
def test_shard_handle_refuses_whole_runs(gpu_lib):
    """A shard handle has no exchange of its own: gpq_phold_run / gpq_phold_step refuse it."""
    import ctypes
    import gpupq_b200 as G
    from gpupq_b200 import shard as S
    with S.PholdShard(_gpu_cfg(GPU_CASES[0], "laq"), 1, 2) as sh:
        sh.populate()
        assert G.lib().gpq_phold_run(sh._h, None) == 1
        assert G.lib().gpq_phold_step(sh._h, 1, ctypes.byref(ctypes.c_int()), None) == 1


@pytest.mark.gpu
def test_outbox_overflow_is_reported(gpu_lib):
    import gpupq_b200 as G
    from gpupq_b200 import shard as S
    c = GPU_CASES[0]
    with S.PholdShard(_gpu_cfg(c, "laq"), 0, 2, outbox_capacity=1) as sh:
        m = sh.populate()
        with pytest.raises(G.GpqError):
            sh.window(m)
