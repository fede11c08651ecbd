"""The multi-GPU bench path on CPU: two gloo ranks reduce their device times and event
counts the way `bench.py --gpus 2` does under torchrun (max of times, sum of events),
and each rank runs its own replica seed.  The bench runs replicas (every rank a whole
instance); one run sharded across ranks, with its per-window exchange, is tested in
test_shard.py."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev_ms = 100.0 + 10.0 * rank          # each rank's device time
        events = 1000.0 * (rank + 1)          # each rank's committed events
        mx = bench.reduce_over_ranks(dist, dev_ms, "max", "cpu")
        sm = bench.reduce_over_ranks(dist, events, "sum", "cpu")
        q.put((rank, mx, sm, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, mx, sm, seed in out:
        assert mx == 110.0 and sm == 3000.0
    assert [seed for *_, seed in out] == [7, 8]


def test_no_group_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(None, 5.0, "max", "cpu") == 5.0
