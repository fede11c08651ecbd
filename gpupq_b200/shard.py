"""Sharded PHOLD: one run's LP space split across GPUs (gpq_phold_shard_* in include/gpq.h).

Each shard (one per rank, or several in one process) holds a contiguous LP range and runs
its safe events on its GPU; between windows the host exchanges the two things a window
needs from the other shards:

* the window minimum: every shard's local minimum (its pending events and all the
  children it made, handed over or not), reduced with MIN;
* the children for other shards' LPs: each shard's outbox, [world][capacity] device items
  with a count per destination, sent with one all-to-all of variable sizes and injected
  into the receiving shard's insert buffers before its next window.

A child is never safe in its parent's window, so the exchange between windows leaves every
result as the unsharded run has it: committed counts, pending events and digests add up,
final minima take the minimum, and every shard runs the same windows.

`run_distributed` drives one shard per rank over torch.distributed: with NCCL the outbox
slices and the received items stay in device memory (the outbox is viewed as a CUDA tensor
through __cuda_array_interface__); with gloo they go through host memory.  `run_local`
drives several shards of one process (on one GPU or several) with the same protocol and an
in-process exchange.  Both take any engine with the methods of `PholdShard`.
"""
import ctypes

import numpy as np

from . import PholdResult, _ptr, check, lib

ITEM_WORDS = 4  # gpq_item: ts (f32 bits), lp, id, aux


class _DeviceView:
    """A device buffer as a CUDA array (int32 words), for torch.as_tensor."""

    def __init__(self, ptr, words):
        self.__cuda_array_interface__ = {"shape": (words,), "typestr": "<i4", "data": (ptr, False),
                                         "version": 3, "strides": None}


class PholdShard:
    """One shard of a PHOLD run (gpq_phold_shard_create): LPs [lp_begin, lp_end)."""

    def __init__(self, cfg, rank, world, outbox_capacity=0):
        self.cfg, self.rank, self.world = cfg, rank, world
        self._h = ctypes.c_void_p()
        check(lib().gpq_phold_shard_create(ctypes.byref(cfg), rank, world, outbox_capacity, ctypes.byref(self._h)),
              "gpq_phold_shard_create")
        b, e, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().gpq_phold_shard_range(self._h, ctypes.byref(b), ctypes.byref(e), ctypes.byref(c)),
              "gpq_phold_shard_range")
        self.lp_begin, self.lp_end, self.capacity = b.value, e.value, c.value
        p = ctypes.c_void_p()
        check(lib().gpq_phold_shard_outbox(self._h, ctypes.byref(p), None), "gpq_phold_shard_outbox")
        self._outbox_ptr = p.value
        self._outbox = None

    def close(self):
        if self._h:
            lib().gpq_phold_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def populate(self):
        m = ctypes.c_float()
        check(lib().gpq_phold_shard_populate(self._h, ctypes.byref(m), None), "gpq_phold_shard_populate")
        return m.value

    def window(self, global_min):
        """Run one window; returns (local minimum, children per destination shard)."""
        m = ctypes.c_float()
        counts = np.zeros(self.world, np.uint32)
        check(lib().gpq_phold_shard_window(self._h, ctypes.c_float(global_min), ctypes.byref(m), _ptr(counts), None),
              "gpq_phold_shard_window")
        return m.value, counts

    def outbox(self, counts, device):
        """The outbox slices as int32 tensors [n, 4], one per destination: views of device
        memory for a CUDA device, host copies for the CPU."""
        import torch
        if self._outbox is None:
            words = self.world * self.capacity * ITEM_WORDS
            self._outbox = torch.as_tensor(_DeviceView(self._outbox_ptr, words), device="cuda").view(
                self.world, self.capacity, ITEM_WORDS)
        out = [self._outbox[d, :int(counts[d])] for d in range(self.world)]
        if torch.device(device).type == "cpu":
            out = [t.cpu() for t in out]
        return out

    def inject(self, items):
        """Hand items (an int32 tensor [n, 4], on the device or the host) to this shard."""
        n = int(items.shape[0])
        if n == 0:
            return
        items = items.contiguous()
        on_device = 1 if items.is_cuda else 0
        if on_device:  # torch's stream made them (cat, all-to-all); the library reads them on its own
            import torch
            torch.cuda.current_stream().synchronize()
        check(lib().gpq_phold_shard_inject(self._h, ctypes.c_void_p(items.data_ptr()), n, on_device, None),
              "gpq_phold_shard_inject")

    def result(self):
        r = PholdResult()
        check(lib().gpq_phold_result_get(self._h, ctypes.byref(r), None), "gpq_phold_result_get")
        return r.as_dict()


def combine(parts):
    """The run's result from its shards' parts: sums modulo 2^64, minimum of the final
    minima; every shard ran the same windows."""
    mask = (1 << 64) - 1
    out = {}
    for k in ("committed", "pending", "pending_csum", "digest"):
        out[k] = sum(int(p[k]) for p in parts) & mask
    out["final_min"] = min(float(p["final_min"]) for p in parts)
    steps = {int(p["steps"]) for p in parts}
    if len(steps) != 1:
        raise RuntimeError(f"shards ran different windows: {sorted(steps)}")
    out["steps"] = steps.pop()
    out["status"] = max(int(p["status"]) for p in parts)
    return out


def connect(shards):
    """Direct hand-over between the bucketed local array queue's shards of one process
    (gpq_phold_shard_connect): a child for another shard's LP is filed straight into that
    shard's buckets by the window that makes it, so windows need no exchange -- only the
    minimum over shards."""
    arr = (ctypes.c_void_p * len(shards))(*[s._h.value for s in shards])
    for s in shards:
        check(lib().gpq_phold_shard_connect(s._h, ctypes.cast(arr, ctypes.c_void_p), len(shards)),
              "gpq_phold_shard_connect")


def run_local_direct(shards, end_time):
    """Drive connected shards of one process (see connect) to the end of the run: per
    window every shard runs with the global minimum, then the minimum over the shards'
    local minima; returns the combined result."""
    m = min(s.populate() for s in shards)
    while m < end_time:
        m = min(s.window(m)[0] for s in shards)
    return combine([s.result() for s in shards])


def run_local(shards, end_time):
    """Drive the shards of one process (shard r at position r) to the end of the run;
    returns the combined result."""
    import torch
    m = min(s.populate() for s in shards)
    while m < end_time:
        mins, sends = [], []
        for s in shards:
            lm, counts = s.window(m)
            mins.append(lm)
            sends.append(s.outbox(counts, "cuda" if torch.cuda.is_available() else "cpu"))
        for d, s in enumerate(shards):
            got = [sends[r][d] for r in range(len(shards)) if r != d and sends[r][d].shape[0]]
            if got:
                s.inject(torch.cat(got))
        m = min(mins)
    return combine([s.result() for s in shards])


def _alltoallv(send, device, group):
    """Variable-size all-to-all of int32 [n, 4] tensors; returns the received items
    (all sources, in rank order) as one tensor."""
    import torch
    import torch.distributed as dist
    n_send = torch.tensor([t.shape[0] for t in send], dtype=torch.int64, device=device)
    n_recv = torch.empty_like(n_send)
    dist.all_to_all_single(n_recv, n_send, group=group)
    inp = torch.cat([t.to(device) for t in send]) if send else torch.empty((0, ITEM_WORDS), dtype=torch.int32)
    out = torch.empty((int(n_recv.sum().item()), ITEM_WORDS), dtype=torch.int32, device=device)
    dist.all_to_all_single(out, inp, output_split_sizes=n_recv.tolist(), input_split_sizes=n_send.tolist(),
                           group=group)
    return out


def run_distributed(shard, end_time, group=None):
    """Drive this rank's shard over torch.distributed (every rank calls it with its own
    shard); returns the combined result on every rank."""
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    m_t = torch.tensor([shard.populate()], dtype=torch.float32, device=device)
    dist.all_reduce(m_t, op=dist.ReduceOp.MIN, group=group)
    m = float(m_t.item())
    while m < end_time:
        lm, counts = shard.window(m)
        got = _alltoallv(shard.outbox(counts, device), device, group)
        shard.inject(got)
        m_t.fill_(lm)
        dist.all_reduce(m_t, op=dist.ReduceOp.MIN, group=group)
        m = float(m_t.item())
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, shard.result(), group=group)
    return combine(parts)
