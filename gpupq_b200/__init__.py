"""gpupq_b200 -- B200-native rebuild of GPUPQ's priority-queue hot path.

Python binding of libgpq.so (ctypes over the C ABI declared in include/gpq.h).  The
compute path is the CUDA library; there is no Python or CPU fallback: importing the
binding succeeds without a GPU, but every call that needs the device fails loudly if
the library is missing or no GPU is present.
"""
import ctypes
import os

import numpy as np

from . import build as _build

__all__ = [
    "GpqError", "ITEM_DTYPE", "PholdConfig", "PholdResult", "Phold", "lib", "presets",
    "QUEUE_LAQ", "QUEUE_GAQ", "QUEUE_HQ", "QUEUE_LHQ", "QUEUE_LSQ", "LOOP_PLAIN", "LOOP_PERSISTENT",
    "DEST_UNIFORM", "DEST_RING", "ring_threshold",
]

QUEUE_LAQ, QUEUE_GAQ, QUEUE_HQ, QUEUE_LHQ, QUEUE_LSQ = range(5)
QUEUE_NAMES = {"laq": QUEUE_LAQ, "gaq": QUEUE_GAQ, "hq": QUEUE_HQ, "lhq": QUEUE_LHQ, "lsq": QUEUE_LSQ}
LOOP_PLAIN, LOOP_PERSISTENT = 0, 1
DEST_UNIFORM, DEST_RING = 0, 1

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "queue full", 4: "insert buffer full",
    5: "device wait timed out", 6: "out of device memory", 7: "unsupported", 8: "not ready",
}

ITEM_DTYPE = np.dtype([("ts", "<f4"), ("lp", "<u4"), ("id", "<u4"), ("aux", "<u4")])


class GpqError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} ({status}) {detail}".strip())


class GpqItem(ctypes.Structure):
    _fields_ = [("ts", ctypes.c_float), ("lp", ctypes.c_uint32), ("id", ctypes.c_uint32), ("aux", ctypes.c_uint32)]


class PholdConfig(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("num_lps", ctypes.c_uint32),
        ("events_per_lp", ctypes.c_uint32),
        ("lookahead", ctypes.c_float),
        ("end_time", ctypes.c_float),
        ("dest_mode", ctypes.c_uint32),
        ("ring_width", ctypes.c_uint32),
        ("ring_threshold", ctypes.c_uint32),
        ("queue_kind", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32),
        ("insert_capacity", ctypes.c_uint32),
        ("loop_mode", ctypes.c_uint32),
        ("block_threads", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("max_steps", ctypes.c_uint32),
        ("lanes_per_lp", ctypes.c_uint32),
        ("node_size", ctypes.c_uint32),
        ("laq_mode", ctypes.c_uint32),
        ("gaq_engine", ctypes.c_uint32),
    ]


class PholdResult(ctypes.Structure):
    _fields_ = [
        ("committed", ctypes.c_uint64),
        ("steps", ctypes.c_uint64),
        ("pending", ctypes.c_uint64),
        ("pending_csum", ctypes.c_uint64),
        ("digest", ctypes.c_uint64),
        ("final_min", ctypes.c_float),
        ("elapsed_ms", ctypes.c_float),
        ("status", ctypes.c_int32),
        ("reserved", ctypes.c_uint32 * 3),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_LIB = None

# Exported symbols and their ctypes signatures (kept in step with include/gpq.h).
_VP = ctypes.c_void_p
_SIGS = {
    "gpq_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "gpq_version": ([], ctypes.c_char_p),
    "gpq_last_error": ([], ctypes.c_char_p),
    "gpq_set_spin_limit": ([ctypes.c_uint64], ctypes.c_int),
    "gpq_phold_create": ([ctypes.POINTER(PholdConfig), ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_phold_destroy": ([_VP], ctypes.c_int),
    "gpq_phold_populate": ([_VP, _VP, ctypes.c_uint64, _VP], ctypes.c_int),
    "gpq_phold_run": ([_VP, _VP], ctypes.c_int),
    "gpq_phold_step": ([_VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int), _VP], ctypes.c_int),
    "gpq_phold_result_get": ([_VP, ctypes.POINTER(PholdResult), _VP], ctypes.c_int),
    "gpq_phold_lp_stats": ([_VP, _VP, _VP, _VP, _VP], ctypes.c_int),
    "gpq_phold_initial_events": ([ctypes.POINTER(PholdConfig), _VP, ctypes.c_uint64], ctypes.c_int),
    "gpq_phold_children": ([ctypes.POINTER(PholdConfig), _VP, _VP, ctypes.c_uint64], ctypes.c_int),
    "gpq_phold_snapshot": ([_VP, _VP, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), _VP], ctypes.c_int),
    "gpq_phold_restore": ([_VP, _VP, ctypes.c_uint64, _VP], ctypes.c_int),
    "gpq_phold_shard_create": ([_VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_VP)],
                               ctypes.c_int),
    "gpq_phold_shard_range": ([_VP, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                              ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_phold_shard_populate": ([_VP, ctypes.POINTER(ctypes.c_float), _VP], ctypes.c_int),
    "gpq_phold_shard_window": ([_VP, ctypes.c_float, ctypes.POINTER(ctypes.c_float), _VP, _VP], ctypes.c_int),
    "gpq_phold_shard_outbox": ([_VP, ctypes.POINTER(_VP), ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_phold_shard_inject": ([_VP, _VP, ctypes.c_uint64, ctypes.c_int, _VP], ctypes.c_int),
    "gpq_phold_shard_connect": ([_VP, _VP, ctypes.c_uint32], ctypes.c_int),
    "gpq_phold_launch_info": ([_VP, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                               ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_phold_run_static": ([ctypes.POINTER(PholdConfig), _VP, _VP, _VP, _VP, ctypes.POINTER(PholdResult), _VP],
                             ctypes.c_int),
    "gpq_astar_ref_create": ([_VP, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_astar_ref_destroy": ([_VP], ctypes.c_int),
    "gpq_astar_ref_solve": ([_VP, _VP, _VP, ctypes.c_uint32, _VP, _VP], ctypes.c_int),
    "gpq_astar_ref_last_ms": ([_VP, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "gpq_astar_ref_map": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_uint64, _VP],
                          ctypes.c_int),
    "gpq_astar_ref_agents": ([_VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _VP],
                             ctypes.c_int),
    "gpq_legacy_configure": ([_VP, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "gpq_legacy_init": ([ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_legacy_queue": ([], _VP),
    "gpq_legacy_pre": ([], ctypes.c_int),
    "gpq_legacy_post": ([], ctypes.c_int),
    "gpq_legacy_get_min_ts": ([], ctypes.c_float),
    "gpq_legacy_counts": ([ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "gpq_legacy_finish": ([], ctypes.c_int),
    "gpq_legacy_status": ([], ctypes.c_int),
    "gpq_host_alloc": ([ctypes.c_uint64, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_host_free": ([_VP], ctypes.c_int),
    "gpq_queue_create": ([ctypes.c_void_p, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_queue_destroy": ([_VP], ctypes.c_int),
    "gpq_queue_insert": ([_VP, _VP, ctypes.c_uint64, ctypes.c_int, _VP], ctypes.c_int),
    "gpq_queue_pre": ([_VP, _VP], ctypes.c_int),
    "gpq_queue_post": ([_VP, _VP], ctypes.c_int),
    "gpq_queue_post_init": ([_VP, _VP], ctypes.c_int),
    "gpq_queue_get_min": ([_VP, ctypes.POINTER(ctypes.c_float), _VP], ctypes.c_int),
    "gpq_queue_dequeue": ([_VP, ctypes.c_float, ctypes.c_uint32, _VP, ctypes.c_uint64,
                           ctypes.POINTER(ctypes.c_uint64), _VP], ctypes.c_int),
    "gpq_queue_length": ([_VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), _VP], ctypes.c_int),
    "gpq_queue_clear": ([_VP, ctypes.c_uint32, _VP], ctypes.c_int),
    "gpq_queue_dump": ([_VP, ctypes.c_uint32, _VP, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), _VP],
                       ctypes.c_int),
    "gpq_queue_counts": ([_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64), _VP],
                         ctypes.c_int),
    "gpq_astar_create": ([_VP, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_astar_destroy": ([_VP], ctypes.c_int),
    "gpq_astar_solve": ([_VP, _VP, ctypes.c_uint32, _VP, _VP], ctypes.c_int),
    "gpq_astar_last_stats": ([_VP, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                              ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64),
                              ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_astar_path": ([_VP, ctypes.c_uint32, _VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), _VP],
                       ctypes.c_int),
    "gpq_astar_gcost": ([_VP, ctypes.c_uint32, _VP, ctypes.c_uint64, _VP], ctypes.c_int),
    "gpq_astar_write_ppm": ([_VP, ctypes.c_uint32, ctypes.c_char_p, _VP], ctypes.c_int),
    "gpq_astar_query": ([ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                         ctypes.c_double, ctypes.c_double, _VP], ctypes.c_int),
    "gpq_astar_session_create": ([_VP, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_VP)],
                                 ctypes.c_int),
    "gpq_astar_session_destroy": ([_VP], ctypes.c_int),
    "gpq_astar_session_admit": ([_VP, _VP, ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_astar_session_step": ([_VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), _VP], ctypes.c_int),
    "gpq_astar_session_collect": ([_VP, _VP, _VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), _VP],
                                  ctypes.c_int),
    "gpq_astar_session_usage": ([_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_astar_session_bytes": ([_VP, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_uint64),
    "gpq_phold_session_create": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_phold_session_create_bucketed": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(_VP)], ctypes.c_int),
    "gpq_phold_session_destroy": ([_VP], ctypes.c_int),
    "gpq_phold_session_admit": ([_VP, ctypes.POINTER(PholdConfig), ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
    "gpq_phold_session_step": ([_VP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), _VP], ctypes.c_int),
    "gpq_phold_session_collect": ([_VP, _VP, ctypes.POINTER(PholdResult), ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_uint32), _VP], ctypes.c_int),
    "gpq_phold_session_snapshot": ([_VP, _VP, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), _VP], ctypes.c_int),
    "gpq_phold_session_restore": ([_VP, _VP, ctypes.c_uint64, _VP], ctypes.c_int),
    "gpq_phold_session_usage": ([_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)],
                                ctypes.c_int),
    "gpq_phold_session_bytes": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32],
                                ctypes.c_uint64),
    "gpq_phold_session_bytes_bucketed": ([ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32],
                                         ctypes.c_uint64),
}


def lib_path():
    return _build.LIB


def lib():
    """Load libgpq.so (building it first if the sources are newer).  Raises if it cannot."""
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not _build.up_to_date():
            try:
                path = _build.build()
            except Exception as e:  # no nvcc on this machine: use the shipped library if any
                if not os.path.exists(path):
                    raise RuntimeError(f"libgpq.so is missing and could not be built: {e}") from e
        L = ctypes.CDLL(path)
        for name, (argtypes, restype) in _SIGS.items():
            f = getattr(L, name, None)
            if f is not None:
                f.argtypes = argtypes
                f.restype = restype
        _LIB = L
    return _LIB


def last_error():
    return lib().gpq_last_error().decode(errors="replace")


def check(status, where):
    if status != 0:
        raise GpqError(status, where, last_error())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def ring_threshold(frac: float) -> int:
    """Probability -> 32-bit threshold floor(frac * 2^32), computed in double."""
    return min(int(frac * 4294967296.0), 0xFFFFFFFF)


def presets():
    """The named workloads (synthetic, seeded).

    phold_plain: 1024 LPs x 16 events, lookahead 1.0, end 100, uniform destinations, seed 42.
    phold_large: 65,536 LPs x 64 events, lookahead 0.1, end 1000, 90% ring +-16 / 10% uniform,
                 per-LP capacity 256, seed 7.
    """
    return {
        "phold_plain": dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42,
                            dest_mode=DEST_UNIFORM, capacity=256, insert_capacity=64),
        "phold_large": dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=1000.0, seed=7,
                            dest_mode=DEST_RING, ring_width=16, ring_frac=0.9, capacity=256,
                            insert_capacity=64),
    }


def make_phold_config(num_lps, events_per_lp, lookahead, end_time, seed, dest_mode=DEST_UNIFORM,
                      ring_width=16, ring_frac=0.9, queue="laq", capacity=256, insert_capacity=64,
                      loop="persistent", block_threads=0, ctas_per_sm=0, max_steps=0, lanes_per_lp=0, node_size=0,
                      laq_mode=0, gaq_engine=0):
    c = PholdConfig()
    c.seed = seed
    c.num_lps = num_lps
    c.events_per_lp = events_per_lp
    c.lookahead = lookahead
    c.end_time = end_time
    c.dest_mode = dest_mode
    c.ring_width = ring_width if dest_mode == DEST_RING else 0
    c.ring_threshold = ring_threshold(ring_frac) if dest_mode == DEST_RING else 0
    c.queue_kind = QUEUE_NAMES[queue] if isinstance(queue, str) else int(queue)
    c.capacity = capacity
    c.insert_capacity = insert_capacity
    c.loop_mode = {"plain": LOOP_PLAIN, "persistent": LOOP_PERSISTENT}[loop] if isinstance(loop, str) else int(loop)
    c.block_threads = block_threads
    c.ctas_per_sm = ctas_per_sm
    c.max_steps = max_steps
    c.lanes_per_lp = lanes_per_lp
    c.node_size = node_size
    c.laq_mode = laq_mode
    c.gaq_engine = gaq_engine
    return c


class Phold:
    """One PHOLD instance on the device (the reference's des_init/des_run/des_finish with
    the PHOLD model, src/des.cu:74-221, src/phold.cu:124-192)."""

    def __init__(self, cfg: PholdConfig):
        self.cfg = cfg
        self._h = ctypes.c_void_p()
        check(lib().gpq_phold_create(ctypes.byref(cfg), ctypes.byref(self._h)), "gpq_phold_create")

    def close(self):
        if self._h:
            lib().gpq_phold_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def populate(self, initial=None, stream=None):
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=ITEM_DTYPE)
            check(lib().gpq_phold_populate(self._h, _ptr(initial), len(initial), stream), "gpq_phold_populate")
        else:
            check(lib().gpq_phold_populate(self._h, None, 0, stream), "gpq_phold_populate")

    def run(self, stream=None):
        check(lib().gpq_phold_run(self._h, stream), "gpq_phold_run")

    def step(self, n, stream=None):
        done = ctypes.c_int(0)
        check(lib().gpq_phold_step(self._h, n, ctypes.byref(done), stream), "gpq_phold_step")
        return bool(done.value)

    def result(self, stream=None):
        r = PholdResult()
        st = lib().gpq_phold_result_get(self._h, ctypes.byref(r), stream)
        d = r.as_dict()
        d["status_code"] = st
        return d

    def snapshot(self, stream=None):
        """The run's whole state between windows (gpq_phold_snapshot) as a uint8 array."""
        n = ctypes.c_uint64()
        check(lib().gpq_phold_snapshot(self._h, None, 0, ctypes.byref(n), stream), "gpq_phold_snapshot")
        buf = np.zeros(n.value, np.uint8)
        check(lib().gpq_phold_snapshot(self._h, _ptr(buf), n.value, ctypes.byref(n), stream), "gpq_phold_snapshot")
        return buf

    def restore(self, buf, stream=None):
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        check(lib().gpq_phold_restore(self._h, _ptr(buf), len(buf), stream), "gpq_phold_restore")

    def launch_info(self):
        g, b, n = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().gpq_phold_launch_info(self._h, ctypes.byref(g), ctypes.byref(b), ctypes.byref(n)),
              "gpq_phold_launch_info")
        return {"grid": g.value, "block": b.value, "launches_per_run": n.value}

    def lp_stats_into(self, count, csum, ohash, stream=None):
        check(lib().gpq_phold_lp_stats(self._h, _ptr(count), _ptr(csum), _ptr(ohash), stream), "gpq_phold_lp_stats")

    def lp_stats(self, stream=None):
        L = self.cfg.num_lps
        count = np.zeros(L, np.uint32)
        csum = np.zeros(L, np.uint64)
        ohash = np.zeros(L, np.uint64)
        check(lib().gpq_phold_lp_stats(self._h, _ptr(count), _ptr(csum), _ptr(ohash), stream), "gpq_phold_lp_stats")
        return {"count": count, "csum": csum, "ohash": ohash}


def initial_events(cfg: PholdConfig):
    n = cfg.num_lps * cfg.events_per_lp
    out = np.zeros(n, ITEM_DTYPE)
    check(lib().gpq_phold_initial_events(ctypes.byref(cfg), _ptr(out), n), "gpq_phold_initial_events")
    return out


def children(cfg: PholdConfig, events):
    events = np.ascontiguousarray(events, dtype=ITEM_DTYPE)
    out = np.zeros(len(events), ITEM_DTYPE)
    check(lib().gpq_phold_children(ctypes.byref(cfg), _ptr(events), _ptr(out), len(events)), "gpq_phold_children")
    return out


class QueueConfig(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("num_lps", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32),
        ("insert_capacity", ctypes.c_uint32),
        ("node_size", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 3),
    ]


class Queue:
    """A queue object (the reference's host queue API, src/queue.h:86-115)."""

    def __init__(self, kind, num_lps, capacity=0, insert_capacity=0, node_size=0):
        c = QueueConfig()
        c.kind = QUEUE_NAMES[kind] if isinstance(kind, str) else int(kind)
        c.num_lps = num_lps
        c.capacity = capacity
        c.insert_capacity = insert_capacity
        c.node_size = node_size
        self.num_lps = num_lps
        self._h = ctypes.c_void_p()
        check(lib().gpq_queue_create(ctypes.byref(c), ctypes.byref(self._h)), "gpq_queue_create")

    def close(self):
        if self._h:
            lib().gpq_queue_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def insert(self, items):
        items = np.ascontiguousarray(items, dtype=ITEM_DTYPE)
        check(lib().gpq_queue_insert(self._h, _ptr(items), len(items), 0, None), "gpq_queue_insert")

    def pre(self):
        check(lib().gpq_queue_pre(self._h, None), "gpq_queue_pre")

    def post(self):
        check(lib().gpq_queue_post(self._h, None), "gpq_queue_post")

    def post_init(self):
        check(lib().gpq_queue_post_init(self._h, None), "gpq_queue_post_init")

    def get_min(self):
        v = ctypes.c_float()
        check(lib().gpq_queue_get_min(self._h, ctypes.byref(v), None), "gpq_queue_get_min")
        return v.value

    def dequeue(self, bound, max_per_lp=0, capacity=None):
        cap = capacity if capacity is not None else 1 << 20
        out = np.zeros(cap, ITEM_DTYPE)
        n = ctypes.c_uint64()
        check(lib().gpq_queue_dequeue(self._h, bound, max_per_lp, _ptr(out), cap, ctypes.byref(n), None),
              "gpq_queue_dequeue")
        return out[: n.value].copy()

    def length(self, lp):
        v = ctypes.c_uint32()
        check(lib().gpq_queue_length(self._h, lp, ctypes.byref(v), None), "gpq_queue_length")
        return v.value

    def clear(self, lp):
        check(lib().gpq_queue_clear(self._h, lp, None), "gpq_queue_clear")

    def dump(self, lp, capacity=1 << 20):
        out = np.zeros(capacity, ITEM_DTYPE)
        n = ctypes.c_uint64()
        check(lib().gpq_queue_dump(self._h, lp, _ptr(out), capacity, ctypes.byref(n), None), "gpq_queue_dump")
        return out[: n.value].copy()

    def counts(self):
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().gpq_queue_counts(self._h, ctypes.byref(a), ctypes.byref(b), None), "gpq_queue_counts")
        return a.value, b.value


class PinnedArray:
    """A numpy array over page-locked host memory (gpq_host_alloc)."""

    def __init__(self, n, dtype):
        dtype = np.dtype(dtype)
        self._p = ctypes.c_void_p()
        check(lib().gpq_host_alloc(n * dtype.itemsize, ctypes.byref(self._p)), "gpq_host_alloc")
        buf = (ctypes.c_char * (n * dtype.itemsize)).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=n)

    def free(self):
        if self._p:
            self.array = None
            lib().gpq_host_free(self._p)
            self._p = ctypes.c_void_p()


# ---- A* grid search (include/gpq/astar.h, gpq_astar_* in include/gpq.h) ----

ASTAR_INF = 0xFFFFFFFF
ASTAR_GRID_DTYPE = np.dtype([("seed", "<u8"), ("width", "<u4"), ("height", "<u4"), ("block_thr", "<u4"),
                             ("conn", "<u4"), ("start", "<u4"), ("goal", "<u4")])
ASTAR_RESULT_DTYPE = np.dtype([("cost", "<u4"), ("path_len", "<u4"), ("expanded", "<u8"), ("gsum", "<u8"),
                               ("path_hash", "<u8"), ("pops", "<u8"), ("windows", "<u4"), ("status", "<i4")])


ASTAR_REF_AGENT_DTYPE = np.dtype([("start", "<u4"), ("goal", "<u4")])
ASTAR_REF_RESULT_DTYPE = np.dtype([("found", "<u4"), ("cost", "<f4"), ("pops", "<u4"), ("rounds", "<u4"),
                                   ("status", "<u4"), ("reserved", "<u4")])


class AstarRefConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("width", "height", "slots", "open_capacity")] + \
        [("reserved", ctypes.c_uint32 * 4)]


def astar_ref_map(width, height, obstacle_frac=0.2, size_mean=1.0, seed=0):
    """The reference's random obstacle map (gpq_astar_ref_map): uint8 [height, width], 1 = wall."""
    m = np.zeros(width * height, np.uint8)
    check(lib().gpq_astar_ref_map(width, height, obstacle_frac, size_mean, seed, _ptr(m)), "gpq_astar_ref_map")
    return m.reshape(height, width)


def astar_ref_agents(map2d, n, seed=0):
    """n agents with random free start and goal cells (gpq_astar_ref_agents)."""
    m = np.ascontiguousarray(map2d, np.uint8)
    out = np.zeros(n, ASTAR_REF_AGENT_DTYPE)
    check(lib().gpq_astar_ref_agents(_ptr(m), m.shape[1], m.shape[0], n, seed, _ptr(out)), "gpq_astar_ref_agents")
    return out


class AStarRef:
    """Reference-semantics A* (gpq_astar_ref_*): the reference's agents (half-precision f,
    eight pops per round, stop at the goal) over a pool of agents on one map."""

    def __init__(self, width, height, slots=0, open_capacity=0):
        c = AstarRefConfig()
        c.width, c.height, c.slots, c.open_capacity = width, height, slots, open_capacity
        self._h = ctypes.c_void_p()
        check(lib().gpq_astar_ref_create(ctypes.byref(c), ctypes.byref(self._h)), "gpq_astar_ref_create")

    def solve(self, map2d, agents):
        m = np.ascontiguousarray(map2d, np.uint8)
        a = np.ascontiguousarray(agents, ASTAR_REF_AGENT_DTYPE)
        out = np.zeros(len(a), ASTAR_REF_RESULT_DTYPE)
        check(lib().gpq_astar_ref_solve(self._h, _ptr(m), _ptr(a), len(a), _ptr(out), None), "gpq_astar_ref_solve")
        return out

    def last_ms(self):
        v = ctypes.c_float()
        check(lib().gpq_astar_ref_last_ms(self._h, ctypes.byref(v)), "gpq_astar_ref_last_ms")
        return v.value

    def close(self):
        if self._h:
            lib().gpq_astar_ref_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AstarConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("tile", "window", "inbox_capacity", "open_capacity",
                                               "frontier_capacity", "block_threads", "ctas_per_sm",
                                               "max_rounds", "tile_worker")] + [("reserved", ctypes.c_uint32 * 3)]


def density_threshold(p: float) -> int:
    """Obstacle density -> the 24-bit threshold of gpq_astar_grid.block_thr."""
    return int(p * 16777216.0)


def astar_grid(width, height, density, seed, conn=4, start=None, goal=None):
    g = np.zeros(1, ASTAR_GRID_DTYPE)
    g[0] = (seed, width, height, density_threshold(density), conn, 0 if start is None else start,
            width * height - 1 if goal is None else goal)
    return g


def astar_queries(base_seed, n, conn, side_lo, side_hi, dens_lo, dens_hi, first=0):
    """Grids of queries first .. first+n-1 of a batch (gpq_astar_query)."""
    out = np.zeros(n, ASTAR_GRID_DTYPE)
    for i in range(n):
        check(lib().gpq_astar_query(base_seed, first + i, conn, side_lo, side_hi, dens_lo, dens_hi,
                                    ctypes.c_void_p(out[i:].ctypes.data)), "gpq_astar_query")
    return out


class AStar:
    """An A* engine handle (gpq_astar_create); solve() runs a batch of grids."""

    def __init__(self, **cfg):
        c = AstarConfig()
        for k, v in cfg.items():
            setattr(c, k, v)
        self._h = ctypes.c_void_p()
        check(lib().gpq_astar_create(ctypes.byref(c), ctypes.byref(self._h)), "gpq_astar_create")

    def close(self):
        if self._h:
            lib().gpq_astar_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, grids, results=None):
        grids = np.ascontiguousarray(grids, ASTAR_GRID_DTYPE)
        if results is None:
            results = np.zeros(len(grids), ASTAR_RESULT_DTYPE)
        check(lib().gpq_astar_solve(self._h, _ptr(grids), len(grids), _ptr(results), None), "gpq_astar_solve")
        return results

    def stats(self):
        t, s = ctypes.c_float(), ctypes.c_float()
        r, g, b = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        v = ctypes.c_uint64()
        check(lib().gpq_astar_last_stats(self._h, ctypes.byref(t), ctypes.byref(s), ctypes.byref(r),
                                         ctypes.byref(v), ctypes.byref(g), ctypes.byref(b)), "gpq_astar_last_stats")
        return {"total_ms": t.value, "search_ms": s.value, "rounds": r.value, "tile_visits": v.value,
                "grid": g.value, "block": b.value}

    def path(self, index, capacity=1 << 20):
        out = np.zeros(capacity, np.uint32)
        n = ctypes.c_uint32()
        check(lib().gpq_astar_path(self._h, index, _ptr(out), capacity, ctypes.byref(n), None), "gpq_astar_path")
        return out[: n.value]

    def gcost(self, index, cells):
        out = np.zeros(cells, np.uint32)
        check(lib().gpq_astar_gcost(self._h, index, _ptr(out), cells, None), "gpq_astar_gcost")
        return out

    def write_ppm(self, index, filename):
        """Binary PPM image of instance `index` of the last solve (gpq_astar_write_ppm)."""
        check(lib().gpq_astar_write_ppm(self._h, index, os.fsencode(filename), None), "gpq_astar_write_ppm")


class AStarSession:
    """Resident A* instances (gpq_astar_session_*): admit, step, collect."""

    def __init__(self, max_cells, max_tiles, max_instances, **cfg):
        c = AstarConfig()
        for k, v in cfg.items():
            setattr(c, k, v)
        self._h = ctypes.c_void_p()
        check(lib().gpq_astar_session_create(ctypes.byref(c), max_cells, max_tiles, max_instances,
                                             ctypes.byref(self._h)), "gpq_astar_session_create")
        self.max_instances = max_instances

    def close(self):
        if self._h:
            lib().gpq_astar_session_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, grid):
        """Slot number, or None when the instance does not fit now."""
        g = np.ascontiguousarray(np.atleast_1d(grid), ASTAR_GRID_DTYPE)
        slot = ctypes.c_uint32()
        st = lib().gpq_astar_session_admit(self._h, _ptr(g), ctypes.byref(slot))
        if st == 6:
            return None
        check(st, "gpq_astar_session_admit")
        return slot.value

    def step(self, rounds=0):
        n = ctypes.c_uint32()
        check(lib().gpq_astar_session_step(self._h, rounds, ctypes.byref(n), None), "gpq_astar_session_step")
        return n.value

    def collect(self):
        slots = np.zeros(self.max_instances, np.uint32)
        res = np.zeros(self.max_instances, ASTAR_RESULT_DTYPE)
        n = ctypes.c_uint32()
        check(lib().gpq_astar_session_collect(self._h, _ptr(slots), _ptr(res), self.max_instances,
                                              ctypes.byref(n), None), "gpq_astar_session_collect")
        return slots[: n.value], res[: n.value]

    def usage(self):
        c, t, i = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        check(lib().gpq_astar_session_usage(self._h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(i)),
              "gpq_astar_session_usage")
        return c.value, t.value, i.value


class PholdSession:
    """Resident PHOLD runs (gpq_phold_session_*): admit, step, collect.

    bucketed=True keeps the LP space as time buckets (gpq_phold_session_create_bucketed,
    `buckets` x `bucket_slots` keys per LP, 0 = 32 x 16) instead of sorted rings
    (capacity, insert_capacity, lanes_per_lp)."""

    def __init__(self, max_lps, max_instances, capacity=256, insert_capacity=64, lanes_per_lp=8, bucketed=False,
                 buckets=0, bucket_slots=0):
        self._h = ctypes.c_void_p()
        if bucketed:
            check(lib().gpq_phold_session_create_bucketed(max_lps, buckets, bucket_slots, max_instances,
                                                          ctypes.byref(self._h)), "gpq_phold_session_create_bucketed")
        else:
            check(lib().gpq_phold_session_create(max_lps, capacity, insert_capacity, max_instances, lanes_per_lp,
                                                 ctypes.byref(self._h)), "gpq_phold_session_create")
        self.max_instances = max_instances

    def close(self):
        if self._h:
            lib().gpq_phold_session_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def admit(self, cfg: PholdConfig):
        slot = ctypes.c_uint32()
        st = lib().gpq_phold_session_admit(self._h, ctypes.byref(cfg), ctypes.byref(slot))
        if st == 6:
            return None
        check(st, "gpq_phold_session_admit")
        return slot.value

    def step(self, windows=0):
        n = ctypes.c_uint32()
        check(lib().gpq_phold_session_step(self._h, windows, ctypes.byref(n), None), "gpq_phold_session_step")
        return n.value

    def collect(self):
        slots = np.zeros(self.max_instances, np.uint32)
        res = (PholdResult * self.max_instances)()
        n = ctypes.c_uint32()
        check(lib().gpq_phold_session_collect(self._h, _ptr(slots), res, self.max_instances, ctypes.byref(n), None),
              "gpq_phold_session_collect")
        return [(int(slots[j]), res[j]) for j in range(n.value)]

    def usage(self):
        a, b = ctypes.c_uint64(), ctypes.c_uint32()
        check(lib().gpq_phold_session_usage(self._h, ctypes.byref(a), ctypes.byref(b)), "gpq_phold_session_usage")
        return a.value, b.value

    def snapshot(self):
        """The whole session's state between steps (gpq_phold_session_snapshot) as a uint8 array."""
        n = ctypes.c_uint64()
        check(lib().gpq_phold_session_snapshot(self._h, None, 0, ctypes.byref(n), None), "gpq_phold_session_snapshot")
        buf = np.zeros(n.value, np.uint8)
        check(lib().gpq_phold_session_snapshot(self._h, _ptr(buf), n.value, ctypes.byref(n), None),
              "gpq_phold_session_snapshot")
        return buf

    def restore(self, buf):
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        check(lib().gpq_phold_session_restore(self._h, _ptr(buf), len(buf), None), "gpq_phold_session_restore")


# ---- serving (gpq_serve_* in include/gpq.h) ----

REQ_ASTAR, REQ_PHOLD = 0, 1
SERVE_BATCHED, SERVE_PLAIN = 0, 1


class AstarGridC(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64)] + [(n, ctypes.c_uint32) for n in
                                              ("width", "height", "block_thr", "conn", "start", "goal")]


class AstarResultC(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_uint32), ("path_len", ctypes.c_uint32), ("expanded", ctypes.c_uint64),
                ("gsum", ctypes.c_uint64), ("path_hash", ctypes.c_uint64), ("pops", ctypes.c_uint64),
                ("windows", ctypes.c_uint32), ("status", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeRequest(ctypes.Structure):
    _fields_ = [("arrival", ctypes.c_double), ("kind", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("astar", AstarGridC), ("phold", PholdConfig)]


class ServeResponse(ctypes.Structure):
    _fields_ = [("admitted", ctypes.c_double), ("finished", ctypes.c_double), ("status", ctypes.c_int32),
                ("reserved", ctypes.c_uint32), ("astar", AstarResultC), ("phold", PholdResult)]


class ServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("mode", ctypes.c_uint32), ("realtime", ctypes.c_uint32),
                ("astar_rounds", ctypes.c_uint32), ("phold_windows", ctypes.c_uint32),
                ("astar_share", ctypes.c_double), ("astar", AstarConfig), ("phold_capacity", ctypes.c_uint32),
                ("phold_insert_capacity", ctypes.c_uint32), ("phold_lanes_per_lp", ctypes.c_uint32),
                ("phold_form", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 4)]


class ServeStats(ctypes.Structure):
    _fields_ = [("makespan", ctypes.c_double), ("throughput", ctypes.c_double), ("p50", ctypes.c_double),
                ("p99", ctypes.c_double), ("p999", ctypes.c_double), ("steps", ctypes.c_uint64),
                ("max_resident", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_SIGS.update({
    "gpq_serve_run": ([ctypes.POINTER(ServeConfig), _VP, ctypes.c_uint32, _VP, ctypes.POINTER(ServeStats)],
                      ctypes.c_int),
    "gpq_serve_stream": ([ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double, _VP,
                          ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
})


def serve_stream(seed, rate, duration, astar_fraction=0.8):
    """The mixed request stream (gpq_serve_stream) as a ctypes array."""
    n = ctypes.c_uint32()
    check(lib().gpq_serve_stream(seed, rate, duration, astar_fraction, None, 0, ctypes.byref(n)), "gpq_serve_stream")
    reqs = (ServeRequest * max(n.value, 1))()
    check(lib().gpq_serve_stream(seed, rate, duration, astar_fraction, ctypes.cast(reqs, ctypes.c_void_p), n.value,
                                 ctypes.byref(n)), "gpq_serve_stream")
    return reqs, n.value


def serve(reqs, n, mode=SERVE_BATCHED, budget=0, realtime=True, astar_rounds=0, phold_windows=0, astar_share=0.0,
          phold_form=0, **astar_cfg):
    """Run gpq_serve_run; returns (responses, stats dict).  phold_form 0 keeps the PHOLD
    runs in sorted rings, 1 in time buckets."""
    c = ServeConfig()
    c.phold_form = phold_form
    c.hbm_budget = budget
    c.astar_share = astar_share
    c.mode = mode
    c.realtime = 1 if realtime else 0
    c.astar_rounds = astar_rounds
    c.phold_windows = phold_windows
    for k, v in astar_cfg.items():
        setattr(c.astar, k, v)
    out = (ServeResponse * max(n, 1))()
    st = ServeStats()
    check(lib().gpq_serve_run(ctypes.byref(c), ctypes.cast(reqs, ctypes.c_void_p), n,
                              ctypes.cast(out, ctypes.c_void_p), ctypes.byref(st)), "gpq_serve_run")
    return out, st.as_dict()
