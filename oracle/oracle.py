"""ctypes wrapper of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the
gpupq_b200 product.  See oracle/phold_oracle.cpp for what is restated from the reference.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_LIB = None


class OraclePholdCfg(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("num_lps", ctypes.c_uint32),
        ("events_per_lp", ctypes.c_uint32),
        ("dest_mode", ctypes.c_uint32),
        ("ring_width", ctypes.c_uint32),
        ("ring_threshold", ctypes.c_uint32),
        ("lookahead", ctypes.c_float),
        ("end_time", ctypes.c_float),
    ]


class OraclePholdSummary(ctypes.Structure):
    _fields_ = [
        ("committed", ctypes.c_uint64),
        ("steps", ctypes.c_uint64),
        ("pending", ctypes.c_uint64),
        ("pending_csum", ctypes.c_uint64),
        ("seconds", ctypes.c_double),
    ]


class OracleAstarGrid(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64)] + [(n, ctypes.c_uint32) for n in
                                              ("width", "height", "block_thr", "conn", "start", "goal")]


class OracleAstarResult(ctypes.Structure):
    _fields_ = [("cost", ctypes.c_uint32), ("path_len", ctypes.c_uint32), ("expanded", ctypes.c_uint64),
                ("gsum", ctypes.c_uint64), ("path_hash", ctypes.c_uint64), ("pops", ctypes.c_uint64),
                ("seconds", ctypes.c_double)]


def lib():
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        _LIB = ctypes.CDLL(path)
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        _LIB.oracle_phold_seq.argtypes = [ctypes.POINTER(OraclePholdCfg), u32p, u64p, u64p,
                                          ctypes.POINTER(OraclePholdSummary)]
        _LIB.oracle_phold_window.argtypes = [ctypes.POINTER(OraclePholdCfg), ctypes.c_int, u32p, u64p,
                                             u64p, ctypes.POINTER(OraclePholdSummary)]
        _LIB.oracle_phold_one_per_lp.argtypes = [ctypes.POINTER(OraclePholdCfg), u32p, u64p, u64p,
                                                 ctypes.POINTER(OraclePholdSummary)]
        _LIB.oracle_phold_digest.argtypes = [ctypes.c_uint32, u32p, u64p, u64p]
        _LIB.oracle_phold_digest.restype = ctypes.c_uint64
        _LIB.oracle_phold_child.argtypes = [ctypes.POINTER(OraclePholdCfg), f32p, u32p, u32p,
                                            ctypes.c_uint64, f32p, u32p]
        _LIB.oracle_phold_initial.argtypes = [ctypes.POINTER(OraclePholdCfg), f32p, u32p, u32p]
        _LIB.oracle_logf.argtypes = [ctypes.c_float]
        _LIB.oracle_logf.restype = ctypes.c_float
        _LIB.oracle_ring_search.argtypes = [i64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64]
        _LIB.oracle_ring_search.restype = ctypes.c_int
        _LIB.oracle_ring_insert_sorted.argtypes = [i64p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int64]
        _LIB.oracle_ring_quicksort.argtypes = [i64p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _LIB.oracle_astar_query.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                            ctypes.POINTER(OracleAstarGrid)]
        _LIB.oracle_astar_solve.argtypes = [ctypes.POINTER(OracleAstarGrid), ctypes.POINTER(OracleAstarResult),
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32]
        _LIB.oracle_astar_solve.restype = ctypes.c_int
        _LIB.oracle_astar_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                            ctypes.c_void_p]
        _LIB.oracle_astar_batch.restype = ctypes.c_double
        _LIB.oracle_astar_ref_run.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p]
        _LIB.oracle_astar_ref_run.restype = ctypes.c_double
        _LIB.oracle_to_half.argtypes = [ctypes.c_float]
        _LIB.oracle_to_half.restype = ctypes.c_float
        _LIB.oracle_half_bits.argtypes = [ctypes.c_float]
        _LIB.oracle_half_bits.restype = ctypes.c_uint32
        _LIB.oracle_astar_ref_h.argtypes = [ctypes.c_int] * 4
        _LIB.oracle_astar_ref_h.restype = ctypes.c_float
    return _LIB


def ring_threshold(frac: float) -> int:
    """Probability -> 32-bit threshold (floor(frac * 2^32)), computed in double."""
    return min(int(frac * 4294967296.0), 0xFFFFFFFF)


def make_cfg(num_lps, events_per_lp, lookahead, end_time, seed, dest_mode=0, ring_width=16, ring_frac=0.9):
    c = OraclePholdCfg()
    c.seed = seed
    c.num_lps = num_lps
    c.events_per_lp = events_per_lp
    c.dest_mode = dest_mode
    c.ring_width = ring_width
    c.ring_threshold = ring_threshold(ring_frac) if dest_mode == 1 else 0
    c.lookahead = lookahead
    c.end_time = end_time
    return c


def phold(cfg, threads=0, one_per_lp=False):
    """Run the oracle. threads=0: sequential global priority queue; >=1: windowed per-LP
    driver; one_per_lp: the reference's schedule (one event per LP per window; its window
    count is the reference loop's)."""
    L = cfg.num_lps
    count = np.zeros(L, np.uint32)
    csum = np.zeros(L, np.uint64)
    ohash = np.zeros(L, np.uint64)
    s = OraclePholdSummary()
    if one_per_lp:
        rc = lib().oracle_phold_one_per_lp(ctypes.byref(cfg), count, csum, ohash, ctypes.byref(s))
    elif threads == 0:
        rc = lib().oracle_phold_seq(ctypes.byref(cfg), count, csum, ohash, ctypes.byref(s))
    else:
        rc = lib().oracle_phold_window(ctypes.byref(cfg), threads, count, csum, ohash, ctypes.byref(s))
    if rc != 0:
        raise RuntimeError("oracle failed")
    return {
        "count": count, "csum": csum, "ohash": ohash,
        "committed": int(s.committed), "steps": int(s.steps), "pending": int(s.pending),
        "pending_csum": int(s.pending_csum), "seconds": float(s.seconds),
        "digest": digest(count, csum, ohash),
    }


def digest(count, csum, ohash):
    """The GPU engine's order-sensitive digest over per-LP outputs."""
    count = np.ascontiguousarray(count, np.uint32)
    csum = np.ascontiguousarray(csum, np.uint64)
    ohash = np.ascontiguousarray(ohash, np.uint64)
    return int(lib().oracle_phold_digest(len(count), count, csum, ohash))


def lp_sha256(count, csum, ohash):
    """sha256 over the per-LP arrays (count u32, csum u64, ohash u64; little endian)."""
    import hashlib
    h = hashlib.sha256()
    for a, dt in ((count, "<u4"), (csum, "<u8"), (ohash, "<u8")):
        h.update(np.ascontiguousarray(a).astype(dt).tobytes())
    return h.hexdigest()


def child(cfg, ts, lp, ids):
    ts = np.ascontiguousarray(ts, np.float32)
    lp = np.ascontiguousarray(lp, np.uint32)
    ids = np.ascontiguousarray(ids, np.uint32)
    out_ts = np.zeros_like(ts)
    out_lp = np.zeros_like(lp)
    lib().oracle_phold_child(ctypes.byref(cfg), ts, lp, ids, len(ts), out_ts, out_lp)
    return out_ts, out_lp


def initial(cfg):
    n = cfg.num_lps * cfg.events_per_lp
    ts = np.zeros(n, np.float32)
    lp = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    lib().oracle_phold_initial(ctypes.byref(cfg), ts, lp, ids)
    return ts, lp, ids


def logf(x):
    return lib().oracle_logf(float(x))


ASTAR_FIELDS = ("seed", "width", "height", "block_thr", "conn", "start", "goal")


def _astar_grid(g):
    o = OracleAstarGrid()
    for k in ASTAR_FIELDS:
        setattr(o, k, int(g[k]))
    return o


def astar_query(base_seed, index, conn, side_lo, side_hi, dens_lo, dens_hi):
    o = OracleAstarGrid()
    lib().oracle_astar_query(base_seed, index, conn, side_lo, side_hi, dens_lo, dens_hi, ctypes.byref(o))
    return {k: getattr(o, k) for k in ASTAR_FIELDS}


def astar(grid, want_g=False, want_path=False):
    """Solve one grid (a mapping with the gpq_astar_grid fields) sequentially."""
    o = _astar_grid(grid)
    r = OracleAstarResult()
    cells = o.width * o.height
    g = np.zeros(cells, np.uint32) if want_g else None
    path = np.zeros(cells, np.uint32) if want_path else None
    rc = lib().oracle_astar_solve(ctypes.byref(o), ctypes.byref(r),
                                  ctypes.c_void_p(g.ctypes.data) if g is not None else None,
                                  ctypes.c_void_p(path.ctypes.data) if path is not None else None,
                                  cells if path is not None else 0)
    if rc != 0:
        raise RuntimeError("A* oracle self-check failed")
    out = {"cost": r.cost, "path_len": r.path_len, "expanded": r.expanded, "gsum": r.gsum,
           "path_hash": r.path_hash, "pops": r.pops, "seconds": r.seconds}
    if g is not None:
        out["g"] = g
    if path is not None:
        out["path"] = path[: r.path_len]
    return out


def astar_batch(grids, threads):
    """Solve many grids, one per host thread at a time; returns (seconds, list of results)."""
    arr = (OracleAstarGrid * len(grids))(*[_astar_grid(g) for g in grids])
    res = (OracleAstarResult * len(grids))()
    sec = lib().oracle_astar_batch(ctypes.cast(arr, ctypes.c_void_p), len(grids), threads,
                                   ctypes.cast(res, ctypes.c_void_p))
    if sec < 0:
        raise RuntimeError("A* oracle self-check failed")
    return sec, [{"cost": r.cost, "path_len": r.path_len, "expanded": r.expanded, "gsum": r.gsum,
                  "path_hash": r.path_hash, "pops": r.pops} for r in res]


ASTAR_REF_RESULT_DTYPE = np.dtype([("found", "<u4"), ("cost", "<f4"), ("pops", "<u4"), ("rounds", "<u4")])


def astar_ref(map2d, agents, threads=1):
    """Reference-semantics A* for every agent ((start, goal) pairs) on a map
    (uint8 [height, width], non-zero = wall); returns (seconds, results)."""
    m = np.ascontiguousarray(map2d, np.uint8)
    sg = np.ascontiguousarray(np.stack([np.asarray(agents["start"], np.uint32),
                                        np.asarray(agents["goal"], np.uint32)], axis=1))
    out = np.zeros(len(sg), ASTAR_REF_RESULT_DTYPE)
    sec = lib().oracle_astar_ref_run(m.shape[1], m.shape[0], ctypes.c_void_p(m.ctypes.data),
                                     ctypes.c_void_p(sg.ctypes.data), len(sg), threads,
                                     ctypes.c_void_p(out.ctypes.data))
    return sec, out
