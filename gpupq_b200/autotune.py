"""Autotuners for the PHOLD engine's launch shape and the A* engine's configuration.

PHOLD: for a workload class it times candidate (lanes_per_lp, block_threads, ctas_per_sm,
insert_capacity) settings -- and, for the local array queue, its sorted and bucketed
forms (laq_mode 0 and 2; the bucketed form ignores lanes_per_lp and insert_capacity, so
only its CTA size is varied) -- on the first `windows` safe windows of the real workload
(same seed, same queues), rejects candidates that overflow or disagree with the others
(every candidate runs the same windows, so committed count and digest must match), and
keeps the fastest.

A*: for a batch of grids it times candidate (tile, window, ctas_per_sm) settings on whole
solves of that batch, rejects candidates whose results differ from the others (every
result field is independent of the schedule), and keeps the fastest.

Results are cached in a JSON file keyed by GPU name and workload class, so later runs
pick the tuned settings without re-timing.
"""
import itertools
import json
import os
import time

import numpy as np

from . import AStar, GpqError, Phold, make_phold_config

DEFAULT_CACHE = os.environ.get("GPQ_TUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                                                              "tune_cache.json"))
# Shapes measured on whole runs (not the tuner's short samples) and shipped with the
# package; consulted when the local cache has no entry for the workload class.
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_shapes.json")

DEFAULT_SPACE = {
    "lanes_per_lp": [8, 16, 32],
    "block_threads": [64, 128, 256, 512],
    "ctas_per_sm": [0],
    "insert_capacity": [32, 64],
}


def _gpu_name():
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "unknown-gpu"


def workload_key(cfgd, queue, loop):
    keys = ("num_lps", "events_per_lp", "lookahead", "dest_mode", "capacity")
    parts = [f"{k}={cfgd.get(k)}" for k in keys]
    return f"{_gpu_name()}|{queue}|{loop}|" + "|".join(parts)


def _load(cache):
    try:
        with open(cache) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(cache, data):
    try:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, cache)
    except OSError:
        pass


def tune_phold(cfgd, queue="laq", loop="persistent", windows=200, space=None, cache=DEFAULT_CACHE,
               force=False, verbose=False):
    """Return the fastest launch-shape settings (a dict of make_phold_config keyword
    arguments) for this workload class, timing candidates if not cached."""
    key = workload_key(cfgd, queue, loop)
    data = _load(cache)
    if not force and key in data:
        return dict(data[key]["best"])
    shipped = _load(SHIPPED)
    if not force and key in shipped:
        return dict(shipped[key]["best"])
    space = dict(DEFAULT_SPACE, **({"laq_mode": [0, 2]} if queue == "laq" else {}), **(space or {}))
    names = list(space.keys())
    results = []
    ref = None
    seen = set()
    for values in itertools.product(*[space[n] for n in names]):
        shape = dict(zip(names, values))
        if shape["block_threads"] < shape["lanes_per_lp"]:
            continue
        if shape.get("laq_mode") == 2:  # the bucketed form: only the CTA size matters
            shape.update(lanes_per_lp=8, insert_capacity=64, ctas_per_sm=0)
            if tuple(sorted(shape.items())) in seen:
                continue
            seen.add(tuple(sorted(shape.items())))
        try:
            cfg = make_phold_config(**cfgd, queue=queue, loop=loop, max_steps=windows, **shape)
            with Phold(cfg) as h:
                h.populate()
                h.run()  # warm-up (module load, first-touch)
                h.populate()
                h.run()
                r = h.result()
        except GpqError as e:
            if verbose:
                print("autotune: reject", shape, e)
            continue
        if r["status_code"] != 0:
            continue
        sig = (r["committed"], r["digest"], r["steps"])
        if ref is None:
            ref = sig
        elif sig != ref:
            raise RuntimeError(f"autotune: candidate {shape} disagrees with the others: {sig} vs {ref}")
        per_window = r["elapsed_ms"] / max(1, r["steps"])
        results.append((per_window, shape))
        if verbose:
            print(f"autotune: {shape} {per_window * 1e3:.1f} us/window")
    if not results:
        raise RuntimeError("autotune: no candidate ran")
    results.sort(key=lambda x: x[0])
    best = results[0][1]
    data[key] = {"best": best, "us_per_window": results[0][0] * 1e3, "when": time.strftime("%Y-%m-%dT%H:%M:%S"),
                 "windows": windows,
                 "all": [{"shape": s, "us_per_window": t * 1e3} for t, s in results]}
    _save(cache, data)
    return dict(best)


ASTAR_SPACE = {
    "tile": [32, 64],
    "window": [2, 4, 10],  # in move costs: 1 for 4-connected grids, 10 for 8-connected ones
    "ctas_per_sm": [0, 1, 2, 4],
}
ASTAR_RESULT_FIELDS = ("status", "cost", "expanded", "gsum", "path_len", "path_hash")


def astar_workload_key(grids):
    """Workload class of an A* batch: instance count, cells, connectivity and density."""
    grids = np.asarray(grids)
    cells = grids["width"].astype(np.int64) * grids["height"]
    conns = "+".join(str(c) for c in sorted(set(int(c) for c in grids["conn"])))
    thr = float(np.mean(grids["block_thr"])) / float(1 << 24)
    return (f"{_gpu_name()}|astar|n={len(grids)}|cells={int(cells.sum())}|max_cells={int(cells.max())}"
            f"|conn={conns}|density={thr:.2f}")


def tune_astar(grids, space=None, repeats=2, cache=DEFAULT_CACHE, force=False, verbose=False):
    """Return the fastest A* configuration (a dict of AStar keyword arguments) for this
    batch's workload class, timing candidates on whole solves of `grids` if not cached."""
    grids = np.asarray(grids)
    key = astar_workload_key(grids)
    data = _load(cache)
    if not force and key in data:
        return dict(data[key]["best"])
    shipped = _load(SHIPPED)
    if not force and key in shipped:
        return dict(shipped[key]["best"])
    space = dict(ASTAR_SPACE, **(space or {}))
    unit = 1 if all(int(c) == 4 for c in grids["conn"]) else 10
    names = list(space.keys())
    results, ref = [], None
    for values in itertools.product(*[space[n] for n in names]):
        shape = dict(zip(names, values))
        kw = dict(shape, window=shape["window"] * unit) if "window" in shape else dict(shape)
        try:
            with AStar(**kw) as a:
                best = None
                for _ in range(max(1, repeats)):
                    r = a.solve(grids)
                    ms = a.stats()["total_ms"]
                    best = ms if best is None else min(best, ms)
        except GpqError as e:
            if verbose:
                print("autotune: reject", kw, e)
            continue
        if np.any(r["status"] != 0):
            if verbose:
                print("autotune: reject", kw, "status", int(np.max(r["status"])))
            continue
        sig = tuple(np.asarray(r[f]).tobytes() for f in ASTAR_RESULT_FIELDS)
        if ref is None:
            ref = sig
        elif sig != ref:
            raise RuntimeError(f"autotune: A* candidate {kw} disagrees with the others")
        results.append((best, kw))
        if verbose:
            print(f"autotune: {kw} {best:.3f} ms")
    if not results:
        raise RuntimeError("autotune: no A* candidate ran")
    results.sort(key=lambda x: x[0])
    best = results[0][1]
    data[key] = {"best": best, "ms": results[0][0], "when": time.strftime("%Y-%m-%dT%H:%M:%S"),
                 "all": [{"config": c, "ms": t} for t, c in results]}
    _save(cache, data)
    return dict(best)
