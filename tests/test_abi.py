"""CPU tests of the C ABI: the library loads, exports every symbol declared in
include/gpq.h, and its host-side model code matches the oracle bit for bit."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import gpupq_b200 as G
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", hdr)).read()
            names += re.findall(r"^GPQ_API\s+[\w\s\*]+?\b(gpq_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_all_declared_symbols():
    lib = G.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", G.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gpq_\w+)", out))
    assert set(names) <= exported, sorted(set(names) - exported)


def test_status_strings_and_version():
    lib = G.lib()
    assert b"sm_100a" in lib.gpq_version()
    for s in range(9):
        assert lib.gpq_status_string(s)


def test_invalid_config_is_rejected_without_gpu():
    cfg = G.make_phold_config(num_lps=0, events_per_lp=1, lookahead=1.0, end_time=1.0, seed=1)
    out = np.zeros(1, G.ITEM_DTYPE)
    st = G.lib().gpq_phold_initial_events(ctypes.byref(cfg), ctypes.c_void_p(out.ctypes.data), 0)
    assert st == 1  # GPQ_ERR_INVALID
    assert b"num_lps" in G.lib().gpq_last_error()


@pytest.mark.parametrize("cfgd", [
    dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42, dest_mode=0),
    dict(num_lps=3000, events_per_lp=7, lookahead=0.1, end_time=1000.0, seed=7, dest_mode=1, ring_width=16),
])
def test_host_initial_events_match_oracle(cfgd):
    cfg = G.make_phold_config(**cfgd)
    ev = G.initial_events(cfg)
    ts, lp, ids = O.initial(O.make_cfg(**cfgd))
    assert np.array_equal(ev["ts"].view(np.uint32), ts.view(np.uint32))
    assert np.array_equal(ev["lp"], lp)
    assert np.array_equal(ev["id"], ids)
    assert (ev["ts"] >= 0).all() and np.isfinite(ev["ts"]).all()


def test_gpu_path_has_no_cpu_fallback():
    """The device entry points must fail (not silently compute on the CPU) without a GPU."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present: covered by the gpu tests")
    except Exception:
        pass
    cfg = G.make_phold_config(num_lps=8, events_per_lp=2, lookahead=1.0, end_time=1.0, seed=1)
    with pytest.raises(G.GpqError):
        G.Phold(cfg)
