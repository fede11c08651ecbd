"""The reference's OWN queues and DES loop against the oracle and this project's engine.

oracle/build_ref.py compiles the reference's unmodified src/des.cu with one of its per-LP
queues (src/local_array_queue.cu + src/sort.cu, src/local_heap_queue.cu,
src/local_splay_queue.cu) and the adapter model (oracle/ref_adapter/), which handles one
event per LP per window like src/phold.cu:81-117 with this project's event function.
Each binary runs on the GPU here; its per-LP committed count, checksum and order-sensitive
hash must equal the CPU oracle's (and so the CUDA engine's, tests/test_phold_full_gpu.py),
and its window count must equal the oracle's one-event-per-LP schedule.  This pins the
engine's trajectories to the reference's own queue code, not only to a restatement.
"""
import json
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import build_ref as B
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "phold_golden.json")) as fh:
    GOLDEN = json.load(fh)
GOLDEN_OF = {"c1": "phold_plain_1024lp_x16_T100", "c2r": "phold_large_65536lp_x64_ring16_T3"}


def run_reference(variant, timeout=600):
    """Runs one reference binary; returns (header dict, count, csum, ohash, stdout)."""
    exe = B.binary_path(variant)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is missing: build it with python oracle/build_ref.py")
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "res.bin")
        p = subprocess.run([exe, out], capture_output=True, text=True, timeout=timeout)
        assert p.returncode == 0, (variant, p.returncode, p.stdout[-2000:], p.stderr[-2000:])
        raw = open(out, "rb").read()
    hdr = np.frombuffer(raw[:64], np.uint64)
    L = int(hdr[0])
    count = np.frombuffer(raw[64:64 + 4 * L], np.uint32)
    csum = np.frombuffer(raw[64 + 4 * L:64 + 12 * L], np.uint64)
    ohash = np.frombuffer(raw[64 + 12 * L:64 + 20 * L], np.uint64)
    h = dict(num_lps=L, committed=int(hdr[1]), windows=int(hdr[2]), pending=int(hdr[3]), pending_csum=int(hdr[4]),
             error=int(hdr[5]))
    return h, count, csum, ohash, p.stdout


def events_per_sec(stdout):
    """The reference's own runtime figure (src/des.cu:122)."""
    m = re.search(r"Events per sec\.:\s*([0-9.]+)", stdout)
    return float(m.group(1)) if m else None


@pytest.mark.gpu
@pytest.mark.parametrize("variant", list(B.VARIANTS))
def test_reference_queue_matches_oracle(gpu_lib, variant):
    _, w = B.VARIANTS[variant]
    g = GOLDEN[GOLDEN_OF[w]]
    g1 = GOLDEN[GOLDEN_OF[w] + "_one_per_lp"]
    h, count, csum, ohash, out = run_reference(variant)
    assert h["error"] == 0, h
    assert h["committed"] == g["committed"]
    assert h["pending"] == g["pending"]
    assert h["pending_csum"] == int(g["pending_csum"])
    assert O.lp_sha256(count, csum, ohash) == g["lp_sha256"]
    assert O.digest(count, csum, ohash) == int(g["digest"])
    # the reference's schedule: one event per LP per window
    assert h["windows"] == g1["windows"]
    assert events_per_sec(out) is not None


def test_generated_config_keeps_reference_names():
    """The generated config.h defines every setting the compiled reference files read."""
    for v in B.VARIANTS:
        txt = B.config_text(v)
        for name in ("NUM_LPS", "NUM_NODES", "DEVICE_MEMORY_MB", "MAX_TS", "MAX_WCT", "MAX_EVENTS", "LOOKAHEAD",
                     "_LAQ_INSERTION_SORT", "LOCAL_ARRAY_QUEUE_BACKWARD", "MAX_THREADS__PHOLD",
                     "MAX_THREADS__LOCAL_ARRAY_QUEUE", "_PHOLD", "CUDA_DEVICE"):
            assert re.search(r"#define " + name + r"\b", txt), (v, name)
        q, w = B.VARIANTS[v]
        assert ("#define " + B.QUEUES[q][0]) in txt
        assert f"#define NUM_LPS {B.WORKLOADS[w]['num_lps']}" in txt
