"""Generates tests/golden/phold_golden.json: PHOLD results of the CPU oracle at full size.

The 65,536-LP ring workload at its full end time (3.8 G committed events) takes the
windowed oracle a few minutes on 8 host threads, too long to repeat inside a GPU test or
the bench; this script runs it once and commits the outputs that pin a run exactly:
committed events, windows, pending events and their checksum, the engine's digest over
the per-LP outputs and a sha256 of the per-LP arrays.  The windowed and the sequential
oracle agree on every output (tests/test_oracle.py); the one-per-LP entries give the
window count of the reference's own schedule (one event per LP per window).

    python tests/golden/make_phold_golden.py [--threads N] [--only NAME]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "phold_golden.json")

# name -> (config, driver); the configs are the PHOLD workloads the tests and bench run
CASES = {
    # 1,024 LPs x 16 events, lookahead 1.0, end 100, uniform destinations, seed 42
    "phold_plain_1024lp_x16_T100": (dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0, seed=42,
                                         dest_mode=0), "window"),
    "phold_plain_1024lp_x16_T100_one_per_lp": (dict(num_lps=1024, events_per_lp=16, lookahead=1.0, end_time=100.0,
                                                    seed=42, dest_mode=0), "one_per_lp"),
    # 65,536 LPs x 64 events, lookahead 0.1, ring +-16 (90 %), end 1000, seed 7
    "phold_large_65536lp_x64_ring16_T1000": (dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=1000.0,
                                                  seed=7, dest_mode=1, ring_width=16), "window"),
    "phold_large_65536lp_x64_ring16_T3": (dict(num_lps=65536, events_per_lp=64, lookahead=0.1, end_time=3.0,
                                               seed=7, dest_mode=1, ring_width=16), "window"),
    # long per-LP queues: 4,096 LPs x 4,096 pending events, lookahead 0.01 (about 40 safe
    # events per LP per window), ring +-16, end 2
    "phold_long_4096lp_x4096_ring16_T2": (dict(num_lps=4096, events_per_lp=4096, lookahead=0.01, end_time=2.0,
                                               seed=23, dest_mode=1, ring_width=16), "window"),
    "phold_large_65536lp_x64_ring16_T3_one_per_lp": (dict(num_lps=65536, events_per_lp=64, lookahead=0.1,
                                                          end_time=3.0, seed=7, dest_mode=1, ring_width=16),
                                                     "one_per_lp"),
}


def run_case(cfgd, driver, threads):
    cfg = O.make_cfg(**cfgd)
    t0 = time.time()
    if driver == "one_per_lp":
        o = O.phold(cfg, one_per_lp=True)
    else:
        o = O.phold(cfg, threads)
    return {
        "config": cfgd, "driver": driver,
        "committed": o["committed"], "windows": o["steps"], "pending": o["pending"],
        "pending_csum": str(o["pending_csum"]), "digest": str(o["digest"]),
        "lp_sha256": O.lp_sha256(o["count"], o["csum"], o["ohash"]),
        "oracle_seconds": round(time.time() - t0, 1),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 8)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as fh:
            data = json.load(fh)
    for name, (cfgd, driver) in CASES.items():
        if a.only and name != a.only:
            continue
        data[name] = run_case(cfgd, driver, a.threads)
        print(name, data[name], flush=True)
        with open(OUT, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
            fh.write("\n")


if __name__ == "__main__":
    main()
