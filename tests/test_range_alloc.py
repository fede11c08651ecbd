"""The first-fit range allocator behind the resident sessions' admission (cell, tile and
LP spaces), against a Python model of first-fit allocation with coalescing frees."""
import os
import random
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not on PATH")
    exe = str(tmp_path_factory.mktemp("ra") / "range_alloc_driver")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "gpupq_b200", "csrc"),
                           os.path.join(HERE, "cpp", "range_alloc_driver.cpp"), "-o", exe])
    return exe


def _model_first_fit(size, cmds):
    free = [(0, size)]  # sorted (start, len)
    out, used = [], 0
    for c in cmds:
        if c[0] == "a":
            n = c[1]
            for i, (s, l) in enumerate(free):
                if l >= n:
                    out.append(s)
                    free[i] = (s + n, l - n)
                    if free[i][1] == 0:
                        free.pop(i)
                    used += n
                    break
            else:
                out.append(-1)
        else:
            s, n = c[1], c[2]
            used -= n
            free.append((s, n))
            free.sort()
            merged = []
            for fs, fl in free:
                if merged and merged[-1][0] + merged[-1][1] == fs:
                    merged[-1] = (merged[-1][0], merged[-1][1] + fl)
                else:
                    merged.append((fs, fl))
            free = merged
    return out, used


@pytest.mark.parametrize("seed", range(6))
def test_random_sequences(driver, seed):
    rng = random.Random(seed)
    size = rng.choice([64, 1000, 1 << 20])
    live, cmds = [], []
    sim_free = size
    for _ in range(400):
        if live and rng.random() < 0.45:
            s, n = live.pop(rng.randrange(len(live)))
            cmds.append(("f", s, n))
            sim_free += n
        else:
            n = rng.randint(1, max(1, size // rng.choice([2, 8, 64])))
            cmds.append(("a", n))
            want, _ = _model_first_fit(size, cmds)
            if want[-1] >= 0:
                live.append((want[-1], n))
    text = f"{size}\n" + "\n".join(" ".join(str(x) for x in c) for c in cmds) + "\n"
    got = subprocess.run([driver], input=text, capture_output=True, text=True, check=True).stdout.split("\n")
    want, used = _model_first_fit(size, cmds)
    assert [int(x) for x in got[:len(want)]] == want
    assert got[len(want)] == f"used {used}"
