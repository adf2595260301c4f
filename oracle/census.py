"""TEST ORACLE — the CPU reference path's cost on a program too large to run on the host: every
instruction class of an exported census (tests/golden/make_c3_census.py) is executed by the
oracle's restated reference routines (liboracle.so) on operands of its shapes, timed, and
multiplied by the class's instruction count.  The sum over classes divided by the host threads
(ideal scaling, which flatters the CPU) estimates one factorization (or one solve) of the
program on the host cores.  Test infrastructure only; it neither imports nor loads the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import lib
from .hodlr import TASK_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
CENSUS = os.path.join(os.path.dirname(HERE), "tests", "golden", "c3_census.npz")
PP_ADAPT_RANK = 2


def _bind(rec, rng):
    """A copy of the record with fresh host buffers for every operand it names (large enough for
    any operand of its shape; diagonally dominant, so factorizations and solves stay finite)."""
    t = rec.copy()
    dims = [int(rec[f]) for f in ("m", "n", "k", "l", "o")]
    D = max(dims + [64])
    keep = []
    for s in range(6):
        ld = int(rec["ld"][s])
        if s > 0 and ld == 0 and s > 3:
            continue
        size = (D + 1) * max(ld, D)
        a = rng.uniform(-1.0, 1.0, size)
        idx = np.arange(D) * max(ld, 1) + np.arange(D)
        a[idx[idx < size]] += 2.0 * D
        keep.append(a)
        t["p"][s] = a.ctypes.data
    if int(rec["flags"]) & PP_ADAPT_RANK:
        w = np.zeros(1)
        keep.append(w)
        t["p"][5] = w.ctypes.data
    tmp = np.zeros(4 * (D + 64) * (D + 64))
    keep.append(tmp)
    t["tmp"] = tmp.ctypes.data
    return t, keep


def time_class(rec, min_s=0.05, rng=None):
    """Seconds one instruction of this class takes on one host core (median-free: the mean over
    at least min_s of repeated runs)."""
    rng = rng or np.random.default_rng(0)
    t, keep = _bind(np.array([rec], dtype=TASK_DTYPE)[0], rng)
    tasks = np.array([t], dtype=TASK_DTYPE)
    reps, t0 = 0, time.perf_counter()
    while True:
        rc = lib().oracle_run_program(tasks.ctypes.data, 1)
        if rc != 0:
            raise RuntimeError(f"oracle: instruction op {int(rec['op'])} unsupported")
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_s:
            break
    del keep
    return el / reps


def program_seconds(which, threads, path=CENSUS, min_s=0.05):
    """(estimated host seconds of one run of the program on `threads` threads, details)."""
    z = np.load(path)
    recs = z[f"records{which}"].reshape(-1).view(TASK_DTYPE)
    counts = z[f"counts{which}"]
    rng = np.random.default_rng(1)
    total_core_s, measured = 0.0, []
    for rec, cnt in zip(recs, counts):
        s = time_class(rec, min_s=min_s, rng=rng)
        total_core_s += s * int(cnt)
        measured.append((int(rec["op"]), int(rec["m"]), int(rec["n"]), int(rec["k"]), int(cnt), s))
    return total_core_s / max(1, threads), {"classes": len(counts), "instructions": int(counts.sum()),
                                            "core_seconds": total_core_s, "per_class": measured,
                                            "flops": int(z[f"total_flops{which}"])}
