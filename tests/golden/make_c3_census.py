"""Instruction census of the mixed-precision benchmark configuration's factorization and solve
programs in their plain FP64 form (N = 65536 points of U[0,1]^3 in Morton order, Laplace kernel
1/(4 pi (r + 1e-3)), standard admissibility eta = 1, leaf 512, adaptive rank <= 32 at 1e-8,
products in 128-wide tiles, 8 right-hand sides).

The CPU reference path cannot execute that program in a bounded time (about 1.3e14 flops), so
bench.py's CPU baseline and reference arm time the oracle on every instruction class of this
census and add the classes up (oracle/census.py).  One row per class: the class's representative
task record (pointers cleared; the timing run binds its own buffers), the instruction count and
the algorithmic flops of one instruction.

Writes tests/golden/c3_census.npz.  Run it where the library is built:
  python tests/golden/make_c3_census.py
"""
import collections
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "c3_census.npz")
CONFIG = dict(n=65536, dim=3, kernel=1, p0=1e-3, leaf=512, admissibility=1, eta=1.0, kmax=32, rank_tol=1e-8,
              gemm_tile=128, nrhs=8, seed=1234)
# the fields that decide an instruction's cost
KEY = ("op", "flags", "m", "n", "k", "l", "o", "ctrl", "prec")


def census(pp, cfg=CONFIG):
    ctx = pp.Context(device=-1)
    rng = np.random.default_rng(cfg["seed"])
    pts = rng.uniform(0.0, 1.0, (cfg["n"], cfg["dim"]))
    pts = pts[pp.morton_order(pts)]
    h = pp.Hierarchical.geometric(ctx, pts, cfg["leaf"], cfg["admissibility"], cfg["eta"], cfg["kmax"])
    h.set_rank_tolerance(cfg["rank_tol"])
    h.set_gemm_tile(cfg["gemm_tile"])
    out = {}
    for which, nrhs in ((0, 1), (1, cfg["nrhs"])):
        tasks, _, _, _ = h.encode_program(which, nrhs, [0] * 5)
        flops = pp_task_flops(tasks)
        groups = collections.OrderedDict()
        for i in range(len(tasks)):
            key = tuple(int(tasks[f][i]) for f in KEY)
            if key not in groups:
                groups[key] = [i, 0]
            groups[key][1] += 1
        reps = tasks[[g[0] for g in groups.values()]].copy()
        reps["p"] = 0
        reps["tmp"] = 0
        reps["succ_begin"] = 0
        reps["n_succ"] = 0
        out[f"records{which}"] = reps.view(np.uint8).reshape(len(reps), 160)
        out[f"counts{which}"] = np.array([g[1] for g in groups.values()], dtype=np.int64)
        out[f"flops{which}"] = np.array([flops[g[0]] for g in groups.values()], dtype=np.int64)
        out[f"total_flops{which}"] = np.array(int(h.program_info(which, nrhs)["flops"]))
    out["config_keys"] = np.array(list(cfg.keys()))
    out["config_vals"] = np.array([float(v) for v in cfg.values()])
    return out


def pp_task_flops(tasks):
    """Algorithmic flops of each task: the generator's count for the classes that dominate, and
    2 m n k for products, m^2 n for triangular solves (the program's own totals are exported too)."""
    op = tasks["op"].astype(np.int64)
    m, n, k = (tasks[f].astype(np.int64) for f in ("m", "n", "k"))
    f = np.zeros(len(tasks), dtype=np.int64)
    f[op == 6] = 2 * m[op == 6] * n[op == 6] * k[op == 6]
    f[op == 1] = (2 * m[op == 1] ** 3) // 3
    tri_l = (op == 2) | (op == 5)
    f[tri_l] = m[tri_l] * m[tri_l] * n[tri_l]
    f[op == 3] = m[op == 3] * n[op == 3] * n[op == 3]
    f[op == 4] = m[op == 4] * m[op == 4] * n[op == 4]
    return f


def main():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_pp
    d = census(load_pp())
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: {len(d['counts0'])} factor classes ({d['counts0'].sum()} instructions), "
          f"{len(d['counts1'])} solve classes ({d['counts1'].sum()} instructions), {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
