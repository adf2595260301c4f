"""Multi-rank path of the bench on CPU (gloo, world size 2): one H-LU is one DAG with no
exchange step, so ranks are independent replicas (seeds offset by rank) whose only collective
is the max of their times; the reference arm runs on rank 0 alone."""
import importlib.util
import os
import socket
import subprocess
import sys
from datetime import timedelta

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cpu_job(pp, oracle, h, prob, tol=1e-10):
    """One factor + solve + FP64 refinement of a replica's problem with the oracle (the program
    the GPU runs, executed on the host); returns (seconds, refinement solves)."""
    import time
    n = prob.n
    b = pp.rhs(n, 1, seed=7)
    A = prob.dense()
    t0 = time.perf_counter()
    fac = oracle.HostArenas(h, 0)
    fac.run(threads=2)
    sol = oracle.HostArenas(h, 1, 1)
    sol.matrix[:] = fac.matrix
    x, r = np.zeros((n, 1)), b.copy()
    for it in range(1, 31):
        sol.rhs[:n] = r.ravel()
        sol.run(threads=1)
        x += sol.rhs[:n].reshape(n, 1)
        r = b - A @ x
        if np.abs(r).max() / (prob.norm_inf * np.abs(x).max() + np.abs(b).max()) <= tol:
            break
    return time.perf_counter() - t0, it


def _replica(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        bench = _bench()
        pp = bench.load_pp()
        import oracle
        ctx = pp.Context(device=-1)
        # this rank's replica: the workload's construction at a small size, seed offset by rank
        h, prob = pp.make_kernel_problem(ctx, 1024, 2, "inv", 1e-3, 256, 16, seed=1234 + rank)
        t, iters = _cpu_job(pp, oracle, h, prob)
        rate, tmax = bench.whole_job_rate(dist, world, t, 1, "cpu")
        q.put((rank, t, iters, rate, tmax, float(prob.points[0, 0])))
    finally:
        dist.destroy_process_group()


def test_replicas_world2_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, it0, rate0, max0, x0), (r1, t1, it1, rate1, max1, x1) = out
    assert (r0, r1) == (0, 1)
    assert x0 != x1  # independent replicas: different seeded problems
    assert 1 <= it0 <= 30 and 1 <= it1 <= 30  # each refined to the tolerance on its own
    assert max0 == max1 == max(t0, t1)  # the slowest rank bounds the job, on every rank
    assert rate0 == rate1 and np.isclose(rate0, 2 / max(t0, t1))


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
