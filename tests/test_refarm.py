"""The CPU reference path (oracle/hodlr.py) that bench.py times as the reference arm and the CPU
baseline: the committed reference-ISA program fixture, the oracle's own construction of the
matrix and its own substitution solve.  No GPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


@pytest.fixture(scope="module")
def job(oracle):
    import oracle.hodlr as oh
    return oh.FixtureJob()


@pytest.fixture(scope="module")
def exported(pp):
    import make_refisa_program as mk
    return mk.export(pp)


def test_fixture_is_what_the_library_generates(job, exported):
    z = np.load(job.__class__.__init__.__defaults__[0])
    assert np.array_equal(z["tasks"], exported["tasks"])
    assert np.array_equal(z["succ"], exported["succ"])
    assert np.array_equal(z["indeg"], exported["indeg"])
    assert np.array_equal(z["blocks"], exported["blocks"])
    assert list(z["meta_keys"]) == list(exported["meta_keys"])
    assert np.array_equal(z["meta_vals"], exported["meta_vals"])


def test_fixture_holds_only_reference_instructions(job):
    ops = set(np.unique(job.tasks["op"]).tolist())
    # getrf, trsml, trsmr, trsmr (transposed B), gemm / gemm_plus, gemm_3x, gemm_4x, accum
    assert ops <= {1, 2, 3, 4, 6, 7, 8, 9}
    assert job.flops > 9e8


def test_oracle_construction_equals_the_library_construction(pp, job):
    ctx = pp.Context(device=-1, seed=int(job.meta["rand_seed"]), reference_isa=1)
    h, prob = pp.make_kernel_problem(ctx, job.n, int(job.meta["dim"]), int(job.meta["kernel"]), job.meta["p0"],
                                     int(job.meta["leaf"]), int(job.meta["rank"]), seed=int(job.meta["seed"]))
    assert np.array_equal(h.host_arena(), job.original)
    assert prob.shift == job.shift and prob.norm_inf == job.norm_inf
    r = h.rand_host()
    assert np.array_equal(r, job.rand[: r.size])


def test_reference_path_reaches_the_tolerance(job):
    A = job.dense()
    b = np.random.default_rng(7).uniform(-1, 1, (job.n, 1))
    x, hist = job.factor_solve(b, A, tol=1e-10, threads=4)
    assert hist[-1] <= 1e-10 and len(hist) <= 6, hist
    # the factors reproduce A to the compression level: ||A - LU|| / ||A|| through the solve
    x_np = np.linalg.solve(A, b)
    assert np.abs(x - x_np).max() <= 1e-9 * np.abs(x_np).max()


def test_substitution_solve_inverts_the_factors(job):
    """The oracle's own solve against the factors multiplied out: L U x = b on the dense image."""
    job.restore()
    job.factor(threads=4)
    n = job.n
    F = np.zeros((n, n))
    for b in range(len(job.blocks)):
        kd, r0, c0, bm, bn = job.blocks[b][:5]
        if kd != 2:
            F[r0:r0 + bm, c0:c0 + bn] = job._apply(b, np.eye(bn))
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    b = np.random.default_rng(3).uniform(-1, 1, (n, 2))
    x = job.solve(b)
    assert np.abs(L @ (U @ x) - b).max() <= 1e-12 * np.abs(b).max() * n
