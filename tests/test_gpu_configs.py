"""Parity at the full benchmark configurations (the sizes bench.py runs), not just small cases.

  config 1  N = 1024 dense, U[-1,1] + N I, 2 x 2 partition to depth 2 (leaf 256), seed 1234:
            the engine's factorization bitwise equal to the textbook no-pivot LU and to the
            reference's own kernel_dynamic running the same program.
  config 2  N = 8192 HODLR (kernel 1/(r + 1e-3) on Morton-sorted U[0,1]^2 points, leaf 256,
            rank 16, seed 1234): the engine's factorization within 1e-12 (relative, Frobenius) of
            the oracle running the same program; the reference-ISA form of the program within
            1e-12 of the reference's kernel_dynamic and of the oracle's CPU path (bench.py's
            reference arm); ||A - LU|| / ||A|| at the compression level.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from test_gpu_vm import factor_on_gpu, rel, run_reference_kernel  # noqa: E402

C2 = dict(n=8192, dim=2, kernel="inv", p0=1e-3, leaf=256, rank=16, seed=1234)


def c2_problem(pp, ctx):
    return pp.make_kernel_problem(ctx, C2["n"], C2["dim"], C2["kernel"], C2["p0"], C2["leaf"], C2["rank"],
                                  seed=C2["seed"])


def lu_relative_error(F, A, n_probe=8, seed=0):
    """||A - L U|| / ||A|| estimated on random probes: ||(A - L U) X||_F / ||A X||_F."""
    X = np.random.default_rng(seed).standard_normal((A.shape[0], n_probe))
    L = np.tril(F, -1) + np.eye(F.shape[0])
    U = np.triu(F)
    return np.linalg.norm(A @ X - L @ (U @ X)) / np.linalg.norm(A @ X)


def test_config1_bitwise_vs_textbook_and_reference_kernel(pp, oracle, gctx):
    h, A = pp.make_dense_problem(gctx, n=1024, leaf=256, seed=1234)
    F_ref = run_reference_kernel(pp, oracle, h)
    F = factor_on_gpu(h)
    assert np.array_equal(F, oracle.dense_getrf(A))
    assert np.array_equal(F, F_ref)
    assert lu_relative_error(F, A) < 1e-14


def test_config2_factor_matches_oracle(pp, oracle, gctx):
    h, prob = c2_problem(pp, gctx)
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=16)
    F = factor_on_gpu(h)
    h.host_arena()[:] = ar.matrix
    Fo = h.to_dense()
    assert rel(F, Fo) < 1e-12
    err = lu_relative_error(F, prob.dense())
    assert err < 1e-3, err  # rank-16 compression of the large off-diagonal blocks (about 2.4e-4)
    print(f"config 2: engine vs oracle {rel(F, Fo):.2e}, ||A - LU|| / ||A|| ~ {err:.2e}")


@pytest.fixture(scope="module")
def rctx(pp):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return pp.Context(device=0, reference_isa=1)


def test_config2_reference_isa_matches_reference_kernel_and_cpu_path(pp, oracle, rctx):
    import oracle.hodlr as oh
    h, prob = c2_problem(pp, rctx)
    ops = np.bincount(h.encode_program(0, 1, [0] * 5)[0]["op"], minlength=16)
    assert ops[10] == 0 and ops[11] == 0  # no split-k sums, no inverses: the reference's set
    F_ref = run_reference_kernel(pp, oracle, h)
    F = factor_on_gpu(h)
    assert rel(F, F_ref) < 1e-12
    # the CPU path bench.py times as the reference arm: the same program from the fixture, on
    # arenas built without this library
    job = oh.FixtureJob()
    assert np.array_equal(job.original, c2_problem(pp, pp.Context(device=-1, reference_isa=1))[0].host_arena())
    job.restore()
    job.factor(threads=16)
    h.host_arena()[:] = job.matrix
    assert rel(F, h.to_dense()) < 1e-12
