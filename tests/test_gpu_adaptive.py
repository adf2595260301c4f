"""Adaptive rank: accumulations truncate to the singular values above a tolerance (Gram
eigen-decomposition by Jacobi, rotation into the singular basis) and record the new rank."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from test_gpu_vm import TaskBench, rel  # noqa: E402


def spectrum_pair(rng, ny, nx, k, decay):
    """U V^T with singular values decay**i (i < k) on random orthonormal bases."""
    qa, _ = np.linalg.qr(rng.standard_normal((ny, k)))
    qb, _ = np.linalg.qr(rng.standard_normal((nx, k)))
    return qa * decay ** np.arange(k), qb


@pytest.mark.parametrize("ny,nx", [(256, 256), (512, 384), (2048, 2048)])
def test_adaptive_accum_truncates_to_tolerance(pp, oracle, gctx, ny, nx):
    rng = np.random.default_rng(ny + nx)
    k1, k2, tol = 16, 16, 1e-7
    tb = TaskBench(pp, seed=3)
    U1, V1 = spectrum_pair(rng, ny, nx, k1, 0.25)        # singular values 4^-i
    U2, V2 = 1e-13 * rng.standard_normal((ny, k2)), rng.standard_normal((nx, k2))
    M = U1 @ V1.T + U2 @ V2.T
    slots = {}
    for s, A in enumerate([U1, V1, U2, V2]):
        tb.host.append(np.ascontiguousarray(A))
        tb.devs.append(torch.from_numpy(tb.host[-1]).cuda())
        slots[s] = (len(tb.host) - 1, A.shape[1])
    tb.host.append(rng.uniform(-1, 1, (nx, k1)))
    tb.devs.append(torch.from_numpy(tb.host[-1]).cuda())
    slots[4] = (len(tb.host) - 1, k1)
    tb.host.append(np.zeros((1, 1)))
    tb.devs.append(torch.from_numpy(tb.host[-1]).cuda())
    slots[5] = (len(tb.host) - 1, 1)
    scratch = 2 * ny * k1 + nx * k1 + k1 * max(k1, k2)
    res = tb.run(gctx, oracle, dict(op=9, m=ny, n=nx, k=k1, l=k2, alpha=1.0, beta=tol, flags=2), slots, tmp_elems=scratch)
    Ud, Vd, rank = res[0][0], res[1][0], res[5][0][0, 0]
    expect = int(np.count_nonzero(np.linalg.svd(M, compute_uv=False)[:k1] > tol * np.linalg.norm(M, 2)))
    assert rank == expect == 12
    assert np.all(Ud[:, expect:] == 0) and np.all(Vd[:, expect:] == 0)
    assert rel(Ud @ Vd.T, M) < 10 * tol
    # the kept directions are orthonormal in U and scaled singular vectors in V
    G = Ud[:, :expect].T @ Ud[:, :expect]
    assert np.abs(G - np.eye(expect)).max() < 1e-12


def test_adaptive_hodlr_factor_refines_and_reports_ranks(pp, gctx):
    n, kmax, tol = 2048, 24, 1e-7
    h, prob = pp.make_kernel_problem(gctx, n, 1, "inv", 1e-3, 128, kmax, seed=77, rank_tol=tol)
    before = h.ranks()
    assert max(before.values()) <= kmax and min(before.values()) < kmax
    h.upload()
    ref = pp.Refiner(h, gctx, prob)
    h.factor()
    b = torch.from_numpy(pp.rhs(n)).cuda()
    x, hist = ref.solve(b, tol=1e-10)
    assert hist[-1] <= 1e-10
    h.sync()
    h.download()
    after = h.ranks()
    assert all(0 <= r <= kmax for r in after.values())
    assert min(after.values()) < kmax  # ranks chosen by the tolerance, not the capacity
    # the factored matrix L U reproduces A to about the truncation tolerance
    A = prob.dense()
    F = h.to_dense()
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    assert rel(L @ U, A) < 1e-5
