"""Partial pivoting inside the GETRF blocks on the GPU (PP_PIVOT) against the oracle running
the same programs (oracle/oracle.cpp o_getrf_piv / o_permute_rows).

* the all-dense tree of N = 1024 with 256-row leaves (64-row GETRF blocks) on U[-1,1] without the diagonal shift
  and with a zero leading entry: the factorization bitwise equal to the oracle's (same pivot
  rows: largest magnitude, first of equal ones), the solve within 1e-12 of the oracle's, and
  FP64 refinement to a backward error <= 1e-12 against the dense matrix;
* a HODLR kernel matrix without the diagonal shift (no dominance): within 1e-12 of the oracle
  (the low-rank accumulations' bar), refined to 1e-10;
* a dominant matrix: the pivoted factorization has the unpivoted bits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def undominated(pp, ctx, n=1024, leaf=256, seed=5):
    h, A = pp.make_dense_problem(ctx, n=n, leaf=leaf, seed=seed, shift=0.0)
    A[0, 0] = 0.0
    for blk in h.blocks():
        if blk["kind"] == pp.DENSE:
            r, c = blk["row0"], blk["col0"]
            h.set_dense(blk["id"], A[r:r + blk["m"], c:c + blk["n"]])
    return h, A


def test_pivoted_dense_factor_bitwise_and_solve(pp, gctx):
    import oracle as O
    h, A = undominated(pp, gctx)
    h.set_pivoting(True)
    ar = O.HostArenas(h, 0)
    ar.run()
    h.upload()
    h.factor()
    h.sync()
    h.download()
    Fg = h.to_dense()
    h.host_arena()[:] = ar.matrix
    Fo = h.to_dense()
    assert np.array_equal(Fg, Fo)
    assert np.all(np.isfinite(Fg))
    # the solve program (TRSML with the block permutations, then TRSMU) against the oracle's
    b = pp.rhs(1024)
    sol = O.HostArenas(h, 1, 1, rhs=b)
    sol.matrix[:] = ar.matrix
    sol.run()
    xo = sol.rhs[:1024].copy()
    bd = torch.from_numpy(b).cuda()
    x = torch.empty_like(bd)
    h.solve(bd, x)
    h.sync()
    xg = x.cpu().numpy().ravel()
    assert np.linalg.norm(xg - xo) <= 1e-12 * np.linalg.norm(xo)
    # FP64 refinement against the dense matrix
    ref = pp.Refiner(h, gctx, dense=A)
    xr, hist = ref.solve(bd, tol=1e-12)
    assert hist[-1] <= 1e-12, hist


def test_pivoted_without_swaps_is_unpivoted(pp, gctx):
    h, A = pp.make_dense_problem(gctx, n=1024, leaf=256, seed=9)
    h.upload()
    h.factor()
    h.sync()
    h.download()
    F0 = h.to_dense()
    h2, _ = pp.make_dense_problem(gctx, n=1024, leaf=256, seed=9)
    h2.set_pivoting(True)
    h2.upload()
    h2.factor()
    h2.sync()
    h2.download()
    assert np.array_equal(h2.to_dense(), F0)


def test_pivoted_hodlr_kernel_matrix(pp, gctx):
    import oracle as O
    h, prob = pp.make_kernel_problem(gctx, 2048, 2, "inv", 1e-3, 128, 16, shift=0.0, seed=12)
    h.set_pivoting(True)
    ar = O.HostArenas(h, 0)
    ar.run()
    h.upload()
    h.factor()
    h.sync()
    h.download()
    Fg = h.to_dense()
    h.host_arena()[:] = ar.matrix
    Fo = h.to_dense()
    assert np.linalg.norm(Fg - Fo) <= 1e-12 * np.linalg.norm(Fo)
    b = torch.from_numpy(pp.rhs(2048, 2)).cuda()
    xr, hist = pp.Refiner(h, gctx, prob).solve(b, tol=1e-10)
    assert hist[-1] <= 1e-10, hist
