"""Partial pivoting inside the GETRF blocks (PP_PIVOT), on the CPU oracle over the engine's
programs (test of the program structure and of the restatement; the GPU parity is in
tests/test_gpu_pivot.py).

* a matrix that is not diagonally dominant (U[-1,1], no shift) and has a zero leading entry:
  the reference's no-pivot LU breaks down, the pivoted program solves it (the oracle runs the
  factor and solve programs; the answer checked against the dense matrix);
* a diagonally dominant matrix needs no swap: the pivoted factorization has the unpivoted bits
  and identity permutations."""
import numpy as np

import oracle as O


def run_factor_solve(pp, h, A, b, pivot):
    h.set_pivoting(pivot)
    f = O.HostArenas(h, 0)
    f.run()
    s = O.HostArenas(h, 1, 1, rhs=b)
    s.matrix[:] = f.matrix
    s.run()
    return f, s.rhs[: len(b)].copy()


def test_pivoted_program_solves_a_matrix_without_dominance(pp, hctx):
    h, A = pp.make_dense_problem(hctx, n=512, leaf=128, seed=5, shift=0.0)
    A[0, :] = A[1, :] * 0.5 + A[0, :] * 0.0  # a_00 is no longer the largest of column 0
    A[0, 0] = 0.0                            # and is zero: no-pivot LU divides by it
    for blk in h.blocks():
        if blk["kind"] == pp.DENSE:
            r, c = blk["row0"], blk["col0"]
            h.set_dense(blk["id"], A[r:r + blk["m"], c:c + blk["n"]])
    b = pp.rhs(512).ravel()
    _, x0 = run_factor_solve(pp, h, A, b, False)
    assert not np.all(np.isfinite(x0))  # the unpivoted program breaks down
    f, x = run_factor_solve(pp, h, A, b, True)
    # one FP64 refinement step with the same pivoted factors
    r = b - A @ x
    s = O.HostArenas(h, 1, 1, rhs=r)
    s.matrix[:] = f.matrix
    s.run()
    x = x + s.rhs[:512]
    be = np.abs(b - A @ x).max() / (np.abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())
    assert be <= 1e-14, be
    info = h.program_info(0)
    assert info["op_count"]["trinv"] == 0  # the pivoted solve substitutes


def dense_blocks(pp, h, arena):
    out = []
    for blk in h.blocks():
        if blk["kind"] == pp.DENSE:
            off = h.block_storage(blk["id"])[0]
            out.append(((blk["row0"], blk["col0"], blk["m"], blk["n"]), arena[off:off + blk["m"] * blk["n"]]))
    return out


def test_pivoted_program_without_swaps_has_the_unpivoted_bits(pp, hctx):
    h, A = pp.make_dense_problem(hctx, n=512, leaf=128, seed=6)
    b = pp.rhs(512).ravel()
    f0, _ = run_factor_solve(pp, h, A, b, False)
    f1, _ = run_factor_solve(pp, h, A, b, True)
    F = O.dense_getrf(A)
    for ((r, c, m, n), x0), (_, x1) in zip(dense_blocks(pp, h, f0.matrix), dense_blocks(pp, h, f1.matrix)):
        assert np.array_equal(x0, x1)
        assert np.array_equal(x1, F[r:r + m, c:c + n].ravel())


def test_block_getrf_piv_matches_lapack():
    """The restated pivoted block LU against LAPACK's dgetrf (scipy): the same pivot rows
    (both take the first row of largest magnitude) and the same factors to rounding (LAPACK
    blocks its updates in another order)."""
    import scipy.linalg as sl
    rng = np.random.default_rng(17)
    for n in (7, 64):
        A = rng.uniform(-1, 1, (n, n))
        F, perm = O.getrf_piv(A)
        lu, piv = sl.lu_factor(A)
        p = np.arange(n)
        for i, r in enumerate(piv):  # LAPACK's swap sequence as a permutation
            p[[i, r]] = p[[r, i]]
        assert np.array_equal(perm, p)
        assert np.abs(F - lu).max() <= 1e-12 * np.abs(lu).max()
        L = np.tril(F, -1) + np.eye(n)
        U = np.triu(F)
        assert np.abs(L @ U - A[perm]).max() <= 1e-13
