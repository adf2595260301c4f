"""The oracle (CPU restatement of the reference's routines) and the host-side H-LU programs.

The oracle is pinned (a) by construction — each routine restates src/kernel.cu's update
order — checked here against independent numpy algebra, (b) against the golden vectors in
tests/golden (outputs of the reference's own kernel_dynamic run on a B200, see
tests/golden/make_golden.py), and (c) on the GPU against the reference kernel directly.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_blocked_program_equals_textbook_lu_bitwise(pp, oracle, hctx):
    # every blocking of the right-looking no-pivot LU applies the same fma sequence per element
    h, A = pp.make_dense_problem(hctx, n=512, leaf=128, seed=5)
    ar = oracle.HostArenas(h, 0)
    ar.run()
    h.host_arena()[:] = ar.matrix
    assert np.array_equal(h.to_dense(), oracle.dense_getrf(A))


def test_parallel_executor_matches_sequential(pp, oracle, hctx):
    h, _ = pp.make_kernel_problem(hctx, 1024, 2, "inv", 1e-3, 128, 8)
    a1 = oracle.HostArenas(h, 0)
    a1.run(threads=1)
    a2 = oracle.HostArenas(h, 0)
    a2.run(threads=6)
    assert np.array_equal(a1.matrix, a2.matrix)


def test_parallel_executor_matches_sequential_standard_admissibility(pp, oracle, hctx):
    """Standard admissibility adds the sketched updates (GEMMs into work buffers, ORTH, COPY):
    running the program over its DAG with 8 threads gives the sequential result bit for bit,
    so every conflicting pair of tasks is ordered by an edge."""
    h, _ = pp.make_kernel_problem(hctx, 1024, 2, "laplace", 1e-3, 32, 8, admissibility=1, eta=1.0, seed=3)
    assert h.program_info(0)["op_count"]["orth"] > 0
    a1 = oracle.HostArenas(h, 0)
    a1.run(threads=1)
    a2 = oracle.HostArenas(h, 0)
    a2.run(threads=8)
    assert np.array_equal(a1.matrix, a2.matrix)


def test_dense_lu_is_an_lu(oracle):
    rng = np.random.default_rng(0)
    n = 200
    A = rng.uniform(-1, 1, (n, n)) + n * np.eye(n)
    F = oracle.dense_getrf(A)
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    assert np.linalg.norm(A - L @ U) / np.linalg.norm(A) < 1e-15


@pytest.mark.parametrize("a_T,b_T", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (1.0, 1.0), (1.0, 0.0)])
def test_gemm_restatement(oracle, a_T, b_T, alpha, beta):
    rng = np.random.default_rng(1)
    m, n, k = 37, 29, 45
    A = rng.standard_normal((k, m) if a_T else (m, k))
    B = rng.standard_normal((n, k) if b_T else (k, n))
    M = rng.standard_normal((m, n))
    want = alpha * ((A.T if a_T else A) @ (B.T if b_T else B)) + beta * M
    oracle.gemm(alpha, beta, M, A, B, a_T, b_T)
    assert np.allclose(M, want, rtol=1e-13, atol=1e-13)


def test_accum_restatement_projects_onto_sketch_range(oracle):
    rng = np.random.default_rng(2)
    ny, nx, k1, k2 = 300, 260, 12, 9
    U1, V1 = rng.standard_normal((ny, k1)), rng.standard_normal((nx, k1))
    U2, V2 = rng.standard_normal((ny, k2)), rng.standard_normal((nx, k2))
    R = rng.uniform(-1, 1, (nx, k1))
    A = U1 @ V1.T + U2 @ V2.T
    Q, _ = np.linalg.qr(A @ R)
    want = Q @ (Q.T @ A)
    oracle.accum(U1, V1, U2, V2, R)
    assert np.linalg.norm(U1 @ V1.T - want) / np.linalg.norm(want) < 1e-12
    assert np.allclose(U1.T @ U1, np.eye(k1), atol=1e-12)


def test_hodlr_program_accuracy_and_solve(pp, oracle, hctx):
    n = 2048
    h, prob = pp.make_kernel_problem(hctx, n, 2, "inv", 1e-3, 256, 16)
    Ah = h.to_dense()
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=4)
    b = pp.rhs(n)
    sol = oracle.HostArenas(h, 1, 1, rhs=b)
    sol.matrix[:] = ar.matrix
    sol.tasks, sol.succ, sol.indeg, sol.ready = h.encode_program(1, 1, sol.bases())
    sol.run()
    h.host_arena()[:] = ar.matrix
    F = h.to_dense()
    L, U = np.tril(F, -1) + np.eye(n), np.triu(F)
    assert np.linalg.norm(Ah - L @ U) / np.linalg.norm(Ah) < 1e-3
    x = sol.rhs[:n].reshape(n, 1)
    assert np.allclose(x, np.linalg.solve(U, np.linalg.solve(L, b)), rtol=1e-12, atol=1e-15)


def _golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not generated yet")
    return np.load(path)


def test_golden_dense_lu_matches_reference_kernel(oracle):
    g = _golden("ref_dense_lu.npz")
    F = oracle.dense_getrf(g["A"])
    assert np.array_equal(F, g["LU"]), "oracle LU differs from the reference kernel's output"


def test_golden_block_routines_match_reference_kernel(oracle):
    g = _golden("ref_routines.npz")
    # gemm (M -= A B) and gemm_plus (M += A B^T) as run by kernel_dynamic
    M = g["M0"].copy()
    oracle.gemm(-1.0, 1.0, M, g["A"], g["B"])
    assert np.array_equal(M, g["M_gemm"])
    M = g["M0"].copy()
    oracle.gemm(1.0, 1.0, M, g["A"], g["Bt"], False, True)
    assert np.array_equal(M, g["M_gemm_plus_bT"])


def test_golden_accum_matches_reference_kernel(oracle):
    g = _golden("ref_accum.npz")
    U1, V1 = g["U1"].copy(), g["V1"].copy()
    oracle.accum(U1, V1, g["U2"], g["V2"], g["R"])
    want = g["U1_out"] @ g["V1_out"].T
    assert np.linalg.norm(U1 @ V1.T - want) / np.linalg.norm(want) < 1e-12


def test_standard_admissibility_program_solves(pp, oracle, hctx):
    """The sketched updates of standard admissibility (products of hierarchical blocks into
    low-rank blocks) give a factorization whose solve is accurate (oracle executor)."""
    n = 2048
    h, prob = pp.make_kernel_problem(hctx, n, 2, "laplace", 1e-3, 64, 16, admissibility=1, eta=1.0, seed=3)
    assert h.program_info(0)["op_count"]["orth"] > 0
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=4)
    b = pp.rhs(n, 1)
    sol = oracle.HostArenas(h, 1, 1, rhs=b)
    sol.matrix[:] = ar.matrix
    sol.tasks, sol.succ, sol.indeg, sol.ready = h.encode_program(1, 1, sol.bases())
    sol.run()
    x = sol.rhs[:n].reshape(n, 1)
    r = b - prob.dense() @ x
    assert np.abs(r).max() / (prob.norm_inf * np.abs(x).max() + np.abs(b).max()) < 1e-6


def test_trmv_row_block_restatement(pp, oracle):
    """The oracle's TRMV against numpy: the whole product in place, and rows [o, o + l) of it
    out of place (the parts of a split solve step), for both triangles."""
    rng = np.random.default_rng(3)
    m, n = 200, 3
    M = rng.standard_normal((m, m + 2))
    B = rng.standard_normal((m, n + 1))

    def run(**fields):
        t = np.zeros(1, dtype=pp.TASK_DTYPE)
        for k, v in fields.items():
            if k in ("p", "ld"):
                for i, x in enumerate(v):
                    t[0][k][i] = x
            else:
                t[0][k] = v
        assert oracle.lib().oracle_run_program(t.ctypes.data, 1) == 0

    for upper in (0, 1):
        T = np.triu(M[:, :m]) if upper else np.tril(M[:, :m])
        want = T @ B[:, :n]
        for r0, l in ((0, 64), (64, 70), (150, 50)):
            O = np.zeros((l, n + 2))
            run(op=12, m=m, n=n, ctrl=upper, o=r0, l=l, p=[O.ctypes.data, M.ctypes.data, B.ctypes.data],
                ld=[n + 2, m + 2, n + 1])
            assert np.allclose(O[:, :n], want[r0:r0 + l], rtol=1e-13, atol=1e-12)
            assert not O[:, n:].any()
        Bc = B.copy()
        run(op=12, m=m, n=n, ctrl=upper, p=[Bc.ctypes.data, M.ctypes.data], ld=[n + 1, m + 2])
        assert np.allclose(Bc[:, :n], want, rtol=1e-13, atol=1e-12)
        assert np.array_equal(Bc[:, n:], B[:, n:])
