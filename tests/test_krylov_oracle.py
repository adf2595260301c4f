"""The numpy GMRES restatement (oracle/krylov.py) that the GPU kernels are checked against:
on a dense system with a deliberately coarse preconditioner (so plain refinement diverges)
it reaches the tolerance, and its least-squares estimate equals the true residual norm."""
import numpy as np
import scipy.linalg as sl

from oracle import krylov as K


def test_restatement_solves_with_a_coarse_preconditioner():
    rng = np.random.default_rng(3)
    n = 300
    A = np.eye(n) * 3.0 + rng.uniform(-1, 1, (n, n)) / np.sqrt(n)
    P = A + rng.uniform(-1, 1, (n, n)) * 0.05  # a coarse approximation of A
    lu = sl.lu_factor(P)
    E = np.linalg.solve(P, A) - np.eye(n)
    b = rng.uniform(-1, 1, n)
    x, hist = K.gmres(A, b, lambda v: sl.lu_solve(lu, v), m=20, tol=1e-13, max_cycles=10)
    assert hist[-1] <= 1e-13
    assert np.linalg.norm(x - np.linalg.solve(A, b)) <= 1e-10 * np.linalg.norm(x)
    assert max(abs(np.linalg.eigvals(E))) > 0.1  # the preconditioner really is coarse


def test_estimate_is_the_residual_norm():
    rng = np.random.default_rng(4)
    n, m = 120, 15
    A = np.eye(n) * 2.0 + rng.uniform(-1, 1, (n, n)) / np.sqrt(n)
    b = rng.uniform(-1, 1, n)
    S = K.GmresState(n, m)
    K.start(S, b)
    for j in range(m):
        S.Z[j] = S.V[j]
        K.arnoldi(S, j, A @ S.Z[j])
        x = K.finish(S, np.zeros(n))
        assert abs(np.linalg.norm(b - A @ x) - S.meta[3]) <= 1e-12 * np.linalg.norm(b)
    # orthonormal basis
    G = S.V @ S.V.T
    assert np.abs(G - np.eye(m + 1)).max() <= 1e-12


def test_zero_residual_freezes():
    S = K.GmresState(10, 4)
    K.start(S, np.zeros(10))
    assert S.meta[1] == 1.0 and S.meta[0] == 0
    K.arnoldi(S, 0, np.ones(10))
    assert np.array_equal(K.finish(S, np.ones(10)), np.ones(10))


def test_perturbed_products_inside_cycles_still_converge():
    """Products inside a cycle with a relative error of 1e-7 (what FP32-evaluated kernel
    entries give): each cycle stalls near that error times the conditioning, but the FP64
    residual at the restart carries the answer on, so restarted GMRES still reaches 1e-12."""
    import scipy.linalg as sl
    rng = np.random.default_rng(8)
    n = 400
    A = np.eye(n) * 3.0 + rng.uniform(-1, 1, (n, n)) / np.sqrt(n)
    E = rng.uniform(-1, 1, (n, n)) * 1e-7 * np.abs(A)  # entry-wise relative perturbation
    P = A + rng.uniform(-1, 1, (n, n)) * 0.05
    lu = sl.lu_factor(P)
    b = rng.uniform(-1, 1, n)
    x = np.zeros(n)
    S = K.GmresState(n, 30)
    nA = np.abs(A).sum(axis=1).max()
    hist = []
    for _ in range(6):
        r = b - A @ x  # FP64 residual with the exact operator
        K.start(S, r)
        for j in range(30):
            S.Z[j] = sl.lu_solve(lu, S.V[j])
            K.arnoldi(S, j, (A + E) @ S.Z[j])  # the cycle's products: perturbed
        x = K.finish(S, x)
        hist.append(np.abs(b - A @ x).max() / (nA * np.abs(x).max() + np.abs(b).max()))
    assert hist[0] > 1e-10  # one cycle stalls at the products' error level
    assert hist[-1] <= 1e-12, hist
