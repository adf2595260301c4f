"""TEST ORACLE — numpy restatement of the batched GMRES kernels (engine csrc/krylov.cu).

Test infrastructure only (tests/ import it; the product never does).  The reference has no
solve or refinement path, so there is nothing of it to follow here: this restates the
textbook restarted GMRES with classical Gram-Schmidt and one re-orthogonalisation pass
(CGS2) and Givens rotations on the Hessenberg columns, in the state layout the kernels use,
so a test can feed both the same vectors and compare every state word.

State of one instance (m = restart length), as csrc/krylov.cu stores it:
  H  (m + 1) x m column-major, cs (m), sn (m), g (m + 1),
  meta = [active dimension, frozen flag, beta, |g_k|].
"""
from __future__ import annotations

import numpy as np


class GmresState:
    def __init__(self, n, m):
        self.n, self.m = n, m
        self.V = np.zeros((m + 1, n))
        self.Z = np.zeros((m, n))
        self.H = np.zeros((m, m + 1))  # row c = column c of the Hessenberg matrix
        self.cs = np.zeros(m)
        self.sn = np.zeros(m)
        self.g = np.zeros(m + 1)
        self.meta = np.zeros(4)

    def flat(self):
        """The state words in the kernels' order."""
        return np.concatenate([self.H.ravel(), self.cs, self.sn, self.g, self.meta])


def start(S: GmresState, r):
    beta = float(np.sqrt(np.dot(r, r)))
    ok = beta > 0.0 and np.isfinite(beta)
    S.V[0] = r / beta if ok else 0.0
    S.g[:] = 0.0
    if ok:
        S.g[0] = beta
    S.meta[:] = [0.0, 0.0 if ok else 1.0, beta, beta if ok else 0.0]


def arnoldi(S: GmresState, j, Az):
    """Step j with w = A z_j given directly (the kernel receives -A z_j)."""
    if S.meta[1] != 0.0:
        S.V[j + 1] = 0.0
        return
    w = np.array(Az, dtype=np.float64)
    h = np.zeros(j + 1)
    for _ in range(2):
        hp = S.V[: j + 1] @ w
        w = w - hp @ S.V[: j + 1]
        h += hp
    hn = float(np.sqrt(np.dot(w, w)))
    col = S.H[j]
    col[: j + 1] = h
    for i in range(j):
        a, b = col[i], col[i + 1]
        col[i] = S.cs[i] * a + S.sn[i] * b
        col[i + 1] = -S.sn[i] * a + S.cs[i] * b
    a = col[j]
    r = float(np.hypot(a, hn))
    if r > 0.0 and np.isfinite(r):
        c, s = a / r, hn / r
        S.cs[j], S.sn[j] = c, s
        col[j], col[j + 1] = r, 0.0
        S.g[j + 1] = -s * S.g[j]
        S.g[j] = c * S.g[j]
        S.meta[0] = j + 1
        S.meta[3] = abs(S.g[j + 1])
        if hn > 1e-300:
            S.V[j + 1] = w / hn
            return
    S.meta[1] = 1.0
    S.V[j + 1] = 0.0


def finish(S: GmresState, x):
    k = int(S.meta[0])
    y = np.zeros(k)
    for i in range(k - 1, -1, -1):
        t = S.g[i] - sum(S.H[c, i] * y[c] for c in range(i + 1, k))
        y[i] = t / S.H[i, i]
    return x + y @ S.Z[:k] if k else x.copy()


def gmres(A, b, M_solve, m=30, tol=1e-12, max_cycles=50):
    """Restarted right-preconditioned GMRES on a dense A (float64); returns (x, backward
    errors after each cycle).  M_solve(v) applies the preconditioner."""
    n = len(b)
    x = np.zeros(n)
    S = GmresState(n, m)
    hist = []
    nA = np.abs(A).sum(axis=1).max()
    for _ in range(max_cycles):
        r = b - A @ x
        start(S, r)
        for j in range(m):
            S.Z[j] = M_solve(S.V[j])
            arnoldi(S, j, A @ S.Z[j])
        x = finish(S, x)
        r = b - A @ x
        e = np.abs(r).max() / (nA * np.abs(x).max() + np.abs(b).max())
        hist.append(e)
        if e <= tol:
            break
    return x, hist
