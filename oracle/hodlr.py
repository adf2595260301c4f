"""TEST ORACLE — the reference's factor path on the CPU, for the timed reference arm and the CPU
baseline of bench.py.  Test infrastructure only; it neither imports nor loads the engine.

What runs:
  * the matrix, built here from its recipe (seeded points, Morton order, kernel entries, diagonal
    shift, truncated-SVD low-rank blocks): the same construction steps as the engine's problem
    helpers, restated in numpy;
  * the factorization program exported once to a fixture (tests/golden/make_refisa_program.py):
    the reference's instruction set only (getrf / trsml / trsmr / gemm / gemm_plus / gemm_3x /
    gemm_4x / accum, the operations of src/kernel.cu:1404-1501), executed by liboracle.so's
    restatement of the reference's block routines (src/kernel.cu:104-955, 1160-1280) over the
    program's DAG with host threads;
  * the solve: forward and backward substitution over the factored block tree (dense leaves by
    triangular solves, low-rank and hierarchical blocks by their products), written here: the
    reference has no solve;
  * FP64 iterative refinement against the dense matrix until the normwise backward error
    ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) meets the tolerance.
"""
from __future__ import annotations

import os

import numpy as np

from . import lib

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(os.path.dirname(HERE), "tests", "golden", "hodlr8192_refisa_program.npz")

# pp_task.h record layout (160 bytes), as numpy sees it
TASK_DTYPE = np.dtype(
    [("op", "<i4"), ("flags", "<i4"), ("m", "<i4"), ("n", "<i4"), ("k", "<i4"), ("l", "<i4"), ("o", "<i4"),
     ("ctrl", "<i4"), ("ld", "<i4", 6), ("p", "<u8", 6), ("tmp", "<u8"), ("alpha", "<f8"), ("beta", "<f8"),
     ("succ_begin", "<i4"), ("n_succ", "<i4"), ("prec", "<i4"), ("instance", "<i4"), ("aux", "<i4"),
     ("pad", "<i4", 3)])
assert TASK_DTYPE.itemsize == 160

DENSE, LOWRANK, HIER = 0, 1, 2


# ----------------------------------------------------------------------------- construction
def kernel_eval(kind, d, p0):
    """0: 1/(r + p0); 1: Laplace 1/(4 pi (r + p0)); 2: exp(-r / p0); 3: Matern-3/2, length p0."""
    if kind == 0:
        return 1.0 / (d + p0)
    if kind == 1:
        return 1.0 / (4.0 * np.pi * (d + p0))
    if kind == 2:
        return np.exp(-d / p0)
    s = np.sqrt(3.0) * d / p0
    return (1.0 + s) * np.exp(-s)


def distances(X, Y):
    from scipy.spatial.distance import cdist
    return cdist(X, Y)


def morton_order(pts):
    """Z-order of points in [0,1]^d: 21 bits per coordinate, bits interleaved low to high."""
    n, dim = pts.shape
    bits = 21 if dim <= 3 else 10
    q = np.clip((pts * (1 << bits)).astype(np.uint64), 0, (1 << bits) - 1)
    key = np.zeros(n, dtype=np.uint64)
    for b in range(bits):
        for d in range(dim):
            key |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + d)
    return np.argsort(key, kind="stable")


def offdiag_rowsum_max(pts, kind, p0, block=2048):
    n = pts.shape[0]
    best = 0.0
    for i0 in range(0, n, block):
        X = pts[i0:i0 + block]
        s = np.zeros(X.shape[0])
        for j0 in range(0, n, block):
            K = np.abs(kernel_eval(kind, distances(X, pts[j0:j0 + block]), p0))
            if i0 == j0:
                np.fill_diagonal(K, 0.0)
            s += K.sum(1)
        best = max(best, float(s.max()))
    return best


def truncated_svd(A, k, rng):
    """Rank-k truncation of A as (U * s, V): exact SVD for small blocks, else a randomized range
    finder (oversampling 10, two power iterations) and the SVD of the projection."""
    m, n = A.shape
    k = min(k, m, n)
    if min(m, n) <= 2 * k + 16:
        u, s, vt = np.linalg.svd(A, full_matrices=False)
        return u[:, :k] * s[:k], vt[:k].T.copy()
    p = min(k + 10, min(m, n))
    Y = A @ rng.standard_normal((n, p))
    Q, _ = np.linalg.qr(Y)
    for _ in range(2):
        Q, _ = np.linalg.qr(A.T @ Q)
        Q, _ = np.linalg.qr(A @ Q)
    ub, s, vt = np.linalg.svd(Q.T @ A, full_matrices=False)
    return (Q @ ub[:, :k]) * s[:k], vt[:k].T.copy()


def splitmix_uniform(seed, count):
    """count uniforms in [-1, 1) from the splitmix64 sequence of `seed` (53 random bits each):
    the random sketch the accumulations read."""
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + (np.arange(1, count + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        z = (s ^ (s >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = (z ^ (z >> np.uint64(31))) & M
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


# ----------------------------------------------------------------------------- the job
class FixtureJob:
    """One factor + solve job of the exported configuration on the host cores."""

    def __init__(self, path=FIXTURE):
        z = np.load(path)
        self.meta = {str(k): float(v) for k, v in zip(z["meta_keys"], z["meta_vals"])}
        m = self.meta
        self.n = int(m["n"])
        self.tasks_tagged = z["tasks"].reshape(-1).view(TASK_DTYPE).copy()
        self.succ = np.ascontiguousarray(z["succ"], dtype=np.int32)
        self.indeg = np.ascontiguousarray(z["indeg"], dtype=np.int32)
        self.blocks = z["blocks"]
        self.root = int(m["root"])
        self.flops = int(m["flops"])
        self.tol = 1e-10
        self._build_matrix()
        self.work = np.zeros(max(int(m["work_elems"]), 1))
        self.scratch = np.zeros(max(int(m["scratch_elems"]), 1))
        self.rhs = np.zeros(max(int(m["rhs_elems"]), 1))
        self.rand = splitmix_uniform(int(m["rand_seed"]), max(int(m["rand_elems"]), 1))
        self.tasks = self._bind()

    # construction: the recipe of the exported configuration
    def _build_matrix(self):
        m = self.meta
        n, dim, kind, p0 = self.n, int(m["dim"]), int(m["kernel"]), m["p0"]
        seed = int(m["seed"])
        pts = np.random.default_rng(seed).uniform(0.0, 1.0, (n, dim))
        self.points = pts[morton_order(pts)]
        off = offdiag_rowsum_max(self.points, kind, p0)
        self.shift = m["shift_factor"] * off
        self.norm_inf = float(kernel_eval(kind, 0.0, p0)) + self.shift + off
        self.original = np.zeros(int(m["matrix_elems"]))
        rng = np.random.default_rng(seed + 1)
        for kd, r0, c0, bm, bn, kmax, rank, o, ov, orank, *_ in self.blocks:
            if kd == HIER:
                continue
            A = self.entries(r0, bm, c0, bn)
            if kd == DENSE:
                self.original[o:o + bm * bn] = A.ravel()
                continue
            U, V = truncated_svd(A, int(kmax), rng)
            Uf, Vf = np.zeros((bm, kmax)), np.zeros((bn, kmax))
            Uf[:, :U.shape[1]] = U
            Vf[:, :V.shape[1]] = V
            self.original[o:o + bm * kmax] = Uf.ravel()
            self.original[ov:ov + bn * kmax] = Vf.ravel()
            if orank >= 0:
                self.original[orank] = U.shape[1]
        self.matrix = self.original.copy()

    def entries(self, r0, m, c0, n):
        A = kernel_eval(int(self.meta["kernel"]), distances(self.points[r0:r0 + m], self.points[c0:c0 + n]),
                        self.meta["p0"])
        ri = np.arange(r0, r0 + m)[:, None]
        ci = np.arange(c0, c0 + n)[None, :]
        return A + self.shift * (ri == ci)

    def dense(self):
        return self.entries(0, self.n, 0, self.n)

    def _bind(self):
        """Task records with the tagged operand pointers replaced by host addresses."""
        t = self.tasks_tagged.copy()
        shift = np.uint64(int(self.meta["tag_shift"]))
        mask = np.uint64((1 << int(self.meta["tag_shift"])) - 1)
        bases = [a.ctypes.data for a in (self.matrix, self.work, self.scratch, self.rhs, self.rand)]
        for field in ("p", "tmp"):
            p = t[field]
            live = p != 0
            kind = (p >> shift).astype(np.int64) - 1
            if np.any(live & ((kind < 0) | (kind > 4))):
                raise ValueError("fixture: operand pointer outside the tagged arenas")
            addr = np.zeros_like(p)
            for a in range(5):
                sel = live & (kind == a)
                addr[sel] = np.uint64(bases[a]) + (p[sel] & mask)
            t[field] = addr
        return t

    # factorization: the exported program over its DAG
    def restore(self):
        self.matrix[:] = self.original

    def factor(self, threads=None):
        threads = threads or os.cpu_count() or 1
        self.work[:] = 0.0
        rc = lib().oracle_run_parallel(self.tasks.ctypes.data, len(self.tasks), self.succ.ctypes.data,
                                       self.indeg.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError(f"oracle: task {rc - 1} unsupported")

    # solve: substitution over the factored block tree
    def _blk(self, b):
        return self.blocks[b]

    def _apply(self, b, x):
        """A_b x for a block of the factored matrix (its stored, not its original, data)."""
        kd, r0, c0, bm, bn, kmax, rank, o, ov, orank = self.blocks[b][:10]
        if kd == DENSE:
            return self.matrix[o:o + bm * bn].reshape(bm, bn) @ x
        if kd == LOWRANK:
            r = int(self.matrix[orank]) if orank >= 0 else int(rank)
            U = self.matrix[o:o + bm * kmax].reshape(bm, kmax)[:, :r]
            V = self.matrix[ov:ov + bn * kmax].reshape(bn, kmax)[:, :r]
            return U @ (V.T @ x)
        ch = self.blocks[b][10:14]
        out = np.zeros((bm, x.shape[1]))
        for i in range(2):
            for j in range(2):
                c = self.blocks[ch[2 * i + j]]
                rr, cc = c[1] - r0, c[2] - c0
                out[rr:rr + c[3]] += self._apply(ch[2 * i + j], x[cc:cc + c[4]])
        return out

    def _lower(self, b, x):
        """x := L_b^-1 x in place (unit lower triangle of a diagonal block)."""
        from scipy.linalg import solve_triangular
        kd, r0, c0, bm, bn, kmax, rank, o = self.blocks[b][:8]
        if kd == DENSE:
            x[:] = solve_triangular(self.matrix[o:o + bm * bn].reshape(bm, bn), x, lower=True, unit_diagonal=True)
            return
        ch = self.blocks[b][10:14]
        s = self.blocks[ch[0]][3]
        self._lower(ch[0], x[:s])
        x[s:] -= self._apply(ch[2], x[:s])
        self._lower(ch[3], x[s:])

    def _upper(self, b, x):
        """x := U_b^-1 x in place (upper triangle with the diagonal)."""
        from scipy.linalg import solve_triangular
        kd, r0, c0, bm, bn, kmax, rank, o = self.blocks[b][:8]
        if kd == DENSE:
            x[:] = solve_triangular(self.matrix[o:o + bm * bn].reshape(bm, bn), x, lower=False)
            return
        ch = self.blocks[b][10:14]
        s = self.blocks[ch[0]][3]
        self._upper(ch[3], x[s:])
        x[:s] -= self._apply(ch[1], x[s:])
        self._upper(ch[0], x[:s])

    def solve(self, b):
        x = np.array(b, dtype=np.float64, copy=True).reshape(self.n, -1)
        self._lower(self.root, x)
        self._upper(self.root, x)
        return x

    def factor_solve(self, b, A, tol=None, max_iter=30, threads=None):
        """restore + factor + solve + FP64 refinement against A until the backward error meets
        tol; returns (x, backward errors per solve)."""
        tol = self.tol if tol is None else tol
        self.restore()
        self.factor(threads)
        b = np.asarray(b, dtype=np.float64).reshape(self.n, -1)
        x = np.zeros_like(b)
        r = b.copy()
        bn = np.abs(b).max()
        hist = []
        for _ in range(max_iter):
            x += self.solve(r)
            r = b - A @ x
            hist.append(float(np.abs(r).max() / (self.norm_inf * np.abs(x).max() + bn)))
            if hist[-1] <= tol:
                break
        return x, hist
