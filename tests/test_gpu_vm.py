"""GPU parity of the persistent VM (sm_100a) against the oracle and the reference kernel.

Bar: dense instructions bitwise equal to the oracle (= the reference's update order);
programs containing the randomized accumulation within 1e-12 relative (Frobenius) of the
oracle and of the reference's own kernel_dynamic on the same instruction stream.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


# ----------------------------------------------------------------------------- single tasks
class TaskBench:
    """Builds one-task tables twice: device operands for the VM, host operands for the oracle."""

    def __init__(self, pp, seed=0):
        self.pp = pp
        self.rng = np.random.default_rng(seed)
        self.host, self.devs = [], []

    def operand(self, rows, cols, kind="normal", ld_pad=3):
        ld = cols + ld_pad
        a = self.rng.standard_normal((rows, ld)) if kind == "normal" else self.rng.uniform(-1, 1, (rows, ld))
        if kind == "diag":
            a[:, :cols] += np.eye(rows, cols) * (2 * max(rows, cols))
        self.host.append(a)
        self.devs.append(dev(a))
        return len(self.host) - 1, ld

    def run(self, gctx, oracle, fields, slots, tmp_elems=0):
        pp = self.pp
        t_dev = np.zeros(1, dtype=pp.TASK_DTYPE)
        t_host = np.zeros(1, dtype=pp.TASK_DTYPE)
        for k, v in fields.items():
            t_dev[0][k] = v
            t_host[0][k] = v
        for s, (idx, ld) in slots.items():
            t_dev[0]["p"][s] = self.devs[idx].data_ptr()
            t_host[0]["p"][s] = self.host[idx].ctypes.data
            t_dev[0]["ld"][s] = ld
            t_host[0]["ld"][s] = ld
        if tmp_elems:
            td = torch.zeros(tmp_elems, dtype=torch.float64, device="cuda")
            th = np.zeros(tmp_elems)
            t_dev[0]["tmp"] = td.data_ptr()
            t_host[0]["tmp"] = th.ctypes.data
        gctx.vm_execute(t_dev, np.zeros(0, np.int32), np.zeros(1, np.int32))
        rc = oracle.lib().oracle_run_program(t_host.ctypes.data, 1)
        assert rc == 0
        return [(d.cpu().numpy(), h) for d, h in zip(self.devs, self.host)]


@pytest.mark.parametrize("tA,tB", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (1.0, 1.0), (1.0, 0.0)])
@pytest.mark.parametrize("m,n,k", [(64, 64, 64), (37, 91, 130), (256, 16, 16), (5, 3, 0), (128, 128, 16),
                                   (130, 140, 20), (200, 256, 9)])
def test_gemm_task_bitwise(pp, oracle, gctx, tA, tB, alpha, beta, m, n, k):
    tb = TaskBench(pp, seed=m * 7 + n)
    c = tb.operand(m, n)
    a = tb.operand(k, m) if tA else tb.operand(m, k)
    b = tb.operand(n, k) if tB else tb.operand(k, n)
    flags = (tA << 5) | (tB << 6)
    out = tb.run(gctx, oracle, dict(op=6, flags=flags, m=m, n=n, k=k, alpha=alpha, beta=beta), {0: c, 1: a, 2: b})
    d, h = out[c[0]]
    assert np.array_equal(d, h)


@pytest.mark.parametrize("m,n", [(64, 64), (37, 50), (1, 1), (64, 17)])
def test_getrf_task_bitwise(pp, oracle, gctx, m, n):
    tb = TaskBench(pp, seed=m + n)
    a = tb.operand(m, n, kind="diag")
    d, h = tb.run(gctx, oracle, dict(op=1, m=m, n=n), {0: a})[a[0]]
    assert np.array_equal(d, h)


@pytest.mark.parametrize("tA,tB", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (1.0, 0.0)])
@pytest.mark.parametrize("m,n,k", [(64, 64, 16), (256, 16, 16), (37, 91, 130), (64, 16, 64)])
def test_gemm_task_free_order(pp, oracle, gctx, tA, tB, alpha, beta, m, n, k):
    """GEMM with the free-order flag (products into work buffers): within rounding of the
    oracle's ascending-k sum."""
    tb = TaskBench(pp, seed=m * 7 + n + k)
    c = tb.operand(m, n)
    a = tb.operand(k, m) if tA else tb.operand(m, k)
    b = tb.operand(n, k) if tB else tb.operand(k, n)
    flags = 1 | (16 << 1 if tA else 0) | (16 << 2 if tB else 0)
    d, h = tb.run(gctx, oracle, dict(op=6, flags=flags, m=m, n=n, k=k, alpha=alpha, beta=beta), {0: c, 1: a, 2: b})[c[0]]
    assert rel(d[:, :n], h[:, :n]) < 1e-14
    assert np.array_equal(d[:, n:], h[:, n:])  # the padding columns are untouched


@pytest.mark.parametrize("op", [2, 3, 4, 5])
@pytest.mark.parametrize("m,n", [(64, 16), (64, 64), (33, 70), (1, 5)])
def test_triangular_tasks_bitwise(pp, oracle, gctx, op, m, n):
    tb = TaskBench(pp, seed=op * 100 + m)
    tri = n if op == 3 else m  # trsmr: U is n x n; others: m x m
    if op == 3 and n > 64:
        pytest.skip("trsmr keeps U (n x n) in shared memory: n <= 64")
    b = tb.operand(m, n)
    t = tb.operand(tri, tri, kind="diag")
    d, h = tb.run(gctx, oracle, dict(op=op, m=m, n=n), {0: b, 1: t})[b[0]]
    assert np.array_equal(d, h)


@pytest.mark.parametrize("upper", [0, 1])
@pytest.mark.parametrize("m,c0,w", [(256, 0, 64), (256, 192, 64), (128, 64, 64), (40, 0, 40)])
def test_trinv_task(pp, oracle, gctx, upper, m, c0, w):
    """TRINV: a column block of L^-1 / U^-1 of a factored leaf, against the oracle and
    against numpy's inverse of the triangular factor."""
    tb = TaskBench(pp, seed=7 * m + c0)
    a = tb.operand(m, m, kind="diag")
    inv = tb.operand(m, m)  # the whole inverse object; the task writes one column block
    res = tb.run(gctx, oracle, dict(op=11, m=m, n=w, o=c0, ctrl=upper), {0: (inv[0], inv[1]), 1: a})
    A = tb.host[a[0]][:, :m]
    d, h = res[inv[0]]
    blk_d, blk_h = d[:, :w], h[:, :w]
    assert rel(blk_d, blk_h) < 1e-13
    T = np.triu(A) if upper else np.tril(A, -1) + np.eye(m)
    assert rel(blk_d, np.linalg.inv(T)[:, c0:c0 + w]) < 1e-10


@pytest.mark.parametrize("upper", [0, 1])
@pytest.mark.parametrize("m,n", [(256, 1), (256, 3), (128, 16), (37, 2)])
def test_trmv_task(pp, oracle, gctx, upper, m, n):
    """TRMV: B := M B with M triangular, against the oracle and numpy."""
    tb = TaskBench(pp, seed=11 * m + n)
    b = tb.operand(m, n)
    mm = tb.operand(m, m)
    B0 = tb.host[b[0]][:, :n].copy()
    M = tb.host[mm[0]][:, :m]
    d, h = tb.run(gctx, oracle, dict(op=12, m=m, n=n, ctrl=upper), {0: b, 1: mm})[b[0]]
    T = np.triu(M) if upper else np.tril(M)
    assert rel(d[:, :n], h[:, :n]) < 1e-14
    assert rel(d[:, :n], T @ B0) < 1e-13


@pytest.mark.parametrize("upper", [0, 1])
@pytest.mark.parametrize("m,n,r0,l", [(256, 1, 0, 128), (256, 1, 181, 41), (256, 3, 222, 34), (200, 16, 17, 100)])
def test_trmv_task_row_block_bitwise(pp, oracle, gctx, upper, m, n, r0, l):
    """TRMV rows [o, o + l) out of place (one part of a split solve step): the same bits as
    those rows of the whole in-place product, the oracle within rounding, the source intact."""
    rng = np.random.default_rng(m + n + r0 + upper)
    M0, B0 = rng.standard_normal((m, m)), rng.standard_normal((m, n))

    def setup(tb, pairs):
        for (idx, _), val in pairs:
            tb.host[idx][:, :val.shape[1]] = val
            tb.devs[idx].copy_(torch.from_numpy(tb.host[idx]))

    tb = TaskBench(pp, seed=1)
    b, mm = tb.operand(m, n), tb.operand(m, m)
    setup(tb, [(b, B0), (mm, M0)])
    full, _ = tb.run(gctx, oracle, dict(op=12, m=m, n=n, ctrl=upper), {0: b, 1: mm})[b[0]]
    tb2 = TaskBench(pp, seed=2)
    o, s, mm2 = tb2.operand(l, n), tb2.operand(m, n), tb2.operand(m, m)
    setup(tb2, [(s, B0), (mm2, M0)])
    out = tb2.run(gctx, oracle, dict(op=12, m=m, n=n, ctrl=upper, o=r0, l=l), {0: o, 1: mm2, 2: s})
    d, h = out[o[0]]
    assert np.array_equal(d[:, :n], full[r0:r0 + l, :n])
    assert rel(d[:, :n], h[:, :n]) < 1e-14
    assert np.array_equal(out[s[0]][0][:, :n], B0)


@pytest.mark.parametrize("ctrl", [0, 1])
def test_gemm3_task_bitwise(pp, oracle, gctx, ctrl):
    tb = TaskBench(pp, seed=ctrl + 50)
    m, n, k, l = 70, 40, 16, 90
    c, a, b, d_ = tb.operand(m, n), tb.operand(m, k), tb.operand(k, l), tb.operand(l, n)
    out = tb.run(gctx, oracle, dict(op=7, m=m, n=n, k=k, l=l, ctrl=ctrl, alpha=-1.0, beta=1.0),
                 {0: c, 1: a, 2: b, 3: d_}, tmp_elems=max(m * l, k * n))
    d, h = out[c[0]]
    assert np.array_equal(d, h)


@pytest.mark.parametrize("ctrl", [0, 1, 2, 3, 4])
def test_gemm4_task_bitwise(pp, oracle, gctx, ctrl):
    tb = TaskBench(pp, seed=ctrl + 60)
    m, n, k, l, o = 48, 40, 16, 80, 12
    c = tb.operand(m, n)
    a, b, cc, dd = tb.operand(m, k), tb.operand(k, l), tb.operand(l, o), tb.operand(o, n)
    big = max(m, k, l) * max(n, l, o)
    out = tb.run(gctx, oracle, dict(op=8, m=m, n=n, k=k, l=l, o=o, ctrl=ctrl, alpha=-1.0, beta=1.0, aux=big),
                 {0: c, 1: a, 2: b, 3: cc, 4: dd}, tmp_elems=2 * big)
    d, h = out[c[0]]
    assert np.array_equal(d, h)


@pytest.mark.parametrize("ny,nx,k1,k2,sign", [(300, 260, 16, 16, 1.0), (129, 64, 8, 24, 1.0), (64, 512, 16, 16, -1.0)])
def test_accum_task_matches_reference_algorithm(pp, oracle, gctx, ny, nx, k1, k2, sign):
    tb = TaskBench(pp, seed=ny + nx)
    u1, v1, u2, v2 = tb.operand(ny, k1), tb.operand(nx, k1), tb.operand(ny, k2), tb.operand(nx, k2)
    r = tb.operand(nx, k1, kind="uniform", ld_pad=0)
    A0 = tb.host[u1[0]][:, :k1] @ tb.host[v1[0]][:, :k1].T + sign * tb.host[u2[0]][:, :k2] @ tb.host[v2[0]][:, :k2].T
    tmp = 2 * ny * k1 + nx * k1 + k1 * max(k1, k2)
    out = tb.run(gctx, oracle, dict(op=9, m=ny, n=nx, k=k1, l=k2, alpha=sign), {0: u1, 1: v1, 2: u2, 3: v2, 4: r},
                 tmp_elems=tmp)
    Ud, Uh = out[u1[0]]
    Vd, Vh = out[v1[0]]
    Pd = Ud[:, :k1] @ Vd[:, :k1].T
    Ph = Uh[:, :k1] @ Vh[:, :k1].T
    assert rel(Pd, Ph) < 1e-12
    Q, _ = np.linalg.qr(A0 @ tb.host[r[0]][:, :k1])
    assert rel(Pd, Q @ (Q.T @ A0)) < 1e-12
    assert np.allclose(Ud[:, :k1].T @ Ud[:, :k1], np.eye(k1), atol=1e-12)


# ----------------------------------------------------------------------------- programs
def factor_on_gpu(h, grid_blocks=0):
    h.upload()
    if grid_blocks:
        import importlib
        pp = importlib.import_module("pastel_palettes_b200")
        pp.dev_hierarchical_GETRF(h, grid_blocks, 256, 0)
    else:
        h.factor()
        h.sync()
    h.download()
    return h.to_dense()


def test_dense_config1_bitwise_vs_textbook_lu(pp, oracle, gctx):
    h, A = pp.make_dense_problem(gctx, n=1024, leaf=256)
    assert np.array_equal(factor_on_gpu(h), oracle.dense_getrf(A))


def test_single_cta_equals_full_grid(pp, gctx):
    h1, _ = pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16)
    h2, _ = pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16)
    F1 = factor_on_gpu(h1)
    F2 = factor_on_gpu(h2, grid_blocks=1)
    assert np.array_equal(F1, F2)


def test_hodlr_factor_matches_oracle(pp, oracle, gctx):
    h, prob = pp.make_kernel_problem(gctx, 2048, 2, "inv", 1e-3, 256, 16)
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=8)
    F = factor_on_gpu(h)
    h.host_arena()[:] = ar.matrix
    assert rel(F, h.to_dense()) < 1e-12


def test_gemm_tile_128_factor_bitwise(pp, gctx):
    """Products split into 128 x 128 output tiles: fewer GEMM instructions, the same bits (each
    element keeps its ascending-k chain and the DAG keeps the update order)."""
    h1, _ = pp.make_kernel_problem(gctx, 2048, 2, "inv", 1e-3, 256, 16)
    h2, _ = pp.make_kernel_problem(gctx, 2048, 2, "inv", 1e-3, 256, 16)
    h2.set_gemm_tile(128)
    with pytest.raises(pp.PPError):
        h2.set_gemm_tile(96)
    F1 = factor_on_gpu(h1)
    F2 = factor_on_gpu(h2)
    assert h2.program_info(0)["n_tasks"] < h1.program_info(0)["n_tasks"]
    assert np.array_equal(F1, F2)


def run_reference_kernel(pp, oracle, h):
    """The reference's kernel_dynamic (1 worker) on the reference-format stream of h."""
    ref = oracle.ref_vm()
    if ref is None:
        pytest.skip("reference kernel not built")
    words, lengths, tmp = h.refstreams(1)
    info = h.program_info(0)
    el = info["arena_elems"]
    arena = dev(h.host_arena())
    work = torch.zeros(max(el["work"], 1), dtype=torch.float64, device="cuda")
    scratch = torch.zeros(max(el["scratch"], 1), dtype=torch.float64, device="cuda")
    rhs = torch.zeros(max(el["rhs"], 1), dtype=torch.float64, device="cuda")
    rnd = dev(h.rand_host() if el["rand"] else np.zeros(1))
    import ctypes as C
    ptrs = (C.c_void_p * 5)(*[C.c_void_p(t.data_ptr()) for t in (arena, work, scratch, rhs, rnd)])
    words = np.ascontiguousarray(words, dtype=np.int32)
    lengths = np.ascontiguousarray(lengths, dtype=np.int32)
    rc = ref.ref_vm_run(1, words.ctypes.data, lengths.ctypes.data, C.cast(ptrs, C.c_void_p), 5, info["n_tasks"],
                        rnd.data_ptr(), max(tmp, 1), 256)
    assert rc == 0, f"reference kernel failed: cuda error {rc}"
    out = arena.cpu().numpy()
    saved = h.host_arena().copy()
    h.host_arena()[:] = out
    F = h.to_dense()
    h.host_arena()[:] = saved
    return F


def test_dense_matches_reference_kernel_bitwise(pp, oracle, gctx):
    h, A = pp.make_dense_problem(gctx, n=512, leaf=128, seed=3)
    F_ref = run_reference_kernel(pp, oracle, h)
    F = factor_on_gpu(h)
    assert np.array_equal(F, F_ref)
    assert np.array_equal(F, oracle.dense_getrf(A))


def test_hodlr_matches_reference_kernel(pp, oracle, gctx):
    h, _ = pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16)
    F_ref = run_reference_kernel(pp, oracle, h)
    F = factor_on_gpu(h)
    assert rel(F, F_ref) < 1e-12


def test_solve_matches_oracle(pp, oracle, gctx):
    n = 2048
    h, prob = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16)
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=8)
    b = pp.rhs(n, 3)
    sol = oracle.HostArenas(h, 1, 3, rhs=b)
    sol.matrix[:] = ar.matrix
    sol.tasks, sol.succ, sol.indeg, sol.ready = h.encode_program(1, 3, sol.bases())
    sol.run()
    x_or = sol.rhs[: n * 3].reshape(n, 3)
    h.upload()
    h.factor()
    bd = dev(b)
    xd = torch.empty_like(bd)
    h.solve(bd, xd)
    h.sync()
    assert rel(xd.cpu().numpy(), x_or) < 1e-12


def test_dense_solve_matches_oracle(pp, oracle, gctx):
    """The solve applies the explicit inverses of the leaf factors (TRMV); the oracle runs
    the same program with its own summation order, so the bar is a tolerance."""
    n = 512
    h, A = pp.make_dense_problem(gctx, n=n, leaf=128)
    ar = oracle.HostArenas(h, 0)
    ar.run()
    b = pp.rhs(n, 2)
    sol = oracle.HostArenas(h, 1, 2, rhs=b)
    sol.matrix[:] = ar.matrix
    sol.tasks, sol.succ, sol.indeg, sol.ready = h.encode_program(1, 2, sol.bases())
    sol.run()
    h.upload()
    h.factor()
    bd = dev(b)
    xd = torch.empty_like(bd)
    h.solve(bd, xd)
    h.sync()
    assert rel(xd.cpu().numpy(), sol.rhs[: n * 2].reshape(n, 2)) < 1e-13


def test_refinement_reaches_1e10(pp, gctx):
    n = 4096
    h, prob = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16)
    h.upload()
    h.factor()
    b_h = pp.rhs(n)
    ref = pp.Refiner(h, gctx, prob)
    x, hist = ref.solve(dev(b_h), tol=1e-10)
    assert hist[-1] <= 1e-10, hist
    A = prob.dense()
    xh = x.cpu().numpy()
    assert abs(np.abs(A).sum(1).max() - prob.norm_inf) < 1e-9 * prob.norm_inf
    berr = np.abs(b_h - A @ xh).max() / (prob.norm_inf * np.abs(xh).max() + np.abs(b_h).max())
    assert berr <= 1e-10, berr


def test_dense_refinement(pp, gctx):
    n = 1024
    h, A = pp.make_dense_problem(gctx, n=n, leaf=256)
    h.upload()
    h.factor()
    b_h = pp.rhs(n)
    x, hist = pp.Refiner(h, gctx, dense=A).solve(dev(b_h), tol=1e-12)
    assert hist[-1] <= 1e-12


@pytest.mark.parametrize("kernel,p0,dim", [("inv", 1e-3, 2), ("laplace", 1e-3, 3), ("exp", 0.1, 2),
                                           ("matern32", 0.2, 3)])
@pytest.mark.parametrize("nrhs", [1, 3, 8])
def test_kernel_residual_matches_dense_fp64(pp, gctx, kernel, p0, dim, nrhs):
    n = 1500
    rng = np.random.default_rng(5)
    pts = rng.uniform(0, 1, (n, dim))
    kid = pp.KERNELS[kernel]
    prob = pp.KernelProblem(n, dim, kid, p0, 3.0, pts)
    A = prob.dense()
    x = rng.standard_normal((n, nrhs))
    b = rng.standard_normal((n, nrhs))
    r = torch.empty((n, nrhs), dtype=torch.float64, device="cuda")
    gctx.kernel_residual(kid, p0, 3.0, dev(pts), dev(x), dev(b), r)
    want = b - A @ x
    scale = np.abs(A).sum(1).max() * np.abs(x).max()
    assert np.abs(r.cpu().numpy() - want).max() <= 1e-14 * scale


def _resid_job(pp, rng, kernel, p0, dim, n, nrhs, dup=False):
    pts = rng.uniform(0, 1, (n, dim))
    if dup and n > 4:
        pts[n // 2] = pts[1]  # coincident points: distance 0 off the diagonal
    x, dx, b = (rng.standard_normal((n, nrhs)) for _ in range(3))
    return (pp.KERNELS[kernel], p0, 3.0, dev(pts), dev(x), dev(dx), dev(b),
            torch.empty((n, nrhs), dtype=torch.float64, device="cuda")), pts


def test_kernel_residual_batch_equals_single_calls(pp, gctx):
    """The batched update + residual gives each job the bits of its own single call on x + dx,
    across kernels, dimensions, RHS widths (tile-pair and row-block paths), ragged sizes and
    more jobs than one launch holds."""
    rng = np.random.default_rng(11)
    shapes = [("inv", 1e-3, 2, 1500, 1), ("laplace", 1e-3, 3, 300, 3), ("exp", 0.1, 2, 129, 1),
              ("matern32", 0.2, 3, 700, 8), ("inv", 1e-3, 2, 1, 1), ("inv", 1e-3, 2, 257, 4),
              ("exp", 0.1, 1, 64, 16)] + [("inv", 1e-3, 2, 40 + q, 1) for q in range(66)]
    jobs = [_resid_job(pp, rng, *sh, dup=(q % 3 == 0))[0] for q, sh in enumerate(shapes)]
    want_x = [(x + dx).clone() for (_, _, _, _, x, dx, _, _) in jobs]
    launches = gctx.kernel_residual_batch(jobs)
    torch.cuda.synchronize()
    assert launches == pp.residual_batch_launches([(j[0], j[3].shape[1], j[4].shape[1], True) for j in jobs])
    for (kid, p0, shift, pts, x, dx, b, r), wx in zip(jobs, want_x):
        assert torch.equal(x, wx)
        r1 = torch.empty_like(r)
        gctx.kernel_residual(kid, p0, shift, pts, x, b, r1)
        torch.cuda.synchronize()
        assert torch.equal(r, r1)


@pytest.mark.parametrize("kernel,p0,dim", [("inv", 1e-3, 2), ("laplace", 1e-3, 3), ("exp", 0.1, 2),
                                           ("matern32", 0.2, 3)])
def test_kernel_residual_coincident_points(pp, gctx, kernel, p0, dim):
    """Distance 0 off the diagonal and points far apart take the exact square-root path."""
    rng = np.random.default_rng(8)
    n = 400
    pts = rng.uniform(0, 1, (n, dim))
    pts[7] = pts[300]
    pts[9] = pts[10]
    pts[20] = 0.0
    pts[21] = 0.0
    pts[21, 0] = 1e-20  # squared distance 1e-40: below the float range of the estimates
    pts[30] = 1e19  # squared distances near 1e38: above it
    kid = pp.KERNELS[kernel]
    prob = pp.KernelProblem(n, dim, kid, p0, 3.0, pts)
    A = prob.dense()
    x = rng.standard_normal((n, 1))
    b = rng.standard_normal((n, 1))
    r = torch.empty((n, 1), dtype=torch.float64, device="cuda")
    gctx.kernel_residual_batch([(kid, p0, 3.0, dev(pts), dev(x), None, dev(b), r)])
    want = b - A @ x
    scale = np.abs(A).sum(1).max() * np.abs(x).max()
    assert np.abs(r.cpu().numpy() - want).max() <= 1e-14 * scale


def test_kernel_residual_rejects_p0_out_of_range(pp, gctx):
    rng = np.random.default_rng(2)
    job, _ = _resid_job(pp, rng, "inv", 1e-3, 2, 64, 1)
    bad = (job[0], -1.0) + job[2:]
    with pytest.raises(RuntimeError, match="p0"):
        gctx.kernel_residual_batch([bad])


def test_dense_residual_kernel(pp, gctx):
    rng = np.random.default_rng(0)
    n = 300
    A = rng.standard_normal((n, n))
    x = rng.standard_normal((n, 2))
    b = rng.standard_normal((n, 2))
    r = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    gctx.dense_residual(dev(A), dev(x), dev(b), r)
    assert np.allclose(r.cpu().numpy(), b - A @ x, rtol=1e-12, atol=1e-12)


def test_timeout_is_reported_not_hung(pp, gctx):
    # host-side fault: task 1 claims two predecessors but only task 0 precedes it, so
    # its ready slot is never filled; the VM must give up and report PP_TIMEOUT
    t = np.zeros(2, dtype=pp.TASK_DTYPE)
    t[0]["op"] = 0
    t[0]["succ_begin"], t[0]["n_succ"] = 0, 1
    t[1]["op"] = 0
    succ = np.array([1], np.int32)
    indeg = np.array([0, 2], np.int32)
    with pytest.raises(pp.PPError) as e:
        gctx.vm_execute(t, succ, indeg, spin_limit=20000)
    assert e.value.status == pp.PP_TIMEOUT
    # the context stays usable
    indeg_ok = np.array([0, 1], np.int32)
    gctx.vm_execute(t, succ, indeg_ok)
