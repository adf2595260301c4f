"""Batched restarted GMRES around the H-LU solve (csrc/krylov.cu, BatchGMRES).

1. The three kernels against the numpy restatement (oracle/krylov.py) on the same vectors:
   dense systems, identity preconditioner, three instances of uneven size in one launch each.
2. Kernel problems whose plain refinement stalls (exp(-r/0.1) + 1e-2 I on 2-D points, weak
   admissibility, ranks capped below what 1e-7 needs, so rho(I - (LU)^-1 A) > 1): GMRES
   reaches a backward error <= 1e-10 against the dense FP64 matrix, every instance of an
   uneven batch, alone-equal-mix not required (the batch shares the stopping point)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_gmres_kernels_match_restatement(pp, gctx):
    from oracle import krylov as K
    rng = np.random.default_rng(5)
    ns, m = [517, 200, 333], 12
    As = [np.eye(n) * 4.0 + rng.uniform(-1, 1, (n, n)) / np.sqrt(n) for n in ns]
    bs = [rng.uniform(-1, 1, n) for n in ns]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    V = [torch.zeros(m + 1, n, dtype=torch.float64, device="cuda") for n in ns]
    Z = [torch.zeros(m, n, dtype=torch.float64, device="cuda") for n in ns]
    x = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in ns]
    r = [dev(b) for b in bs]
    Ad = [dev(A) for A in As]
    k = len(ns)
    vp = lambda ts: (C.c_void_p * k)(*[C.c_void_p(t.data_ptr()) for t in ts])
    h = C.c_void_p()
    L = pp.lib()
    gctx.check(L.pp_gmres_create(gctx.handle, k, (C.c_int * k)(*ns), m, vp(V), vp(Z), vp(x), vp(r), C.byref(h)),
               "gmres_create")
    try:
        S = [K.GmresState(n, m) for n in ns]
        gctx.check(L.pp_gmres_start(h, None), "start")
        for s, b in zip(S, bs):
            K.start(s, b)
        for j in range(m):
            for i in range(k):
                Z[i][j].copy_(V[i][j])
                V[i][j + 1].copy_(-(Ad[i] @ Z[i][j]))
                S[i].Z[j] = S[i].V[j]
                K.arnoldi(S[i], j, As[i] @ S[i].Z[j])
            gctx.check(L.pp_gmres_arnoldi(h, j, None), "arnoldi")
        gctx.check(L.pp_gmres_finish(h, None), "finish")
        torch.cuda.synchronize()
        st = np.zeros(2 * k)
        gctx.check(L.pp_gmres_status(h, st.ctypes.data_as(C.POINTER(C.c_double))), "status")
        for i in range(k):
            xo = K.finish(S[i], np.zeros(ns[i]))
            xg = x[i].cpu().numpy()
            assert np.linalg.norm(xg - xo) <= 1e-11 * np.linalg.norm(xo)
            Vg = V[i].cpu().numpy()
            assert np.abs(Vg - S[i].V).max() <= 1e-11
            assert st[2 * i] == m
            assert abs(st[2 * i + 1] - S[i].meta[3]) <= 1e-9 * S[i].meta[2]
            # the estimate is the true residual norm of the cycle's answer
            res = np.linalg.norm(bs[i] - As[i] @ xg)
            assert abs(res - st[2 * i + 1]) <= 1e-9 * np.linalg.norm(bs[i])
    finally:
        L.pp_gmres_destroy(h)


def stalled_instances(pp, ctx):
    # (n, rank cap): with these caps the spectral radius of I - (LU)^-1 A is far above 1
    spec = [(2048, 8), (4096, 16), (3072, 12)]
    out = []
    for i, (n, cap) in enumerate(spec):
        h, prob = pp.make_kernel_problem(ctx, n, 2, "exp", 0.1, 128, cap, shift=1e-2, seed=7 + i, rank_tol=1e-7)
        out.append((h, prob))
    return out


@pytest.mark.parametrize("kernel,p0,dim", [("inv", 1e-3, 2), ("laplace", 1e-3, 3), ("exp", 0.1, 2), ("matern32", 0.2, 3)])
def test_lowp_products_within_their_bound(pp, gctx, kernel, p0, dim):
    """FP32-evaluated entries: the product is within 5e-6 * |A| |x| of the FP64 one (which is
    checked against the dense matrix elsewhere)."""
    probs = [pp.make_kernel_problem(gctx, n, dim, kernel, p0, 128, 8, seed=21 + n)[1] for n in (700, 1536)]
    jobs64, jobs32, want = [], [], []
    for p in probs:
        pts = torch.from_numpy(np.ascontiguousarray(p.points)).cuda()
        for nr in (1, 3):
            x = torch.from_numpy(np.random.default_rng(p.n + nr).uniform(-1, 1, (p.n, nr))).cuda()
            b = torch.zeros_like(x)
            r64, r32 = torch.empty_like(x), torch.empty_like(x)
            jobs64.append((p.kernel, p.p0, p.shift, pts, x, None, b, r64))
            jobs32.append((p.kernel, p.p0, p.shift, pts, x, None, b, r32))
            want.append((np.abs(p.dense()) @ np.abs(x.cpu().numpy())))
    gctx.kernel_residual_batch(jobs64)
    gctx.kernel_residual_batch(jobs32, lowp=True)
    torch.cuda.synchronize()
    for j64, j32, bound in zip(jobs64, jobs32, want):
        d = np.abs(j64[7].cpu().numpy() - j32[7].cpu().numpy())
        assert np.all(d <= 5e-6 * bound), (d / bound).max()
        assert (d > 0).any()  # really the FP32 path


@pytest.mark.parametrize("lowp", [False, True])
def test_gmres_converges_where_refinement_stalls(pp, gctx, lowp):
    inst = stalled_instances(pp, gctx)
    hs = [h for h, _ in inst]
    probs = [p for _, p in inst]
    s = torch.cuda.Stream()
    for h in hs:
        h.upload(s)
    batch = pp.Batch(gctx, hs)
    batch.factor(s)
    bs = [torch.from_numpy(pp.rhs(p.n, 1, seed=3 + i)).cuda() for i, p in enumerate(probs)]
    # plain refinement does not get there
    ir = pp.BatchRefiner(batch, probs, stream=s)
    with torch.cuda.stream(s):
        _, hist = ir.solve(bs, tol=1e-10, max_iter=30)
    assert hist[-1] > 1e-8
    gm = pp.BatchGMRES(batch, probs, m=32, stream=s, lowp=lowp)
    with torch.cuda.stream(s):
        xs, ghist = gm.solve(bs, tol=1e-10, max_cycles=12)
    batch.sync(s)
    assert ghist[-1] <= 1e-10, ghist
    for p, x, b in zip(probs, xs, bs):
        A = p.dense()
        xh, bh = x.cpu().numpy(), b.cpu().numpy()
        r = bh - A @ xh
        be = np.abs(r).max() / (np.abs(A).sum(axis=1).max() * np.abs(xh).max() + np.abs(bh).max())
        assert be <= 1e-10, be
    # the same cycles replayed from a CUDA graph reach the same tolerance (the solve sums its
    # products in free order, so the bits may differ)
    cycles = len(ghist)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            out, outr = gm.run(bs, cycles)
    with torch.cuda.stream(s):
        g.replay()
    s.synchronize()
    assert max(gm.errors(bs, out, outr)) <= 1e-10
    del g
