"""Batched launches: many H-matrices of uneven size in one persistent VM launch.

Each instance's result must be the same alone and in the mix (bitwise: every task is
deterministic given its inputs, and the merged DAG keeps each instance's dependencies)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def mixed_instances(pp, ctx):
    probs = [
        pp.make_kernel_problem(ctx, 1024, 2, "inv", 1e-3, 128, 16, seed=1),
        pp.make_kernel_problem(ctx, 1536, 2, "exp", 0.1, 128, 12, shift=1.0, seed=2),
        pp.make_kernel_problem(ctx, 2048, 3, "laplace", 1e-3, 256, 16, seed=3),
    ]
    hd, A = pp.make_dense_problem(ctx, n=512, leaf=128, seed=4)
    return probs, (hd, A)


def test_batch_factor_alone_equals_mix(pp, gctx):
    probs, (hd, A) = mixed_instances(pp, gctx)
    hs = [h for h, _ in probs] + [hd]
    alone = []
    for h in hs:
        h.upload()
        h.factor()
        h.sync()
        h.download()
        alone.append(h.host_arena().copy())
    # fresh uploads of the same matrices, factored together
    probs2, (hd2, _) = mixed_instances(pp, gctx)
    hs2 = [h for h, _ in probs2] + [hd2]
    for h in hs2:
        h.upload()
    b = pp.Batch(gctx, hs2)
    assert b.program_info(0)["n_tasks"] == sum(h.program_info(0)["n_tasks"] for h in hs2)
    b.factor()
    b.sync()
    for h, ref in zip(hs2, alone):
        h.download()
        assert np.array_equal(h.host_arena(), ref)


def test_batch_solve_and_refinement(pp, gctx):
    probs, _ = mixed_instances(pp, gctx)
    hs = [h for h, _ in probs]
    for h in hs:
        h.upload()
        h.keep_original()
    b = pp.Batch(gctx, hs)
    b.factor()
    bs = [dev(pp.rhs(h.n, 2, seed=10 + i)) for i, h in enumerate(hs)]
    xs = [torch.empty_like(x) for x in bs]
    b.solve(bs, xs)
    b.sync()
    # alone: the same solve on each instance's own plan
    for h, bb, xx in zip(hs, bs, xs):
        x1 = torch.empty_like(bb)
        h.solve(bb, x1)
        h.sync()
        assert torch.equal(x1, xx)
    # refinement of the whole batch to 1e-10 (restore, factor again, refine)
    b.restore()
    b.factor()
    ref = pp.BatchRefiner(b, [p for _, p in probs])
    xs, hist = ref.solve(bs, tol=1e-10)
    assert hist[-1] <= 1e-10, hist
    for (h, p), x, bb in zip(probs, xs, bs):
        Ad = p.dense()
        xh, bh = x.cpu().numpy(), bb.cpu().numpy()
        berr = np.abs(bh - Ad @ xh).max() / (p.norm_inf * np.abs(xh).max() + np.abs(bh).max())
        assert berr <= 1e-10, berr


def test_batch_graph_capture_replays(pp, gctx):
    probs, _ = mixed_instances(pp, gctx)
    hs = [h for h, _ in probs]
    for h in hs:
        h.upload()
        h.keep_original()
    b = pp.Batch(gctx, hs)
    bs = [dev(pp.rhs(h.n, 1, seed=20 + i)) for i, h in enumerate(hs)]
    ref = pp.BatchRefiner(b, [p for _, p in probs])
    # eager warm-up allocates every plan; then the fixed step is captured once
    b.restore()
    b.factor()
    xs_eager, hist = ref.solve(bs, tol=1e-10)
    iters = len(hist)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        ref.stream = s
        b.restore(s)
        b.factor(s)
        with torch.cuda.graph(g, stream=s):
            b.restore(s)
            b.factor(s)
            out = ref.run(bs, iters)
    torch.cuda.current_stream().wait_stream(s)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        errs = ref.errors(bs, *out)
        assert max(errs) <= 1e-10, errs
        for xe, xg in zip(xs_eager, out[0]):
            assert torch.equal(xe, xg)


def test_batch_autotune_keeps_results(pp, gctx):
    """The autotuner times tile x product tile x grid candidates and keeps the fastest; the
    factorization it then runs equals the untuned one (dense blocks are blocking-invariant,
    the low-rank work is decomposed independently of the tile)."""
    hs = [pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 128, 16, seed=11 + i)[0] for i, n in enumerate([1024, 1536])]
    ref = []
    for h in hs:
        h.upload()
        h.keep_original()
    b0 = pp.Batch(gctx, hs)
    b0.factor()
    b0.sync()
    for h in hs:
        h.download()
        ref.append(h.to_dense())
    b = pp.Batch(gctx, hs)
    choice = b.autotune()
    assert choice["tile"] in (32, 64) and choice["gemm_tile"] in (64, 128) and choice["grid"] > 0
    assert choice["trials"] == 12
    b.factor()
    b.sync()
    for h, F in zip(hs, ref):
        h.download()
        assert rel(h.to_dense(), F) < 1e-12


def test_batch_set_tuning_applies_a_tuning(pp, gctx):
    """A tuning found on one batch, applied to a second batch of the same shapes, gives the
    same factors; bad tunings are refused."""
    hs = [pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16, seed=5 + i)[0] for i in range(2)]
    hs2 = [pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16, seed=5 + i)[0] for i in range(2)]
    for h in hs + hs2:
        h.upload()
        h.keep_original()
    b = pp.Batch(gctx, hs)
    tune = b.autotune()
    b2 = pp.Batch(gctx, hs2)
    b2.set_tuning(**tune)
    with pytest.raises(pp.PPError):
        b2.set_tuning(tile=64, gemm_tile=100, grid=0)
    b2.set_tuning(**tune)
    for bt in (b, b2):
        bt.factor()
        bt.sync()
    for h, h2 in zip(hs, hs2):
        h.download()
        h2.download()
        assert np.array_equal(h.to_dense(), h2.to_dense())
