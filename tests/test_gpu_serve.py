"""Serving loop on the GPU: requests of different sizes admitted by HBM budget and free slots,
overlapping on the device, each refined in FP64 to 1e-10; a request's result is the same
alone and in a mix (the bar: 1e-12 relative; the engine is deterministic, so it is equal)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def request(pp, ctx, n, kernel, p0, seed, nrhs=2, n_sets=2, leaf=128, rank=16):
    h, prob = pp.make_kernel_problem(ctx, n, 3, kernel, p0, leaf, rank, seed=seed)
    rhs = np.random.default_rng(seed + 1).uniform(-1, 1, (n_sets, n, nrhs))
    return h, prob, rhs


def dense_backward_error(prob, x, b):
    A = prob.dense()
    r = b - A @ x
    return np.abs(r).max() / (prob.norm_inf * np.abs(x).max() + np.abs(b).max())


def test_serve_converges_and_matches_dense(pp, gctx):
    srv = pp.Server(gctx, hbm_budget_bytes=8 << 30, max_inflight=3)
    jobs = [request(pp, gctx, n, k, p0, 40 + i) for i, (n, k, p0) in
            enumerate([(1024, "laplace", 1e-3), (1536, "exp", 0.1), (2048, "matern32", 0.2)])]
    ids = [srv.submit(h, prob, rhs, tol=1e-10) for h, prob, rhs in jobs]
    srv.wait_all()
    for rid, (_, prob, rhs) in zip(ids, jobs):
        st = srv.poll(rid)
        assert st["status"] == "done", st["message"]
        assert st["backward_error"] <= 1e-10
        x = srv.result(rid)
        for s in range(rhs.shape[0]):  # every set, checked against the dense FP64 matrix
            assert dense_backward_error(prob, x[s], rhs[s]) <= 1e-10
    srv.close()


def test_serve_result_same_alone_and_in_mix(pp, gctx):
    def run(mix):
        srv = pp.Server(gctx, hbm_budget_bytes=8 << 30, max_inflight=4)
        h, prob, rhs = request(pp, gctx, 2048, "exp", 0.1, 7)
        others = [request(pp, gctx, n, k, p0, 100 + i) for i, (n, k, p0) in
                  enumerate([(1024, "laplace", 1e-3), (3072, "matern32", 0.2), (1536, "exp", 0.1),
                             (2048, "laplace", 1e-3)])] if mix else []
        ids = []
        if mix:  # two requests are on the GPU before the watched one arrives, two come after
            ids += [srv.submit(*others[0]), srv.submit(*others[1])]
            time.sleep(0.002)
        rid = srv.submit(h, prob, rhs, tol=1e-10)
        if mix:
            ids += [srv.submit(*others[2]), srv.submit(*others[3])]
        srv.wait_all()
        for i in ids + [rid]:
            assert srv.poll(i)["status"] == "done", srv.poll(i)["message"]
        x = srv.result(rid).copy()
        srv.close()
        return x

    alone = run(False)
    mixed = run(True)
    assert rel(mixed, alone) <= 1e-12


def test_serve_admission_respects_budget(pp, gctx):
    jobs = [request(pp, gctx, 1024, "laplace", 1e-3, 60 + i, n_sets=1) for i in range(3)]
    # learn one request's device bytes, then allow only one at a time
    probe = pp.Server(gctx, hbm_budget_bytes=8 << 30, max_inflight=4)
    h0, p0_, r0 = request(pp, gctx, 1024, "laplace", 1e-3, 59, n_sets=1)
    rid0 = probe.submit(h0, p0_, r0)
    probe.wait_all()
    one = probe.poll(rid0)["device_bytes"]
    probe.close()
    srv = pp.Server(gctx, hbm_budget_bytes=int(one * 1.5), max_inflight=4)
    ids = [srv.submit(h, prob, rhs) for h, prob, rhs in jobs]
    srv.wait_all()
    st = [srv.poll(i) for i in ids]
    assert all(s["status"] == "done" for s in st)
    spans = sorted((s["t_admit_ms"], s["t_done_ms"]) for s in st)
    for (a0, d0), (a1, _) in zip(spans, spans[1:]):
        assert a1 >= d0  # never two requests on the device at once
    srv.close()


def test_serve_rejects_request_over_budget(pp, gctx):
    srv = pp.Server(gctx, hbm_budget_bytes=1 << 20, max_inflight=2)
    h, prob, rhs = request(pp, gctx, 1024, "laplace", 1e-3, 5, n_sets=1)
    with pytest.raises(pp.PPError, match="OOM"):
        srv.submit(h, prob, rhs)
    srv.close()


def test_serve_builds_unfilled_matrices_on_the_device(pp, gctx):
    """Requests whose H-matrices were never filled on the host: the server builds them on the
    device from the request's points at admission, and the results meet the tolerance against
    the dense FP64 matrix; the same request alone and in a mix gives the same solution."""
    def unbuilt(n, kernel, p0, seed):
        h, prob = pp.make_kernel_problem(gctx, n, 3, kernel, p0, 128, 24, seed=seed, rank_tol=1e-7,
                                         construct="none")
        rhs = np.random.default_rng(seed + 1).uniform(-1, 1, (2, n, 3))
        return h, prob, rhs

    srv = pp.Server(gctx, hbm_budget_bytes=8 << 30, max_inflight=3)
    jobs = [unbuilt(n, k, p0, 70 + i) for i, (n, k, p0) in
            enumerate([(2048, "laplace", 1e-3), (3072, "exp", 0.1), (2560, "matern32", 0.2)])]
    ids = [srv.submit(h, prob, rhs, tol=1e-10) for h, prob, rhs in jobs]
    srv.wait_all()
    xs = []
    for rid, (_, prob, rhs) in zip(ids, jobs):
        st = srv.poll(rid)
        assert st["status"] == "done", st["message"]
        x = srv.result(rid)
        xs.append(x)
        for s in range(rhs.shape[0]):
            assert dense_backward_error(prob, x[s], rhs[s]) <= 1e-10
    h, prob, rhs = unbuilt(2048, "laplace", 1e-3, 70)
    rid = srv.submit(h, prob, rhs, tol=1e-10)
    srv.wait_all()
    assert rel(srv.result(rid), xs[0]) <= 1e-12
    srv.close()
