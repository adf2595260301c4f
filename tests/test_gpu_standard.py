"""Standard admissibility on the GPU: low-rank blocks updated by products of hierarchical
blocks (sketched update: GEMMs into work buffers, ORTH, COPY)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from test_gpu_vm import TaskBench, rel  # noqa: E402


@pytest.mark.parametrize("m,k", [(512, 16), (1000, 8), (300, 32)])
def test_orth_task_spans_the_input(pp, oracle, gctx, m, k):
    tb = TaskBench(pp, seed=m + k)
    y = tb.operand(m, k, ld_pad=0)
    Y0 = tb.host[y[0]].copy()
    d, h = tb.run(gctx, oracle, dict(op=13, m=m, n=k), {0: y})[y[0]]
    assert np.abs(d.T @ d - np.eye(k)).max() < 1e-13
    assert rel(d @ (d.T @ Y0), Y0) < 1e-13  # same range
    assert rel(d, h) < 1e-12


def test_standard_admissibility_factor_matches_oracle_and_refines(pp, oracle, gctx):
    n = 4096
    h, prob = pp.make_kernel_problem(gctx, n, 2, "laplace", 1e-3, 128, 16, admissibility=1, eta=1.0, seed=3)
    info = h.program_info(0)
    assert info["op_count"]["orth"] > 0
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=8)
    h.upload()
    h.factor()
    h.sync()
    h.download()
    F = h.to_dense()
    h.host_arena()[:] = ar.matrix
    assert rel(F, h.to_dense()) < 1e-10
    h.upload()
    ref = pp.Refiner(h, gctx, prob)
    h.factor()
    x, hist = ref.solve(torch.from_numpy(pp.rhs(n)).cuda(), tol=1e-10)
    assert hist[-1] <= 1e-10
