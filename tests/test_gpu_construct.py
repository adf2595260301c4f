"""Building an H-matrix on the device: dense blocks assembled from the points (the first step
of the construction; the low-rank blocks still come from the host's truncated SVD)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("kernel,p0,dim,adm", [("inv", 1e-3, 2, 0), ("matern32", 0.2, 3, 0), ("exp", 0.1, 2, 1),
                                               ("laplace", 1e-3, 1, 0)])
def test_assemble_dense_blocks_on_device(pp, gctx, kernel, p0, dim, adm):
    n = 1024
    h, prob = pp.make_kernel_problem(gctx, n, dim, kernel, p0, 128, 16, admissibility=adm)
    saved = h.host_arena().copy()
    h.host_arena()[:] = 0.0  # the device copy starts without the host's dense blocks
    h.upload()
    h.host_arena()[:] = saved
    h.assemble_dense(prob)
    torch.cuda.synchronize()
    h.download()
    F = h.to_dense()
    A = prob.dense()
    dense = [b for b in h.blocks() if b["kind"] == pp.DENSE]
    assert dense
    for b in dense:
        r, c = slice(b["row0"], b["row0"] + b["m"]), slice(b["col0"], b["col0"] + b["n"])
        assert np.abs(F[r, c] - A[r, c]).max() <= 1e-14 * np.abs(A[r, c]).max()


def test_factor_after_device_assembly_matches_host_assembly(pp, gctx):
    h1, prob = pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16)
    h2, _ = pp.make_kernel_problem(gctx, 1024, 2, "inv", 1e-3, 128, 16)
    for h in (h1, h2):
        h.upload()
    h2.assemble_dense(prob)
    for h in (h1, h2):
        h.factor()
        h.sync()
        h.download()
    F1, F2 = h1.to_dense(), h2.to_dense()
    assert np.linalg.norm(F1 - F2) <= 1e-13 * np.linalg.norm(F1)
