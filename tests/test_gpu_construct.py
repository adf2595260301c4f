"""Building an H-matrix on the device: dense blocks assembled from the points, low-rank blocks
compressed by a randomized range finder on the VM (KMUL / ORTH / LRTRUNC instructions).  Parity
for the compression is by accuracy against the host's truncated SVD of the same blocks."""
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


def _block_errors(h, A):
    """Relative Frobenius error of every low-rank block of h (host image) against A."""
    F = h.to_dense()
    out = []
    for b in h.blocks():
        if b["kind"] == 1:
            r, c = slice(b["row0"], b["row0"] + b["m"]), slice(b["col0"], b["col0"] + b["n"])
            out.append(np.linalg.norm(F[r, c] - A[r, c]) / np.linalg.norm(A[r, c]))
    return np.array(out)


def test_device_construction_matches_host_svd_accuracy(pp, gctx):
    """Low-rank blocks compressed on the device (randomized range finder with one power step on
    the VM) against the host's truncated SVD of the same blocks: the same accuracy class."""
    n = 2048
    h1, p1 = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16)
    h2, p2 = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16, construct="device")
    assert abs(p2.shift - p1.shift) <= 1e-12 * p1.shift
    h2.sync()
    h2.download()
    A = p1.dense()
    e_host, e_dev = _block_errors(h1, A), _block_errors(h2, A)
    assert e_dev.size == e_host.size > 0
    assert np.all(e_dev <= 20 * e_host + 1e-13), (e_dev.max(), e_host.max())
    F = h2.to_dense()
    for b in h2.blocks():
        if b["kind"] == 0:
            r, c = slice(b["row0"], b["row0"] + b["m"]), slice(b["col0"], b["col0"] + b["n"])
            assert np.abs(F[r, c] - A[r, c]).max() <= 1e-14 * np.abs(A[r, c]).max()


def test_device_construction_adaptive_rank_factor_and_refine(pp, gctx):
    n = 8192  # 2-D: standard admissibility gives low-rank blocks at this size (3-D barely does)
    h, prob = pp.make_kernel_problem(gctx, n, 2, "laplace", 1e-3, 256, 32, admissibility=1, eta=1.0,
                                     rank_tol=1e-8, construct="device")
    h.sync()
    h.download()
    ranks = [r for r in h.ranks().values() if r >= 0]
    assert ranks and max(ranks) <= 32 and min(ranks) >= 1
    h.factor()
    b = pp.rhs(n, 4)
    x, hist = pp.Refiner(h, gctx, prob).solve(torch.from_numpy(b).cuda(), tol=1e-10)
    assert hist[-1] <= 1e-10, hist


def test_device_assembly_refuses_wrong_point_dimension(pp, gctx):
    """Points of another dimension than the tree's would be read past their end: refused."""
    h, prob = pp.make_kernel_problem(gctx, 512, 2, "inv", 1e-3, 128, 16)
    h.upload()
    pts = torch.zeros(512, 3, dtype=torch.float64, device="cuda")
    L = pp.lib()
    assert L.pp_hmatrix_assemble_dense_dev(h.handle, int(prob.kernel), float(prob.p0), float(prob.shift),
                                           pts.data_ptr(), 3, None) == pp.PP_INVALID_ARG
    assert L.pp_hmatrix_construct_dev(h.handle, int(prob.kernel), float(prob.p0), float(prob.shift),
                                      pts.data_ptr(), 3, None) == pp.PP_INVALID_ARG
