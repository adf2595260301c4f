"""Dependency DAG built on the device (csrc/dag.cu) against the host build.

The device build must give the same program to the VM: every task record, successor list
(order included: successors are sorted by bottom level, ties in program order), in-degree and
initial ready order, for the factor and solve programs of the benchmark configurations' trees
(all-dense N = 1024 with 256 leaves; HODLR N = 8192 with 256 leaves and rank 16; 3-D Laplace
N = 8192 with 512 leaves, eta 1, rank <= 32, in FP64 and BF16 form; standard admissibility in
2-D, N = 4096 with 128 leaves).  Only the tree matters to the DAG, so no matrix is
filled."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def tree(pp, ctx, case):
    if case == "dense_n1024_leaf256":
        return pp.Hierarchical.dense(ctx, 1024, 256), 1
    rng = np.random.default_rng(1234)
    if case == "hodlr_n8192_leaf256":
        pts = rng.uniform(0, 1, (8192, 2))
        return pp.Hierarchical.geometric(ctx, pts[pp.morton_order(pts)], 256, 0, 1.0, 16), 1
    if case in ("laplace3d_n8192_leaf512_fp64", "laplace3d_n8192_leaf512_bf16"):
        pts = rng.uniform(0, 1, (8192, 3))
        h = pp.Hierarchical.geometric(ctx, pts[pp.morton_order(pts)], 512, 1, 1.0, 32)
        h.set_rank_tolerance(1e-8)
        if case.endswith("bf16"):
            h.set_precision(pp.BF16)
        return h, 8
    if case == "standard2d_n4096_leaf128":
        pts = rng.uniform(0, 1, (4096, 2))
        h = pp.Hierarchical.geometric(ctx, pts[pp.morton_order(pts)], 128, 1, 1.0, 24)
        h.set_rank_tolerance(1e-7)
        return h, 1
    raise ValueError(case)


@pytest.mark.parametrize("case", ["dense_n1024_leaf256", "hodlr_n8192_leaf256", "laplace3d_n8192_leaf512_fp64",
                                  "laplace3d_n8192_leaf512_bf16", "standard2d_n4096_leaf128"])
def test_device_dag_equals_host_dag(pp, case):
    ctx_h, ctx_d = pp.Context(device=0), pp.Context(device=0)
    ctx_d.set_device_dag(True)
    hh, nrhs = tree(pp, ctx_h, case)
    hd, _ = tree(pp, ctx_d, case)
    for which in (0, 1):
        ih, idv = hh.program_info(which, nrhs), hd.program_info(which, nrhs)
        assert ih["n_tasks"] == idv["n_tasks"] and ih["n_edges"] == idv["n_edges"]
        _, on_dev = hd.dag_info(which, nrhs)
        assert on_dev, ctx_d.last_error()
        assert not hh.dag_info(which, nrhs)[1]
        bases = [0x100000 * (k + 1) for k in range(5)]
        th, sh, dh, rh = hh.encode_program(which, nrhs, bases)
        td, sd, dd, rd = hd.encode_program(which, nrhs, bases)
        assert th.tobytes() == td.tobytes()
        assert np.array_equal(sh, sd) and np.array_equal(dh, dd) and np.array_equal(rh, rd)
        fh, toh, tyh = hh.edges(which, nrhs)
        fd, tod, tyd = hd.edges(which, nrhs)
        assert np.array_equal(fh, fd) and np.array_equal(toh, tod) and np.array_equal(tyh, tyd)

