"""The device DAG build's walk rule (restated on the CPU in oracle/dagwalk.py) gives exactly
the host build's typed edges (Program::build_dag, the reference's dependency semantics) on the
factor and solve programs of several trees: all-dense, HODLR, the 3-D leaf-512 tree in FP64
and BF16 form (whole-leaf products, shadows), standard admissibility in 2-D, pivoted.  The GPU
test (tests/test_gpu_dag.py) checks the kernel against the same host build."""
import numpy as np
import pytest

from oracle import dagwalk


def trees(pp, ctx):
    rng = np.random.default_rng(3)
    out = [("dense_n512_leaf128", pp.Hierarchical.dense(ctx, 512, 128), 1)]
    p2 = rng.uniform(0, 1, (2048, 2))
    out.append(("hodlr_n2048_leaf128", pp.Hierarchical.geometric(ctx, p2[pp.morton_order(p2)], 128, 0, 1.0, 16), 1))
    p8 = rng.uniform(0, 1, (8192, 2))
    h8 = pp.Hierarchical.geometric(ctx, p8[pp.morton_order(p8)], 256, 0, 1.0, 16)
    h8.set_gemm_tile(128)
    out.append(("hodlr_n8192_leaf256", h8, 1))
    p3 = rng.uniform(0, 1, (2048, 3))
    for form, label in ((pp.FP64, "fp64"), (pp.BF16, "bf16")):
        h = pp.Hierarchical.geometric(ctx, p3[pp.morton_order(p3)], 512, 1, 1.0, 32)
        h.set_rank_tolerance(1e-8)
        h.set_precision(form)
        out.append((f"laplace3d_n2048_leaf512_{label}", h, 8))
    p4 = rng.uniform(0, 1, (1024, 2))
    h = pp.Hierarchical.geometric(ctx, p4[pp.morton_order(p4)], 64, 1, 1.0, 16)
    h.set_rank_tolerance(1e-7)
    out.append(("standard2d_n1024_leaf64", h, 1))
    hp = pp.Hierarchical.dense(ctx, 512, 128)
    hp.set_pivoting(True)
    out.append(("dense_n512_leaf128_pivoted", hp, 2))
    return out


def test_walk_rule_gives_the_host_edges(pp, hctx):
    for name, h, nrhs in trees(pp, hctx):
        for which in (0, 1):
            f, t, ty = h.edges(which, nrhs)
            host = {(int(a), int(b)): int(c) for a, b, c in zip(f, t, ty)}
            walk = dagwalk.walk_edges(h.regions(which, nrhs))
            assert walk == host, (name, which, len(walk), len(host))
            assert len(host) == h.program_info(which, nrhs)["n_edges"]
