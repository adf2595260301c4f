"""Mixed-precision factorization: GEMM instructions on the tcgen05 tensor cores (TF32
operands, FP32 accumulation in tensor memory, FP64 result), FP64 everywhere else.

Bars:
  * one TF32 GEMM task: |C_tc - C_fp64| <= 2^-9 |alpha| (|op(A)| |op(B)|)_ij elementwise
    (operand rounding to TF32 costs 2^-11 each, FP32 accumulation k 2^-24) and not
    bitwise FP64 (the tensor-core path really ran);
  * a mixed H-LU followed by FP64 iterative refinement reaches backward error <= 1e-10;
  * ||A - LU|| / ||A|| of the mixed factor stays below 1e-2 and its factors differ from
    the FP64 factors at TF32 level (1e-9 .. 1e-2).  (With low-rank blocks the FP64 H-LU is
    not exact either: the fixed-rank recompression of the accumulated updates truncates.)
"""
import numpy as np
import pytest

from test_gpu_vm import TaskBench, dev, rel

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PREC_TF32 = 1


@pytest.mark.parametrize("tA,tB", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(128, 64, 32), (37, 91, 130), (256, 16, 16), (300, 200, 70), (5, 3, 0)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (1.0, 0.0)])
def test_tf32_gemm_task_within_bound(pp, oracle, gctx, tA, tB, m, n, k, alpha, beta):
    tb = TaskBench(pp, seed=3 * m + n + k)
    c = tb.operand(m, n)
    a = tb.operand(k, m) if tA else tb.operand(m, k)
    b = tb.operand(n, k) if tB else tb.operand(k, n)
    flags = (tA << 5) | (tB << 6)
    fields = dict(op=6, flags=flags, m=m, n=n, k=k, alpha=alpha, beta=beta, prec=PREC_TF32)
    out = tb.run(gctx, oracle, fields, {0: c, 1: a, 2: b})
    d, h = out[c[0]]
    A = tb.host[a[0]][:, : (m if tA else k)]
    B = tb.host[b[0]][:, : (k if tB else n)]
    opA = A.T if tA else A
    opB = B.T if tB else B
    bound = 2.0 ** -9 * abs(alpha) * (np.abs(opA) @ np.abs(opB)) + 1e-300
    err = np.abs(d[:, :n] - h[:, :n])
    assert np.all(err <= bound), float((err / bound).max())
    # the padding columns of C are untouched
    assert np.array_equal(d[:, n:], h[:, n:])
    if k >= 8:
        assert not np.array_equal(d[:, :n], h[:, :n])


def lu_error(h, F, A):
    """||A - L U||_F / ||A||_F from the dense image of the factors."""
    n = F.shape[0]
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    return np.linalg.norm(A - L @ U) / np.linalg.norm(A)


def factor_dense_image(h, precision):
    h.set_precision(precision)
    h.upload()
    h.factor()
    h.sync()
    h.download()
    return h.to_dense()


def test_mixed_factor_error_and_refinement(pp, gctx):
    n = 2048
    h, prob = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16)
    A_h = h.to_dense()  # the H-matrix operator (before factorization)
    F64 = factor_dense_image(h, pp.FP64)
    e64 = lu_error(h, F64, A_h)
    h2, _ = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 256, 16)
    assert np.array_equal(h2.to_dense(), A_h)
    F32 = factor_dense_image(h2, pp.TF32)
    assert h2.precision == pp.TF32
    e32 = lu_error(h2, F32, A_h)
    assert e64 <= 1e-3, e64
    assert e32 <= 1e-2, e32
    assert 1e-9 <= rel(F32, F64) <= 1e-2, rel(F32, F64)
    # FP64 refinement around the mixed factors, residual against the exact kernel matrix
    h2.upload()
    h2.factor()
    b = pp.rhs(n, 2, seed=11)
    x, hist = pp.Refiner(h2, gctx, prob).solve(dev(b), tol=1e-10, max_iter=20)
    assert hist[-1] <= 1e-10, hist
    A = prob.dense()
    xh = x.cpu().numpy()
    berr = np.abs(b - A @ xh).max() / (prob.norm_inf * np.abs(xh).max() + np.abs(b).max())
    assert berr <= 1e-10, berr


def test_precision_switch_restores_fp64_parity(pp, oracle, gctx):
    # TF32 -> FP64 again rebuilds the FP64 program: the factor matches the oracle to 1e-12
    n = 1024
    h, _ = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 128, 16)
    h.set_precision(pp.TF32)
    h.upload()
    h.factor()
    h.sync()
    h.set_precision(pp.FP64)
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=8)
    F = factor_dense_image(h, pp.FP64)
    h.host_arena()[:] = ar.matrix
    assert rel(F, h.to_dense()) < 1e-12


def test_mixed_batch_equals_alone(pp, gctx):
    # instances of a mixed batch give the same factors as each factored alone (mixed)
    hs, alone = [], []
    for j, n in enumerate([1024, 2048]):
        h, _ = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 128, 16, seed=40 + j)
        alone.append(factor_dense_image(h, pp.TF32))
        h2, _ = pp.make_kernel_problem(gctx, n, 2, "inv", 1e-3, 128, 16, seed=40 + j)
        h2.set_precision(pp.TF32)
        h2.upload()
        hs.append(h2)
    bt = pp.Batch(gctx, hs)
    bt.factor()
    bt.sync()
    for h, F in zip(hs, alone):
        h.download()
        assert np.array_equal(h.to_dense(), F)
