"""Mixed-precision Schur updates of large leaves (PP_PRECISION_BF16) on the tcgen05 tensor cores.

  SHADOW   the BF16 copy of an operand in the tiled layout: bitwise equal to the oracle's.
  GEMM     (BF16 shadows, FP32 accumulation in tensor memory, FP64 result) against the oracle's
           FP64 sum of the same BF16 products: relative error <= 1e-5 (FP32 accumulation over
           k = 512 terms); several such tasks in one launch on one CTA (the pipeline's barrier
           phases continue from task to task) and on the whole grid.
  programs the FP64 form with whole-leaf Schur instructions bitwise equal to the textbook LU;
           the BF16 form within 1e-4 of the oracle running the same program, and refined to a
           1e-10 backward error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from test_gpu_vm import dev, factor_on_gpu, rel  # noqa: E402

SHADOW, GEMM, BF16 = 15, 6, 2


@pytest.fixture(scope="module")
def bctx(pp):
    """A context whose device waits give up after 20 s (instead of 120 s)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return pp.Context(device=0, spin_limit=20_000_000)


def shadow_pair(pp, rng, rows, k, transposed=False):
    """An FP64 operand (host + device) and zeroed shadow buffers (host + device) for it."""
    src = rng.standard_normal((k, rows) if transposed else (rows, k))
    sh_h = np.zeros(rows * k // 4)
    sh_d = torch.zeros(rows * k // 4, dtype=torch.float64, device="cuda")
    return src, dev(src), sh_h, sh_d


def shadow_task(pp, sh, src, rows, k, transposed, ld):
    t = np.zeros(1, dtype=pp.TASK_DTYPE)
    t[0]["op"], t[0]["m"], t[0]["k"] = SHADOW, rows, k
    t[0]["flags"] = pp_T(1) if transposed else 0
    t[0]["p"][0], t[0]["p"][1] = sh, src
    t[0]["ld"][1] = ld
    return t


def pp_T(i):
    return 1 << (4 + i)


def ptr(x):
    return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data


@pytest.mark.parametrize("transposed", [False, True])
def test_shadow_bitwise_vs_oracle(pp, oracle, bctx, transposed):
    rng = np.random.default_rng(11)
    rows, k = 256, 512
    src, src_d, sh_h, sh_d = shadow_pair(pp, rng, rows, k, transposed)
    ld = src.shape[1]
    bctx.vm_execute(shadow_task(pp, ptr(sh_d), ptr(src_d), rows, k, transposed, ld), np.zeros(0, np.int32),
                    np.zeros(1, np.int32))
    th = shadow_task(pp, ptr(sh_h), ptr(src), rows, k, transposed, ld)
    assert oracle.lib().oracle_run_program(th.ctypes.data, 1) == 0
    assert np.array_equal(sh_d.cpu().numpy().view(np.uint16), sh_h.view(np.uint16))


def _gemm_case(pp, rng, m, n, k):
    """Host and device copies of C, the A / B^T operands and their (empty) shadows."""
    C = rng.standard_normal((m, n))
    A = rng.standard_normal((m, k))
    Bt = rng.standard_normal((n, k))
    return dict(C=C, Cd=dev(C), A=A, Ad=dev(A), Bt=Bt, Btd=dev(Bt), As=np.zeros(m * k // 4),
                Asd=torch.zeros(m * k // 4, dtype=torch.float64, device="cuda"), Bs=np.zeros(n * k // 4),
                Bsd=torch.zeros(n * k // 4, dtype=torch.float64, device="cuda"), m=m, n=n, k=k)


def _gemm_tasks(pp, cases, device):
    """Per case: SHADOW of A, SHADOW of B^T, then the BF16 GEMM C -= A B (successors wired)."""
    recs, succ = [], []
    for c in cases:
        s = "d" if device else ""
        a_sh = shadow_task(pp, ptr(c["As" + s]), ptr(c["A" + s]), c["m"], c["k"], False, c["k"])
        b_sh = shadow_task(pp, ptr(c["Bs" + s]), ptr(c["Bt" + s]), c["n"], c["k"], False, c["k"])
        g = np.zeros(1, dtype=pp.TASK_DTYPE)
        g[0]["op"], g[0]["prec"] = GEMM, BF16
        g[0]["m"], g[0]["n"], g[0]["k"] = c["m"], c["n"], c["k"]
        g[0]["alpha"], g[0]["beta"] = -1.0, 1.0
        g[0]["p"][0], g[0]["p"][1], g[0]["p"][2] = ptr(c["C" + s]), ptr(c["As" + s]), ptr(c["Bs" + s])
        g[0]["ld"][0] = c["n"]
        recs += [a_sh, b_sh, g]
    tasks = np.concatenate(recs)
    indeg = np.zeros(len(tasks), np.int32)
    for i in range(len(cases)):
        g = 3 * i + 2
        for j in (3 * i, 3 * i + 1):
            tasks[j]["succ_begin"], tasks[j]["n_succ"] = len(succ), 1
            succ.append(g)
        indeg[g] = 2
    return tasks, np.array(succ, np.int32), indeg


@pytest.mark.parametrize("grid", [1, 0])
def test_bf16_gemm_tasks_vs_oracle(pp, oracle, bctx, grid):
    rng = np.random.default_rng(21)
    cases = [_gemm_case(pp, rng, m, n, k) for m, n, k in [(512, 512, 512), (128, 256, 64), (256, 768, 192)]]
    C0 = [c["C"].copy() for c in cases]
    td, sd, ind = _gemm_tasks(pp, cases, True)
    bctx.vm_execute(td, sd, ind, grid=grid)
    th, _, _ = _gemm_tasks(pp, cases, False)
    assert oracle.lib().oracle_run_program(th.ctypes.data, len(th)) == 0
    for c, c0 in zip(cases, C0):
        assert np.array_equal(c["Asd"].cpu().numpy(), c["As"]) and np.array_equal(c["Bsd"].cpu().numpy(), c["Bs"])
        # the update C - C0 = -A B: tensor cores (FP32 sums) against the oracle (FP64 sums) of
        # the same BF16 products
        assert rel(c["Cd"].cpu().numpy() - c0, c["C"] - c0) < 1e-5


def test_bf16_gemm_matches_fp64_product_of_rounded_operands(pp, bctx):
    rng = np.random.default_rng(3)
    c = _gemm_case(pp, rng, 256, 512, 512)
    C0 = c["C"].copy()
    td, sd, ind = _gemm_tasks(pp, [c], True)
    bctx.vm_execute(td, sd, ind)
    Cg = c["Cd"].cpu().numpy()

    def bf16(x):
        u = x.astype(np.float32).view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
        return u.astype(np.uint32).view(np.float32).astype(np.float64)

    want = C0 - bf16(c["A"]) @ bf16(c["Bt"]).T
    assert np.abs(Cg - want).max() <= 1e-5 * np.abs(bf16(c["A"])).sum(1).max() * np.abs(bf16(c["Bt"])).max()


def test_fp64_whole_leaf_program_bitwise(pp, oracle, bctx):
    h, A = pp.make_dense_problem(bctx, n=2048, leaf=512, seed=8)
    h.set_gemm_tile(128)
    ops = h.program_info(0)["op_count"]
    assert ops["gemm"] > 0 and ops["shadow"] == 0
    assert np.array_equal(factor_on_gpu(h), oracle.dense_getrf(A))


def test_bf16_program_matches_oracle_and_refines(pp, oracle, bctx):
    n = 4096
    h, prob = pp.make_kernel_problem(bctx, n, 3, "laplace", 1e-3, 512, 32, admissibility=1, eta=1.0, seed=5,
                                     rank_tol=1e-8)
    h.set_gemm_tile(128)
    h.set_precision(pp.BF16)
    info = h.program_info(0)
    assert info["op_count"]["shadow"] > 0
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=16)
    F = factor_on_gpu(h)
    h.host_arena()[:] = ar.matrix
    assert rel(F, h.to_dense()) < 1e-4
    # refinement with the FP64 matrix-free residual to 1e-10
    h2, prob2 = pp.make_kernel_problem(bctx, n, 3, "laplace", 1e-3, 512, 32, admissibility=1, eta=1.0, seed=5,
                                       rank_tol=1e-8)
    h2.set_gemm_tile(128)
    h2.set_precision(pp.BF16)
    h2.upload()
    h2.factor()
    b = pp.rhs(n, 8)
    x, hist = pp.Refiner(h2, bctx, prob2).solve(dev(b), tol=1e-10)
    assert hist[-1] <= 1e-10, hist


def _shadow_task_ex(pp, sh, src, rows, k_src, ld, cr):
    """SHADOW with the inner dimension padded to a multiple of 64 and chunks of cr rows."""
    K = (k_src + 63) // 64 * 64
    t = shadow_task(pp, sh, src, rows, K, False, ld)
    t[0]["n"] = k_src if k_src < K else 0
    t[0]["ctrl"] = 0 if cr == 128 else cr
    return t, K


@pytest.mark.parametrize("m,n,k", [(512, 32, 512), (256, 64, 128), (512, 512, 32), (128, 128, 64)])
def test_bf16_skinny_and_padded_products_vs_oracle(pp, oracle, bctx, m, n, k):
    """Products the mixed form runs beside the Schur updates: a dense leaf times a low-rank factor
    (n = 32: B shadow of 32-row chunks) and rank-k updates of a leaf (k = 32 padded to 64)."""
    rng = np.random.default_rng(m + n + k)
    C, A, Bt = rng.standard_normal((m, n)), rng.standard_normal((m, k)), rng.standard_normal((n, k))
    K = (k + 63) // 64 * 64
    cr = 128 if n % 256 == 0 else n
    out = {}
    for side in ("dev", "host"):
        mk = (lambda x: dev(x)) if side == "dev" else (lambda x: x.copy())
        Cx, Ax, Bx = mk(C), mk(A), mk(Bt)
        As = torch.zeros(m * K // 4, dtype=torch.float64, device="cuda") if side == "dev" else np.zeros(m * K // 4)
        Bs = torch.zeros(n * K // 4, dtype=torch.float64, device="cuda") if side == "dev" else np.zeros(n * K // 4)
        ta, _ = _shadow_task_ex(pp, ptr(As), ptr(Ax), m, k, k, 128)
        tb, _ = _shadow_task_ex(pp, ptr(Bs), ptr(Bx), n, k, k, cr)
        g = np.zeros(1, dtype=pp.TASK_DTYPE)
        g[0]["op"], g[0]["prec"] = GEMM, BF16
        g[0]["m"], g[0]["n"], g[0]["k"] = m, n, K
        g[0]["alpha"], g[0]["beta"] = -1.0, 1.0
        g[0]["p"][0], g[0]["p"][1], g[0]["p"][2] = ptr(Cx), ptr(As), ptr(Bs)
        g[0]["ld"][0] = n
        tasks = np.concatenate([ta, tb, g])
        tasks[0]["succ_begin"], tasks[0]["n_succ"] = 0, 1
        tasks[1]["succ_begin"], tasks[1]["n_succ"] = 1, 1
        if side == "dev":
            bctx.vm_execute(tasks, np.array([2, 2], np.int32), np.array([0, 0, 2], np.int32))
            out[side] = (Cx.cpu().numpy(), As.cpu().numpy(), Bs.cpu().numpy())
        else:
            assert oracle.lib().oracle_run_program(tasks.ctypes.data, 3) == 0
            out[side] = (Cx, As, Bs)
    (Cd, Asd, Bsd), (Ch, Ash, Bsh) = out["dev"], out["host"]
    assert np.array_equal(Asd, Ash) and np.array_equal(Bsd, Bsh)
    assert rel(Cd - C, Ch - C) < 1e-5


SPLIT_A, SPLIT_B = (3 << 8) | 2, (3 << 8) | 4


@pytest.mark.parametrize("transposed,split,cr", [(False, SPLIT_A, 128), (True, SPLIT_A, 128),
                                                 (False, SPLIT_B, 128), (True, SPLIT_B, 32)])
def test_split_shadow_bitwise_vs_oracle(pp, oracle, bctx, transposed, split, cr):
    """Split shadows (three segments: bf16(x) or the residual bf16(x - bf16(x))), the operands of
    the mixed form's products with explicit inverses; 480 source columns padded to 512."""
    rng = np.random.default_rng(12 + split)
    rows, k_src = 256, 480
    K = 512
    src = rng.standard_normal((k_src, rows) if transposed else (rows, k_src)) * 10.0 ** rng.integers(-3, 3)
    ld = src.shape[1]
    out = []
    for side in ("dev", "host"):
        sh = torch.zeros(rows * 3 * K // 4, dtype=torch.float64, device="cuda") if side == "dev" else \
            np.zeros(rows * 3 * K // 4)
        s = dev(src) if side == "dev" else src
        t = shadow_task(pp, ptr(sh), ptr(s), rows, 3 * K, transposed, ld)
        t[0]["n"], t[0]["o"], t[0]["ctrl"] = k_src, split, 0 if cr == 128 else cr
        if side == "dev":
            bctx.vm_execute(t, np.zeros(0, np.int32), np.zeros(1, np.int32))
            out.append(sh.cpu().numpy())
        else:
            assert oracle.lib().oracle_run_program(t.ctypes.data, 1) == 0
            out.append(sh)
    assert np.array_equal(out[0].view(np.uint16), out[1].view(np.uint16))


@pytest.mark.parametrize("m,n,k", [(512, 512, 512), (512, 32, 512), (256, 256, 256)])
def test_split_product_accuracy(pp, oracle, bctx, m, n, k):
    """C := A B (beta 0) from split shadows [hi lo hi] x [hi hi lo] (K = 3 k): within 2e-5 of the
    FP64 product relative to |A| |B| (BF16 alone: about 4e-3), and within 1e-5 of the oracle's
    FP64 sum of the same products (the tensor cores sum the 3 k terms in FP32)."""
    rng = np.random.default_rng(m + n + k)
    A, Bt = rng.standard_normal((m, k)), rng.standard_normal((n, k))
    cr = 128 if n % 256 == 0 else n
    out = {}
    for side in ("dev", "host"):
        mk = (lambda x: dev(x)) if side == "dev" else (lambda x: x.copy())
        Cx, Ax, Bx = mk(np.full((m, n), 7.0)), mk(A), mk(Bt)
        z = lambda e: torch.zeros(e, dtype=torch.float64, device="cuda") if side == "dev" else np.zeros(e)
        As, Bs = z(m * 3 * k // 4), z(n * 3 * k // 4)
        ta = shadow_task(pp, ptr(As), ptr(Ax), m, 3 * k, False, k)
        ta[0]["o"] = SPLIT_A
        tb = shadow_task(pp, ptr(Bs), ptr(Bx), n, 3 * k, False, k)
        tb[0]["o"], tb[0]["ctrl"] = SPLIT_B, 0 if cr == 128 else cr
        g = np.zeros(1, dtype=pp.TASK_DTYPE)
        g[0]["op"], g[0]["prec"] = GEMM, BF16
        g[0]["m"], g[0]["n"], g[0]["k"] = m, n, 3 * k
        g[0]["alpha"], g[0]["beta"] = 1.0, 0.0
        g[0]["p"][0], g[0]["p"][1], g[0]["p"][2] = ptr(Cx), ptr(As), ptr(Bs)
        g[0]["ld"][0] = n
        tasks = np.concatenate([ta, tb, g])
        tasks[0]["succ_begin"], tasks[0]["n_succ"] = 0, 1
        tasks[1]["succ_begin"], tasks[1]["n_succ"] = 1, 1
        if side == "dev":
            bctx.vm_execute(tasks, np.array([2, 2], np.int32), np.array([0, 0, 2], np.int32))
            out[side] = Cx.cpu().numpy()
        else:
            assert oracle.lib().oracle_run_program(tasks.ctypes.data, 3) == 0
            out[side] = Cx
    want = A @ Bt.T
    scale = np.abs(A) @ np.abs(Bt).T
    assert (np.abs(out["dev"] - want) / scale).max() < 2e-5
    assert (np.abs(out["host"] - want) / scale).max() < 2e-5
    assert rel(out["dev"], out["host"]) < 1e-5


@pytest.mark.parametrize("m,n,k1,k2", [(512, 512, 512, 512), (256, 512, 512, 64), (512, 32, 64, 512)])
def test_bf16_gemm_two_pairs_vs_oracle(pp, oracle, bctx, m, n, k1, k2):
    """C -= A1 B1 + A2 B2 in one pass over C (the merged form of two consecutive updates of one
    leaf): against the oracle's FP64 sums of the same BF16 products, within 1e-5 of the update."""
    rng = np.random.default_rng(m + n + k1 + 7 * k2)
    C = rng.standard_normal((m, n))
    ops = [(rng.standard_normal((m, k)), rng.standard_normal((n, k)), k) for k in (k1, k2)]
    cr = 128 if n % 256 == 0 else n
    out = {}
    for side in ("dev", "host"):
        mk = (lambda x: dev(x)) if side == "dev" else (lambda x: x.copy())
        z = (lambda e: torch.zeros(e, dtype=torch.float64, device="cuda")) if side == "dev" else np.zeros
        Cx = mk(C)
        recs, sh = [], []
        for A, Bt, k in ops:
            Ax, Bx = mk(A), mk(Bt)
            As, Bs = z(m * k // 4), z(n * k // 4)
            ta = shadow_task(pp, ptr(As), ptr(Ax), m, k, False, k)
            tb = shadow_task(pp, ptr(Bs), ptr(Bx), n, k, False, k)
            tb[0]["ctrl"] = 0 if cr == 128 else cr
            recs += [ta, tb]
            sh += [As, Bs, Ax, Bx]
        g = np.zeros(1, dtype=pp.TASK_DTYPE)
        g[0]["op"], g[0]["prec"] = GEMM, BF16
        g[0]["m"], g[0]["n"], g[0]["k"], g[0]["l"] = m, n, k1, k2
        g[0]["alpha"], g[0]["beta"] = -1.0, 1.0
        g[0]["p"][0], g[0]["p"][1], g[0]["p"][2] = ptr(Cx), ptr(sh[0]), ptr(sh[1])
        g[0]["p"][3], g[0]["p"][4] = ptr(sh[4]), ptr(sh[5])
        g[0]["ld"][0] = n
        tasks = np.concatenate(recs + [g])
        for i in range(4):
            tasks[i]["succ_begin"], tasks[i]["n_succ"] = i, 1
        if side == "dev":
            bctx.vm_execute(tasks, np.full(4, 4, np.int32), np.array([0, 0, 0, 0, 4], np.int32))
            out[side] = Cx.cpu().numpy()
        else:
            assert oracle.lib().oracle_run_program(tasks.ctypes.data, 5) == 0
            out[side] = Cx
    assert rel(out["dev"] - C, out["host"] - C) < 1e-5
    want = C - sum(A @ Bt.T for A, Bt, _ in ops)
    assert rel(out["host"], want) < 1e-2  # BF16 rounding of the operands
