"""Programs of large leaves (512 rows and more) on the CPU: whole-leaf Schur updates are one
instruction each, triangular solves of such leaves take 256-row triangles, and the BF16 form
adds one SHADOW instruction per operand block.  The oracle's run of the FP64 program is the
textbook no-pivot LU bit for bit (every element keeps its ascending update chain)."""
import numpy as np


def test_whole_leaf_fp64_program_is_textbook_lu(pp, oracle, hctx):
    h, A = pp.make_dense_problem(hctx, n=1024, leaf=512, seed=5)
    h.set_gemm_tile(128)
    tasks, _, _, _ = h.encode_program(0, 1, [0] * 5)
    big = tasks[(tasks["op"] == 6) & (tasks["m"] == 512) & (tasks["n"] == 512) & (tasks["k"] == 512)]
    assert len(big) == 1  # the Schur update of the trailing leaf
    assert tasks[tasks["op"] == 2]["m"].max() == 256  # 256-row triangles for the 512-column target
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=4)
    h.host_arena()[:] = ar.matrix
    assert np.array_equal(h.to_dense(), oracle.dense_getrf(A))


def test_bf16_program_shadows_each_operand_once(pp, oracle, hctx):
    h, A = pp.make_dense_problem(hctx, n=2048, leaf=512, seed=6)
    h.set_gemm_tile(128)
    h.set_precision(pp.BF16)
    tasks, succ, indeg, _ = h.encode_program(0, 1, [0] * 5)
    g = tasks[(tasks["op"] == 6) & (tasks["prec"] == 2)]
    n_blocks = 4
    # Schur updates of whole leaves: sum over k of (n_blocks - 1 - k)^2
    assert len(g) == sum((n_blocks - 1 - k) ** 2 for k in range(n_blocks))
    # one shadow per L-panel and per U-panel block: 2 * sum over k of (n_blocks - 1 - k)
    assert (tasks["op"] == 15).sum() == 2 * sum(n_blocks - 1 - k for k in range(n_blocks))
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=4)
    h.host_arena()[:] = ar.matrix
    F = h.to_dense()
    ref = oracle.dense_getrf(A)
    assert np.linalg.norm(F - ref) / np.linalg.norm(ref) < 1e-4
