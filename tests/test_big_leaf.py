"""Programs of large leaves (512 rows and more) on the CPU: whole-leaf Schur updates are one
instruction each, triangular solves of such leaves take 256-row triangles, and the BF16 form
adds one SHADOW instruction per operand block and solves each panel block with one product
against the diagonal leaf's explicit inverse from split shadows.  The oracle's run of the FP64
program is the textbook no-pivot LU bit for bit (every element keeps its ascending update
chain)."""
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
    panels = sum(n_blocks - 1 - k for k in range(n_blocks))  # per side
    # Schur updates of whole leaves: sum over k of (n_blocks - 1 - k)^2, consecutive updates of the
    # same leaf two to a task (a second operand pair, inner dimension l)
    schur = g[g["k"] == 512]
    assert len(schur) + (schur["l"] > 0).sum() == sum((n_blocks - 1 - k) ** 2 for k in range(n_blocks))
    assert (schur["l"] == 512).sum() > 0 and set(np.unique(schur["l"])) <= {0, 512}
    # panel solves: one split product (K = 3 x 512) per L-panel and per U-panel block, and no
    # triangular solve task on a whole leaf
    assert (g["k"] == 3 * 512).sum() == 2 * panels
    assert tasks[np.isin(tasks["op"], (2, 3))]["m"].max() <= 64 and tasks[np.isin(tasks["op"], (2, 3))]["n"].max() <= 64
    sh = tasks[tasks["op"] == 15]
    # one plain shadow per L-panel and per U-panel block (the Schur operands); split shadows of
    # every panel target and of both inverses of each leaf that has panels
    assert (sh["o"] == 0).sum() == 2 * panels
    assert (sh["o"] != 0).sum() == 2 * panels + 2 * (n_blocks - 1)
    assert set(np.unique(sh["o"][sh["o"] != 0])) == {(3 << 8) | 2, (3 << 8) | 4}
    ar = oracle.HostArenas(h, 0)
    ar.run(threads=4)
    h.host_arena()[:] = ar.matrix
    F = h.to_dense()
    ref = oracle.dense_getrf(A)
    assert np.linalg.norm(F - ref) / np.linalg.norm(ref) < 1e-4
