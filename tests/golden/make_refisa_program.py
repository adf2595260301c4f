"""Exports the factorization program of the FP64 HODLR configuration (N = 8192 points of
U[0,1]^2 in Morton order, kernel 1/(r + 1e-3), diagonal shift 2 x max off-diagonal row sum, weak
admissibility, leaf 256, rank 16, seed 1234) restricted to the reference's instruction set
(getrf / trsml / trsmr / gemm / gemm_plus / gemm_3x / gemm_4x / accum: no split-k reductions, no
explicit inverses), so that the oracle can execute it on the CPU without this library.

Writes tests/golden/hodlr8192_refisa_program.npz:
  tasks     the 160-byte task records (pp_task.h); every operand pointer is tagged with its
            arena instead of an address: pointer = ((arena kind + 1) << 44) + byte offset
            (arena kinds: 0 matrix, 1 work, 2 scratch, 3 rhs, 4 random sketch)
  succ, indeg  the DAG (successor lists as the task records index them; in-degrees)
  blocks    one row per block of the tree: kind, row0, col0, m, n, kmax, rank, the element
            offsets of its data (dense data or U), V and rank word (-1: none), children[4]
  meta      the construction recipe and the arena sizes

Run it where the library is built (python tests/golden/make_refisa_program.py); the CPU tests
check that the committed fixture still equals what the library generates.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "hodlr8192_refisa_program.npz")

CONFIG = dict(n=8192, dim=2, kernel=0, p0=1e-3, leaf=256, rank=16, admissibility=0, eta=1.0, seed=1234,
              shift_factor=2.0, rand_seed=0x5EED5EED, tile=64)
TAG_SHIFT = 44


def export(pp, cfg=CONFIG):
    ctx = pp.Context(device=-1, tile=cfg["tile"], seed=cfg["rand_seed"], reference_isa=1)
    h, prob = pp.make_kernel_problem(ctx, cfg["n"], cfg["dim"], cfg["kernel"], cfg["p0"], cfg["leaf"], cfg["rank"],
                                     cfg["admissibility"], cfg["eta"], shift_factor=cfg["shift_factor"],
                                     seed=cfg["seed"])
    info = h.program_info(0, 1)
    bases = [(a + 1) << TAG_SHIFT for a in range(5)]
    tasks, succ, indeg, _ = h.encode_program(0, 1, bases)
    rows = []
    for b in h.blocks():
        off, off_v, off_rank = h.block_storage(b["id"])
        rows.append([b["kind"], b["row0"], b["col0"], b["m"], b["n"], b["kmax"], b["rank"], off, off_v, off_rank,
                     *b["children"]])
    el = info["arena_elems"]
    meta = dict(cfg, shift=prob.shift, norm_inf=prob.norm_inf, root=h.root, matrix_elems=len(h.host_arena()),
                block_elems=int(pp.lib().pp_hmatrix_block_elems(h.handle)), work_elems=el["work"],
                scratch_elems=el["scratch"], rhs_elems=el["rhs"], rand_elems=el["rand"], flops=info["flops"],
                n_tasks=info["n_tasks"], tag_shift=TAG_SHIFT)
    ops = np.bincount(tasks["op"], minlength=16)
    assert ops[10] == 0 and ops[11] == 0 and ops[12] == 0, "reference-ISA program holds engine-only instructions"
    return dict(tasks=tasks.view(np.uint8).reshape(len(tasks), 160), succ=succ, indeg=indeg,
                blocks=np.array(rows, dtype=np.int64), meta_keys=np.array(list(meta.keys())),
                meta_vals=np.array([float(v) for v in meta.values()]))


def main():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_pp
    d = export(load_pp())
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: {d['tasks'].shape[0]} tasks, {d['succ'].size} edges, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
