"""rts layer: overlap predicate, dependency classification, dependency table, DAG.

Pinned against the reference's own rts/ops.cpp and rts/dependency.cpp, compiled unmodified
into oracle/_ref/libref_rts.so.  The randomized overlap cases follow the reference's only
test (Pastel-Palettes main.cpp:9-43), seeded here so failures reproduce.
"""
import numpy as np
import pytest


def brute_overlap(a, pa, wa, ha, b, pb, wb, hb):
    sa = {a + i * pa + j for i in range(ha) for j in range(wa)}
    return any((b + i * pb + j) in sa for i in range(hb) for j in range(wb))


def ref_rts_or_skip(oracle):
    r = oracle.ref_rts()
    if r is None:
        pytest.skip("reference rts not built (no reference sources)")
    return r


def test_overlap_main_cpp_cases_vs_reference(pp, oracle):
    ref = ref_rts_or_skip(oracle)
    rng = np.random.default_rng(20190731)
    for _ in range(3000):
        a, b = int(rng.integers(0, 200)), int(rng.integers(0, 200))
        ma, na, oa = int(rng.integers(1, 17)), int(rng.integers(1, 17)), int(rng.integers(0, 16))
        mb, nb, ob = int(rng.integers(1, 17)), int(rng.integers(1, 17)), int(rng.integers(0, 16))
        # main.cpp: DataMap2D(ptr=a, pitch=ma+oa, width=ma, height=na)
        args = (a, ma + oa, ma, na, b, mb + ob, mb, nb)
        mine = pp.lib().pp_datamap2d_check_overlap(*args)
        theirs = ref.ref_check_overlap(*args)
        assert mine == theirs == brute_overlap(*args), args


def test_overlap_large_pitched_regions_vs_reference(pp, oracle):
    ref = ref_rts_or_skip(oracle)
    rng = np.random.default_rng(7)
    base = 1 << 20
    for _ in range(3000):
        pa = 8 * int(rng.integers(1, 600))
        pb = pa if rng.random() < 0.5 else 8 * int(rng.integers(1, 600))
        wa, wb = 8 * int(rng.integers(1, pa // 8 + 1)), 8 * int(rng.integers(1, pb // 8 + 1))
        ha, hb = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        a = base + 8 * int(rng.integers(0, 20000))
        b = base + 8 * int(rng.integers(0, 20000))
        args = (a, pa, wa, ha, b, pb, wb, hb)
        assert pp.lib().pp_datamap2d_check_overlap(*args) == ref.ref_check_overlap(*args), args


def test_overlap_empty_regions_overlap_nothing(pp):
    assert pp.DataMap2D(64, 64, 0, 4).checkOverlap(pp.DataMap2D(64, 64, 8, 4)) is False
    assert pp.DataMap2D(64, 64, 8, 0).checkOverlap(pp.DataMap2D(64, 64, 8, 4)) is False
    assert pp.DataMap2D(64, 64, 8, 1).checkOverlap(pp.DataMap2D(64, 64, 8, 1)) is True


def test_operation_dependency_classification(pp, oracle):
    ref = ref_rts_or_skip(oracle)
    rng = np.random.default_rng(3)

    def region():
        p = 8 * int(rng.integers(1, 40))
        return pp.DataMap2D(8 * int(rng.integers(0, 400)), p, 8 * int(rng.integers(1, p // 8 + 1)),
                            int(rng.integers(1, 20)))

    for _ in range(500):
        f = pp.Operation([(bool(rng.integers(0, 2)), region()) for _ in range(int(rng.integers(1, 4)))])
        t = pp.Operation([(bool(rng.integers(0, 2)), region()) for _ in range(int(rng.integers(1, 4)))])
        want = 0
        for rof, df in f.data:
            for rot, dt in t.data:
                if ref.ref_check_overlap(df.ptr, df.pitch, df.width, df.height, dt.ptr, dt.pitch, dt.width, dt.height):
                    if not rof and rot:
                        want = ref.ref_dependency_combine(want, 1)
                    if rof and not rot:
                        want = ref.ref_dependency_combine(want, 2)
                    if not rof and not rot:
                        want = ref.ref_dependency_combine(want, 4)
        assert t.checkDependencyFrom(f) == want
        assert f.checkDependencyTo(t) == want


def test_dependency_table_semantics_vs_reference(oracle):
    ref = ref_rts_or_skip(oracle)
    rng = np.random.default_rng(11)
    tab = ref.ref_table_create()
    model = {}
    try:
        for _ in range(400):
            f, t, d = int(rng.integers(0, 30)), int(rng.integers(0, 30)), int(rng.integers(1, 8))
            ref.ref_table_update(tab, f, t, d)
            model[(f, t)] = d
        for f in range(30):
            assert ref.ref_table_count_from(tab, f) == sum(1 for (a, _) in model if a == f)
            assert ref.ref_table_count_to(tab, f) == sum(1 for (_, b) in model if b == f)
            for t in range(30):
                assert ref.ref_table_lookup(tab, f, t) == model.get((f, t), 0)
    finally:
        ref.ref_table_destroy(tab)


# ----------------------------------------------------------------------------- DAG validator
def task_regions(T):
    """(ptr, pitch, width, height, read_only) byte regions an instruction touches
    (the random sketch of accum is read-only shared data and excluded)."""
    op, m, n, k, l = int(T["op"]), int(T["m"]), int(T["n"]), int(T["k"]), int(T["l"])
    ld, p, fl = T["ld"], T["p"], int(T["flags"])

    def reg(i, rows, cols, ro):
        if (fl >> (4 + i)) & 1:
            rows, cols = cols, rows
        return (int(p[i]), 8 * int(ld[i]), 8 * cols, rows, ro)

    if op == 1:
        return [reg(0, m, n, False)]
    if op in (2, 4, 5):
        return [reg(0, m, n, False), reg(1, m, m, True)]
    if op == 3:
        return [reg(0, m, n, False), reg(1, n, n, True)]
    if op == 6:
        return [reg(0, m, n, False), reg(1, m, k, True), reg(2, k, n, True)]
    if op == 9:
        return [reg(0, m, k, False), reg(1, n, k, False), reg(2, m, l, True), reg(3, n, l, True)]
    if op == 10:
        return [reg(0, m, n, False), reg(1, k * m, n, True)]
    if op == 11:  # TRINV: an m x n column block of an inverse from the m x m leaf factors
        return [reg(0, m, n, False), reg(1, m, m, True)]
    if op == 12:  # TRMV: B (m x n) := M B, M m x m; l > 0: rows [o, o + l) of M S (S at p[2])
        if l > 0:
            return [reg(0, l, n, False), reg(1, m, m, True), reg(2, m, n, True)]
        return [reg(0, m, n, False), reg(1, m, m, True)]
    if op == 13:  # ORTH: Y (m x n) in place
        return [reg(0, m, n, False)]
    if op == 14:  # COPY: C (m x n) := A
        return [reg(0, m, n, False), reg(1, m, n, True)]
    raise AssertionError(f"unexpected op {op}")


def check_dag(pp, h, which, nrhs, overlap):
    info = h.program_info(which, nrhs)
    sizes = info["arena_elems"]
    # disjoint fake address ranges per arena (no memory behind them: regions only)
    bases, at = [], 1 << 32
    for a in pp.ARENAS:
        bases.append(at)
        at += 8 * (sizes[a] + 4096) + (1 << 20)
    tasks, succ, indeg, ready = h.encode_program(which, nrhs, bases)
    n = len(tasks)
    regs = [task_regions(t) for t in tasks]
    # reachability (program order is topological): bitset of descendants
    reach = [0] * n
    for t in range(n - 1, -1, -1):
        r = 0
        for q in range(tasks[t]["n_succ"]):
            s = int(succ[tasks[t]["succ_begin"] + q])
            assert s > t
            r |= (1 << s) | reach[s]
        reach[t] = r
    # byte spans for a fast pre-filter
    spans = [[(g[0], g[0] + (g[3] - 1) * g[1] + g[2]) for g in rs] for rs in regs]
    conflicts = 0
    for i in range(n):
        for j in range(i + 1, n):
            hit = False
            for gi, si in zip(regs[i], spans[i]):
                for gj, sj in zip(regs[j], spans[j]):
                    if si[1] <= sj[0] or sj[1] <= si[0] or (gi[4] and gj[4]):
                        continue
                    if overlap(gi[0], gi[1], gi[2], gi[3], gj[0], gj[1], gj[2], gj[3]):
                        hit = True
                        break
                if hit:
                    break
            if hit:
                conflicts += 1
                assert (reach[i] >> j) & 1, f"conflicting tasks {i} -> {j} are not ordered"
    assert sum(indeg == 0) == len(ready)
    return conflicts


def test_dag_orders_every_conflict_dense(pp, oracle, hctx):
    ref = oracle.ref_rts()
    overlap = ref.ref_check_overlap if ref is not None else pp.lib().pp_datamap2d_check_overlap
    h, _ = pp.make_dense_problem(hctx, n=512, leaf=128)
    assert check_dag(pp, h, 0, 1, overlap) > 0


def test_dag_orders_every_conflict_hodlr(pp, oracle, hctx):
    ref = oracle.ref_rts()
    overlap = ref.ref_check_overlap if ref is not None else pp.lib().pp_datamap2d_check_overlap
    h, _ = pp.make_kernel_problem(hctx, 1024, 2, "inv", 1e-3, 128, 8)
    assert check_dag(pp, h, 0, 1, overlap) > 0
    assert check_dag(pp, h, 1, 2, overlap) > 0


def test_edge_types_match_classification(pp, hctx):
    h, _ = pp.make_kernel_problem(hctx, 512, 2, "inv", 1e-3, 64, 8)
    f, t, ty = h.edges(0)
    assert len(f) == h.program_info(0)["n_edges"] > 0
    assert np.all(f < t) and np.all((ty >= 1) & (ty <= 7))


def test_scheduler_streams_cover_every_instruction(pp, hctx):
    h, _ = pp.make_kernel_problem(hctx, 1024, 2, "inv", 1e-3, 128, 8)
    tasks, _, _, _ = h.encode_program(0, 1, [0x1000000 * (i + 1) for i in range(5)])
    # every instruction of the factorization proper; TRINV (the solves' inverse
    # preparation, no reference counterpart) is left out of the reference streams
    expect = [i for i in range(len(tasks)) if int(tasks["op"][i]) != pp.OP_NAMES.index("trinv")]
    assert len(expect) < len(tasks)
    for workers in (1, 3, 16):
        words, lengths, tmp = h.refstreams(workers)
        seen, at = [], 0
        for w in range(workers):
            s = words[at: at + lengths[w]]
            at += lengths[w]
            pc = 0
            while s[pc] != 0:
                if s[pc] == 1:
                    seen.append(int(s[pc + 1]))
                    pc += {1: 8, 2: 13, 3: 13, 4: 17, 5: 17, 6: 23, 7: 29, 8: 21}[int(s[pc + 2])]
                else:
                    assert s[pc] == 2 and workers > 1
                    pc += 3
            assert pc == lengths[w] - 1
        assert sorted(seen) == expect
        if workers == 1:
            assert len(words) > 0 and tmp > 0


def test_solve_program_splits_leaf_products(pp, hctx):
    """Every leaf product of the solve program on a triangle of 128 rows or more is cut into
    out-of-place parts of at most 64 rows that cover the triangle's rows once, each followed by
    one copy back into the right-hand side."""
    h, _ = pp.make_kernel_problem(hctx, 2048, 2, "inv", 1e-3, 256, 16)
    info = h.program_info(1, 1)
    bases, at = [], 1 << 32
    for a in pp.ARENAS:
        bases.append(at)
        at += 8 * (info["arena_elems"][a] + 4096) + (1 << 20)
    tasks, succ, indeg, ready = h.encode_program(1, 1, bases)
    parts = {}
    for t in tasks:
        if int(t["op"]) == 12:
            assert int(t["l"]) > 0 and int(t["m"]) >= 128
            parts.setdefault((int(t["p"][1]), int(t["p"][2])), []).append((int(t["o"]), int(t["l"]), int(t["m"])))
    copies = sum(1 for t in tasks if int(t["op"]) == 14)
    assert parts and copies == len(parts)
    for rows in parts.values():
        rows.sort()
        m = rows[0][2]
        assert all(l <= 64 for _, l, _ in rows)
        assert rows[0][0] == 0 and all(a[0] + a[1] == b[0] for a, b in zip(rows, rows[1:]))
        assert rows[-1][0] + rows[-1][1] == m
