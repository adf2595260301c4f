"""C ABI: the library loads, exports what include/pastel_palettes.h declares, validates
arguments, and never computes on the host (no CPU fallback)."""
import ctypes as C
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(pp):
    lib = pp.lib()
    declared = pp.exported_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", pp.LIB_PATH], capture_output=True, text=True).stdout
    for s in declared:
        assert f" T {s}" in out, s


def test_host_context_refuses_compute(pp, hctx):
    h, _ = pp.make_dense_problem(hctx, n=256, leaf=64)
    with pytest.raises(pp.PPError) as e:
        h.upload()
    assert e.value.status == pp.PP_CUDA_ERROR
    with pytest.raises(pp.PPError) as e:
        h.factor()
    assert e.value.status in (pp.PP_CUDA_ERROR, pp.PP_INVALID_ARG)


def test_invalid_arguments(pp, hctx):
    lib = pp.lib()
    out = C.c_void_p()
    assert lib.pp_hmatrix_create_dense(hctx.handle, 0, 64, C.byref(out)) == pp.PP_INVALID_ARG
    pts = np.zeros((4, 2))
    assert lib.pp_hmatrix_create_geometric(hctx.handle, 4, 2, pts.ctypes.data_as(C.POINTER(C.c_double)), 2, 0, 1.0,
                                           0, C.byref(out)) == pp.PP_INVALID_ARG
    with pytest.raises(pp.PPError):
        pp.Context(device=-1, tile=4)
    h, _ = pp.make_dense_problem(hctx, n=128, leaf=64)
    with pytest.raises(pp.PPError):
        h.set_lowrank(h.root, np.zeros((2, 2)), np.zeros((2, 2)))


def test_block_tree_of_configurations(pp, hctx):
    h, _ = pp.make_dense_problem(hctx, n=1024, leaf=256)
    blocks = h.blocks()
    assert sum(b["kind"] == pp.DENSE for b in blocks) == 16
    assert h.getNy_abs() == h.getNx_abs() == 1024
    pts = np.random.default_rng(0).uniform(0, 1, (8192, 2))
    pts = pts[pp.morton_order(pts)]
    hg = pp.Hierarchical.geometric(hctx, pts, 256, 0, 1.0, 16)
    kinds = [b["kind"] for b in hg.blocks()]
    assert kinds.count(pp.DENSE) == 32 and kinds.count(pp.LOWRANK) == 62


def test_factor_program_flops_match_dense_count(pp, hctx):
    h, _ = pp.make_dense_problem(hctx, n=1024, leaf=256)
    n = 1024
    assert h.program_info(0)["flops"] == 2 * n ** 3 // 3 - n ** 2 // 2 - n // 6 == 715303424


def test_reference_isa_switch(pp):
    # split-k reductions (SUM) speed up long-k products but have no reference form
    fast = pp.Context(device=-1)
    h, _ = pp.make_kernel_problem(fast, 2048, 2, "inv", 1e-3, 256, 16)
    assert h.program_info(0)["op_count"]["sum"] > 0
    with pytest.raises(pp.PPError) as e:
        h.refstreams(1)
    assert e.value.status == pp.PP_UNSUPPORTED
    ref = pp.Context(device=-1, reference_isa=1)
    h2, _ = pp.make_kernel_problem(ref, 2048, 2, "inv", 1e-3, 256, 16)
    assert h2.program_info(0)["op_count"]["sum"] == 0
    words, lengths, tmp = h2.refstreams(1)
    assert len(words) > 0


def test_refstream_rejects_solve_only_instruction(pp, hctx):
    # the factor program is expressible in the reference's instruction set
    h, _ = pp.make_kernel_problem(hctx, 512, 2, "inv", 1e-3, 64, 8)
    words, lengths, tmp = h.refstreams(1)
    assert words[0] == 1 and words[-1] == 0


def test_precision_switch_marks_gemm_instructions(pp, hctx):
    h, _ = pp.make_kernel_problem(hctx, 1024, 2, "inv", 1e-3, 128, 16)
    bases = [0x1000000 * (i + 1) for i in range(5)]
    t64, _, _, _ = h.encode_program(0, 1, bases)
    assert h.precision == pp.FP64
    assert np.all(t64["prec"] == pp.FP64)
    h.set_precision(pp.TF32)
    t32, s32, _, _ = h.encode_program(0, 1, bases)
    gemm = t32["op"] == pp.OP_NAMES.index("gemm")
    # the tensor-core form goes to the GEMMs of at least 64 in every dimension (dense Schur
    # updates); skinny low-rank products stay FP64
    big = gemm & (t32["m"] >= 64) & (t32["n"] >= 64) & (t32["k"] >= 64)
    assert big.any() and (gemm & ~big).any()
    assert np.all(t32["prec"][big] == pp.TF32)
    assert np.all(t32["prec"][~big] == pp.FP64)
    # same program otherwise; the solve program stays FP64
    assert np.array_equal(t32["op"], t64["op"])
    ts, _, _, _ = h.encode_program(1, 1, bases)
    assert np.all(ts["prec"] == pp.FP64)
    assert pp.lib().pp_hmatrix_set_precision(h.handle, 7) == pp.PP_INVALID_ARG
    h.set_precision(pp.FP64)
    assert np.array_equal(h.encode_program(0, 1, bases)[0], t64)


def test_residual_batch_refuses_without_device_and_counts_launches(pp, hctx):
    """The batched residual refuses a host context, and the launch count the refiners report
    follows the library's grouping (update and reduction per 64 jobs, residual per group of
    kernel / dimension / RHS width per 64 jobs, one per job above 4 RHS)."""
    job = pp._ResidualJob(0, 2, 8, 1, 1e-3, 0.0, 1, 1, None, 1, 1)
    assert pp.lib().pp_kernel_residual_batch_dev(hctx._h, 1, C.byref(job), None) == pp.PP_CUDA_ERROR
    count = pp.residual_batch_launches
    assert count([]) == 0
    assert count([(0, 2, 1, True)] * 64) == 3
    assert count([(0, 2, 1, True)] * 65) == 6
    assert count([(0, 2, 1, False), (0, 2, 3, False), (2, 3, 1, False)]) == 4
    assert count([(0, 2, 8, True), (0, 2, 16, True), (1, 3, 4, True)]) == 1 + 1 + 2 + 1


def test_gemm_tile_option_shrinks_the_factor_program(pp, hctx):
    """128 x 128 product tiles: fewer GEMM instructions and the same flops; only 64 and 128."""
    h1, _ = pp.make_kernel_problem(hctx, 2048, 2, "inv", 1e-3, 256, 16)
    h2, _ = pp.make_kernel_problem(hctx, 2048, 2, "inv", 1e-3, 256, 16)
    h2.set_gemm_tile(128)
    with pytest.raises(pp.PPError):
        h2.set_gemm_tile(32)
    i1, i2 = h1.program_info(0), h2.program_info(0)
    assert i2["op_count"]["gemm"] < i1["op_count"]["gemm"]
    assert i2["flops"] == i1["flops"]
    assert h2.program_info(1)["n_tasks"] == h1.program_info(1)["n_tasks"]  # the solve keeps 64


def test_device_assembly_refuses_host_context(pp, hctx):
    """Dense-block assembly on the device needs a device context (no host fallback)."""
    h, prob = pp.make_kernel_problem(hctx, 512, 2, "inv", 1e-3, 128, 16)
    pts = np.ascontiguousarray(prob.points)
    st = pp.lib().pp_hmatrix_assemble_dense_dev(h.handle, int(prob.kernel), float(prob.p0), float(prob.shift),
                                                pts.ctypes.data, 2, None)
    assert st == pp.PP_CUDA_ERROR


def test_device_dag_needs_device_context(pp, hctx):
    """The device DAG build is refused for a host-only context (no silent host build claim)."""
    with pytest.raises(pp.PPError):
        hctx.set_device_dag(True)
    h = pp.Hierarchical.dense(hctx, 512, 128)
    ms, on_dev = h.dag_info(0)
    assert not on_dev and ms >= 0.0


def test_gmres_and_pivot_entry_points_validate_arguments(pp, hctx):
    """Host-side argument checks of the GMRES, low-precision product and pivoting entry points:
    refused before anything reaches a device."""
    import ctypes as C
    L = pp.lib()
    g = C.c_void_p()
    n = (C.c_int * 1)(128)
    ptrs = (C.c_void_p * 1)(C.c_void_p(0x1000))
    # a host-only context has no device to run on
    assert L.pp_gmres_create(hctx.handle, 1, n, 8, ptrs, ptrs, ptrs, ptrs, C.byref(g)) == pp.PP_CUDA_ERROR
    assert L.pp_gmres_start(None, None) == pp.PP_INVALID_ARG
    assert L.pp_gmres_arnoldi(None, 0, None) == pp.PP_INVALID_ARG
    assert L.pp_gmres_finish(None, None) == pp.PP_INVALID_ARG
    job = pp._ResidualJob()
    assert L.pp_kernel_residual_batch_lowp_dev(hctx.handle, 1, C.byref(job), None) == pp.PP_CUDA_ERROR
    h = pp.Hierarchical.dense(hctx, 256, 64)
    assert L.pp_hmatrix_set_pivoting(h.handle, 2) == pp.PP_INVALID_ARG
    assert L.pp_hmatrix_set_pivoting(None, 1) == pp.PP_INVALID_ARG
    h.set_pivoting(True)
    info = h.program_info(0)
    assert info["op_count"]["trinv"] == 0 and info["op_count"]["getrf"] > 0
    h.set_pivoting(False)
    assert h.program_info(0)["op_count"]["trinv"] > 0


def test_pivoted_programs_have_no_reference_stream(pp):
    """The reference's int32 stream format has no pivoting: export is refused, not silently
    unpivoted."""
    ctx = pp.Context(device=-1, reference_isa=1)
    h = pp.Hierarchical.dense(ctx, 256, 64)
    h.set_pivoting(True)
    with pytest.raises(pp.PPError):
        h.refstreams(1)
