"""TEST ORACLE — CPU restatement of the reference's FP64 block routines and loaders for the
reference's own compiled pieces.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py.  The product never imports it.

  liboracle.so        oracle.cpp: DenseGetrf / DenseTrsmL / DenseTrsmR / _transposeB /
                      blockDenseGemm / _3x / _4x / blockLowRankAccum (Givens) restated from
                      Pastel-Palettes src/kernel.cu, plus a sequential and a threaded executor
                      of task tables (pp_task.h)
  _ref/libref_rts.so  the reference's rts/ops.cpp + rts/dependency.cpp, compiled unmodified
  _ref/libref_vm.so   the reference's src/kernel.cu (kernel_dynamic) compiled for sm_100a
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref_rts = None
_ref_vm = None


def build():
    subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.oracle_run_program.argtypes = [vp, i]
        L.oracle_run_program.restype = i
        L.oracle_run_parallel.argtypes = [vp, i, vp, vp, i]
        L.oracle_run_parallel.restype = i
        L.oracle_dense_getrf.argtypes = [vp, i, i]
        L.oracle_dense_getrf.restype = None
        L.oracle_getrf_piv.argtypes = [vp, i, i, vp]
        L.oracle_getrf_piv.restype = None
        L.oracle_gemm.argtypes = [d, d, vp, vp, vp, i, i, i, i, i, i, i, i]
        L.oracle_gemm.restype = None
        L.oracle_accum.argtypes = [vp, vp, vp, vp, i, i, i, i, i, i, i, i, d, vp, i]
        L.oracle_accum.restype = None
        _lib = L
    return _lib


def ref_rts():
    """The reference's own rts (None when it was not built: no reference sources)."""
    global _ref_rts
    if _ref_rts is None:
        path = os.path.join(HERE, "_ref", "libref_rts.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        u64, sz = C.c_uint64, C.c_size_t
        L.ref_check_overlap.argtypes = [u64, sz, sz, sz, u64, sz, sz, sz]
        L.ref_check_overlap.restype = C.c_int
        L.ref_dependency_combine.argtypes = [C.c_int, C.c_int]
        L.ref_dependency_combine.restype = C.c_int
        L.ref_table_create.restype = C.c_void_p
        L.ref_table_destroy.argtypes = [C.c_void_p]
        L.ref_table_update.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong, C.c_int]
        L.ref_table_lookup.argtypes = [C.c_void_p, C.c_longlong, C.c_longlong]
        L.ref_table_lookup.restype = C.c_int
        L.ref_table_count_from.argtypes = [C.c_void_p, C.c_longlong]
        L.ref_table_count_from.restype = C.c_longlong
        L.ref_table_count_to.argtypes = [C.c_void_p, C.c_longlong]
        L.ref_table_count_to.restype = C.c_longlong
        L.ref_table_list.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_longlong]
        L.ref_table_list.restype = C.c_longlong
        _ref_rts = L
    return _ref_rts


def ref_vm():
    """The reference's own kernel_dynamic launcher (None when not built)."""
    global _ref_vm
    if _ref_vm is None:
        path = os.path.join(HERE, "_ref", "libref_vm.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_vm_run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                 C.c_longlong, C.c_int]
        L.ref_vm_run.restype = C.c_int
        _ref_vm = L
    return _ref_vm


class HostArenas:
    """Host copies of the five arenas of an encoded program (matrix, work, scratch, rhs, rand)."""

    def __init__(self, h, which=0, nrhs=1, rhs=None):
        info = h.program_info(which, nrhs)
        el = info["arena_elems"]
        self.matrix = h.host_arena().copy()
        self.work = np.zeros(max(el["work"], 1))
        self.scratch = np.zeros(max(el["scratch"], 1))
        self.rhs = np.zeros(max(el["rhs"], 1))
        if rhs is not None:
            self.rhs[: rhs.size] = np.ascontiguousarray(rhs).ravel()
        self.rand = h.rand_host() if el["rand"] > 0 else np.zeros(1)
        if self.rand.size == 0:
            self.rand = np.zeros(1)
        self.tasks, self.succ, self.indeg, self.ready = h.encode_program(which, nrhs, self.bases())

    def bases(self):
        return [a.ctypes.data for a in (self.matrix, self.work, self.scratch, self.rhs, self.rand)]

    def run(self, threads=1):
        # the programs accumulate intermediate products into zero-filled work buffers
        # (the device launch clears them too)
        self.work[:] = 0.0
        if threads <= 1:
            rc = lib().oracle_run_program(self.tasks.ctypes.data, len(self.tasks))
        else:
            rc = lib().oracle_run_parallel(self.tasks.ctypes.data, len(self.tasks), self.succ.ctypes.data,
                                           self.indeg.ctypes.data, threads)
        if rc != 0:
            raise RuntimeError(f"oracle: task {rc - 1} unsupported")


def dense_getrf(A):
    """Textbook right-looking LU without pivoting, L\\U in place of a copy of A."""
    M = np.ascontiguousarray(A, dtype=np.float64).copy()
    lib().oracle_dense_getrf(M.ctypes.data, M.shape[0], M.shape[1])
    return M


def getrf_piv(A):
    """One block's LU with partial pivoting (largest magnitude, first of equal ones): returns
    (L\\U of P A, perm) with row i of P A = row perm[i] of A."""
    M = np.ascontiguousarray(A, dtype=np.float64).copy()
    perm = np.zeros(M.shape[0])
    lib().oracle_getrf_piv(M.ctypes.data, M.shape[0], M.shape[1], perm.ctypes.data)
    return M, perm.astype(np.int64)


def gemm(alpha, beta, M, A, B, a_T=False, b_T=False):
    """blockDenseGemm restated: M = alpha op(A) op(B) + beta M (in place)."""
    m, n = M.shape
    k = A.shape[0] if a_T else A.shape[1]
    lib().oracle_gemm(alpha, beta, M.ctypes.data, A.ctypes.data, B.ctypes.data, m, n, k, M.shape[1], A.shape[1],
                      B.shape[1], int(a_T), int(b_T))


def accum(U1, V1, U2, V2, rnd, sign=1.0):
    """blockLowRankAccum restated (in place on U1, V1); rnd is nx x k1 row-major."""
    ny, k1 = U1.shape
    nx, k2 = V2.shape
    lib().oracle_accum(U1.ctypes.data, V1.ctypes.data, U2.ctypes.data, V2.ctypes.data, nx, ny, k1, k2, U1.shape[1],
                       V1.shape[1], U2.shape[1], V2.shape[1], sign, rnd.ctypes.data, k1)
