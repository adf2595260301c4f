"""pastel_palettes_b200 — Python host mirror of the B200 H-LU engine.

Thin ctypes layer over libpastel_palettes.so (C ABI: include/pastel_palettes.h).  The
names follow the reference's host interface (Pastel-Palettes matrix/Dense.h,
matrix/Hierarchical.h, rts/ops.h, include/launcher.cuh):

  Hierarchical        block tree + device copy        (matrix/Hierarchical.h:4-7; usage
                                                        src/launcher.cu:126,138-139)
  dev_hierarchical_GETRF(h, num_blocks, num_threads, kernel_size)
                                                       (include/launcher.cuh:18)
  DataMap2D.checkOverlap                               (rts/ops.h:9-20, rts/ops.cpp:7-40)
  Operation.checkDependencyFrom                        (rts/ops.h:22-36, rts/ops.cpp:42-61)

plus what the reference lacks: solve, FP64 residuals, and the synthetic problem builders
of the benchmark configurations.  There is no CPU fallback: compute calls go to the CUDA
library or raise.
"""
from __future__ import annotations

import collections
import ctypes as C
import os
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpastel_palettes.so")

PP_OK, PP_INVALID_ARG, PP_OOM, PP_TIMEOUT, PP_NUMERICAL, PP_CUDA_ERROR, PP_UNSUPPORTED, PP_INTERNAL = range(8)
STATUS_NAMES = ["OK", "INVALID_ARG", "OOM", "TIMEOUT", "NUMERICAL", "CUDA_ERROR", "UNSUPPORTED", "INTERNAL"]
OP_NAMES = ["nop", "getrf", "trsml", "trsmr", "trsmrt", "trsmu", "gemm", "gemm3", "gemm4", "accum", "sum", "trinv",
            "trmv", "orth", "copy", "shadow", "kmul", "lrtrunc"]
DENSE, LOWRANK, HIER = 0, 1, 2
FP64, TF32, BF16 = 0, 1, 2  # contraction precision of the factor's GEMM instructions
ARENAS = ["matrix", "work", "scratch", "rhs", "rand"]

# pp_task (pastel-palettes_b200/csrc/pp_task.h), 160 bytes
TASK_DTYPE = np.dtype(
    [("op", "<i4"), ("flags", "<i4"), ("m", "<i4"), ("n", "<i4"), ("k", "<i4"), ("l", "<i4"), ("o", "<i4"),
     ("ctrl", "<i4"), ("ld", "<i4", 6), ("p", "<u8", 6), ("tmp", "<u8"), ("alpha", "<f8"), ("beta", "<f8"),
     ("succ_begin", "<i4"), ("n_succ", "<i4"), ("prec", "<i4"), ("instance", "<i4"), ("aux", "<i4"),
     ("pad", "<i4", 3)])
assert TASK_DTYPE.itemsize == 160


class PPError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else status}: {msg}")
        self.status = status


class _Config(C.Structure):
    _fields_ = [("tile", C.c_int), ("ctas_per_sm", C.c_int), ("spin_limit", C.c_longlong), ("seed", C.c_ulonglong),
                ("reference_isa", C.c_int)]


class _BlockInfo(C.Structure):
    _fields_ = [("kind", C.c_int), ("row0", C.c_int), ("col0", C.c_int), ("m", C.c_int), ("n", C.c_int),
                ("rank", C.c_int), ("kmax", C.c_int), ("level", C.c_int), ("children", C.c_int * 4)]


class _ServeConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_longlong), ("max_inflight", C.c_int), ("grid_per_request", C.c_int)]


class _RequestDesc(C.Structure):
    _fields_ = [("kernel", C.c_int), ("p0", C.c_double), ("shift", C.c_double), ("norm_inf", C.c_double),
                ("dim", C.c_int), ("points", C.c_void_p), ("rhs", C.c_void_p), ("nrhs", C.c_int),
                ("n_sets", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int), ("x_out", C.c_void_p)]


def residual_batch_launches(jobs, per_launch=64):
    """Kernel launches of one pp_kernel_residual_batch_dev call; jobs: (kernel, dim, nrhs,
    has_dx) tuples.  Update and reduction run in chunks of `per_launch` jobs, the residual once
    per chunk of a (kernel, dim, nrhs 1 | 2-4) group and once per job of more than 4 RHS."""
    if not jobs:
        return 0
    chunks = lambda c: (c + per_launch - 1) // per_launch
    groups = collections.Counter((k, d, 1 if r == 1 else 4) for k, d, r, _ in jobs if r <= 4)
    return (chunks(sum(1 for j in jobs if j[3])) + sum(chunks(c) for c in groups.values())
            + sum(1 for j in jobs if j[2] > 4) + chunks(len(jobs)))


class _ResidualJob(C.Structure):
    _fields_ = [("kernel", C.c_int), ("dim", C.c_int), ("n", C.c_int), ("nrhs", C.c_int), ("p0", C.c_double),
                ("shift", C.c_double), ("points", C.c_void_p), ("x", C.c_void_p), ("dx", C.c_void_p),
                ("b", C.c_void_p), ("r", C.c_void_p)]


class _RequestStats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("backward_error", C.c_double),
                ("t_submit_ms", C.c_double), ("t_admit_ms", C.c_double), ("t_done_ms", C.c_double),
                ("t_enqueued_ms", C.c_double),
                ("device_bytes", C.c_longlong), ("message", C.c_char * 128)]


class _TuneResult(C.Structure):
    _fields_ = [("tile", C.c_int), ("grid", C.c_int), ("trials", C.c_int), ("factor_ms", C.c_double),
                ("gemm_tile", C.c_int)]


class _ProgramInfo(C.Structure):
    _fields_ = [("n_tasks", C.c_int), ("n_edges", C.c_longlong), ("flops", C.c_longlong),
                ("op_count", C.c_longlong * 24), ("arena_elems", C.c_longlong * 5), ("host_build_ms", C.c_double)]


_lib = None


def lib():
    """The loaded C library; raises if it was not built (no silent fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C pastel-palettes_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        vp, i, ll, d, dp = C.c_void_p, C.c_int, C.c_longlong, C.c_double, C.POINTER(C.c_double)
        sig = {
            "pp_context_create": (i, [i, C.POINTER(_Config), C.POINTER(vp)]),
            "pp_context_destroy": (None, [vp]),
            "pp_last_error": (i, [vp, C.c_char_p, C.c_size_t]),
            "pp_device_sm_count": (i, [vp]),
            "pp_hmatrix_create_dense": (i, [vp, i, i, C.POINTER(vp)]),
            "pp_hmatrix_create_geometric": (i, [vp, i, i, dp, i, i, d, i, C.POINTER(vp)]),
            "pp_hmatrix_destroy": (None, [vp]),
            "pp_hmatrix_num_blocks": (i, [vp]),
            "pp_hmatrix_root": (i, [vp]),
            "pp_hmatrix_block_info": (i, [vp, i, C.POINTER(_BlockInfo)]),
            "pp_hmatrix_block_storage": (i, [vp, i, C.POINTER(ll), C.POINTER(ll), C.POINTER(ll)]),
            "pp_hmatrix_set_dense": (i, [vp, i, dp, i]),
            "pp_hmatrix_set_lowrank": (i, [vp, i, dp, i, dp, i, i]),
            "pp_hmatrix_upload": (i, [vp, vp]),
            "pp_hmatrix_download": (i, [vp, vp]),
            "pp_hmatrix_pin_host": (i, [vp]),
            "pp_hmatrix_keep_original": (i, [vp, vp]),
            "pp_hmatrix_restore": (i, [vp, vp]),
            "pp_hmatrix_to_dense": (i, [vp, dp]),
            "pp_hmatrix_storage_elems": (ll, [vp]),
            "pp_hmatrix_host_arena": (dp, [vp, C.POINTER(ll)]),
            "pp_hmatrix_device_arena": (vp, [vp]),
            "pp_hmatrix_block_elems": (ll, [vp]),
            "pp_hlu_factor": (i, [vp, vp]),
            "pp_hlu_solve": (i, [vp, vp, vp, i, vp]),
            "pp_hmatrix_sync": (i, [vp, vp]),
            "pp_hmatrix_program_info": (i, [vp, i, i, C.POINTER(_ProgramInfo)]),
            "pp_dev_hierarchical_getrf": (i, [vp, i, i, i]),
            "pp_dense_residual_dev": (i, [vp, vp, i, i, vp, vp, vp, i, vp]),
            "pp_kernel_residual_dev": (i, [vp, i, d, d, vp, i, i, vp, vp, vp, i, vp]),
            "pp_kernel_residual_batch_dev": (i, [vp, i, C.POINTER(_ResidualJob), vp]),
            "pp_kernel_residual_batch_lowp_dev": (i, [vp, i, C.POINTER(_ResidualJob), vp]),
            "pp_hmatrix_assemble_dense_dev": (i, [vp, i, d, d, vp, i, vp]),
            "pp_hmatrix_construct_dev": (i, [vp, i, d, d, vp, i, vp]),
            "pp_datamap2d_check_overlap": (i, [C.c_uint64, C.c_size_t, C.c_size_t, C.c_size_t,
                                               C.c_uint64, C.c_size_t, C.c_size_t, C.c_size_t]),
            "pp_operation_dependency": (i, [i, vp, vp, i, vp, vp]),
            "pp_hmatrix_encode_program": (i, [vp, i, i, vp, vp, vp, vp, vp]),
            "pp_hmatrix_rand_host": (i, [vp, dp, ll]),
            "pp_hmatrix_program_edges": (i, [vp, i, i, vp, vp, vp]),
            "pp_hmatrix_trace": (i, [vp, i, i, i, vp]),
            "pp_vm_execute": (i, [vp, vp, i, vp, ll, vp, ll, i, vp]),
            "pp_lowrank_accum_noalloc": (i, [vp, vp, i, vp, i, vp, i, vp, i, vp, i, i, i, i, i, d, vp]),
            "pp_gmres_create": (i, [vp, i, vp, i, vp, vp, vp, vp, C.POINTER(vp)]),
            "pp_context_set_device_dag": (i, [vp, i]),
            "pp_hmatrix_set_pivoting": (i, [vp, i]),
            "pp_hmatrix_program_regions": (i, [vp, i, i, C.POINTER(ll), vp]),
            "pp_hmatrix_dag_info": (i, [vp, i, i, C.POINTER(d), C.POINTER(i)]),
            "pp_gmres_destroy": (None, [vp]),
            "pp_gmres_start": (i, [vp, vp]),
            "pp_gmres_arnoldi": (i, [vp, i, vp]),
            "pp_gmres_finish": (i, [vp, vp]),
            "pp_gmres_status": (i, [vp, dp]),
            "pp_batch_create": (i, [vp, vp, i, C.POINTER(vp)]),
            "pp_batch_destroy": (None, [vp]),
            "pp_batch_factor": (i, [vp, vp]),
            "pp_batch_solve": (i, [vp, vp, vp, i, vp]),
            "pp_batch_restore": (i, [vp, vp]),
            "pp_batch_sync": (i, [vp, vp]),
            "pp_batch_program_info": (i, [vp, i, i, C.POINTER(_ProgramInfo)]),
            "pp_batch_trace": (i, [vp, i, i, i, vp]),
            "pp_batch_autotune": (i, [vp, vp, C.POINTER(_TuneResult)]),
            "pp_batch_set_tuning": (i, [vp, i, i, i]),
            "pp_refstream_encode": (i, [vp, i, vp, ll, vp, C.POINTER(ll)]),
            "pp_server_create": (i, [vp, C.POINTER(_ServeConfig), C.POINTER(vp)]),
            "pp_server_submit": (i, [vp, vp, C.POINTER(_RequestDesc), C.POINTER(ll)]),
            "pp_server_poll": (i, [vp, ll, C.POINTER(_RequestStats)]),
            "pp_server_wait_all": (i, [vp, d]),
            "pp_server_clock_ms": (d, [vp]),
            "pp_server_destroy": (None, [vp]),
            "pp_hmatrix_set_precision": (i, [vp, i]),
            "pp_hmatrix_set_gemm_tile": (i, [vp, i]),
            "pp_hmatrix_set_rank_tolerance": (i, [vp, d]),
            "pp_hmatrix_block_rank": (i, [vp, i]),
            "pp_hmatrix_get_precision": (i, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _stream_handle(stream):
    if stream is None:
        return None
    return C.c_void_p(getattr(stream, "cuda_stream", stream))


def exported_symbols():
    """Names declared in include/pastel_palettes.h (for the load test)."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "pastel_palettes.h")
    import re
    src = open(hdr).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return sorted(set(re.findall(r"\b(pp_[a-z0-9_]+)\s*\(", src)))


class Context:
    """Device context (device >= 0) or host-only planning context (device = -1)."""

    def __init__(self, device=0, tile=64, ctas_per_sm=0, spin_limit=0, seed=0x5EED5EED, reference_isa=0):
        cfg = _Config(tile, ctas_per_sm, spin_limit, seed, reference_isa)
        h = C.c_void_p()
        st = lib().pp_context_create(device, C.byref(cfg), C.byref(h))
        if st != PP_OK:
            raise PPError(st, f"pp_context_create(device={device}) failed")
        self._h = h
        self.device = device

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pp_context_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def last_error(self):
        buf = C.create_string_buffer(1024)
        lib().pp_last_error(self._h, buf, 1024)
        return buf.value.decode()

    def check(self, st, what):
        if st != PP_OK:
            raise PPError(st, f"{what}: {self.last_error()}")

    @property
    def sm_count(self):
        return lib().pp_device_sm_count(self._h)

    def set_device_dag(self, on=True):
        """Build the dependency DAG of programs made from now on on the device (same edges,
        types and orders as the host build; the host build runs when the device one cannot)."""
        self.check(lib().pp_context_set_device_dag(self._h, int(bool(on))), "set_device_dag")

    # --- FP64 residuals (device pointers of torch tensors)
    def dense_residual(self, A, x, b, r, stream=None):
        n, nrhs = x.shape
        self.check(lib().pp_dense_residual_dev(self._h, A.data_ptr(), A.stride(0), n, x.data_ptr(), b.data_ptr(),
                                               r.data_ptr(), nrhs, _stream_handle(stream)), "dense_residual")

    def vm_execute(self, tasks, succ, indeg, spin_limit=0, grid=0, stream=None):
        """Run a task table (TASK_DTYPE array with device pointers) on the VM and wait."""
        tasks = np.ascontiguousarray(tasks, dtype=TASK_DTYPE)
        succ = np.ascontiguousarray(succ, dtype=np.int32)
        indeg = np.ascontiguousarray(indeg, dtype=np.int32)
        self.check(lib().pp_vm_execute(self._h, tasks.ctypes.data, len(tasks), succ.ctypes.data if succ.size else None,
                                       succ.size, indeg.ctypes.data, spin_limit, grid, _stream_handle(stream)),
                   "vm_execute")

    def kernel_residual(self, kernel, p0, shift, pts, x, b, r, stream=None):
        n, nrhs = x.shape
        self.check(lib().pp_kernel_residual_dev(self._h, kernel, p0, shift, pts.data_ptr(), pts.shape[1], n,
                                                x.data_ptr(), b.data_ptr(), r.data_ptr(), nrhs,
                                                _stream_handle(stream)), "kernel_residual")

    def kernel_residual_batch(self, jobs, stream=None, lowp=False):
        """jobs: (kernel, p0, shift, pts, x, dx or None, b, r) per problem (device tensors);
        every job does x += dx (when given), then r = b - A x, in a few batched launches.
        lowp: entries of jobs with <= 4 right-hand sides evaluated in FP32 (Krylov products
        only; a residual that certifies a result must not use it)."""
        arr = (_ResidualJob * max(1, len(jobs)))()
        for q, (kernel, p0, shift, pts, x, dx, b, r) in enumerate(jobs):
            n, nrhs = x.shape
            arr[q] = _ResidualJob(int(kernel), int(pts.shape[1]), int(n), int(nrhs), float(p0), float(shift),
                                  pts.data_ptr(), x.data_ptr(), None if dx is None else dx.data_ptr(),
                                  b.data_ptr(), r.data_ptr())
        fn = lib().pp_kernel_residual_batch_lowp_dev if lowp else lib().pp_kernel_residual_batch_dev
        self.check(fn(self._h, len(jobs), arr, _stream_handle(stream)), "kernel_residual_batch")
        return residual_batch_launches([(j[0], j[3].shape[1], j[4].shape[1], j[5] is not None) for j in jobs])


class Hierarchical:
    """A block tree (dense / low-rank / 2x2 hierarchical blocks) and its device copy."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self._h = handle

    @classmethod
    def dense(cls, ctx, n, leaf):
        h = C.c_void_p()
        ctx.check(lib().pp_hmatrix_create_dense(ctx.handle, n, leaf, C.byref(h)), "create_dense")
        return cls(ctx, h)

    @classmethod
    def geometric(cls, ctx, points, leaf, admissibility=0, eta=1.0, kmax=16):
        pts = np.ascontiguousarray(points, dtype=np.float64)
        n, dim = pts.shape
        h = C.c_void_p()
        ctx.check(lib().pp_hmatrix_create_geometric(ctx.handle, n, dim, _ptr(pts), leaf, admissibility, eta, kmax,
                                                    C.byref(h)), "create_geometric")
        return cls(ctx, h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pp_hmatrix_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    # --- structure (getNy_abs / getNx_abs / getRootIndex)
    def blocks(self):
        out = []
        for b in range(lib().pp_hmatrix_num_blocks(self._h)):
            info = _BlockInfo()
            lib().pp_hmatrix_block_info(self._h, b, C.byref(info))
            out.append(dict(id=b, kind=info.kind, row0=info.row0, col0=info.col0, m=info.m, n=info.n,
                            rank=info.rank, kmax=info.kmax, level=info.level, children=list(info.children)))
        return out

    def block_storage(self, block):
        """Arena element offsets of a block: dense data / U, V and the rank word (-1: none)."""
        o, ov, orank = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self.ctx.check(lib().pp_hmatrix_block_storage(self._h, block, C.byref(o), C.byref(ov), C.byref(orank)),
                       "block_storage")
        return o.value, ov.value, orank.value

    @property
    def n(self):
        info = _BlockInfo()
        lib().pp_hmatrix_block_info(self._h, self.root, C.byref(info))
        return info.m

    def getNy_abs(self):
        return self.n

    def getNx_abs(self):
        return self.n

    @property
    def root(self):
        return lib().pp_hmatrix_root(self._h)

    def getRootIndex(self):
        return self.root

    def storage_elems(self):
        return lib().pp_hmatrix_storage_elems(self._h)

    # --- data
    def set_dense(self, block, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.ctx.check(lib().pp_hmatrix_set_dense(self._h, block, _ptr(a), a.shape[1]), "set_dense")

    def set_lowrank(self, block, U, V):
        U = np.ascontiguousarray(U, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        self.ctx.check(lib().pp_hmatrix_set_lowrank(self._h, block, _ptr(U), U.shape[1], _ptr(V), V.shape[1],
                                                    U.shape[1]), "set_lowrank")

    def host_arena(self):
        """Writable numpy view of the host image of the block arena."""
        n = C.c_longlong()
        p = lib().pp_hmatrix_host_arena(self._h, C.byref(n))
        return np.ctypeslib.as_array(p, shape=(max(n.value, 1),))[: n.value]

    def to_dense(self):
        out = np.zeros((self.n, self.n))
        self.ctx.check(lib().pp_hmatrix_to_dense(self._h, _ptr(out)), "to_dense")
        return out

    def upload(self, stream=None):
        self.ctx.check(lib().pp_hmatrix_upload(self._h, _stream_handle(stream)), "upload")

    def download(self, stream=None):
        self.ctx.check(lib().pp_hmatrix_download(self._h, _stream_handle(stream)), "download")

    def device_arena_ptr(self):
        return lib().pp_hmatrix_device_arena(self._h)

    def pin_host(self):
        self.ctx.check(lib().pp_hmatrix_pin_host(self._h), "pin_host")

    def keep_original(self, stream=None):
        self.ctx.check(lib().pp_hmatrix_keep_original(self._h, _stream_handle(stream)), "keep_original")

    def restore(self, stream=None):
        self.ctx.check(lib().pp_hmatrix_restore(self._h, _stream_handle(stream)), "restore")

    def arena_bytes(self):
        """Bytes of the matrix blocks: what upload, download and restore copy."""
        return 8 * int(lib().pp_hmatrix_block_elems(self._h))

    # --- factor / solve
    @property
    def precision(self):
        return lib().pp_hmatrix_get_precision(self._h)

    def set_precision(self, precision):
        """FP64 (default) or TF32: the factor's GEMM instructions on the tensor cores with
        FP32 accumulation; GETRF / TRSM / accumulation stay FP64."""
        self.ctx.check(lib().pp_hmatrix_set_precision(self._h, precision), "set_precision")

    def assemble_dense(self, prob, pts=None, stream=None):
        """Dense blocks evaluated on the device from the kernel problem's points (after upload);
        pts: the points as a device tensor (n x dim), made from prob when not given."""
        import torch
        if pts is None:
            pts = torch.from_numpy(np.ascontiguousarray(prob.points, dtype=np.float64)).cuda()
        if hasattr(stream, "wait_stream"):  # the points were written on the current stream
            stream.wait_stream(torch.cuda.current_stream())
        self.ctx.check(lib().pp_hmatrix_assemble_dense_dev(self._h, int(prob.kernel), float(prob.p0),
                                                           float(prob.shift), pts.data_ptr(), int(pts.shape[1]),
                                                           _stream_handle(stream)), "assemble_dense")
        return pts

    def construct(self, prob, pts=None, stream=None):
        """The whole H-matrix built on the device from the problem's points (no host image):
        dense blocks evaluated, low-rank blocks compressed by a randomized range finder on the
        VM and truncated at the rank tolerance.  pts: the points as a device tensor (n x dim),
        made from prob when not given; returned (keep it alive until the stream has run)."""
        import torch
        if pts is None:
            pts = torch.from_numpy(np.ascontiguousarray(prob.points, dtype=np.float64)).cuda()
        if hasattr(stream, "wait_stream"):  # the points were written on the current stream
            stream.wait_stream(torch.cuda.current_stream())
        self.ctx.check(lib().pp_hmatrix_construct_dev(self._h, int(prob.kernel), float(prob.p0), float(prob.shift),
                                                      pts.data_ptr(), int(pts.shape[1]), _stream_handle(stream)),
                       "construct")
        return pts

    def set_pivoting(self, on=True):
        """Partial pivoting inside every GETRF block (block-local row permutations applied by
        the triangular solves against that block); drops the built programs."""
        self.ctx.check(lib().pp_hmatrix_set_pivoting(self._h, int(bool(on))), "set_pivoting")

    def set_gemm_tile(self, edge):
        """Output tile edge (64 or 128) of the product instructions; results do not change."""
        self.ctx.check(lib().pp_hmatrix_set_gemm_tile(self._h, edge), "set_gemm_tile")

    def set_rank_tolerance(self, tol):
        """Adaptive rank (tol > 0): accumulations truncate to singular values > tol * largest."""
        self.ctx.check(lib().pp_hmatrix_set_rank_tolerance(self._h, float(tol)), "set_rank_tolerance")

    def ranks(self):
        """{block id: numerical rank} of the low-rank blocks (host image)."""
        return {b["id"]: lib().pp_hmatrix_block_rank(self._h, b["id"]) for b in self.blocks() if b["kind"] == LOWRANK}

    def factor(self, stream=None):
        self.ctx.check(lib().pp_hlu_factor(self._h, _stream_handle(stream)), "hlu_factor")

    def solve(self, b, x, stream=None):
        """x := A^-1 b with device tensors (n x nrhs row-major, float64)."""
        nrhs = b.shape[1] if b.dim() == 2 else 1
        self.ctx.check(lib().pp_hlu_solve(self._h, b.data_ptr(), x.data_ptr(), nrhs, _stream_handle(stream)),
                       "hlu_solve")

    def sync(self, stream=None):
        self.ctx.check(lib().pp_hmatrix_sync(self._h, _stream_handle(stream)), "sync")

    def program_info(self, which=0, nrhs=1):
        info = _ProgramInfo()
        self.ctx.check(lib().pp_hmatrix_program_info(self._h, which, nrhs, C.byref(info)), "program_info")
        return dict(n_tasks=info.n_tasks, n_edges=info.n_edges, flops=info.flops,
                    op_count={OP_NAMES[i]: info.op_count[i] for i in range(len(OP_NAMES))},
                    arena_elems={ARENAS[i]: info.arena_elems[i] for i in range(5)},
                    host_build_ms=info.host_build_ms)

    def regions(self, which=0, nrhs=1):
        """Every instruction's data regions: int32 rows (task, object, row0, col0, rows, cols,
        read_only) in program order."""
        k = C.c_longlong()
        self.ctx.check(lib().pp_hmatrix_program_regions(self._h, which, nrhs, C.byref(k), None), "program_regions")
        out = np.zeros((max(k.value, 1), 7), dtype=np.int32)
        self.ctx.check(lib().pp_hmatrix_program_regions(self._h, which, nrhs, C.byref(k), out.ctypes.data),
                       "program_regions")
        return out[: k.value]

    def dag_info(self, which=0, nrhs=1):
        """(DAG build milliseconds, built on the device) of the factor / solve program."""
        ms, dev = C.c_double(), C.c_int()
        self.ctx.check(lib().pp_hmatrix_dag_info(self._h, which, nrhs, C.byref(ms), C.byref(dev)), "dag_info")
        return ms.value, bool(dev.value)

    def encode_program(self, which, nrhs, bases):
        """Task table bound to the given arena base addresses (ints); returns
        (tasks structured array, succ, indeg, ready)."""
        info = self.program_info(which, nrhs)
        n, e = info["n_tasks"], info["n_edges"]
        tasks = np.zeros(n, dtype=TASK_DTYPE)
        succ = np.zeros(max(e, 1), dtype=np.int32)
        indeg = np.zeros(n, dtype=np.int32)
        order = np.zeros(n, dtype=np.int32)
        b = (C.c_void_p * 5)(*[C.c_void_p(int(x)) for x in bases])
        self.ctx.check(lib().pp_hmatrix_encode_program(self._h, which, nrhs, b, tasks.ctypes.data,
                                                       succ.ctypes.data, indeg.ctypes.data, order.ctypes.data),
                       "encode_program")
        ready = order[order >= 0]
        return tasks, succ[:e], indeg, ready

    def edges(self, which=0, nrhs=1):
        """Typed DAG edges (from, to, dependency_t bits) of the factor / solve program."""
        e = self.program_info(which, nrhs)["n_edges"]
        f = np.zeros(max(e, 1), dtype=np.int64)
        t = np.zeros(max(e, 1), dtype=np.int64)
        ty = np.zeros(max(e, 1), dtype=np.int32)
        self.ctx.check(lib().pp_hmatrix_program_edges(self._h, which, nrhs, f.ctypes.data, t.ctypes.data,
                                                      ty.ctypes.data), "program_edges")
        return f[:e], t[:e], ty[:e]

    def enable_trace(self, which=0, nrhs=1, enable=True):
        self.ctx.check(lib().pp_hmatrix_trace(self._h, which, nrhs, int(enable), None), "trace")

    def read_trace(self, which=0, nrhs=1):
        """(n_tasks, 3) uint64: start ns, end ns, sm | cta << 32 of the last traced launch."""
        n = self.program_info(which, nrhs)["n_tasks"]
        out = np.zeros((n, 3), dtype=np.uint64)
        self.ctx.check(lib().pp_hmatrix_trace(self._h, which, nrhs, 1, out.ctypes.data), "trace")
        return out

    def rand_host(self):
        n = self.program_info(0)["arena_elems"]["rand"]
        out = np.zeros(max(n, 1))
        self.ctx.check(lib().pp_hmatrix_rand_host(self._h, _ptr(out), n), "rand_host")
        return out[:n]

    def refstreams(self, workers=1):
        """Reference-format instruction streams of the factor program (one per worker)."""
        lengths = np.zeros(workers, dtype=np.int32)
        tmp = C.c_longlong()
        self.ctx.check(lib().pp_refstream_encode(self._h, workers, None, 0, lengths.ctypes.data, C.byref(tmp)),
                       "refstream size")
        words = np.zeros(int(lengths.sum()), dtype=np.int32)
        self.ctx.check(lib().pp_refstream_encode(self._h, workers, words.ctypes.data, words.size,
                                                 lengths.ctypes.data, C.byref(tmp)), "refstream")
        return words, lengths, tmp.value


class Batch:
    """Several uploaded H-matrices (any sizes) factored / solved by one persistent launch
    over their merged task tables.  Each instance's result equals its result alone."""

    def __init__(self, ctx, hs):
        arr = (C.c_void_p * len(hs))(*[h.handle for h in hs])
        h = C.c_void_p()
        ctx.check(lib().pp_batch_create(ctx.handle, arr, len(hs), C.byref(h)), "batch_create")
        self.ctx, self.hs, self._h = ctx, list(hs), h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pp_batch_destroy(self._h)
            self._h = None

    def factor(self, stream=None):
        self.ctx.check(lib().pp_batch_factor(self._h, _stream_handle(stream)), "batch_factor")

    def solve(self, Bs, Xs, stream=None):
        nrhs = Bs[0].shape[1]
        b = (C.c_void_p * len(Bs))(*[C.c_void_p(t.data_ptr()) for t in Bs])
        x = (C.c_void_p * len(Xs))(*[C.c_void_p(t.data_ptr()) for t in Xs])
        self.ctx.check(lib().pp_batch_solve(self._h, b, x, nrhs, _stream_handle(stream)), "batch_solve")

    def restore(self, stream=None):
        self.ctx.check(lib().pp_batch_restore(self._h, _stream_handle(stream)), "batch_restore")

    def sync(self, stream=None):
        self.ctx.check(lib().pp_batch_sync(self._h, _stream_handle(stream)), "batch_sync")

    def program_info(self, which=0, nrhs=1):
        info = _ProgramInfo()
        self.ctx.check(lib().pp_batch_program_info(self._h, which, nrhs, C.byref(info)), "batch_program_info")
        return dict(n_tasks=info.n_tasks, n_edges=info.n_edges, flops=info.flops,
                    op_count={OP_NAMES[i]: info.op_count[i] for i in range(len(OP_NAMES))},
                    host_build_ms=info.host_build_ms)

    def autotune(self, stream=None):
        """Picks the dense tile and persistent grid of this batch by timing its factor launch
        (instances need keep_original); returns the choice and its time."""
        r = _TuneResult()
        self.ctx.check(lib().pp_batch_autotune(self._h, _stream_handle(stream), C.byref(r)), "batch_autotune")
        return dict(tile=r.tile, gemm_tile=r.gemm_tile, grid=r.grid, trials=r.trials, factor_ms=r.factor_ms)

    def set_tuning(self, tile, gemm_tile, grid, **_):
        """Applies an autotune() result (of a batch of the same shapes) without timing."""
        self.ctx.check(lib().pp_batch_set_tuning(self._h, int(tile), int(gemm_tile), int(grid)), "batch_set_tuning")

    def enable_trace(self, which=0, nrhs=1):
        self.ctx.check(lib().pp_batch_trace(self._h, which, nrhs, 1, None), "batch_trace")

    def read_trace(self, which=0, nrhs=1):
        n = self.program_info(which, nrhs)["n_tasks"]
        out = np.zeros((n, 3), dtype=np.uint64)
        self.ctx.check(lib().pp_batch_trace(self._h, which, nrhs, 1, out.ctypes.data), "batch_trace")
        return out


class BatchRefiner:
    """FP64 iterative refinement for every instance of a Batch (kernel problems); one batched
    solve launch per iteration, residuals per instance, until all backward errors <= tol."""

    def __init__(self, batch, probs, stream=None):
        import torch
        self.batch, self.probs, self.stream = batch, probs, stream
        self.pts = [torch.from_numpy(np.ascontiguousarray(p.points)).cuda() for p in probs]
        self.launches = 0

    def _iterate(self, xs, rs, dxs, bs):
        self.batch.solve(rs, dxs, self.stream)
        self.launches += 2
        # x += dx and r = b - A x of every instance: update, residual (one launch per group of
        # instances with the same kernel, dimension and RHS width) and reduction launches
        self.launches += self.batch.ctx.kernel_residual_batch(
            [(p.kernel, p.p0, p.shift, pts, x, dx, b, r)
             for p, pts, x, dx, b, r in zip(self.probs, self.pts, xs, dxs, bs, rs)], self.stream)

    def errors(self, bs, xs, rs):
        """Normwise backward error of every instance (one device-to-host read)."""
        import torch
        bn = torch.stack([b.abs().max() for b in bs])
        nA = torch.tensor([p.norm_inf for p in self.probs], dtype=torch.float64, device=bs[0].device)
        err = torch.stack([r.abs().max() for r in rs]) / (nA * torch.stack([x.abs().max() for x in xs]) + bn)
        return err.cpu().tolist()

    def run(self, bs, iters):
        """Exactly `iters` refinement solves without host synchronization (capturable in a
        CUDA graph); returns (xs, rs) with rs the final residuals."""
        import torch
        xs = [torch.zeros_like(b) for b in bs]
        rs = [b.clone() for b in bs]
        dxs = [torch.empty_like(b) for b in bs]
        for _ in range(iters):
            self._iterate(xs, rs, dxs, bs)
        return xs, rs

    def solve(self, bs, tol=1e-10, max_iter=30):
        """Refine until every instance's backward error <= tol; bs: device n_i x nrhs."""
        import torch
        xs = [torch.zeros_like(b) for b in bs]
        rs = [b.clone() for b in bs]
        dxs = [torch.empty_like(b) for b in bs]
        hist = []
        for _ in range(max_iter):
            self._iterate(xs, rs, dxs, bs)
            e = max(self.errors(bs, xs, rs))
            hist.append(e)
            if e <= tol:
                break
        return xs, hist


class BatchGMRES:
    """Restarted GMRES (FP64) for every instance of a Batch of kernel problems, right
    preconditioned by the batch's H-LU solve: A (LU)^-1 y = b, x = (LU)^-1 y.  No reference
    counterpart.  Where plain refinement (BatchRefiner) stalls because the factors are too
    coarse (ranks capped below what the tolerance needs), this converges whenever the
    preconditioned spectrum is clustered.  A cycle of m steps is one batched solve, one batched
    matrix-free product and one Arnoldi launch per step, then x += Z y and the true residual
    r = b - A x from the points; no host synchronization inside a cycle (capturable).  The
    Krylov bases are torch tensors owned here: (2 m + 1) n doubles per instance.
    lowp: the products inside a cycle evaluate the kernel entries in FP32 (a few 1e-7 relative,
    far below what one cycle gains when rho(I - (LU)^-1 A) is large); the residual at every
    restart, which decides convergence and certifies the answer, stays FP64."""

    def __init__(self, batch, probs, m=32, stream=None, lowp=True):
        import torch
        self.batch, self.probs, self.stream, self.m = batch, probs, stream, int(m)
        self.lowp = bool(lowp)
        dev = torch.device("cuda", torch.cuda.current_device())
        f64 = torch.float64
        self.pts = [torch.from_numpy(np.ascontiguousarray(p.points)).to(dev) for p in probs]
        self.V = [torch.zeros(self.m + 1, p.n, dtype=f64, device=dev) for p in probs]
        self.Z = [torch.zeros(self.m, p.n, dtype=f64, device=dev) for p in probs]
        self.x = [torch.zeros(p.n, 1, dtype=f64, device=dev) for p in probs]
        self.r = [torch.zeros(p.n, 1, dtype=f64, device=dev) for p in probs]
        self.zero = torch.zeros(max(p.n for p in probs), 1, dtype=f64, device=dev)
        k = len(probs)
        vp = lambda ts: (C.c_void_p * k)(*[C.c_void_p(t.data_ptr()) for t in ts])
        ns = (C.c_int * k)(*[p.n for p in probs])
        h = C.c_void_p()
        batch.ctx.check(lib().pp_gmres_create(batch.ctx.handle, k, ns, self.m, vp(self.V), vp(self.Z), vp(self.x),
                                              vp(self.r), C.byref(h)), "gmres_create")
        self._h = h
        self.launches = 0

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pp_gmres_destroy(self._h)
            self._h = None

    def _residual(self, bs):
        self.launches += self.batch.ctx.kernel_residual_batch(
            [(p.kernel, p.p0, p.shift, pts, x, None, b, r)
             for p, pts, x, b, r in zip(self.probs, self.pts, self.x, bs, self.r)], self.stream)

    def cycle(self, bs):
        """One restart cycle from the current r = b - A x (left as the new residual)."""
        L, ctx, sh = lib(), self.batch.ctx, _stream_handle(self.stream)
        ctx.check(L.pp_gmres_start(self._h, sh), "gmres_start")
        for j in range(self.m):
            vj = [V[j].view(-1, 1) for V in self.V]
            zj = [Z[j].view(-1, 1) for Z in self.Z]
            self.batch.solve(vj, zj, self.stream)
            self.launches += 2
            self.launches += ctx.kernel_residual_batch(
                [(p.kernel, p.p0, p.shift, pts, z, None, self.zero[:p.n], V[j + 1].view(-1, 1))
                 for p, pts, z, V in zip(self.probs, self.pts, zj, self.V)], self.stream, lowp=self.lowp)
            ctx.check(L.pp_gmres_arnoldi(self._h, j, sh), "gmres_arnoldi")
        ctx.check(L.pp_gmres_finish(self._h, sh), "gmres_finish")
        self.launches += 2 + self.m
        self._residual(bs)

    def reset(self, bs):
        """x = 0, r = b (on the current stream)."""
        for x, r, b in zip(self.x, self.r, bs):
            x.zero_()
            r.copy_(b)

    def run(self, bs, cycles):
        """Exactly `cycles` restart cycles from x = 0 without host synchronization (capturable);
        returns (xs, rs)."""
        self.reset(bs)
        for _ in range(cycles):
            self.cycle(bs)
        return self.x, self.r

    def errors(self, bs, xs=None, rs=None):
        """Normwise backward error of every instance (one device-to-host read)."""
        import torch
        xs = self.x if xs is None else xs
        rs = self.r if rs is None else rs
        bn = torch.stack([b.abs().max() for b in bs])
        nA = torch.tensor([p.norm_inf for p in self.probs], dtype=torch.float64, device=bs[0].device)
        err = torch.stack([r.abs().max() for r in rs]) / (nA * torch.stack([x.abs().max() for x in xs]) + bn)
        return err.cpu().tolist()

    def status(self):
        """Per instance: (active dimension, residual estimate) of the last cycle."""
        out = np.zeros(2 * len(self.probs))
        self.batch.ctx.check(lib().pp_gmres_status(self._h, _ptr(out)), "gmres_status")
        return out.reshape(-1, 2)

    def solve(self, bs, tol=1e-10, max_cycles=20):
        """Cycles until every instance's backward error <= tol; returns (xs, history)."""
        self.reset(bs)
        hist = []
        for _ in range(max_cycles):
            self.cycle(bs)
            e = max(self.errors(bs))
            hist.append(e)
            if e <= tol:
                break
        return self.x, hist


SERVE_STATUS = ["queued", "running", "done", "failed"]


class Server:
    """Request loop with continuous admission (C++ worker thread in the library; no reference
    counterpart).  submit() hands over an H-matrix (built and filled, not uploaded) with its
    kernel problem and one or more right-hand-side sets; the server admits requests by HBM
    budget and free slots, runs each on its own stream (their work overlaps on the device),
    keeps the factors resident for the request's follow-up sets and refines every set in FP64
    to `tol`."""

    def __init__(self, ctx, hbm_budget_bytes, max_inflight=4, grid_per_request=0):
        cfg = _ServeConfig(int(hbm_budget_bytes), int(max_inflight), int(grid_per_request))
        h = C.c_void_p()
        ctx.check(lib().pp_server_create(ctx.handle, C.byref(cfg), C.byref(h)), "server_create")
        self.ctx, self._h = ctx, h
        self._bufs = {}

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.pp_server_destroy(self._h)
            self._h = None

    def clock_ms(self):
        return lib().pp_server_clock_ms(self._h)

    def submit(self, h, prob, rhs_sets, tol=1e-10, max_iter=30):
        """rhs_sets: (n_sets, n, nrhs) array; returns the request id.  h is owned by the
        server from here on."""
        rhs_sets = np.ascontiguousarray(rhs_sets, dtype=np.float64)
        if rhs_sets.ndim == 2:
            rhs_sets = rhs_sets[None]
        n_sets, n, nrhs = rhs_sets.shape
        pts = np.ascontiguousarray(prob.points, dtype=np.float64)
        x = np.zeros_like(rhs_sets)
        d = _RequestDesc(int(prob.kernel), float(prob.p0), float(prob.shift), float(prob.norm_inf), int(prob.dim),
                         pts.ctypes.data, rhs_sets.ctypes.data, int(nrhs), int(n_sets), float(tol), int(max_iter),
                         x.ctypes.data)
        rid = C.c_longlong()
        self.ctx.check(lib().pp_server_submit(self._h, h.handle, C.byref(d), C.byref(rid)), "server_submit")
        h._h = None  # ownership moved to the server
        self._bufs[rid.value] = (x, rhs_sets, pts)
        return rid.value

    def poll(self, rid):
        st = _RequestStats()
        self.ctx.check(lib().pp_server_poll(self._h, int(rid), C.byref(st)), "server_poll")
        return dict(status=SERVE_STATUS[st.status], iterations=st.iterations, backward_error=st.backward_error,
                    t_submit_ms=st.t_submit_ms, t_admit_ms=st.t_admit_ms, t_done_ms=st.t_done_ms,
                    t_enqueued_ms=st.t_enqueued_ms,
                    device_bytes=st.device_bytes, message=st.message.decode(errors="replace"))

    def result(self, rid):
        """(n_sets, n, nrhs) solutions (valid once the request is done)."""
        return self._bufs[rid][0]

    def wait_all(self, timeout_ms=600000.0):
        self.ctx.check(lib().pp_server_wait_all(self._h, float(timeout_ms)), "server_wait_all")


def dev_hierarchical_GETRF(h, num_blocks=0, num_threads=0, kernel_size=0):
    """Reference signature (include/launcher.cuh:18): factor h in place and wait."""
    h.ctx.check(lib().pp_dev_hierarchical_getrf(h.handle, num_blocks, num_threads, kernel_size),
                "dev_hierarchical_GETRF")


class DataMap2D:
    """Pitched 2-D byte region (rts/ops.h:9-20)."""

    def __init__(self, ptr, pitch, width, height):
        self.ptr, self.pitch, self.width, self.height = int(ptr), int(pitch), int(width), int(height)

    def checkOverlap(self, other):
        return bool(lib().pp_datamap2d_check_overlap(self.ptr, self.pitch, self.width, self.height, other.ptr,
                                                     other.pitch, other.width, other.height))


class Operation:
    """R/W region list of one operation (rts/ops.h:22-36); `data` holds (read_only, DataMap2D)."""

    def __init__(self, data=()):
        self.data = list(data)

    def _flat(self):
        r = np.array([[d.ptr, d.pitch, d.width, d.height] for _, d in self.data], dtype=np.uint64).reshape(-1, 4)
        ro = np.array([1 if f else 0 for f, _ in self.data], dtype=np.int32)
        return np.ascontiguousarray(r), ro

    def checkDependencyFrom(self, op_from):
        rf, rof = op_from._flat()
        rt, rot = self._flat()
        return lib().pp_operation_dependency(len(op_from.data), rf.ctypes.data, rof.ctypes.data, len(self.data),
                                             rt.ctypes.data, rot.ctypes.data)

    def checkDependencyTo(self, op_to):
        return op_to.checkDependencyFrom(self)


# --------------------------------------------------------------------------- problems
KERNELS = {"inv": 0, "laplace": 1, "exp": 2, "matern32": 3}


def kernel_eval(kind, d, p0):
    if kind == 0:
        return 1.0 / (d + p0)
    if kind == 1:
        return 1.0 / (4.0 * np.pi * (d + p0))
    if kind == 2:
        return np.exp(-d / p0)
    s = np.sqrt(3.0) * d / p0
    return (1.0 + s) * np.exp(-s)


def morton_order(pts):
    """Indices sorting points of [0,1]^d along a Z-order (Morton) curve."""
    n, dim = pts.shape
    bits = 21 if dim <= 3 else 10
    q = np.clip((pts * (1 << bits)).astype(np.uint64), 0, (1 << bits) - 1)
    key = np.zeros(n, dtype=np.uint64)
    for b in range(bits):
        for d in range(dim):
            key |= ((q[:, d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim + d)
    return np.argsort(key, kind="stable")


def truncated_svd(A, k, rng, with_s=False):
    """Rank-k truncated SVD of A as (U*s, V) (and s): exact for small blocks, randomized with
    oversampling 10 and two power iterations otherwise."""
    m, n = A.shape
    k = min(k, m, n)
    if min(m, n) <= 2 * k + 16:
        u, s, vt = np.linalg.svd(A, full_matrices=False)
        out = (u[:, :k] * s[:k], vt[:k].T.copy())
        return out + (s[:k],) if with_s else out
    p = min(k + 10, min(m, n))
    Y = A @ rng.standard_normal((n, p))
    Q, _ = np.linalg.qr(Y)
    for _ in range(2):
        Q, _ = np.linalg.qr(A.T @ Q)
        Q, _ = np.linalg.qr(A @ Q)
    B = Q.T @ A
    ub, s, vt = np.linalg.svd(B, full_matrices=False)
    U = (Q @ ub[:, :k]) * s[:k]
    return (U, vt[:k].T.copy(), s[:k]) if with_s else (U, vt[:k].T.copy())


class KernelProblem:
    """Points, kernel and diagonal shift of a kernel-matrix configuration."""

    def __init__(self, n, dim, kernel, p0, shift, points, offdiag_max=None):
        self.n, self.dim, self.kernel, self.p0, self.shift, self.points = n, dim, kernel, p0, shift, points
        if offdiag_max is None:
            offdiag_max = offdiag_rowsum_max(points, kernel, p0)
        # all kernels here are positive: max row sum of |A| = K(0) + shift + off-diagonal row sum
        self.norm_inf = float(kernel_eval(kernel, 0.0, p0)) + shift + offdiag_max

    def entries(self, rows, cols):
        X, Y = self.points[rows], self.points[cols]
        A = kernel_eval(self.kernel, pairwise_distances(X, Y), self.p0)
        ri = np.asarray(rows)[:, None] if not isinstance(rows, slice) else np.arange(rows.start, rows.stop)[:, None]
        ci = np.asarray(cols)[None, :] if not isinstance(cols, slice) else np.arange(cols.start, cols.stop)[None, :]
        return A + self.shift * (ri == ci)

    def dense(self):
        return self.entries(slice(0, self.n), slice(0, self.n))


def pairwise_distances(X, Y):
    """|x_i - y_j| for all pairs (scipy's compiled cdist when present: the same bits as the
    numpy form below, 10-17x faster)."""
    try:
        from scipy.spatial.distance import cdist
    except ImportError:
        return np.sqrt(np.maximum(((X[:, None, :] - Y[None, :, :]) ** 2).sum(-1), 0.0))
    return cdist(X, Y)


def offdiag_rowsum_max(points, kernel, p0, block=2048):
    n = points.shape[0]
    best = 0.0
    for i0 in range(0, n, block):
        X = points[i0:i0 + block]
        s = np.zeros(X.shape[0])
        for j0 in range(0, n, block):
            Y = points[j0:j0 + block]
            K = np.abs(kernel_eval(kernel, pairwise_distances(X, Y), p0))
            if i0 == j0:
                np.fill_diagonal(K, 0.0)
            s += K.sum(1)
        best = max(best, float(s.max()))
    return best


def fill_kernel_hmatrix(h, prob, seed=7, rank_tol=None):
    """Dense blocks evaluated exactly; low-rank blocks by truncated SVD at their kmax, or (with
    rank_tol) at the number of singular values above rank_tol times the largest, at most kmax."""
    rng = np.random.default_rng(seed)
    for b in h.blocks():
        if b["kind"] == DENSE:
            h.set_dense(b["id"], prob.entries(slice(b["row0"], b["row0"] + b["m"]),
                                              slice(b["col0"], b["col0"] + b["n"])))
        elif b["kind"] == LOWRANK:
            A = prob.entries(slice(b["row0"], b["row0"] + b["m"]), slice(b["col0"], b["col0"] + b["n"]))
            U, V, s = truncated_svd(A, b["kmax"], rng, with_s=True)
            if rank_tol:
                r = int(np.count_nonzero(s > rank_tol * s[0])) if s.size and s[0] > 0 else 0
                U, V = U[:, :r], V[:, :r]
            h.set_lowrank(b["id"], U, V)


def make_dense_problem(ctx, n=1024, leaf=256, seed=1234, shift=None):
    """Configuration 1: A = U[-1,1]^{n x n} + shift I (shift n by default: strictly diagonally
    dominant), all-dense 2x2 tree down to `leaf`."""
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1.0, 1.0, (n, n)) + (n if shift is None else shift) * np.eye(n)
    h = Hierarchical.dense(ctx, n, leaf)
    for b in h.blocks():
        if b["kind"] == DENSE:
            h.set_dense(b["id"], A[b["row0"]:b["row0"] + b["m"], b["col0"]:b["col0"] + b["n"]])
    return h, A


def offdiag_rowsum_max_dev(ctx, pts_dev, kernel, p0, stream=None):
    """max_i sum_{j != i} |K(p_i, p_j)| on the device (the kernels here are positive): the
    matrix-free residual of the unshifted matrix applied to ones, minus the diagonal K(0)."""
    import torch
    n = pts_dev.shape[0]
    x = torch.ones((n, 1), dtype=torch.float64, device=pts_dev.device)
    b = torch.zeros_like(x)
    r = torch.empty_like(x)
    ctx.kernel_residual(kernel, p0, 0.0, pts_dev, x, b, r, stream)
    if stream is not None:
        stream.synchronize()
    else:
        torch.cuda.synchronize()
    return float((-r).max().item()) - float(kernel_eval(kernel, 0.0, p0))


def make_kernel_problem(ctx, n, dim, kernel, p0, leaf, rank, admissibility=0, eta=1.0, shift=None,
                        shift_factor=2.0, seed=1234, rank_tol=None, construct="host", stream=None):
    """Kernel-matrix configuration: points U[0,1]^dim (Morton order), A_ij = K(|x_i - x_j|),
    diagonal shifted by `shift` or by shift_factor * max off-diagonal row sum.
    construct="host": blocks filled on the host (exact dense blocks, truncated SVD of the
    low-rank ones) for a later upload; "device": the row sums and every block computed on the
    device (Hierarchical.construct), no host image; prob.points_dev holds the device points;
    "none": the row sums on the device, the blocks left unbuilt (a served request: the server
    builds them on the device at admission)."""
    rng = np.random.default_rng(seed)
    pts = rng.uniform(0.0, 1.0, (n, dim))
    pts = pts[morton_order(pts)]
    kid = KERNELS[kernel] if isinstance(kernel, str) else kernel
    pts_dev = None
    if construct in ("device", "none"):
        import torch
        pts_dev = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
        off = offdiag_rowsum_max_dev(ctx, pts_dev, kid, p0, stream)
    else:
        off = offdiag_rowsum_max(pts, kid, p0)
    if shift is None:
        shift = shift_factor * off
    prob = KernelProblem(n, dim, kid, p0, shift, pts, off)
    prob.points_dev = pts_dev
    h = Hierarchical.geometric(ctx, pts, leaf, admissibility, eta, rank)
    if rank_tol:
        h.set_rank_tolerance(rank_tol)
    if construct == "device":
        h.construct(prob, pts_dev, stream)
    elif construct == "host":
        fill_kernel_hmatrix(h, prob, seed + 1, rank_tol=rank_tol)
    return h, prob


def rhs(n, nrhs=1, seed=99):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, (n, nrhs))


class Refiner:
    """FP64 iterative refinement around the H-LU solve (no reference counterpart):
    x_0 = (LU)^-1 b;  r = b - A x (FP64, A evaluated exactly: kernel entries on the fly or
    the dense FP64 matrix);  x += (LU)^-1 r; until the normwise backward error
    ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol."""

    def __init__(self, h, ctx, prob=None, dense=None, norm_inf=None, stream=None):
        import torch
        self.h, self.ctx, self.prob, self.stream = h, ctx, prob, stream
        if prob is not None:
            self.pts = torch.from_numpy(np.ascontiguousarray(prob.points)).cuda()
            self.norm_inf = prob.norm_inf
        else:
            self.A = torch.from_numpy(np.ascontiguousarray(dense)).cuda()
            self.norm_inf = float(np.abs(dense).sum(1).max()) if norm_inf is None else norm_inf
        self.launches = 0

    def residual(self, x, b, r):
        if self.prob is not None:
            self.ctx.kernel_residual(self.prob.kernel, self.prob.p0, self.prob.shift, self.pts, x, b, r, self.stream)
        else:
            self.ctx.dense_residual(self.A, x, b, r, self.stream)
        self.launches += 1

    def solve(self, b, tol=1e-10, max_iter=30, x=None):
        import torch
        x = torch.zeros_like(b) if x is None else x
        r = b.clone()
        dx = torch.empty_like(b)
        bn = b.abs().max().item()
        hist = []
        for it in range(max_iter):
            self.h.solve(r, dx, self.stream)
            self.launches += 2
            if self.prob is not None:  # update and residual in one batched call
                self.launches += self.ctx.kernel_residual_batch(
                    [(self.prob.kernel, self.prob.p0, self.prob.shift, self.pts, x, dx, b, r)], self.stream)
            else:
                x += dx
                self.residual(x, b, r)
            err = r.abs().max().item() / (self.norm_inf * x.abs().max().item() + bn)
            hist.append(err)
            if err <= tol:
                break
        return x, hist


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
