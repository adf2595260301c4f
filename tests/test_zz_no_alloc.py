"""pp_lowrank_accum_noalloc: the low-rank accumulation for callers that cannot allocate
device memory (stream capture in progress, a fully reserved memory budget, a framework that
owns the device pool).  It must give what the ACCUM instruction gives through pp_vm_execute,
call after call, although every call reuses the same static scratch array.

Kept in its own file so pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-12  # relative Frobenius tolerance the accumulation tests use


def _inputs(rng, ny, nx, k1, k2):
    mk = lambda r, c: torch.from_numpy(rng.standard_normal((r, c))).cuda()
    return dict(U1=mk(ny, k1), V1=mk(nx, k1), U2=mk(ny, k2), V2=mk(nx, k2),
                R=torch.from_numpy(rng.uniform(-1, 1, (nx, k1))).cuda())


def _via_vm_execute(pp, gctx, d, ny, nx, k1, k2, sign):
    U1, V1 = d["U1"].clone(), d["V1"].clone()
    scratch = torch.zeros(2 * ny * k1 + nx * k1 + k1 * max(k1, k2), dtype=torch.float64, device="cuda")
    t = np.zeros(1, dtype=pp.TASK_DTYPE)
    t[0]["op"] = 9
    t[0]["m"], t[0]["n"], t[0]["k"], t[0]["l"] = ny, nx, k1, k2
    t[0]["alpha"], t[0]["beta"] = sign, 1.0
    for s, (x, ld) in enumerate([(U1, k1), (V1, k1), (d["U2"], k2), (d["V2"], k2), (d["R"], k1)]):
        t[0]["p"][s] = x.data_ptr()
        t[0]["ld"][s] = ld
    t[0]["tmp"] = scratch.data_ptr()
    gctx.vm_execute(t, np.zeros(0, np.int32), np.zeros(1, np.int32))
    return U1, V1


def _via_noalloc(pp, gctx, d, ny, nx, k1, k2, sign):
    U1, V1 = d["U1"].clone(), d["V1"].clone()
    torch.cuda.synchronize()
    st = pp.lib().pp_lowrank_accum_noalloc(gctx.handle, U1.data_ptr(), k1, V1.data_ptr(), k1, d["U2"].data_ptr(), k2,
                                           d["V2"].data_ptr(), k2, d["R"].data_ptr(), k1, ny, nx, k1, k2, sign, None)
    assert st == pp.PP_OK, gctx.last_error()
    torch.cuda.synchronize()
    return U1, V1


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


def test_noalloc_accum_matches_vm_accum_on_consecutive_calls(pp, gctx):
    rng = np.random.default_rng(4242)
    cases = [(700, 520, 16, 16, 1.0), (300, 900, 24, 8, -1.0)]
    for ny, nx, k1, k2, sign in cases:  # two calls in a row on the shared scratch
        d = _inputs(rng, ny, nx, k1, k2)
        U_ref, V_ref = _via_vm_execute(pp, gctx, d, ny, nx, k1, k2, sign)
        U_new, V_new = _via_noalloc(pp, gctx, d, ny, nx, k1, k2, sign)
        assert _rel(U_new @ V_new.T, U_ref @ V_ref.T) < TOL
        assert _rel(U_new, U_ref) < TOL and _rel(V_new, V_ref) < TOL


def test_noalloc_accum_rejects_oversized_requests(pp, gctx):
    cap = 1 << 20
    ny, nx, k1, k2 = 40000, 40000, 16, 16  # needs 2*ny*k1 + nx*k1 + k1*k1 > cap doubles
    assert 2 * ny * k1 + nx * k1 + k1 * k1 > cap
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    st = pp.lib().pp_lowrank_accum_noalloc(gctx.handle, p, k1, p, k1, p, k2, p, k2, p, k1, ny, nx, k1, k2, 1.0, None)
    assert st == pp.PP_INVALID_ARG
    assert "scratch" in gctx.last_error()
