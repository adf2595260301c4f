"""pp_lowrank_accum_noalloc: the low-rank accumulation for callers that cannot allocate
device memory (stream capture in progress, a fully reserved memory budget, a framework that
owns the device pool).  It must give what the ACCUM instruction gives through pp_vm_execute,
and what the reference's blockLowRankAccum (restated by the oracle) gives, call after call,
although every call reuses the same static scratch array.

The accumulation keeps its ny x k1 sketch in shared memory while it fits; the cases below are
sized so that the sketch does not fit and goes through the static array, and they run back to
back so that each call finds the previous call's data in it.

Kept in its own file so pytest collects it last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-12  # relative Frobenius tolerance the accumulation tests use
# shared memory holds the sketch (dev_accum) while ny * (k1 + 1) (rows padded by one double) is
# at most 21328 doubles when k1, k2 <= 16, 17856 otherwise
YCAP = {16: 21328, 32: 17856}


def _inputs(rng, ny, nx, k1, k2):
    h = dict(U1=rng.standard_normal((ny, k1)), V1=rng.standard_normal((nx, k1)), U2=rng.standard_normal((ny, k2)),
             V2=rng.standard_normal((nx, k2)), R=rng.uniform(-1, 1, (nx, k1)))
    return h, {k: torch.from_numpy(v).cuda() for k, v in h.items()}


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


def _via_oracle(oracle, h, sign):
    U1, V1 = h["U1"].copy(), h["V1"].copy()
    oracle.accum(U1, V1, h["U2"], h["V2"], np.ascontiguousarray(h["R"]), sign)
    return U1 @ V1.T


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_accum_matches_vm_accum_and_oracle_on_consecutive_calls(pp, oracle, gctx):
    rng = np.random.default_rng(4242)
    cases = [(4000, 600, 16, 16, 1.0), (2000, 500, 32, 32, -1.0), (3000, 900, 24, 8, 1.0), (700, 520, 16, 16, -1.0)]
    # the first three keep their sketch in the static array (the last one in shared memory)
    for ny, nx, k1, k2, _ in cases[:3]:
        assert ny * (k1 + 1) > YCAP[16 if max(k1, k2) <= 16 else 32]
    for ny, nx, k1, k2, sign in cases:  # calls in a row on the shared scratch
        h, d = _inputs(rng, ny, nx, k1, k2)
        U_ref, V_ref = _via_vm_execute(pp, gctx, d, ny, nx, k1, k2, sign)
        U_new, V_new = _via_noalloc(pp, gctx, d, ny, nx, k1, k2, sign)
        P_new = (U_new @ V_new.T).cpu().numpy()
        assert _rel(P_new, (U_ref @ V_ref.T).cpu().numpy()) < TOL
        assert _rel(U_new.cpu().numpy(), U_ref.cpu().numpy()) < TOL
        assert _rel(V_new.cpu().numpy(), V_ref.cpu().numpy()) < TOL
        # the reference's accumulation (Givens QR where the engine uses Cholesky QR): the same
        # projection of U1 V1^T + sign U2 V2^T onto the range of its sketch
        assert _rel(P_new, _via_oracle(oracle, h, sign)) < TOL


def test_noalloc_accum_rejects_oversized_requests(pp, gctx):
    cap = 1 << 20
    ny, nx, k1, k2 = 40000, 1000, 32, 16  # a 40000 x 32 sketch: more than the array holds
    assert ny * k1 > cap
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    st = pp.lib().pp_lowrank_accum_noalloc(gctx.handle, p, k1, p, k1, p, k2, p, k2, p, k1, ny, nx, k1, k2, 1.0, None)
    assert st == pp.PP_INVALID_ARG
    assert "scratch" in gctx.last_error()


def test_noalloc_accum_rejects_ranks_above_32(pp, gctx):
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    for k1, k2 in [(16, 33), (33, 16)]:
        st = pp.lib().pp_lowrank_accum_noalloc(gctx.handle, p, k1, p, k1, p, k2, p, k2, p, k1, 500, 500, k1, k2, 1.0,
                                               None)
        assert st == pp.PP_INVALID_ARG
