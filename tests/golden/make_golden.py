"""Generates tests/golden/*.npz: outputs of the REFERENCE's own kernel_dynamic (Pastel-Palettes
src/kernel.cu, compiled for sm_100a by oracle/Makefile into oracle/_ref/libref_vm.so) on small
seeded inputs, one reference-format instruction per run (one worker, so no waits).

Run on a machine with a CUDA device after `make -C oracle`:
    python tests/golden/make_golden.py
The CPU tests compare the oracle against these files (tests/test_oracle.py).
"""
import ctypes as C
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

EXECUTE, FINISH = 1, 0
GETRF, GEMM, GEMM_PLUS, ACCUM = 1, 4, 5, 8


def run(stream_words, arrays, rnd=None, tmp_elems=1):
    ref = oracle.ref_vm()
    assert ref is not None, "build the reference kernel first: make -C oracle"
    devs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]
    rnd_d = torch.from_numpy(np.ascontiguousarray(rnd)).cuda() if rnd is not None else torch.zeros(1, dtype=torch.float64, device="cuda")
    words = np.array(stream_words + [FINISH], dtype=np.int32)
    lengths = np.array([len(words)], dtype=np.int32)
    ptrs = (C.c_void_p * len(devs))(*[C.c_void_p(d.data_ptr()) for d in devs])
    rc = ref.ref_vm_run(1, words.ctypes.data, lengths.ctypes.data, C.cast(ptrs, C.c_void_p), len(devs), 1,
                        rnd_d.data_ptr(), tmp_elems, 256)
    assert rc == 0, rc
    return [d.cpu().numpy() for d in devs]


def main():
    rng = np.random.default_rng(20191117)
    # dense LU of a 128 x 128 diagonally dominant block (blockDenseGetrf, two 64-panels)
    n = 128
    A = rng.uniform(-1, 1, (n, n)) + n * np.eye(n)
    (LU,) = run([EXECUTE, 0, GETRF, 0, 0, n, n, n], [A])
    np.savez(os.path.join(HERE, "ref_dense_lu.npz"), A=A, LU=LU)

    # gemm: M -= A B ; gemm_plus with transposed B: M += A Bt^T
    m, nn, k = 96, 80, 64
    M0, Am, B = rng.standard_normal((m, nn)), rng.standard_normal((m, k)), rng.standard_normal((k, nn))
    Bt = rng.standard_normal((nn, k))
    M1, _, _ = run([EXECUTE, 0, GEMM, 0, 1, 2, 0, 0, 0, m, nn, k, nn, k, nn, 0, 0], [M0, Am, B])
    M2, _, _ = run([EXECUTE, 0, GEMM_PLUS, 0, 1, 2, 0, 0, 0, m, nn, k, nn, k, k, 0, 1], [M0, Am, Bt])
    np.savez(os.path.join(HERE, "ref_routines.npz"), M0=M0, A=Am, B=B, Bt=Bt, M_gemm=M1, M_gemm_plus_bT=M2)

    # accum: U1 V1^T += U2 V2^T recompressed to rank k1 with the random sketch R
    ny, nx, k1, k2 = 200, 176, 16, 16
    U1, V1 = rng.standard_normal((ny, k1)), rng.standard_normal((nx, k1))
    U2, V2 = 0.1 * rng.standard_normal((ny, k2)), rng.standard_normal((nx, k2))
    R = rng.uniform(-1, 1, (nx, k1))
    off1 = ny * k1
    off2 = off1 + nx * k1
    tmp = off2 + max(ny * k1, k1 * k2)
    U1o, V1o, _, _ = run([EXECUTE, 0, ACCUM, 0, 1, 2, 3, 0, 0, 0, 0, nx, ny, k1, k2, k1, k1, k2, k2, off1, off2],
                         [U1, V1, U2, V2], rnd=R, tmp_elems=tmp)
    np.savez(os.path.join(HERE, "ref_accum.npz"), U1=U1, V1=V1, U2=U2, V2=V2, R=R, U1_out=U1o, V1_out=V1o)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
