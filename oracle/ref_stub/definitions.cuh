/* Stand-in for the reference's missing `definitions.cuh` (Pastel-Palettes
 * src/launcher.cu:3 and src/kernel.cu:3 include it; the file is absent from the
 * snapshot).  Written for this project: every value below is inferred from how
 * src/kernel.cu and src/kernel_cublas.cu use the names, and is only used to
 * compile the reference's own kernel into the test oracle (oracle/_ref).
 *
 * The opcode / operation enum VALUES are this project's choice; the encoder that
 * writes reference-format instruction streams (pp_refstream_*) uses the same
 * values, declared once more in include/pastel_palettes.h.
 */
#pragma once
#include <cuda_runtime.h>

#define DEVICE __device__

typedef double real_t;
typedef double2 vec_t;
#define vec_size 2

/* tile sizes of the reference's block routines; any even values give identical
 * results (every update is a k-ascending fma), these only set the smem footprint:
 * _BLOCK_M^2 + 2*_BLOCK_M*_BLOCK_K doubles must fit in _SHM_SIZE ints. */
#define _BLOCK_M 64
#define _BLOCK_K 16
#define _SHM_SIZE 12288
#define _MAX_INST_LENGTH 32

enum opcode_t { finish = 0, execute = 1, signal_wait = 2 };

enum operation_t { nop = 0, getrf = 1, trsml = 2, trsmr = 3, gemm = 4, gemm_plus = 5,
                   gemm_3x = 6, gemm_4x = 7, accum = 8 };

/* instruction lengths in int32 words (opcode, signal, operation, args...) */
#define nop_l 3
#define getrf_l 8
#define trsml_l 13
#define trsmr_l 13
#define gemm_l 17
#define gemm_plus_l 17
#define gemm_3x_l 23
#define gemm_4x_l 29
#define accum_l 21
