/* pp_task.h — one device instruction of the H-LU virtual machine.
 *
 * The reference encodes its block operations as variable-length int32 words
 * (opcode, signal id, operation, pointer-table indices, int offsets, dims, lds,
 * transpose flags; Pastel-Palettes src/kernel.cu:1404-1501).  This engine keeps
 * the same operation set (getrf / trsm L / trsm R / gemm / gemm_3x / gemm_4x /
 * accum) but stores each instruction as a fixed 160-byte record with absolute
 * 64-bit device pointers, so one task table can mix operands of many H-matrices
 * (batched launches) and no offset overflows past 2^31 elements.
 *
 * The record is read by the VM kernel (vm.cu), written by the host encoder
 * (hops.cpp), and executed on the CPU by the test oracle; it is plain C.
 */
#ifndef PP_TASK_H
#define PP_TASK_H
#include <stdint.h>

enum pp_op {
  PP_OP_NOP = 0,
  PP_OP_GETRF = 1,   /* A[m x n] := L\U in place, no pivoting (kernel.cu:104-147, 820-882)      */
  PP_OP_TRSML = 2,   /* B[m x n] := L^-1 B, L unit lower m x m      (kernel.cu:150-182, 667-715)  */
  PP_OP_TRSMR = 3,   /* B[m x n] := B U^-1, U upper n x n           (kernel.cu:185-226, 718-766)  */
  PP_OP_TRSMRT = 4,  /* V[m x n] := U^-T V, U upper m x m  (trsmr on V^T, kernel.cu:229-285, 769-817) */
  PP_OP_TRSMU = 5,   /* B[m x n] := U^-1 B, U upper m x m (solve only; no reference counterpart;
                        rows are scaled by the reciprocal of the diagonal)                     */
  PP_OP_GEMM = 6,    /* C[m x n] := beta C + alpha op(A)[m x k] op(B)[k x n] (kernel.cu:415-664)    */
  PP_OP_GEMM3 = 7,   /* C += alpha A B D, association by ctrl          (kernel.cu:886-904)         */
  PP_OP_GEMM4 = 8,   /* C += alpha A B D E, association by ctrl 0..4   (kernel.cu:907-955)         */
  PP_OP_ACCUM = 9,   /* U1 V1^T := rank-k1 range of U1 V1^T + alpha U2 V2^T (kernel.cu:1255-1280)   */
  PP_OP_SUM = 10,    /* C[m x n] := beta C + sum_{p<k} T_p, T_p = p-th m x n block (ld n) of p[1]:
                        reduction of split-k partial products (no reference counterpart)       */
  PP_OP_TRINV = 11,  /* columns [o, o + n) of the inverse of a factored diagonal leaf A = L\U
                        (m x m, p[1]) into the m x n column block at p[0] (ld ld[0]):
                        ctrl 0: L^-1 (unit lower), ctrl 1: U^-1 (upper).  Factor phase; no
                        reference counterpart (it serves the solve)                             */
  PP_OP_TRMV = 12,   /* B[m x n] := M B, M (p[1], m x m) lower (ctrl 0) or upper (ctrl 1)
                        triangular with explicit diagonal: a solve step with a precomputed
                        inverse; no reference counterpart.  With l > 0, rows [o, o + l) of
                        M B (B read from p[2], ld[2]) go to the l x n block at p[0]: one part
                        of a product split over several CTAs, each row summed as in the
                        whole product                                                          */
  PP_OP_ORTH = 13,   /* Y[m x k] (ld k, k <= 32) := an orthonormal basis of its range (shifted
                        CholeskyQR3; rank-deficient columns become zero): the range finder of
                        a sketched low-rank update; no reference counterpart                   */
  PP_OP_COPY = 14,   /* C[m x n] := A[m x n] (p[1]); no reference counterpart                   */
  PP_OP_SHADOW = 15, /* BF16 shadow of an FP64 operand for the tensor-core GEMM: the m x k matrix
                        X(r, c) = p[1][r * ld[1] + c] (or p[1][c * ld[1] + r] with PP_T(1)),
                        rounded to BF16 and written at p[0] in the tiled layout below (m a
                        multiple of 128, k of 64); rows from l and columns from n on (when set)
                        are written as zeros (padding).  o != 0: a split shadow (PP_SPLIT_*):
                        the k columns are o >> 8 segments of k / (o >> 8), each a copy of X's
                        columns holding bf16(x), or the residual bf16(x - bf16(x)) where bit s
                        of o & 0xFF is set; no reference counterpart                            */
  PP_OP_KMUL = 16,   /* C[m x k] (p[0]) := K(P_I, P_J) B: a kernel matrix evaluated from points
                        times B (p[3], n x k, k <= 32); P_I = p[1] (m points), P_J = p[2] (n
                        points), rows of dim = l coordinates (ld[1], ld[2]); kernel ctrl (0
                        1/(r + p0), 1 Laplace, 2 exp(-r/p0), 3 Matern-3/2), p0 = alpha; no
                        diagonal shift (the blocks it serves are admissible: disjoint rows and
                        columns).  Randomized compression on the device; no reference
                        counterpart (the reference's matrices come from a Java compressor)   */
  PP_OP_LRTRUNC = 17,/* U V^T (U = p[0] m x k with orthonormal columns, V = p[1] n x k) := its
                        best rank-r form, r the singular values above beta times the largest
                        (at most o), columns beyond r zero; r written to p[5] when set          */
  PP_OP_COUNT = 18
};

/* flags: bit (4+i) = operand i is stored transposed (operand 0 is the target). */
#define PP_T(i) (1 << (4 + (i)))
/* flags bit 0: the contraction may sum its k products in any fixed order (set on
 * products into work buffers, whose results are only compared within a tolerance);
 * without it every element accumulates in ascending k, as the reference does. */
#define PP_FREE_ORDER 1
/* flags bit 1 (ACCUM): adaptive rank — truncate to the singular values above beta times the
 * largest and store the new rank (as a double) at p[5] when p[5] is set */
#define PP_ADAPT_RANK 2
/* flags bit 2 (GETRF, TRSML): partial pivoting inside the block.  GETRF picks, at step i, the
 * row r >= i of largest |a_ri| (the first of equal ones), swaps whole rows i and r of the block,
 * then eliminates as without pivoting; it writes the block's row permutation to p[1] (m doubles
 * holding row indices: row i of the factored block came from row p[1][i]).  TRSML reads the
 * permutation of its L block from p[2] and solves L X = P B, row i of P B being row p[2][i] of
 * B.  The permutations stay block-local and are applied lazily: a solve against the block's L
 * permutes its right-hand side first, the blocks below the pivoted block are left as they are.
 * No reference counterpart in use (the reference's pivot helpers, src/kernel.cu:958-1051, are
 * never called). */
#define PP_PIVOT 4
/* precision of the contraction inside GEMM-class tasks */
#define PP_PREC_FP64 0
#define PP_PREC_TF32 1
/* PP_PREC_BF16: a GEMM whose operands are BF16 shadows (PP_OP_SHADOW) in the tiled layout:
 * p[1] the m x k shadow of op(A), p[2] the n x k shadow of op(B)^T; products summed in FP32 on
 * the tensor cores, C (FP64) := beta C + alpha sum.  m a multiple of 128, k of 64, n 32, 64, 128
 * or a multiple of 256.  l > 0 (a multiple of 64): a second pair p[3] (m x l), p[4] (n x l) whose
 * products join the same sums (two consecutive updates of C in one pass over it). */
#define PP_PREC_BF16 2

/* Split shadows (SHADOW o): a product A B summed over K' = 3 K from the shadows
 * [hi(A) lo(A) hi(A)] and [hi(B) hi(B) lo(B)] is hi hi + lo hi + hi lo, the product of the
 * operands to about 2^-16 of their magnitude instead of BF16's 2^-8 (the mixed form's solves
 * against explicit inverses of the diagonal leaves). */
#define PP_SPLIT_A ((3 << 8) | 0x2)
#define PP_SPLIT_B ((3 << 8) | 0x4)

/* Tiled BF16 layout of an R x K operand (R a multiple of the chunk height h = 128, 64 or 32 — the
 * SHADOW task's ctrl, 0 meaning 128 — and K of 64): chunks of h rows x 64 columns (h * 128 bytes),
 * chunk (R / h block rb, K / 64 block kc) at byte ((rb * (K / 64)) + kc) * h * 128; inside a chunk,
 * element (r, c) at byte ((c / 8) * (h / 8) + r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2 (8 x 8
 * core matrices of 128 contiguous bytes, adjacent along r 128 bytes apart, along c h * 16 bytes
 * apart): the operand layout the tensor core reads from shared memory without swizzling, so one
 * chunk moves with one bulk copy.  A GEMM's A shadow has h = 128; its B shadow has h = 128 when n
 * is a multiple of 256, else h = n (32, 64 or 128). */
#define PP_SHADOW_CHUNK_ROWS 128
#define PP_SHADOW_CHUNK_COLS 64
#define PP_SHADOW_CHUNK_BYTES 16384

typedef struct pp_task {
  int32_t op;
  int32_t flags;
  int32_t m, n, k, l, o; /* dims; meaning per op, documented in vm.cu */
  int32_t ctrl;          /* association order for GEMM3/GEMM4 */
  int32_t ld[6];         /* leading dimension (elements) of each operand */
  double *p[6];          /* operand pointers: p[0] target, p[1..5] inputs */
  double *tmp;           /* task-private scratch (GEMM3/GEMM4/ACCUM) */
  double alpha, beta;
  int32_t succ_begin;    /* successors: succ[succ_begin .. succ_begin + n_succ) */
  int32_t n_succ;
  int32_t prec;          /* PP_PREC_* */
  int32_t instance;      /* owning H-matrix (batched launches) */
  int32_t aux;           /* GEMM4: element offset of the second intermediate in tmp */
  int32_t pad[3];
} pp_task;

#ifdef __cplusplus
static_assert(sizeof(pp_task) == 160, "pp_task layout");
#endif

#endif
