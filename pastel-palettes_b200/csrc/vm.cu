// vm.cu — the persistent H-LU virtual machine for sm_100a, plus FP64 residual kernels.
//
// Replaces the reference's `kernel_dynamic` (Pastel-Palettes src/kernel.cu:1375-1526).
// The reference gives each thread block a fixed, statically scheduled instruction
// stream and makes blocks spin on per-instruction flags in global memory.  Here every
// CTA of a persistent grid pops the next READY task from a device queue; finishing a
// task decrements its successors' dependency counters (acq_rel atomics) and pushes the
// ones that reach zero.  Waits are bounded: a CTA that polls an empty slot for
// `spin_limit` rounds records PP_VM_TIMEOUT and every CTA returns.
//
// Arithmetic contract (FP64 path): every matrix element receives its updates in the
// order the reference's routines apply them, one fma per product with the same
// operands, so dense results are bitwise identical to src/kernel.cu:
//   GETRF  kernel.cu:104-147   l = a_ri / a_ii;  a_rc = fma(a_ic, -l, a_rc), i ascending
//   TRSML  kernel.cu:150-182   b_rc = fma(b_ic, -l_ri, b_rc), i ascending
//   TRSMR  kernel.cu:185-226   x_ri = b_ri / u_ii; b_rc = fma(-x_ri, u_ic, b_rc)
//   TRSMRT kernel.cu:229-285   x_ic = v_ic * (1 / u_ii); v_rc = fma(-u_ir, x_ic, v_rc)
//   GEMM   kernel.cu:288-664   c_ij = fma(alpha a_ik, b_kj, c_ij), k ascending from beta c_ij
// All global loads of data other CTAs may have written use ld.global.cg (L2), never L1.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "vm.cuh"

#define NT PP_VM_THREADS
#define TL PP_VM_TILE
#define LDS (PP_VM_TILE + 1)  /* padded smem row stride (doubles) */
#define KC 16                 /* k-chunk of the GEMM tile loop   */

namespace {

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// ------------------------------------------------------------------------- GEMM
// C[m x n] = beta C + alpha op(A) op(B), alpha in {+1, -1}, beta in {0, 1}.
// 64 x 64 output tiles, 4 x 4 elements per thread, k staged through shared memory
// in chunks of KC; each element's k loop runs in ascending order with one fma.
__device__ void dev_gemm(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda, bool tA,
                         const double* __restrict__ B, int ldb, bool tB, int m, int n, int k, double alpha,
                         double beta, double* smem) {
  double* As = smem;            // [KC][LDS], element (kk, r)
  double* Bs = smem + KC * LDS;  // [KC][LDS], element (kk, c)
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int i0 = 0; i0 < m; i0 += 64)
    for (int j0 = 0; j0 < n; j0 += 64) {
      double acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int r = i0 + ty + 16 * a, c = j0 + tx + 16 * b;
          acc[a][b] = (beta != 0.0 && r < m && c < n) ? ldcg(&C[(size_t)r * ldc + c]) : 0.0;
        }
      for (int k0 = 0; k0 < k; k0 += KC) {
        const int kc = min(KC, k - k0);
        __syncthreads();
        for (int e = tid; e < 64 * KC; e += NT) {
          int kk, r;
          if (!tA) { r = e / KC; kk = e % KC; }
          else { kk = e / 64; r = e % 64; }
          double v = 0.0;
          if (kk < kc && i0 + r < m)
            v = tA ? ldcg(&A[(size_t)(k0 + kk) * lda + i0 + r]) : ldcg(&A[(size_t)(i0 + r) * lda + k0 + kk]);
          As[kk * LDS + r] = v * alpha;  // exact: alpha is +-1
        }
        for (int e = tid; e < 64 * KC; e += NT) {
          int kk, c;
          if (!tB) { kk = e / 64; c = e % 64; }
          else { c = e / KC; kk = e % KC; }
          double v = 0.0;
          if (kk < kc && j0 + c < n)
            v = tB ? ldcg(&B[(size_t)(j0 + c) * ldb + k0 + kk]) : ldcg(&B[(size_t)(k0 + kk) * ldb + j0 + c]);
          Bs[kk * LDS + c] = v;
        }
        __syncthreads();
        for (int kk = 0; kk < kc; ++kk) {
          double av[4], bv[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) av[a] = As[kk * LDS + ty + 16 * a];
#pragma unroll
          for (int b = 0; b < 4; ++b) bv[b] = Bs[kk * LDS + tx + 16 * b];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int r = i0 + ty + 16 * a, c = j0 + tx + 16 * b;
          if (r < m && c < n) C[(size_t)r * ldc + c] = acc[a][b];
        }
      __syncthreads();
    }
}

// ------------------------------------------------------------------------- tiles in smem
__device__ void load_tile(double* S, const double* __restrict__ G, int ld, int rows, int cols) {
  for (int e = threadIdx.x; e < rows * cols; e += NT) {
    const int r = e / cols, c = e % cols;
    S[r * LDS + c] = ldcg(&G[(size_t)r * ld + c]);
  }
}
__device__ void store_tile(double* G, int ld, const double* S, int rows, int cols) {
  for (int e = threadIdx.x; e < rows * cols; e += NT) {
    const int r = e / cols, c = e % cols;
    G[(size_t)r * ld + c] = S[r * LDS + c];
  }
}

// A[m x n] := L\U in place (m, n <= TL), a warp per row like kernel.cu:104-147
__device__ void dev_getrf(double* A, int lda, int m, int n, double* smem) {
  double* S = smem;
  load_tile(S, A, lda, m, n);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mn = min(m, n);
  for (int i = 0; i < mn; ++i) {
    const double piv = S[i * LDS + i];
    for (int r = i + 1 + warp; r < m; r += NT / 32) {
      double l = 0.0;
      if (lane == 0) {
        l = S[r * LDS + i] / piv;
        S[r * LDS + i] = l;
      }
      l = __shfl_sync(0xffffffffu, l, 0);
      for (int c = i + 1 + lane; c < n; c += 32) S[r * LDS + c] = fma(S[i * LDS + c], -l, S[r * LDS + c]);
    }
    __syncthreads();
  }
  store_tile(A, lda, S, m, n);
}

// B[m x n] := L^-1 B, L unit lower m x m (m <= TL); column chunks of TL
__device__ void dev_trsml(double* B, int ldb, const double* L, int ldl, int m, int n, double* smem) {
  double* Ls = smem;
  double* Bs = smem + TL * LDS;
  load_tile(Ls, L, ldl, m, m);
  for (int c0 = 0; c0 < n; c0 += TL) {
    const int w = min(TL, n - c0);
    load_tile(Bs, B + c0, ldb, m, w);
    __syncthreads();
    for (int i = 0; i + 1 < m; ++i) {
      const int cnt = (m - i - 1) * w;
      for (int e = threadIdx.x; e < cnt; e += NT) {
        const int r = i + 1 + e / w, c = e % w;
        Bs[r * LDS + c] = fma(Bs[i * LDS + c], -Ls[r * LDS + i], Bs[r * LDS + c]);
      }
      __syncthreads();
    }
    store_tile(B + c0, ldb, Bs, m, w);
    __syncthreads();
  }
}

// B[m x n] := B U^-1, U upper n x n (n <= TL); rows are independent: a warp per row,
// the row held in registers (lane owns columns lane and lane + 32)
__device__ void dev_trsmr(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  double* Us = smem;
  load_tile(Us, U, ldu, n, n);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < m; r += NT / 32) {
    double* row = B + (size_t)r * ldb;
    double x0 = lane < n ? ldcg(&row[lane]) : 0.0;
    double x1 = lane + 32 < n ? ldcg(&row[lane + 32]) : 0.0;
    for (int i = 0; i < n; ++i) {
      const double bi = __shfl_sync(0xffffffffu, i < 32 ? x0 : x1, i & 31);
      const double xi = bi / Us[i * LDS + i];
      if (lane == (i & 31)) {
        if (i < 32) x0 = xi;
        else x1 = xi;
      }
      const double left = -xi;
      if (lane > i && lane < n) x0 = fma(left, Us[i * LDS + lane], x0);
      if (lane + 32 > i && lane + 32 < n) x1 = fma(left, Us[i * LDS + lane + 32], x1);
    }
    if (lane < n) row[lane] = x0;
    if (lane + 32 < n) row[lane + 32] = x1;
  }
}

// V[m x n] := U^-T V, U upper m x m (m <= TL): the reference's trsmr on a transposed
// B (kernel.cu:229-285) — row i is scaled by the reciprocal of u_ii
__device__ void dev_trsmrt(double* V, int ldv, const double* U, int ldu, int m, int n, double* smem) {
  double* Us = smem;
  double* Vs = smem + TL * LDS;
  load_tile(Us, U, ldu, m, m);
  for (int c0 = 0; c0 < n; c0 += TL) {
    const int w = min(TL, n - c0);
    load_tile(Vs, V + c0, ldv, m, w);
    __syncthreads();
    for (int i = 0; i < m; ++i) {
      const double rd = 1.0 / Us[i * LDS + i];
      for (int c = threadIdx.x; c < w; c += NT) Vs[i * LDS + c] *= rd;
      __syncthreads();
      const int cnt = (m - i - 1) * w;
      for (int e = threadIdx.x; e < cnt; e += NT) {
        const int r = i + 1 + e / w, c = e % w;
        Vs[r * LDS + c] = fma(-Us[i * LDS + r], Vs[i * LDS + c], Vs[r * LDS + c]);
      }
      __syncthreads();
    }
    store_tile(V + c0, ldv, Vs, m, w);
    __syncthreads();
  }
}

// B[m x n] := U^-1 B, U upper m x m (m <= TL), backward substitution (solve phase)
__device__ void dev_trsmu(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  double* Us = smem;
  double* Bs = smem + TL * LDS;
  load_tile(Us, U, ldu, m, m);
  for (int c0 = 0; c0 < n; c0 += TL) {
    const int w = min(TL, n - c0);
    load_tile(Bs, B + c0, ldb, m, w);
    __syncthreads();
    for (int i = m - 1; i >= 0; --i) {
      const double d = Us[i * LDS + i];
      for (int c = threadIdx.x; c < w; c += NT) Bs[i * LDS + c] = Bs[i * LDS + c] / d;
      __syncthreads();
      const int cnt = i * w;
      for (int e = threadIdx.x; e < cnt; e += NT) {
        const int r = e / w, c = e % w;
        Bs[r * LDS + c] = fma(-Us[r * LDS + i], Bs[i * LDS + c], Bs[r * LDS + c]);
      }
      __syncthreads();
    }
    store_tile(B + c0, ldb, Bs, m, w);
    __syncthreads();
  }
}

// ------------------------------------------------------------------------- GEMM3 / GEMM4
// Reference association orders (kernel.cu:886-955), intermediates in task scratch.
__device__ void dev_gemm3(const pp_task& T, double* smem) {
  const bool tA = T.flags & PP_T(1), tB = T.flags & PP_T(2), tC = T.flags & PP_T(3);
  double* t1 = T.tmp;
  const int m = T.m, n = T.n, k = T.k, l = T.l;
  if (T.ctrl) {  // (A B) C, t1: m x l
    dev_gemm(t1, l, T.p[1], T.ld[1], tA, T.p[2], T.ld[2], tB, m, l, k, 1.0, 0.0, smem);
    __syncthreads();
    dev_gemm(T.p[0], T.ld[0], t1, l, false, T.p[3], T.ld[3], tC, m, n, l, T.alpha, 1.0, smem);
  } else {       // A (B C), t1: k x n
    dev_gemm(t1, n, T.p[2], T.ld[2], tB, T.p[3], T.ld[3], tC, k, n, l, 1.0, 0.0, smem);
    __syncthreads();
    dev_gemm(T.p[0], T.ld[0], T.p[1], T.ld[1], tA, t1, n, false, m, n, k, T.alpha, 1.0, smem);
  }
}

__device__ void dev_gemm4(const pp_task& T, double* smem) {
  const bool tA = T.flags & PP_T(1), tB = T.flags & PP_T(2), tC = T.flags & PP_T(3), tD = T.flags & PP_T(4);
  const double *A = T.p[1], *B = T.p[2], *Cm = T.p[3], *D = T.p[4];
  const int la = T.ld[1], lb = T.ld[2], lc = T.ld[3], ld = T.ld[4];
  const int m = T.m, n = T.n, k = T.k, l = T.l, o = T.o;
  double* t1 = T.tmp;
  double* t2 = T.tmp + T.aux;  // second intermediate (reference gemm_4x `offset`)
  double* M = T.p[0];
  const int lm = T.ld[0];
  switch (T.ctrl) {
    case 0:  // ((A B) C) D; t1 m x l, t2 m x o
      dev_gemm(t1, l, A, la, tA, B, lb, tB, m, l, k, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(t2, o, t1, l, false, Cm, lc, tC, m, o, l, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(M, lm, t2, o, false, D, ld, tD, m, n, o, T.alpha, 1.0, smem);
      break;
    case 1:  // (A (B C)) D; t1 k x o, t2 m x o
      dev_gemm(t1, o, B, lb, tB, Cm, lc, tC, k, o, l, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(t2, o, A, la, tA, t1, o, false, m, o, k, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(M, lm, t2, o, false, D, ld, tD, m, n, o, T.alpha, 1.0, smem);
      break;
    case 2:  // A ((B C) D); t1 k x o, t2 k x n
      dev_gemm(t1, o, B, lb, tB, Cm, lc, tC, k, o, l, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(t2, n, t1, o, false, D, ld, tD, k, n, o, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(M, lm, A, la, tA, t2, n, false, m, n, k, T.alpha, 1.0, smem);
      break;
    case 3:  // A (B (C D)); t1 l x n, t2 k x n
      dev_gemm(t1, n, Cm, lc, tC, D, ld, tD, l, n, o, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(t2, n, B, lb, tB, t1, n, false, k, n, l, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(M, lm, A, la, tA, t2, n, false, m, n, k, T.alpha, 1.0, smem);
      break;
    default:  // 4: (A B) (C D); t1 m x l, t2 l x n
      dev_gemm(t1, l, A, la, tA, B, lb, tB, m, l, k, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(t2, n, Cm, lc, tC, D, ld, tD, l, n, o, 1.0, 0.0, smem); __syncthreads();
      dev_gemm(M, lm, t1, l, false, t2, n, false, m, n, l, T.alpha, 1.0, smem);
      break;
  }
}

// ------------------------------------------------------------------------- ACCUM
// Deterministic CTA-wide column sums: thread t accumulates rows r0 + t, r0 + t + NT, ...
// in ascending order; lanes combine by an xor butterfly; warps are added in order.
template <int KM>
__device__ __forceinline__ void cta_sum_cols(double (&v)[KM], int ncols, double* red, double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < KM; ++c) {
    if (c < ncols) {
      double x = v[c];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane == 0) red[warp * KM + c] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x < ncols) {
    double s = red[threadIdx.x];
    for (int w = 1; w < NT / 32; ++w) s += red[w * KM + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Householder QR of Y (m x k, ld k, global scratch) and explicit Q (m x k, ld k).
// Column j: nrm = sqrt(y_jj^2 + sum_{r>j} y_rj^2), beta = -sign(y_jj) nrm,
// v_r = y_rj / (y_jj - beta), tau = (beta - y_jj) / beta.
__device__ void dev_householder_qr(double* Y, double* Q, int m, int k, double* smem) {
  double* red = smem;                  // NT/32 x PP_VM_MAX_RANK
  double* sums = red + (NT / 32) * PP_VM_MAX_RANK;  // PP_VM_MAX_RANK
  double* tau = sums + PP_VM_MAX_RANK;  // PP_VM_MAX_RANK
  __shared__ double s_beta;
  for (int j = 0; j < k; ++j) {
    double v[PP_VM_MAX_RANK];
    // norm of the column below the diagonal
    {
      double s = 0.0;
      for (int r = j + 1 + threadIdx.x; r < m; r += NT) {
        const double y = ldcg(&Y[(size_t)r * k + j]);
        s = fma(y, y, s);
      }
      double one[1] = {s};
      cta_sum_cols<1>(one, 1, red, sums);
    }
    if (threadIdx.x == 0) {
      const double a = ldcg(&Y[(size_t)j * k + j]);
      const double nrm = sqrt(fma(a, a, sums[0]));
      if (nrm == 0.0) { tau[j] = 0.0; s_beta = 0.0; }
      else {
        const double beta = a >= 0.0 ? -nrm : nrm;
        tau[j] = (beta - a) / beta;
        s_beta = a - beta;  // divisor of v
        Y[(size_t)j * k + j] = beta;
      }
    }
    __syncthreads();
    const double div = s_beta;
    if (div != 0.0)
      for (int r = j + 1 + threadIdx.x; r < m; r += NT) Y[(size_t)r * k + j] = ldcg(&Y[(size_t)r * k + j]) / div;
    __syncthreads();
    const double tj = tau[j];
    const int nc = k - j - 1;  // columns j+1 .. k-1
    if (nc > 0 && tj != 0.0) {
#pragma unroll
      for (int c = 0; c < PP_VM_MAX_RANK; ++c) v[c] = 0.0;
      for (int r = j + 1 + threadIdx.x; r < m; r += NT) {
        const double vr = ldcg(&Y[(size_t)r * k + j]);
#pragma unroll
        for (int c = 0; c < PP_VM_MAX_RANK; ++c)
          if (c < nc) v[c] = fma(vr, ldcg(&Y[(size_t)r * k + j + 1 + c]), v[c]);
      }
      cta_sum_cols<PP_VM_MAX_RANK>(v, nc, red, sums);
      // w_c = y_jc + sum;  y_jc -= tau w_c;  y_rc -= tau w_c v_r
      for (int c = threadIdx.x; c < nc; c += NT) {
        const double w = ldcg(&Y[(size_t)j * k + j + 1 + c]) + sums[c];
        sums[c] = tj * w;
        Y[(size_t)j * k + j + 1 + c] = fma(-tj, w, ldcg(&Y[(size_t)j * k + j + 1 + c]));
      }
      __syncthreads();
      for (int r = j + 1 + threadIdx.x; r < m; r += NT) {
        const double vr = ldcg(&Y[(size_t)r * k + j]);
        for (int c = 0; c < nc; ++c) {
          double* p = &Y[(size_t)r * k + j + 1 + c];
          *p = fma(-sums[c], vr, ldcg(p));
        }
      }
      __syncthreads();
    }
  }
  // Q = H_0 ... H_{k-1} [I; 0]
  for (int e = threadIdx.x; e < m * k; e += NT) {
    const int r = e / k, c = e % k;
    Q[e] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int j = k - 1; j >= 0; --j) {
    const double tj = tau[j];
    if (tj == 0.0) continue;
    const int nc = k - j;  // columns j .. k-1
    double v[PP_VM_MAX_RANK];
#pragma unroll
    for (int c = 0; c < PP_VM_MAX_RANK; ++c) v[c] = 0.0;
    for (int r = j + 1 + threadIdx.x; r < m; r += NT) {
      const double vr = ldcg(&Y[(size_t)r * k + j]);
#pragma unroll
      for (int c = 0; c < PP_VM_MAX_RANK; ++c)
        if (c < nc) v[c] = fma(vr, ldcg(&Q[(size_t)r * k + j + c]), v[c]);
    }
    cta_sum_cols<PP_VM_MAX_RANK>(v, nc, red, sums);
    for (int c = threadIdx.x; c < nc; c += NT) {
      const double w = ldcg(&Q[(size_t)j * k + j + c]) + sums[c];
      sums[c] = tj * w;
      Q[(size_t)j * k + j + c] = fma(-tj, w, ldcg(&Q[(size_t)j * k + j + c]));
    }
    __syncthreads();
    for (int r = j + 1 + threadIdx.x; r < m; r += NT) {
      const double vr = ldcg(&Y[(size_t)r * k + j]);
      for (int c = 0; c < nc; ++c) {
        double* p = &Q[(size_t)r * k + j + c];
        *p = fma(-sums[c], vr, ldcg(p));
      }
    }
    __syncthreads();
  }
}

// U1 V1^T := Q Q^T (U1 V1^T + alpha U2 V2^T), Q spanning (U1 V1^T + alpha U2 V2^T) R:
// the reference's randomized accumulation (kernel.cu:1255-1280) with a Householder QR
// in place of its Givens sweeps.  m = ny, n = nx, k = k1 (target rank), l = k2.
__device__ void dev_accum(const pp_task& T, double* smem) {
  const int ny = T.m, nx = T.n, k1 = T.k, k2 = T.l;
  const bool tU2 = T.flags & PP_T(2), tV2 = T.flags & PP_T(3);
  double *U1 = T.p[0], *V1 = T.p[1];
  const double *U2 = T.p[2], *V2 = T.p[3], *R = T.p[4];
  const int lu1 = T.ld[0], lv1 = T.ld[1], lu2 = T.ld[2], lv2 = T.ld[3], lr = T.ld[4];
  const int kp = max(k1, k2);
  double* Ys = T.tmp;                          // ny x k1
  double* P = Ys + (size_t)ny * k1;            // k1 x kp
  double* W = P + (size_t)k1 * kp;             // nx x k1
  double* Q = W + (size_t)nx * k1;             // ny x k1
  const double al = T.alpha;
  dev_gemm(P, kp, R, lr, true, V1, lv1, false, k1, k1, nx, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(Ys, k1, U1, lu1, false, P, kp, true, ny, k1, k1, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(P, kp, R, lr, true, V2, lv2, tV2, k1, k2, nx, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(Ys, k1, U2, lu2, tU2, P, kp, true, ny, k1, k2, al, 1.0, smem); __syncthreads();
  dev_householder_qr(Ys, Q, ny, k1, smem);
  __syncthreads();
  dev_gemm(P, kp, Q, k1, true, U1, lu1, false, k1, k1, ny, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(W, k1, V1, lv1, false, P, kp, true, nx, k1, k1, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(P, kp, Q, k1, true, U2, lu2, tU2, k1, k2, ny, 1.0, 0.0, smem); __syncthreads();
  dev_gemm(W, k1, V2, lv2, tV2, P, kp, true, nx, k1, k2, al, 1.0, smem); __syncthreads();
  for (int e = threadIdx.x; e < ny * k1; e += NT) {
    const int r = e / k1, c = e % k1;
    U1[(size_t)r * lu1 + c] = ldcg(&Q[e]);
  }
  for (int e = threadIdx.x; e < nx * k1; e += NT) {
    const int r = e / k1, c = e % k1;
    V1[(size_t)r * lv1 + c] = ldcg(&W[e]);
  }
}

__device__ bool run_task(const pp_task& T, double* smem) {
  switch (T.op) {
    case PP_OP_NOP: return true;
    case PP_OP_GETRF:
      if (T.m > TL || T.n > TL) return false;
      dev_getrf(T.p[0], T.ld[0], T.m, T.n, smem);
      return true;
    case PP_OP_TRSML:
      if (T.m > TL) return false;
      dev_trsml(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMR:
      if (T.n > TL) return false;
      dev_trsmr(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMRT:
      if (T.m > TL) return false;
      dev_trsmrt(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMU:
      if (T.m > TL) return false;
      dev_trsmu(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_GEMM:
      dev_gemm(T.p[0], T.ld[0], T.p[1], T.ld[1], T.flags & PP_T(1), T.p[2], T.ld[2], T.flags & PP_T(2), T.m, T.n,
               T.k, T.alpha, T.beta, smem);
      return true;
    case PP_OP_GEMM3: dev_gemm3(T, smem); return true;
    case PP_OP_GEMM4: dev_gemm4(T, smem); return true;
    case PP_OP_ACCUM:
      if (T.k > PP_VM_MAX_RANK || T.k < 1) return false;
      dev_accum(T, smem);
      return true;
    default: return false;
  }
}

__global__ void vm_init(const int32_t* __restrict__ indeg, const int32_t* __restrict__ ready, int n_ready, int n,
                        int32_t* counters, int32_t* slots, pp_vm_state* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    counters[i] = indeg[i];
    slots[i] = i < n_ready ? ready[i] : -1;
  }
  if (i == 0) {
    st->head = 0;
    st->tail = n_ready;
    st->done = 0;
    st->error = 0;
    st->err_info = -1;
  }
}

__global__ void __launch_bounds__(NT, 2)
    vm_kernel(const pp_task* __restrict__ tasks, int n_tasks, const int32_t* __restrict__ succ, int32_t* counters,
              int32_t* slots, pp_vm_state* st, long long spin_limit) {
  extern __shared__ double smem[];
  __shared__ __align__(16) pp_task s_task;
  __shared__ int s_id;
  for (;;) {
    if (threadIdx.x == 0) {
      int id = -1;
      const int idx = atomicAdd(&st->head, 1);
      if (idx < n_tasks) {
        long long spins = 0;
        for (;;) {
          id = ld_acquire(&slots[idx]);
          if (id >= 0) break;
          if (ld_relaxed(&st->error)) { id = -1; break; }
          if (++spins > spin_limit) {
            if (atomicCAS(&st->error, 0, PP_VM_TIMEOUT) == 0) st->err_info = idx;
            id = -1;
            break;
          }
          __nanosleep(64);
        }
      }
      s_id = id;
    }
    __syncthreads();
    const int id = s_id;
    if (id < 0) return;
    if (threadIdx.x < (int)(sizeof(pp_task) / 8))
      reinterpret_cast<unsigned long long*>(&s_task)[threadIdx.x] =
          __ldg(reinterpret_cast<const unsigned long long*>(&tasks[id]) + threadIdx.x);
    __syncthreads();
    const bool ok = run_task(s_task, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (!ok && atomicCAS(&st->error, 0, PP_VM_BAD_TASK) == 0) st->err_info = id;
      __threadfence();
      for (int q = 0; q < s_task.n_succ; ++q) {
        const int s = succ[s_task.succ_begin + q];
        if (atom_add_acq_rel(&counters[s], -1) == 1) {
          const int pos = atomicAdd(&st->tail, 1);
          st_release(&slots[pos], s);
        }
      }
      atomicAdd(&st->done, 1);
    }
  }
}

// ------------------------------------------------------------------------- residuals
// r = b - A x, one warp per row; columns of A read once per RHS block
__global__ void dense_residual_kernel(const double* __restrict__ A, int lda, int n, const double* __restrict__ x,
                                      const double* __restrict__ b, double* __restrict__ r, int nrhs) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const double* a = A + (size_t)warp * lda;
  for (int q = 0; q < nrhs; ++q) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s = fma(a[j], x[(size_t)j * nrhs + q], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) r[(size_t)warp * nrhs + q] = b[(size_t)warp * nrhs + q] - s;
  }
}

__device__ __forceinline__ double kernel_eval(int kind, double d, double p0, double p1) {
  switch (kind) {
    case 0: return 1.0 / (d + p0);                                  // 1 / (r + eps)
    case 1: return 1.0 / (4.0 * 3.14159265358979323846 * (d + p0)); // Laplace 3-D
    case 2: return exp(-d / p0);                                     // exponential
    default: {                                                      // Matern 3/2
      const double s = 1.7320508075688772 * d / p0;
      return (1.0 + s) * exp(-s);
    }
  }
}

#define KR_ROWS 128
#define KR_COLS 256
// matrix-free r = b - A x, A_ij = K(|p_i - p_j|) (+ diag_shift on i == j); each CTA owns
// KR_ROWS rows (a thread per row) and sweeps all columns in KR_COLS tiles through smem
__global__ void kernel_residual_kernel(int kind, double p0, double p1, double shift, const double* __restrict__ pts,
                                       int dim, int n, const double* __restrict__ x, const double* __restrict__ b,
                                       double* __restrict__ r, int nrhs) {
  __shared__ double sp[KR_COLS * 3];
  __shared__ double sx[KR_COLS * 16];
  const int i = blockIdx.x * KR_ROWS + threadIdx.x;
  double pi[3] = {0, 0, 0};
  if (i < n)
    for (int d = 0; d < dim; ++d) pi[d] = pts[(size_t)i * dim + d];
  double acc[16];
  for (int q = 0; q < 16; ++q) acc[q] = 0.0;
  for (int j0 = 0; j0 < n; j0 += KR_COLS) {
    const int nj = min(KR_COLS, n - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < nj * dim; e += blockDim.x) sp[e] = pts[(size_t)j0 * dim + e];
    for (int e = threadIdx.x; e < nj * nrhs; e += blockDim.x) sx[e] = x[(size_t)j0 * nrhs + e];
    __syncthreads();
    if (i < n)
      for (int j = 0; j < nj; ++j) {
        double d2 = 0.0;
        for (int d = 0; d < dim; ++d) {
          const double t = pi[d] - sp[j * dim + d];
          d2 = fma(t, t, d2);
        }
        double a = kernel_eval(kind, sqrt(d2), p0, p1);
        if (j0 + j == i) a += shift;
        for (int q = 0; q < nrhs; ++q) acc[q] = fma(a, sx[j * nrhs + q], acc[q]);
      }
  }
  if (i < n)
    for (int q = 0; q < nrhs; ++q) r[(size_t)i * nrhs + q] = b[(size_t)i * nrhs + q] - acc[q];
}

// One ACCUM on caller buffers; its scratch (T.tmp) is the static array below.
__global__ void __launch_bounds__(NT) accum_noalloc_kernel(pp_task T) {
  extern __shared__ double smem[];
  dev_accum(T, smem);
}

}  // namespace

// Scratch of pp_lowrank_accum_noalloc: a file-scope device array, so the entry point never
// allocates.  Every device that loads the library holds it (8 MiB) until the process exits.
// Host code may not use its name as an address: the device address is looked up once per
// device with cudaGetSymbolAddress (below) and passed to the kernel.
#define PP_NOALLOC_SCRATCH_DOUBLES (1 << 20)
static __device__ __align__(256) double g_accum_noalloc_scratch[PP_NOALLOC_SCRATCH_DOUBLES];

long long pp_accum_noalloc_capacity() { return PP_NOALLOC_SCRATCH_DOUBLES; }

cudaError_t pp_accum_noalloc_launch(const pp_task& T, long long scratch_doubles, cudaStream_t s) {
  if (scratch_doubles < 0 || scratch_doubles > PP_NOALLOC_SCRATCH_DOUBLES) return cudaErrorInvalidValue;
  constexpr int kMaxDevices = 64;
  static double* addr[kMaxDevices] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!addr[dev]) {  // set-up, once per device, with that device current
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_accum_noalloc_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = p;
  }
  pp_task t = T;
  t.tmp = addr[dev];
  // shared memory: the GEMM k-chunk tiles, which also hold the QR reductions
  accum_noalloc_kernel<<<1, NT, (size_t)2 * KC * LDS * sizeof(double), s>>>(t);
  return cudaGetLastError();
}

size_t pp_vm_smem_bytes() { return (size_t)2 * TL * LDS * sizeof(double); }

int pp_vm_blocks_per_sm() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, vm_kernel, NT, pp_vm_smem_bytes());
  return nb;
}

cudaError_t pp_vm_prepare() {
  return cudaFuncSetAttribute(vm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pp_vm_smem_bytes());
}

cudaError_t pp_vm_run(const pp_vm_launch& L, cudaStream_t s) {
  if (L.n_tasks <= 0) return cudaSuccess;
  const int ib = 256;
  vm_init<<<(L.n_tasks + ib - 1) / ib, ib, 0, s>>>(L.indeg, L.ready, L.n_ready, L.n_tasks, L.counters, L.slots,
                                                  L.state);
  vm_kernel<<<L.grid, NT, pp_vm_smem_bytes(), s>>>(L.tasks, L.n_tasks, L.succ, L.counters, L.slots, L.state,
                                                   L.spin_limit);
  return cudaGetLastError();
}

cudaError_t pp_dense_residual(const double* A, int lda, int n, const double* x, const double* b, double* r, int nrhs,
                              cudaStream_t s) {
  const int threads = 256, warps = threads / 32;
  dense_residual_kernel<<<(n + warps - 1) / warps, threads, 0, s>>>(A, lda, n, x, b, r, nrhs);
  return cudaGetLastError();
}

cudaError_t pp_kernel_residual(int kernel, double p0, double p1, double diag_shift, const double* pts, int dim, int n,
                               const double* x, const double* b, double* r, int nrhs, cudaStream_t s) {
  if (dim < 1 || dim > 3 || nrhs < 1 || nrhs > 16) return cudaErrorInvalidValue;
  kernel_residual_kernel<<<(n + KR_ROWS - 1) / KR_ROWS, KR_ROWS, 0, s>>>(kernel, p0, p1, diag_shift, pts, dim, n, x, b,
                                                                        r, nrhs);
  return cudaGetLastError();
}
