// vm.cu — the persistent H-LU virtual machine for sm_100a, plus FP64 residual kernels.
//
// Replaces the reference's `kernel_dynamic` (Pastel-Palettes src/kernel.cu:1375-1526).
// The reference gives each thread block a fixed, statically scheduled instruction
// stream and makes blocks spin on per-instruction flags in global memory.  Here every
// CTA of a persistent grid pops the next READY task from a device queue; finishing a
// task decrements its successors' dependency counters (acq_rel atomics) and pushes the
// ones that reach zero.  Waits are bounded: a CTA that polls an empty slot for
// longer than its time limit (globaltimer) records PP_VM_TIMEOUT and every CTA returns.
//
// Arithmetic contract (FP64 path): every matrix element receives its updates in the
// order the reference's routines apply them, one fma per product with the same
// operands, so dense results are bitwise identical to src/kernel.cu:
//   GETRF  kernel.cu:104-147   l = a_ri / a_ii;  a_rc = fma(a_ic, -l, a_rc), i ascending
//   TRSML  kernel.cu:150-182   b_rc = fma(b_ic, -l_ri, b_rc), i ascending
//   TRSMR  kernel.cu:185-226   x_ri = b_ri / u_ii; b_rc = fma(-x_ri, u_ic, b_rc)
//   TRSMRT kernel.cu:229-285   x_ic = v_ic * (1 / u_ii); v_rc = fma(-u_ir, x_ic, v_rc)
//   GEMM   kernel.cu:288-664   c_ij = fma(alpha a_ik, b_kj, c_ij), k ascending from beta c_ij
// Work distribution does not touch that order: GEMM tiles are shaped to the operands
// (square, skinny, single column, small output with a long k), the triangular routines
// keep each column (or row) in registers across four lanes of a warp and broadcast the
// finished pivot entry with a shuffle, so they need no CTA barrier per step.
// All global loads of data other CTAs may have written use ld.global.cg (L2), never L1.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>
#include <stdint.h>

#include "vm.cuh"

#define NT PP_VM_THREADS
#define TL PP_VM_TILE
#define LDS (PP_VM_TILE + 1)   /* padded smem row stride (doubles) */
#define VM_SMEM_BYTES 184320   /* 180 KB, one CTA per SM: ACCUM keeps its ny x k1 sketch on chip;
                                  the BF16 GEMM holds 3 stages of 48 KB + its epilogue's buffers */

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
// CTA tile TM x TN, thread micro-tile RM x RN (rows ty + TY a, columns tx + TX b), k in
// chunks of KCH staged through shared memory; the next chunk is fetched into registers
// while the current one is consumed.  Each element's k loop runs in ascending order.
template <int TM, int TN, int RM, int RN, int KCH>
__device__ __noinline__ void gemm_cfg(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda,
                                         bool tA, const double* __restrict__ B, int ldb, bool tB, int m, int n, int k,
                                         double alpha, double beta, double* smem) {
  constexpr int TX = TN / RN, TY = TM / RM;
  static_assert(TX * TY == NT, "thread layout");
  constexpr int LA = TM + 1, LB = TN + 1;
  constexpr int AE = TM * KCH, BE = KCH * TN;
  constexpr int AP = (AE + NT - 1) / NT, BP = (BE + NT - 1) / NT;
  static_assert((KCH * LA + KCH * LB) * 8 <= VM_SMEM_BYTES, "smem");
  double* As = smem;             // [KCH][LA]
  double* Bs = smem + KCH * LA;  // [KCH][LB]
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int nch = (k + KCH - 1) / KCH;
  for (int i0 = 0; i0 < m; i0 += TM)
    for (int j0 = 0; j0 < n; j0 += TN) {
      double acc[RM][RN];
#pragma unroll
      for (int a = 0; a < RM; ++a)
#pragma unroll
        for (int b = 0; b < RN; ++b) {
          const int r = i0 + ty + TY * a, c = j0 + tx + TX * b;
          acc[a][b] = (beta != 0.0 && r < m && c < n) ? ldcg(&C[(size_t)r * ldc + c]) : 0.0;
        }
      double ra[AP], rb[BP];
#define PP_GEMM_FETCH(K0)                                                                                     \
  do {                                                                                                        \
    const int k0_ = (K0);                                                                                     \
    _Pragma("unroll") for (int p = 0; p < AP; ++p) {                                                          \
      const int e = tid + p * NT;                                                                             \
      int r, kk;                                                                                              \
      if (!tA) { r = e / KCH; kk = e % KCH; }                                                                 \
      else { kk = e / TM; r = e % TM; }                                                                       \
      double v = 0.0;                                                                                         \
      if (e < AE && k0_ + kk < k && i0 + r < m)                                                               \
        v = tA ? ldcg(&A[(size_t)(k0_ + kk) * lda + i0 + r]) : ldcg(&A[(size_t)(i0 + r) * lda + k0_ + kk]);   \
      ra[p] = v * alpha; /* exact: alpha is +-1 */                                                            \
    }                                                                                                         \
    _Pragma("unroll") for (int p = 0; p < BP; ++p) {                                                          \
      const int e = tid + p * NT;                                                                             \
      int c, kk;                                                                                              \
      if (!tB) { kk = e / TN; c = e % TN; }                                                                   \
      else { c = e / KCH; kk = e % KCH; }                                                                     \
      double v = 0.0;                                                                                         \
      if (e < BE && k0_ + kk < k && j0 + c < n)                                                               \
        v = tB ? ldcg(&B[(size_t)(j0 + c) * ldb + k0_ + kk]) : ldcg(&B[(size_t)(k0_ + kk) * ldb + j0 + c]);   \
      rb[p] = v;                                                                                              \
    }                                                                                                         \
  } while (0)
      if (nch > 0) PP_GEMM_FETCH(0);
      for (int ch = 0; ch < nch; ++ch) {
        __syncthreads();
#pragma unroll
        for (int p = 0; p < AP; ++p) {
          const int e = tid + p * NT;
          if (e < AE) {
            int r, kk;
            if (!tA) { r = e / KCH; kk = e % KCH; }
            else { kk = e / TM; r = e % TM; }
            As[kk * LA + r] = ra[p];
          }
        }
#pragma unroll
        for (int p = 0; p < BP; ++p) {
          const int e = tid + p * NT;
          if (e < BE) {
            int c, kk;
            if (!tB) { kk = e / TN; c = e % TN; }
            else { c = e / KCH; kk = e % KCH; }
            Bs[kk * LB + c] = rb[p];
          }
        }
        __syncthreads();
        if (ch + 1 < nch) PP_GEMM_FETCH((ch + 1) * KCH);
        const int kc = min(KCH, k - ch * KCH);
        for (int kk = 0; kk < kc; ++kk) {
          double av[RM], bv[RN];
#pragma unroll
          for (int a = 0; a < RM; ++a) av[a] = As[kk * LA + ty + TY * a];
#pragma unroll
          for (int b = 0; b < RN; ++b) bv[b] = Bs[kk * LB + tx + TX * b];
#pragma unroll
          for (int a = 0; a < RM; ++a)
#pragma unroll
            for (int b = 0; b < RN; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
      }
#pragma unroll
      for (int a = 0; a < RM; ++a)
#pragma unroll
        for (int b = 0; b < RN; ++b) {
          const int r = i0 + ty + TY * a, c = j0 + tx + TX * b;
          if (r < m && c < n) C[(size_t)r * ldc + c] = acc[a][b];
        }
    }
  __syncthreads();
}

// C[m x n] (m, n <= 16) = beta C + alpha op(A) op(B) for a long k, in free order: each warp
// sums a contiguous k slice (ascending, 8 outputs per lane), the slices are then added in
// warp order.  Deterministic, but not the reference's single ascending chain per element.
__device__ __noinline__ void gemm_splitk(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda,
                                         bool tA, const double* __restrict__ B, int ldb, bool tB, int m, int n, int k,
                                         double alpha, double beta, double* smem) {
  constexpr int KW = 16, NW = NT / 32, LW = 17;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* As = smem + w * (2 * KW * LW);  // [KW][LW] (kk, r), this warp's
  double* Bs = As + KW * LW;              // [KW][LW] (kk, c)
  const int kseg = (k + NW - 1) / NW;
  const int kb = min(k, w * kseg), ke = min(k, kb + kseg);
  const int c_out = lane & 15;
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) acc[q] = 0.0;
  double ra[8], rb[8];
#define PP_SPLITK_FETCH(K0)                                                                                   \
  do {                                                                                                        \
    const int k0_ = (K0);                                                                                     \
    _Pragma("unroll") for (int p = 0; p < 8; ++p) {                                                           \
      const int e = lane + 32 * p;                                                                            \
      const int kk = tA ? (e >> 4) : (e & 15), r = tA ? (e & 15) : (e >> 4);                                  \
      double v = 0.0;                                                                                         \
      if (r < m && k0_ + kk < ke)                                                                             \
        v = tA ? ldcg(&A[(size_t)(k0_ + kk) * lda + r]) : ldcg(&A[(size_t)r * lda + k0_ + kk]);               \
      ra[p] = v * alpha;                                                                                      \
      const int kb_ = tB ? (e & 15) : (e >> 4), c = tB ? (e >> 4) : (e & 15);                                 \
      double u = 0.0;                                                                                         \
      if (c < n && k0_ + kb_ < ke)                                                                            \
        u = tB ? ldcg(&B[(size_t)c * ldb + k0_ + kb_]) : ldcg(&B[(size_t)(k0_ + kb_) * ldb + c]);            \
      rb[p] = u;                                                                                              \
    }                                                                                                         \
  } while (0)
  if (kb < ke) PP_SPLITK_FETCH(kb);
  for (int k0 = kb; k0 < ke; k0 += KW) {
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int e = lane + 32 * p;
      As[(tA ? (e >> 4) : (e & 15)) * LW + (tA ? (e & 15) : (e >> 4))] = ra[p];
      Bs[(tB ? (e & 15) : (e >> 4)) * LW + (tB ? (e >> 4) : (e & 15))] = rb[p];
    }
    __syncwarp();
    if (k0 + KW < ke) PP_SPLITK_FETCH(k0 + KW);
    const int kc = min(KW, ke - k0);
    for (int kk = 0; kk < kc; ++kk) {
      const double b = Bs[kk * LW + c_out];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] = fma(As[kk * LW + ((lane + 32 * q) >> 4)], b, acc[q]);
    }
    __syncwarp();
  }
#undef PP_SPLITK_FETCH
  __syncthreads();
  double* red = smem;  // [NW][256] partial sums, output o = r * 16 + c
#pragma unroll
  for (int q = 0; q < 8; ++q) red[w * 256 + lane + 32 * q] = acc[q];
  __syncthreads();
  {
    const int o = threadIdx.x, r = o >> 4, c = o & 15;
    if (r < m && c < n) {
      double s = red[o];
      for (int ww = 1; ww < NW; ++ww) s += red[ww * 256 + o];
      double* p = &C[(size_t)r * ldc + c];
      *p = beta != 0.0 ? ldcg(p) + s : s;
    }
  }
  __syncthreads();
}

// C[1 x n] (n <= 32) = beta C + alpha op(A)[1 x k] op(B)[k x n] in free order (a row vector
// times a tall skinny matrix, e.g. x^T V in a solve): thread t sums k = t, t + NT, ... into
// n partial sums, then warps and the CTA reduce them.
__device__ __noinline__ void gemv_row(double* __restrict__ C, const double* __restrict__ A, int lda, bool tA,
                                      const double* __restrict__ B, int ldb, bool tB, int n, int k, double alpha,
                                      double beta, double* smem) {
  constexpr int NC = 32;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
#pragma unroll 2
  for (int kk = threadIdx.x; kk < k; kk += NT) {
    const double a = tA ? ldcg(&A[(size_t)kk * lda]) : ldcg(&A[kk]);
#pragma unroll
    for (int c = 0; c < NC; ++c)
      if (c < n) acc[c] = fma(a, tB ? ldcg(&B[(size_t)c * ldb + kk]) : ldcg(&B[(size_t)kk * ldb + c]), acc[c]);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (c < n) {
      double v = acc[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) smem[w * NC + c] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < n) {
    double v = 0.0;
    for (int q = 0; q < NT / 32; ++q) v += smem[q * NC + threadIdx.x];
    v *= alpha;
    C[threadIdx.x] = beta != 0.0 ? ldcg(&C[threadIdx.x]) + v : v;
  }
  __syncthreads();
}

template <int NB, int RU, int TC>
__device__ __noinline__ void trmv_impl(double* O, int ldo, const double* S, int lds, const double* M, int ldm, int m,
                                       int n, int mode, int rbeg, int rows, double* smem, double alpha = 1.0,
                                       double beta = 0.0);

__device__ __forceinline__ void dev_gemm(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda, bool tA,
                         const double* __restrict__ B, int ldb, bool tB, int m, int n, int k, double alpha,
                         double beta, double* smem, bool free_order = false) {
  if (free_order && m == 1 && n <= 32 && k >= 64)
    gemv_row(C, A, lda, tA, B, ldb, tB, n, k, alpha, beta, smem);
  else if (free_order && !tA && !tB && m > 16 && n <= 16 && k >= 64 && k <= 512) {
    // rows of A times a skinny B (the solves' products): B staged in shared memory, warps take
    // rows of A with lanes along k and every load of a row batch issued first, a warp reduction
    // per row and column; no per-element ascending-k order (work and right-hand-side targets)
    if (k <= 256) {
      if (n <= 4) trmv_impl<4, 4, 8>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
      else if (n <= 8) trmv_impl<8, 2, 8>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
      else trmv_impl<16, 2, 8>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
    } else {
      if (n <= 4) trmv_impl<4, 2, 16>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
      else if (n <= 8) trmv_impl<8, 2, 16>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
      else trmv_impl<16, 1, 16>(C, ldc, B, ldb, A, lda, k, n, 2, 0, m, smem, alpha, beta);
    }
  }
  else if (free_order && m <= 16 && n <= 16 && k >= 256)
    gemm_splitk(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (m <= 16 && n <= 16) gemm_cfg<16, 16, 1, 1, 128>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (m <= 32 && n <= 32) gemm_cfg<32, 32, 2, 2, 64>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (n == 1) gemm_cfg<256, 1, 1, 1, 16>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (n <= 16) gemm_cfg<128, 16, 8, 1, 32>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (m <= 16) gemm_cfg<16, 128, 1, 8, 32>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  // tall or wide skinny products over a long k (a dense block times a low-rank factor): 10 loads
  // in flight per thread, 16 FMAs per thread and k step
  else if (n <= 32 && m >= 128) gemm_cfg<128, 32, 4, 4, 16>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (m <= 32 && n >= 128) gemm_cfg<32, 128, 4, 4, 16>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else if (m > 64 && n > 64) gemm_cfg<128, 128, 8, 8, 16>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
  else gemm_cfg<64, 64, 4, 4, 32>(C, ldc, A, lda, tA, B, ldb, tB, m, n, k, alpha, beta, smem);
}

// ------------------------------------------------------------------------- tensor-core GEMM
// Mixed-precision contraction on the 5th-generation tensor cores:
//   C[m x n] (FP64) = beta C + alpha op(A) op(B),  op(A), op(B) rounded to TF32,
//   products summed in FP32 in tensor memory (TMEM), the sum added to C in FP64.
// Tile 128 x 64 (tcgen05.mma.cta_group::1.kind::tf32, M = 128, N = 64, K = 8 per
// instruction), k in chunks of 32.  Operands are staged in shared memory in the canonical
// K-major layout without swizzle: 8-row x 16-byte core matrices, core matrices 128 B apart
// along M/N (SBO) and one k16-column of core matrices apart along K (LBO).  One thread
// issues the MMAs and commits them to an mbarrier; the CTA waits on it (bounded) before
// reusing the staging buffers or reading the accumulators with tcgen05.ld.
#define TC_M 128
#define TC_N 64
#define TC_K 32
#define TC_A_BYTES (TC_M * TC_K * 4)
#define TC_B_BYTES (TC_N * TC_K * 4)
#define TC_LBO_A (TC_M / 8 * 128)  /* bytes between k16 columns of A's core matrices */
#define TC_LBO_B (TC_N / 8 * 128)
#define TC_TMEM_COLS 512  /* all of an SM's tensor memory: the VM runs one CTA per SM */

struct TcCtx {
  uint32_t tmem;      // accumulator base address in tensor memory
  uint32_t mbar;      // shared address of the MMA-completion mbarrier
  uint32_t phase;     // parity of the next completion
  long long limit;    // nanoseconds before a wait for the tensor core gives up
  int pending;        // a commit whose completion was not observed (after a timeout)
  int active;         // tensor memory and the mbarrier were set up for this CTA
  // BF16 pipeline (dev_gemm_bf16): shared address of its 10 mbarriers, the number of stage
  // fills and accumulator tiles used so far (every thread counts the same), an abort flag in
  // shared memory, and the last stage fill / tile commit whose completion nobody waited for
  uint32_t bars;
  uint32_t q;
  uint32_t u;
  int* abort;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100; layout type 0 = no swizzle
  return d;
}

// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2), both
// K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                                ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(double v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(__double2float_rn(v)));
  return r;
}

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the completion of phase `phase` of an mbarrier: false after `limit_ns`
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase, long long limit_ns) {
  const unsigned long long t0 = gtimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
    if ((long long)(gtimer_ns() - t0) > limit_ns) return false;
  }
}

__device__ __noinline__ bool dev_gemm_tc(double* __restrict__ C, int ldc, const double* __restrict__ A, int lda,
                                         bool tA, const double* __restrict__ B, int ldb, bool tB, int m, int n, int k,
                                         double alpha, double beta, double* smem, TcCtx& tc) {
  uint8_t* sbase = reinterpret_cast<uint8_t*>(smem);
  const uint32_t s0 = smem_u32(sbase);
  const uint32_t pad = ((s0 + 1023u) & ~1023u) - s0;  // core matrices from a 1 KB boundary
  uint32_t* As = reinterpret_cast<uint32_t*>(sbase + pad);
  uint32_t* Bs = reinterpret_cast<uint32_t*>(sbase + pad + TC_A_BYTES);
  const uint32_t a_addr = s0 + pad, b_addr = s0 + pad + TC_A_BYTES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nch = (k + TC_K - 1) / TC_K;
  bool ok = true;
  for (int i0 = 0; i0 < m; i0 += TC_M)
    for (int j0 = 0; j0 < n; j0 += TC_N) {
      for (int ch = 0; ch < nch && ok; ++ch) {
        const int k0 = ch * TC_K;
        for (int e = tid; e < TC_M * TC_K; e += NT) {
          int r, kk;
          if (!tA) { r = e / TC_K; kk = e % TC_K; }
          else { kk = e / TC_M; r = e % TC_M; }
          double v = 0.0;
          if (i0 + r < m && k0 + kk < k)
            v = tA ? ldcg(&A[(size_t)(k0 + kk) * lda + i0 + r]) : ldcg(&A[(size_t)(i0 + r) * lda + k0 + kk]);
          As[((kk >> 2) * TC_LBO_A + (r >> 3) * 128 + (r & 7) * 16 + (kk & 3) * 4) >> 2] = to_tf32(v);
        }
        for (int e = tid; e < TC_N * TC_K; e += NT) {
          int c, kk;
          if (!tB) { kk = e / TC_N; c = e % TC_N; }
          else { c = e / TC_K; kk = e % TC_K; }
          double v = 0.0;
          if (j0 + c < n && k0 + kk < k)
            v = tB ? ldcg(&B[(size_t)(j0 + c) * ldb + k0 + kk]) : ldcg(&B[(size_t)(k0 + kk) * ldb + j0 + c]);
          Bs[((kk >> 2) * TC_LBO_B + (c >> 3) * 128 + (c & 7) * 16 + (kk & 3) * 4) >> 2] = to_tf32(v);
        }
        // generic-proxy smem writes become visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
          for (int ks = 0; ks < TC_K / 8; ++ks) {
            const uint64_t ad = umma_desc(a_addr + ks * 2 * TC_LBO_A, TC_LBO_A, 128);
            const uint64_t bd = umma_desc(b_addr + ks * 2 * TC_LBO_B, TC_LBO_B, 128);
            const uint32_t acc = (ch > 0 || ks > 0) ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tc.tmem),
                "l"(ad), "l"(bd), "r"(kIdescTf32), "r"(acc)
                : "memory");
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc.mbar)
                       : "memory");
        }
        // one verdict for the whole CTA, so that every thread takes the same path below
        ok = __syncthreads_and(mbar_wait(tc.mbar, tc.phase, tc.limit) ? 1 : 0) != 0;
        tc.phase ^= 1u;
        if (!ok) tc.pending = 1;
      }
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // accumulators: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), columns 32 (w / 4) .. + 31
      const int q = warp & 3, h = warp >> 2;
      const int row = i0 + 32 * q + lane;
      uint32_t v[32];
      if (nch > 0) {
        const uint32_t taddr = tc.tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * h);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] = 0u;
      }
      if (row < m) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int col = j0 + 32 * h + c;
          if (col < n) {
            double* p = &C[(size_t)row * ldc + col];
            const double s = alpha * (double)__uint_as_float(v[c]);
            *p = beta != 0.0 ? ldcg(p) + s : s;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
  return ok;
}

// ------------------------------------------------------------------------- BF16 Schur GEMM
// Operands are BF16 shadows in the tiled layout of pp_task.h (PP_OP_SHADOW writes them), so
// every 128-row x 64-column chunk of an operand moves into shared memory with ONE bulk copy of
// 16 KB (the TMA engine's untiled mode: no tensor map, no per-element work) and lands in the
// canonical no-swizzle K-major layout tcgen05.mma reads.
//
// C[m x n] (FP64) = beta C + alpha A B, tile loop over 128 x 256 sub-tiles of C, k in chunks of
// 64 through a 3-stage ring of shared-memory stages (A chunk + two B chunks = 48 KB each).
// Roles inside the CTA (warp specialised):
//   warp 0, one lane   producer: waits for a free stage, posts the expected bytes on the
//                      stage's "full" mbarrier and issues the three bulk copies;
//   warp 1, one lane   MMA issuer: per stage four K=16 steps x two 128 x 128 MMAs
//                      (kind::f16, BF16 inputs, FP32 accumulators in tensor memory), then
//                      tcgen05.commit to the stage's "empty" mbarrier; after a sub-tile's last
//                      stage, a commit to the accumulator buffer's "full" mbarrier;
//   warps 4..7         epilogue: tcgen05.ld of the accumulator buffer (warp w reads TMEM lanes
//                      32 (w % 4) ..), C += alpha acc in FP64, then an arrive on the buffer's
//                      "empty" mbarrier.
// Two accumulator buffers of 256 TMEM columns: the epilogue of one sub-tile overlaps the MMAs
// of the next, and the producer runs up to three stages ahead of the MMAs.
#define BG_STAGES 3
#define BG_CHUNK PP_SHADOW_CHUNK_BYTES
#define BG_STAGE_BYTES (3 * BG_CHUNK)
#define BG_TILE_N 256
// instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both
// K-major, M = 128 (bits 24-28 = M >> 4); N (bits 17-22 = N >> 3) is added per task
constexpr uint32_t kIdescBf16Base = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ uint32_t bf16_bits(double x) {
  // round to nearest even through FP32 (finite values; NaN stays a quiet NaN)
  uint32_t u = __float_as_uint(__double2float_rn(x));
  if ((u & 0x7F800000u) == 0x7F800000u) return (u >> 16) | ((u & 0xFFFFu) ? 0x40u : 0u);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return u >> 16;
}

// byte offset of element (r, c) of an R x K operand in the tiled layout with chunks of cr rows
// (32, 64 or 128) and 64 columns
__device__ __forceinline__ size_t tiled_at(int r, int c, int K, int cr) {
  const size_t chunk = (size_t)(r / cr) * (K >> 6) + (c >> 6);
  const int rr = r % cr, cc = c & 63;
  return chunk * ((size_t)cr * 128) + (size_t)((((cc >> 3) * (cr >> 3)) + (rr >> 3)) << 7) + ((rr & 7) << 4) +
         ((cc & 7) << 1);
}

// S := the tiled BF16 shadow of X (m x k, padded with zeros beyond the source's mr rows and nc
// columns), X(r, c) = A[r lda + c] or A[c lda + r] (tA).  Each thread converts 8 consecutive
// columns of a row and stores them as one 16-byte word, lanes along the rows (the stores of 32
// consecutive rows fill 512 contiguous bytes).  With tA the loads are coalesced as they stand
// (four words per thread at a time: 32 loads in flight); otherwise 128 x 64 blocks of X are
// staged in shared memory with coalesced loads, 32 per thread in flight, the loads of the next
// block issued before the current one is converted.  A split shadow (split = PP_SPLIT_*, k = nseg
// segments of ks columns) writes each word once per segment: bf16(x), or the residual
// bf16(x - bf16(x)) in the segments of the low mask.
__device__ __forceinline__ void shadow_word(uint8_t* S, int r, int c, int k, int ks, int cr, int split,
                                            const double* x) {
  uint32_t h[8], l[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    h[q] = bf16_bits(x[q]);
    l[q] = split ? bf16_bits(x[q] - (double)__uint_as_float(h[q] << 16)) : 0u;
  }
  uint4 vh, vl;
  vh.x = h[0] | (h[1] << 16);
  vh.y = h[2] | (h[3] << 16);
  vh.z = h[4] | (h[5] << 16);
  vh.w = h[6] | (h[7] << 16);
  if (!split) {
    *reinterpret_cast<uint4*>(S + tiled_at(r, c, k, cr)) = vh;
    return;
  }
  vl.x = l[0] | (l[1] << 16);
  vl.y = l[2] | (l[3] << 16);
  vl.z = l[4] | (l[5] << 16);
  vl.w = l[6] | (l[7] << 16);
  const int nseg = split >> 8;
  for (int sg = 0; sg < nseg; ++sg)
    *reinterpret_cast<uint4*>(S + tiled_at(r, c + sg * ks, k, cr)) = ((split >> sg) & 1) ? vl : vh;
}

__device__ __noinline__ void dev_shadow(uint8_t* S, const double* A, int lda, bool tA, int m, int k, int mr, int nc,
                                       int cr, int split, double* smem) {
  const int ks = split ? k / (split >> 8) : k;  // source columns (one segment)
  if (tA) {
    constexpr int W = 4;
    const int units = m * (ks >> 3);
    for (int u0 = threadIdx.x; u0 < units; u0 += W * NT) {
      double x[W][8];
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const int u = u0 + j * NT, r = u % m, c = (u / m) << 3;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          x[j][q] = (u < units && r < mr && c + q < nc) ? ldcg(&A[(size_t)(c + q) * lda + r]) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const int u = u0 + j * NT, r = u % m, c = (u / m) << 3;
        if (u >= units) break;
        shadow_word(S, r, c, k, ks, cr, split, x[j]);
      }
    }
  } else {
    constexpr int BR = 128, BC = 64, LD = BC + 1, PER = BR * BC / NT;
    const int nbc = ks / BC, nb = ((m + BR - 1) / BR) * nbc;
    double v[PER];
    auto fetch = [&](int b) {
      const int r0 = (b / nbc) * BR, c0 = (b % nbc) * BC;
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int e = threadIdx.x + p * NT, r = r0 + e / BC, c = c0 + e % BC;
        v[p] = (r < m && r < mr && c < nc) ? ldcg(&A[(size_t)r * lda + c]) : 0.0;
      }
    };
    fetch(0);
    for (int b = 0; b < nb; ++b) {
      const int r0 = (b / nbc) * BR, c0 = (b % nbc) * BC, rows = min(BR, m - r0);
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int e = threadIdx.x + p * NT;
        smem[(e / BC) * LD + e % BC] = v[p];
      }
      __syncthreads();
      if (b + 1 < nb) fetch(b + 1);
      for (int u = threadIdx.x; u < rows * (BC >> 3); u += NT) {
        const int rr = u % rows, cg = (u / rows) << 3;
        double x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = smem[rr * LD + cg + q];
        shadow_word(S, r0 + rr, c0 + cg, k, ks, cr, split, x);
      }
      __syncthreads();
    }
  }
  // the shadow is read by bulk copies (the async proxy) of other CTAs
  asm volatile("fence.proxy.async.global;" ::: "memory");
  __syncthreads();
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(addr) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(addr),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// bounded wait that also gives up when another role of the CTA has given up
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t addr, uint32_t phase, long long limit_ns,
                                                   volatile int* abort) {
  const unsigned long long t0 = gtimer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
    if (*abort) return false;
    if ((long long)(gtimer_ns() - t0) > limit_ns) {
      *abort = 1;
      return false;
    }
  }
}
__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void red_add_f64(double* p, double v) {
  asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// C[r][lane] = beta C + alpha T[r][lane] for the warp's 32 rows (row stride ldc), T the 32 x 32
// FP32 transpose buffer (row stride 33).  With beta = 1 and alpha = +-1 (every Schur update) the
// sum goes to the L2 as a fire-and-forget FP64 reduction: one rounding of C + alpha T, the value
// fma(alpha, T, C) gives, with no load latency on the epilogue's path.  Otherwise 32 coalesced
// loads in flight per lane, then the stores.
__device__ __noinline__ void bg_rows_update(double* __restrict__ cp, int ldc, const float* tb, int lane, double alpha,
                                            double beta) {
  if (beta == 1.0 && (alpha == 1.0 || alpha == -1.0)) {
#pragma unroll
    for (int rr = 0; rr < 32; ++rr) red_add_f64(cp + (size_t)rr * ldc, alpha * (double)tb[rr * 33 + lane]);
    return;
  }
  double cv[32];
#pragma unroll
  for (int rr = 0; rr < 32; ++rr) cv[rr] = beta != 0.0 ? __ldcg(cp + (size_t)rr * ldc) : 0.0;
#pragma unroll
  for (int rr = 0; rr < 32; ++rr) cp[(size_t)rr * ldc] = fma(alpha, (double)tb[rr * 33 + lane], beta * cv[rr]);
}

// the same for two adjacent 32-column pieces (buffers T and T + 32 x 33): 64 loads in flight
__device__ __noinline__ void bg_rows_update2(double* __restrict__ cp, int ldc, const float* tb, int lane, double alpha,
                                             double beta) {
  if (beta == 1.0 && (alpha == 1.0 || alpha == -1.0)) {
#pragma unroll
    for (int rr = 0; rr < 32; ++rr) {
      red_add_f64(cp + (size_t)rr * ldc, alpha * (double)tb[rr * 33 + lane]);
      red_add_f64(cp + (size_t)rr * ldc + 32, alpha * (double)tb[32 * 33 + rr * 33 + lane]);
    }
    return;
  }
  double cv[64];
#pragma unroll
  for (int rr = 0; rr < 32; ++rr) {
    cv[rr] = beta != 0.0 ? __ldcg(cp + (size_t)rr * ldc) : 0.0;
    cv[32 + rr] = beta != 0.0 ? __ldcg(cp + (size_t)rr * ldc + 32) : 0.0;
  }
#pragma unroll
  for (int rr = 0; rr < 32; ++rr) {
    cp[(size_t)rr * ldc] = fma(alpha, (double)tb[rr * 33 + lane], beta * cv[rr]);
    cp[(size_t)rr * ldc + 32] = fma(alpha, (double)tb[32 * 33 + rr * 33 + lane], beta * cv[32 + rr]);
  }
}

// With a second pair (As2, Bs2, inner dimension k2 > 0) the k loop runs over the chunks of both
// pairs into the same accumulator: C := beta C + alpha (A B + A2 B2), one pass over C.
__device__ __noinline__ bool dev_gemm_bf16(double* __restrict__ C, int ldc, const uint8_t* __restrict__ As,
                                           const uint8_t* __restrict__ Bs, int m, int n, int k, double alpha,
                                           double beta, double* smem, TcCtx& tc, const uint8_t* __restrict__ As2,
                                           const uint8_t* __restrict__ Bs2, int k2) {
  uint8_t* sbase = reinterpret_cast<uint8_t*>(smem);
  const uint32_t s0 = smem_u32(sbase);
  const uint32_t stage0 = (s0 + 1023u) & ~1023u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kchunks = k >> 6, kchunks2 = k2 >> 6, nch = kchunks + kchunks2;
  // tile width: 256 (two 128-column MMAs) when n is a multiple of 256, else n itself (32, 64, 128:
  // one MMA of that width reading the first n rows of one B chunk)
  const int tw = (n % BG_TILE_N == 0) ? BG_TILE_N : n, nbc = tw > 128 ? 2 : 1;
  const int tiles_n = n / tw, tiles = (m >> 7) * tiles_n;
  // B chunks of cb_rows rows (the B shadow's chunk height: 128, or n itself below 128)
  const int cb_rows = tw > 128 ? 128 : tw;
  const uint32_t b_chunk = (uint32_t)cb_rows * 128u, b_lbo = (uint32_t)cb_rows * 16u;
  const uint32_t stage_bytes = BG_CHUNK + (uint32_t)nbc * b_chunk;
  const uint32_t idesc = kIdescBf16Base | ((uint32_t)((tw > 128 ? 128 : tw) >> 3) << 17);
  volatile int* abort = tc.abort;
  if (tid == 0) *abort = 0;
  // shared memory written by earlier tasks (generic proxy) is overwritten by bulk copies
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  auto full = [&](uint32_t s) { return tc.bars + 8u * s; };
  auto empty = [&](uint32_t s) { return tc.bars + 8u * (BG_STAGES + s); };
  auto tfull = [&](uint32_t b) { return tc.bars + 8u * (2 * BG_STAGES + b); };
  auto tempty = [&](uint32_t b) { return tc.bars + 8u * (2 * BG_STAGES + 2 + b); };
  if (warp == 0) {
    if (lane == 0) {  // producer
      // the shadows were written with ordinary stores by other CTAs (acquired through the
      // dependency counters); order them before this thread's bulk copies read them
      asm volatile("fence.proxy.async.global;" ::: "memory");
      uint32_t q = tc.q;
      for (int t = 0; t < tiles && !*abort; ++t) {
        const int rb = (t / tiles_n), cb = (t % tiles_n) * nbc;
        for (int kc = 0; kc < nch; ++kc, ++q) {
          const uint32_t s = q % BG_STAGES, ph = (q / BG_STAGES) & 1u;
          if (!mbar_wait_or_abort(empty(s), ph ^ 1u, tc.limit, abort)) break;
          const uint32_t dst = stage0 + s * BG_STAGE_BYTES;
          mbar_expect_tx(full(s), stage_bytes);
          const bool first = kc < kchunks;  // chunk of the first pair, else of the second
          const uint8_t* a = first ? As : As2;
          const uint8_t* b = first ? Bs : Bs2;
          const int kcp = first ? kc : kc - kchunks, kch = first ? kchunks : kchunks2;
          bulk_g2s(dst, a + ((size_t)rb * kch + kcp) * BG_CHUNK, BG_CHUNK, full(s));
          bulk_g2s(dst + BG_CHUNK, b + ((size_t)cb * kch + kcp) * b_chunk, b_chunk, full(s));
          if (nbc == 2)
            bulk_g2s(dst + BG_CHUNK + b_chunk, b + ((size_t)(cb + 1) * kch + kcp) * b_chunk, b_chunk, full(s));
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      uint32_t q = tc.q, u = tc.u;
      for (int t = 0; t < tiles && !*abort; ++t, ++u) {
        const uint32_t b = u & 1u;
        if (!mbar_wait_or_abort(tempty(b), ((u >> 1) & 1u) ^ 1u, tc.limit, abort)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc0 = tc.tmem + b * BG_TILE_N;
        bool ok = true;
        for (int kc = 0; kc < nch; ++kc, ++q) {
          const uint32_t s = q % BG_STAGES, ph = (q / BG_STAGES) & 1u;
          if (!mbar_wait_or_abort(full(s), ph, tc.limit, abort)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a = stage0 + s * BG_STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
            const uint64_t ad = umma_desc(a + ks * 4096u, 2048u, 128u);
            tc_mma_bf16(acc0, ad, umma_desc(a + BG_CHUNK + ks * 2u * b_lbo, b_lbo, 128u), idesc, acc);
            if (nbc == 2)
              tc_mma_bf16(acc0 + 128u, ad, umma_desc(a + BG_CHUNK + b_chunk + ks * 2u * b_lbo, b_lbo, 128u), idesc,
                          acc);
          }
          tc_commit(empty(s));  // the stage is free once these MMAs have read it
        }
        if (!ok) break;
        tc_commit(tfull(b));  // the accumulator tile is complete
      }
    }
  } else if (warp >= 4) {  // epilogue
    // per warp two 32 x 32 FP32 transpose buffers (row stride 33: conflict-free both ways): the
    // warp reads its 32 accumulator rows from TMEM (a thread per row), then updates C a row at a
    // time with the lanes along the columns, so every load and store of C is coalesced; two
    // 32-column pieces at a time, so each lane has 64 loads of C in flight
    const int qd = warp & 3;
    float* tb = reinterpret_cast<float*>(sbase + (stage0 - s0) + BG_STAGES * BG_STAGE_BYTES) + qd * (2 * 32 * 33);
    uint32_t u = tc.u;
    for (int t = 0; t < tiles; ++t, ++u) {
      const uint32_t b = u & 1u;
      const bool ok = mbar_wait_or_abort(tfull(b), (u >> 1) & 1u, tc.limit, abort);
      if (__any_sync(0xffffffffu, !ok)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int i0 = (t / tiles_n) << 7, j0 = (t % tiles_n) * tw;
      double* cblk = C + (size_t)(i0 + 32 * qd) * ldc + j0 + lane;
      const int pieces = tw / 32;
#pragma unroll 1
      for (int p = 0; p < pieces; p += 2) {
        const int np = pieces - p >= 2 ? 2 : 1;
        for (int h = 0; h < np; ++h) {
          uint32_t v[32];
          const uint32_t taddr = tc.tmem + ((uint32_t)(32 * qd) << 16) + b * BG_TILE_N + 32u * (p + h);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
              "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
              : "r"(taddr)
              : "memory");
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          float* th = tb + h * (32 * 33);
#pragma unroll
          for (int c = 0; c < 32; ++c) th[lane * 33 + c] = __uint_as_float(v[c]);
        }
        __syncwarp();
        if (np == 2) bg_rows_update2(cblk + 32 * p, ldc, tb, lane, alpha, beta);
        else bg_rows_update(cblk + 32 * p, ldc, tb, lane, alpha, beta);
        __syncwarp();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty(b));
    }
  }
  __syncthreads();
  const bool ok = !*abort;
  // every thread advances the pipeline counters alike (the next BF16 task continues the phases)
  tc.q += (uint32_t)(tiles * nch);
  tc.u += (uint32_t)tiles;
  if (!ok) tc.pending = 1;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  return ok;
}

// ------------------------------------------------------------------------- tiles in smem
// rows x cols (<= TL x TL) from global (L2) into S (ld LDS); every thread issues its up to
// sixteen loads before it stores any, so a tile costs one memory latency, not sixteen
__device__ void load_tile(double* S, const double* __restrict__ G, int ld, int rows, int cols) {
  const int total = rows * cols;
  for (int e0 = 0; e0 < total; e0 += 16 * NT) {
    double v[16];
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      const int e = e0 + threadIdx.x + p * NT;
      v[p] = e < total ? ldcg(&G[(size_t)(e / cols) * ld + e % cols]) : 0.0;
    }
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      const int e = e0 + threadIdx.x + p * NT;
      if (e < total) S[(e / cols) * LDS + e % cols] = v[p];
    }
  }
}

// ------------------------------------------------------------------------- GETRF
// A[m x n] := L\U in place (m, n <= TL), like kernel.cu:104-147: step i divides the entries
// below the pivot by a_ii and applies a_rc = fma(a_ic, -l_r, a_rc) to the trailing block.
// Thread t = 16 ty + tx holds rows ty + 16 a and columns tx + 16 b (a, b < 4).  The pivot
// row and the raw pivot column of step i are published to shared memory (double buffered)
// by their owners at the end of step i - 1, so a step needs one CTA barrier; lanes tx < 4
// of each half-warp form the multipliers of the half-warp's rows (one division each) and
// share them by shuffles.  The steps run in four blocks of sixteen whose block index is a
// compile-time constant: register selection, the shrinking trailing region and most
// bounds tests then cost nothing at run time.
struct GetrfState {
  double x[4][4];
  double* prow;  // [2][TL]
  double* pcol;  // [2][TL]
  int tx, ty, lane, m;
};

template <int JB>
__device__ __forceinline__ void getrf_publish(GetrfState& S, int j, int buf) {
  const int jj = j & 15;
  if (S.ty == jj) {
#pragma unroll
    for (int b = JB; b < 4; ++b) S.prow[buf * TL + S.tx + 16 * b] = S.x[JB][b];
  }
  if (S.tx == jj) {
#pragma unroll
    for (int a = JB; a < 4; ++a) S.pcol[buf * TL + S.ty + 16 * a] = S.x[a][JB];
  }
}

template <int IB>
__device__ __forceinline__ void getrf_step(GetrfState& S, int i, int i_end, int mn) {
  const int ii = i & 15, buf = i & 1;
  __syncthreads();
  const double piv = S.prow[buf * TL + i];
  double lm = 0.0;
  if (S.tx >= IB && S.tx < 4) {
    const int r = S.ty + 16 * S.tx;
    if (r > i && r < S.m) lm = S.pcol[buf * TL + r] / piv;
  }
  double l[4], u[4];
#pragma unroll
  for (int a = IB; a < 4; ++a) l[a] = __shfl_sync(0xffffffffu, lm, (S.lane & 16) | a);
#pragma unroll
  for (int b = IB; b < 4; ++b) u[b] = S.prow[buf * TL + S.tx + 16 * b];
  const bool row_below = S.ty > ii, col_right = S.tx > ii;
#pragma unroll
  for (int a = IB; a < 4; ++a)
#pragma unroll
    for (int b = IB; b < 4; ++b) {
      const bool live = (a > IB || row_below) && (b > IB || col_right);
      if (live) S.x[a][b] = fma(u[b], -l[a], S.x[a][b]);
    }
  if (S.tx == ii) {  // column i keeps its multipliers (the L part)
#pragma unroll
    for (int a = IB; a < 4; ++a)
      if (a > IB || row_below) S.x[a][IB] = l[a];
  }
  if (i + 1 < i_end) getrf_publish<IB>(S, i + 1, buf ^ 1);
  else if constexpr (IB < 3) {
    if (i + 1 < mn) getrf_publish<IB + 1>(S, i + 1, buf ^ 1);
  }
}

template <int IB>
__device__ __forceinline__ void getrf_block(GetrfState& S, int mn) {
  const int i_end = min(mn, 16 * IB + 16);
  if (i_end == 16 * IB + 16) {
#pragma unroll
    for (int t = 0; t < 16; ++t) getrf_step<IB>(S, 16 * IB + t, i_end, mn);
  } else {
#pragma unroll 1
    for (int i = 16 * IB; i < i_end; ++i) getrf_step<IB>(S, i, i_end, mn);
  }
}

__device__ __noinline__ void dev_getrf(double* A, int lda, int m, int n, double* smem) {
  GetrfState S;
  S.prow = smem;
  S.pcol = smem + 2 * TL;
  S.tx = threadIdx.x & 15;
  S.ty = threadIdx.x >> 4;
  S.lane = threadIdx.x & 31;
  S.m = m;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = S.ty + 16 * a, c = S.tx + 16 * b;
      S.x[a][b] = (r < m && c < n) ? ldcg(&A[(size_t)r * lda + c]) : 0.0;
    }
  const int mn = min(m, n);
  if (mn > 0) getrf_publish<0>(S, 0, 0);
  getrf_block<0>(S, mn);
  getrf_block<1>(S, mn);
  getrf_block<2>(S, mn);
  getrf_block<3>(S, mn);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = S.ty + 16 * a, c = S.tx + 16 * b;
      if (r < m && c < n) A[(size_t)r * lda + c] = S.x[a][b];
    }
  __syncthreads();
}

// A[m x n] := L\U of P A with partial pivoting inside the block (m, n <= TL), P written to
// Pout (m doubles of row indices).  Step i: the row r >= i of largest |a_ri| (the first of
// equal ones; warp 0 scans, lanes take rows i + lane + 32 t in ascending order, the shuffle
// tree keeps the larger value and, on a tie, the smaller row), whole rows i and r swapped,
// then l_r = a_ri / a_ii and a_rc = fma(a_ic, -l_r, a_rc) for r, c > i — the elimination of
// the unpivoted routine, so a block that needs no swap gets the same bits.  The block lives in
// shared memory (row stride LDS) for the whole factorization.
__device__ __noinline__ void dev_getrf_piv(double* A, int lda, int m, int n, double* Pout, double* smem) {
  double* S = smem;
  int* perm = reinterpret_cast<int*>(smem + TL * LDS);
  int* pivot = perm + TL;
  load_tile(S, A, lda, m, n);
  for (int i = threadIdx.x; i < m; i += NT) perm[i] = i;
  __syncthreads();
  const int mn = min(m, n), lane = threadIdx.x & 31;
  for (int i = 0; i < mn; ++i) {
    if (threadIdx.x < 32) {
      double best = -1.0;
      int bi = i;
      for (int r = i + lane; r < m; r += 32) {
        const double v = fabs(S[r * LDS + i]);
        if (v > best) { best = v; bi = r; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
      }
      if (lane == 0) *pivot = bi;
    }
    __syncthreads();
    const int r = *pivot;
    if (r != i) {
      for (int c = threadIdx.x; c < n; c += NT) {
        const double t = S[i * LDS + c];
        S[i * LDS + c] = S[r * LDS + c];
        S[r * LDS + c] = t;
      }
      if (threadIdx.x == 0) {
        const int t = perm[i];
        perm[i] = perm[r];
        perm[r] = t;
      }
    }
    __syncthreads();
    const double d = S[i * LDS + i];
    for (int rr = i + 1 + threadIdx.x; rr < m; rr += NT) S[rr * LDS + i] = S[rr * LDS + i] / d;
    __syncthreads();
    const int w = n - i - 1;
    for (int e = threadIdx.x; e < (m - i - 1) * w; e += NT) {
      const int rr = i + 1 + e / w, c = i + 1 + e % w;
      S[rr * LDS + c] = fma(S[i * LDS + c], -S[rr * LDS + i], S[rr * LDS + c]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * n; e += NT) {
    const int rr = e / n, c = e % n;
    A[(size_t)rr * lda + c] = S[rr * LDS + c];
  }
  for (int i = threadIdx.x; i < m; i += NT) Pout[i] = (double)perm[i];
  __syncthreads();
}

// ------------------------------------------------------------------------- TRSM sweeps
// One triangular sweep over independent lines (the columns of B for TRSML / TRSMRT /
// TRSMU, the rows of B for TRSMR) against a triangle T staged in shared memory (ld LDS).
// Line q is held by R consecutive lanes of a warp: lane R cc + g holds positions g + R j
// (j < TL / R); position p of step i is eliminated as x_p = fma(-coef(i, p), x_i, x_p),
// the operand order of the reference's routines up to the commutation of the product
// (exact inside an fma).  The finished x_i reaches the line's lanes by a shuffle; no CTA
// barrier inside the sweep.  Steps run in TL / R blocks of R with a compile-time block
// index (register selection and the live range of positions resolved at compile time).
//   PIV 0: unit diagonal, x_i unchanged                     (TRSML, kernel.cu:150-182)
//   PIV 1: x_i = x_i * rd[i], rd = 1 / diagonal              (TRSMRT kernel.cu:229-285, TRSMU)
//   PIV 2: x_i = x_i / t_ii                                  (TRSMR, kernel.cu:185-226)
//   CT: coef(i, p) = T[i][p] (row i of T) when true, T[p][i] (column i) when false.
template <int R, int PIV, bool CT, bool BACK>
struct Sweep {
  static constexpr int NJ = TL / R;
  double x[NJ];
  const double* T;
  const double* rd;
  int g, src0, len;

  template <int J>
  __device__ __forceinline__ void step(int i) {
    const int ii = i - R * J;
    double v = __shfl_sync(0xffffffffu, x[J], ii, R);
    if (PIV == 1) v = v * rd[i];
    if (PIV == 2) v = v / T[i * LDS + i];
    if (PIV != 0 && g == ii) x[J] = v;
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const bool live = BACK ? (j < J || (j == J && g < ii)) : (j > J || (j == J && g > ii));
      if (live) {
        const int p = g + R * j;
        const double c = CT ? T[i * LDS + p] : T[p * LDS + i];
        x[j] = fma(-c, v, x[j]);
      }
    }
  }
  template <int J>
  __device__ __forceinline__ void block() {
    if (R * J + R <= len) {  // a whole block: steps unrolled, coefficient loads scheduled early
#pragma unroll
      for (int t = 0; t < R; ++t) step<J>(BACK ? R * J + R - 1 - t : R * J + t);
    } else {
      const int i0 = BACK ? len - 1 : R * J;
      const int i1 = BACK ? R * J - 1 : len;
#pragma unroll 1
      for (int i = i0; i != i1; i += BACK ? -1 : 1) step<J>(i);
    }
  }
  template <int J>
  __device__ __forceinline__ void run_from() {
    if constexpr (J >= 0 && J < NJ) {
      if (R * J < len) block<J>();
      run_from<BACK ? J - 1 : J + 1>();
    }
  }
  __device__ __forceinline__ void run() {
    if constexpr (BACK) run_from<NJ - 1>();
    else run_from<0>();
  }
};

// B: lines of length len (<= TL), line q at B + q * lstride, position p at + p * pstride.
// perm (shared memory, optional): position p of a line is loaded from position perm[p] (the
// row permutation of a pivoted L block); results are stored in natural order.  A line lives in
// the registers of its lanes between its loads and its stores, so the permuted load is safe in
// place.
template <int R, int PIV, bool CT, bool BACK>
__device__ __forceinline__ void tri_sweep(double* B, size_t lstride, size_t pstride, int nlines, int len,
                                          const double* T, const double* rd, const int* perm = nullptr) {
  constexpr int LPP = NT / R;  // lines per pass
  const int lane = threadIdx.x & 31, g = lane % R;
  const int q_in = (threadIdx.x / 32) * (32 / R) + lane / R;
  for (int q0 = 0; q0 < nlines; q0 += LPP) {
    if (q0 + (threadIdx.x / 32) * (32 / R) >= nlines) continue;  // warp without a live line
    const int q = q0 + q_in;
    Sweep<R, PIV, CT, BACK> S;
    S.T = T;
    S.rd = rd;
    S.g = g;
    S.src0 = 0;
    S.len = len;
#pragma unroll
    for (int j = 0; j < Sweep<R, PIV, CT, BACK>::NJ; ++j) {
      const int p = g + R * j;
      const int src = (perm && p < len) ? perm[p] : p;
      S.x[j] = (q < nlines && p < len) ? ldcg(&B[q * lstride + src * pstride]) : 0.0;
    }
    S.run();
#pragma unroll
    for (int j = 0; j < Sweep<R, PIV, CT, BACK>::NJ; ++j) {
      const int p = g + R * j;
      if (q < nlines && p < len) B[q * lstride + p * pstride] = S.x[j];
    }
  }
}

template <int PIV, bool CT, bool BACK>
__device__ __forceinline__ void tri_lines(double* B, size_t lstride, size_t pstride, int nlines, int len,
                                          const double* T, const double* rd, const int* perm = nullptr) {
  if (nlines <= 16) tri_sweep<16, PIV, CT, BACK>(B, lstride, pstride, nlines, len, T, rd, perm);
  else tri_sweep<4, PIV, CT, BACK>(B, lstride, pstride, nlines, len, T, rd, perm);
}

// B[m x n] := L^-1 B, L unit lower m x m (m <= TL); columns independent
__device__ __noinline__ void dev_trsml(double* B, int ldb, const double* L, int ldl, int m, int n, double* smem) {
  load_tile(smem, L, ldl, m, m);
  __syncthreads();
  tri_lines<0, false, false>(B, 1, (size_t)ldb, n, m, smem, nullptr);
  __syncthreads();
}

// B[m x n] := L^-1 P B (m <= TL), P the row permutation of a pivoted GETRF of L's block
// (P[i]: the row of B that row i of P B takes; m doubles holding indices)
__device__ __noinline__ void dev_trsml_piv(double* B, int ldb, const double* L, int ldl, const double* P, int m, int n,
                                           double* smem) {
  int* perm = reinterpret_cast<int*>(smem + TL * LDS);
  load_tile(smem, L, ldl, m, m);
  for (int i = threadIdx.x; i < m; i += NT) {
    const int v = (int)ldcg(&P[i]);
    perm[i] = (v >= 0 && v < m) ? v : i;  // indices come from the block's GETRF; guard anyway
  }
  __syncthreads();
  tri_lines<0, false, false>(B, 1, (size_t)ldb, n, m, smem, nullptr, perm);
  __syncthreads();
}

// V[m x n] := U^-T V, U upper m x m (m <= TL): the reference's trsmr on a transposed B
// (kernel.cu:229-285) — row i is scaled by the reciprocal of u_ii, then eliminated below
__device__ __noinline__ void dev_trsmrt(double* V, int ldv, const double* U, int ldu, int m, int n, double* smem) {
  double* rd = smem + TL * LDS;
  load_tile(smem, U, ldu, m, m);
  __syncthreads();
  if (threadIdx.x < m) rd[threadIdx.x] = 1. / smem[threadIdx.x * LDS + threadIdx.x];
  __syncthreads();
  tri_lines<1, true, false>(V, 1, (size_t)ldv, n, m, smem, rd);
  __syncthreads();
}

// B[m x n] := U^-1 B, U upper m x m (m <= TL), backward substitution (solve phase; no
// reference counterpart): x_i = b_i * (1 / u_ii), then b_r -= u_ri x_i for r < i
__device__ __noinline__ void dev_trsmu(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  double* rd = smem + TL * LDS;
  load_tile(smem, U, ldu, m, m);
  __syncthreads();
  if (threadIdx.x < m) rd[threadIdx.x] = 1. / smem[threadIdx.x * LDS + threadIdx.x];
  __syncthreads();
  tri_lines<1, false, true>(B, 1, (size_t)ldb, n, m, smem, rd);
  __syncthreads();
}

// B[m x n] := B U^-1, U upper n x n (n <= TL); rows independent
__device__ __noinline__ void dev_trsmr(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  load_tile(smem, U, ldu, n, n);
  __syncthreads();
  tri_lines<2, true, false>(B, (size_t)ldb, 1, m, n, smem, nullptr);
  __syncthreads();
}

// Triangular solves on blocks up to 4 x TL rows, inside one CTA: diagonal TL-blocks by the
// routines above, the coupling between blocks by ordered GEMMs.  Every element gets the same
// update sequence as the tiled DAG would apply (i ascending), so results are identical.
__device__ __noinline__ void dev_trsml_big(double* B, int ldb, const double* L, int ldl, int m, int n, double* smem) {
  for (int d = 0; d < m; d += TL) {
    const int md = min(TL, m - d);
    dev_trsml(B + (size_t)d * ldb, ldb, L + (size_t)d * ldl + d, ldl, md, n, smem);
    if (d + md < m)  // B_below -= L(below, d) B_d
      dev_gemm(B + (size_t)(d + md) * ldb, ldb, L + (size_t)(d + md) * ldl + d, ldl, false, B + (size_t)d * ldb, ldb,
               false, m - d - md, n, md, -1.0, 1.0, smem);
  }
}

__device__ __noinline__ void dev_trsmu_big(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  const int nb = (m + TL - 1) / TL;
  for (int bi = nb - 1; bi >= 0; --bi) {
    const int d = bi * TL, md = min(TL, m - d);
    dev_trsmu(B + (size_t)d * ldb, ldb, U + (size_t)d * ldu + d, ldu, md, n, smem);
    if (d > 0)  // B_above -= U(above, d) B_d
      dev_gemm(B, ldb, U + d, ldu, false, B + (size_t)d * ldb, ldb, false, d, n, md, -1.0, 1.0, smem);
  }
}

__device__ __noinline__ void dev_trsmr_big(double* B, int ldb, const double* U, int ldu, int m, int n, double* smem) {
  for (int d = 0; d < n; d += TL) {
    const int nd = min(TL, n - d);
    dev_trsmr(B + d, ldb, U + (size_t)d * ldu + d, ldu, m, nd, smem);
    if (d + nd < n)  // B(:, right) -= B_d U(d, right)
      dev_gemm(B + d + nd, ldb, B + d, ldb, false, U + (size_t)d * ldu + d + nd, ldu, false, m, n - d - nd, nd, -1.0,
               1.0, smem);
  }
}

__device__ __noinline__ void dev_trsmrt_big(double* V, int ldv, const double* U, int ldu, int m, int n, double* smem) {
  for (int d = 0; d < m; d += TL) {
    const int md = min(TL, m - d);
    dev_trsmrt(V + (size_t)d * ldv, ldv, U + (size_t)d * ldu + d, ldu, md, n, smem);
    if (d + md < m)  // V_below -= U(d, below)^T V_d
      dev_gemm(V + (size_t)(d + md) * ldv, ldv, U + (size_t)d * ldu + d + md, ldu, true, V + (size_t)d * ldv, ldv,
               false, m - d - md, n, md, -1.0, 1.0, smem);
  }
}

// ------------------------------------------------------------------------- TRINV / TRMV
// Explicit inverses of a factored diagonal leaf (factor phase) and their application (solve
// phase).  A solve then costs one triangular matrix-vector product per leaf, whose loads are
// all independent, instead of a substitution whose steps form a chain.

// Columns [c0, c0 + w) of L^-1 (upper = 0) or U^-1 (upper = 1), A = L\U (m x m, ld lda),
// into I (the column block, m x w, ld ldi): identity columns, then the blocked sweep on the
// sub-triangle the block needs (rows c0.. of L^-1 are the only nonzeros; rows ..c0+w of U^-1).
__device__ __noinline__ void dev_trinv(double* I, int ldi, const double* A, int lda, int m, int w, int c0, int upper,
                                       double* smem) {
  for (int e = threadIdx.x; e < m * w; e += NT) {
    const int r = e / w, j = e % w;
    I[(size_t)r * ldi + j] = r == c0 + j ? 1.0 : 0.0;
  }
  __syncthreads();
  if (!upper) dev_trsml_big(I + (size_t)c0 * ldi, ldi, A + (size_t)c0 * lda + c0, lda, m - c0, w, smem);
  else dev_trsmu_big(I, ldi, A, lda, c0 + w, w, smem);
}

// Rows [r0, r0 + rows) of M S into O (row r at O row r - r0), M (m x m, m <= 32 TC) lower
// (mode 0) or upper (mode 1) triangular or full (mode 2, then any number of rows), S (m x n);
// O := beta O + alpha (M S) (alpha 1, beta 0 for the solves' inverses).  S is staged in shared memory first (so O may be S itself);
// warp w takes RU rows at a time, lanes stride the columns, and every load of the RU rows is
// issued before the first product; a warp reduction per row and right-hand side finishes the
// dot products, so a row's result does not depend on which rows the call covers.
template <int NB, int RU, int TC>
__device__ __noinline__ void trmv_impl(double* O, int ldo, const double* S, int lds, const double* M, int ldm, int m,
                                       int n, int mode, int rbeg, int rows, double* smem, double alpha,
                                       double beta) {
  // S staged as m rows of NB values, row stride NB + 1 for NB > 1: the lanes of a warp read
  // consecutive rows, which then fall in distinct shared-memory banks
  constexpr int SB = NB > 1 ? NB + 1 : 1;
  double* Bs = smem;
  for (int e = threadIdx.x; e < m * NB; e += NT) {
    const int r = e / NB, q = e % NB;
    Bs[r * SB + q] = q < n ? ldcg(&S[(size_t)r * lds + q]) : 0.0;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rend = rbeg + rows;
  for (int r0 = rbeg + w * RU; r0 < rend; r0 += (NT / 32) * RU) {
    double v[RU][TC];
#pragma unroll
    for (int u = 0; u < RU; ++u)
#pragma unroll
      for (int t = 0; t < TC; ++t) {
        const int r = r0 + u, c = lane + 32 * t;
        const bool in = r < rend && c < m && (mode == 2 || (mode == 1 ? c >= r : c <= r));
        v[u][t] = in ? ldcg(&M[(size_t)r * ldm + c]) : 0.0;
      }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      double acc[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q) acc[q] = 0.0;
#pragma unroll
      for (int t = 0; t < TC; ++t) {
        const int c = lane + 32 * t;
        if (c < m) {
#pragma unroll
          for (int q = 0; q < NB; ++q) acc[q] = fma(v[u][t], Bs[c * SB + q], acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      }
      const int r = r0 + u;
      if (lane == 0 && r < rend) {
#pragma unroll
        for (int q = 0; q < NB; ++q)
          if (q < n) {
            double* o = &O[(size_t)(r - rbeg) * ldo + q];
            *o = beta != 0.0 ? fma(alpha, acc[q], ldcg(o)) : alpha * acc[q];
          }
      }
    }
  }
  __syncthreads();
}

// TRMV: the whole product in place (l == 0) or rows [o, o + l) of it out of place (l > 0)
__device__ __forceinline__ bool dev_trmv(const pp_task& T, double* smem) {
  const int m = T.m, n = T.n;
  if (m > PP_VM_INV || n < 1 || n > 16) return false;
  const bool part = T.l > 0;
  if (part && (T.o < 0 || T.o + T.l > m || !T.p[2])) return false;
  const double* S = part ? T.p[2] : T.p[0];
  const int lds = part ? T.ld[2] : T.ld[0], r0 = part ? T.o : 0, rows = part ? T.l : m;
  if (m <= 256) {
    if (n == 1) trmv_impl<1, 8, 8>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else if (n <= 4) trmv_impl<4, 4, 8>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else if (n <= 8) trmv_impl<8, 2, 8>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else trmv_impl<16, 2, 8>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
  } else {  // leaves of up to 512 rows: 16 columns per lane, half the rows per pass of loads
    if (n == 1) trmv_impl<1, 4, 16>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else if (n <= 4) trmv_impl<4, 2, 16>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else if (n <= 8) trmv_impl<8, 2, 16>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
    else trmv_impl<16, 1, 16>(T.p[0], T.ld[0], S, lds, T.p[1], T.ld[1], m, n, T.ctrl, r0, rows, smem);
  }
  return true;
}

// ------------------------------------------------------------------------- GEMM3 / GEMM4
// Reference association orders (kernel.cu:886-955), intermediates in task scratch.
__device__ __noinline__ void dev_gemm3(const pp_task& T, double* smem) {
  const bool tA = T.flags & PP_T(1), tB = T.flags & PP_T(2), tC = T.flags & PP_T(3);
  double* t1 = T.tmp;
  const int m = T.m, n = T.n, k = T.k, l = T.l;
  if (T.ctrl) {  // (A B) C, t1: m x l
    dev_gemm(t1, l, T.p[1], T.ld[1], tA, T.p[2], T.ld[2], tB, m, l, k, 1.0, 0.0, smem);
    dev_gemm(T.p[0], T.ld[0], t1, l, false, T.p[3], T.ld[3], tC, m, n, l, T.alpha, 1.0, smem);
  } else {       // A (B C), t1: k x n
    dev_gemm(t1, n, T.p[2], T.ld[2], tB, T.p[3], T.ld[3], tC, k, n, l, 1.0, 0.0, smem);
    dev_gemm(T.p[0], T.ld[0], T.p[1], T.ld[1], tA, t1, n, false, m, n, k, T.alpha, 1.0, smem);
  }
}

__device__ __noinline__ void dev_gemm4(const pp_task& T, double* smem) {
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
      dev_gemm(t1, l, A, la, tA, B, lb, tB, m, l, k, 1.0, 0.0, smem);
      dev_gemm(t2, o, t1, l, false, Cm, lc, tC, m, o, l, 1.0, 0.0, smem);
      dev_gemm(M, lm, t2, o, false, D, ld, tD, m, n, o, T.alpha, 1.0, smem);
      break;
    case 1:  // (A (B C)) D; t1 k x o, t2 m x o
      dev_gemm(t1, o, B, lb, tB, Cm, lc, tC, k, o, l, 1.0, 0.0, smem);
      dev_gemm(t2, o, A, la, tA, t1, o, false, m, o, k, 1.0, 0.0, smem);
      dev_gemm(M, lm, t2, o, false, D, ld, tD, m, n, o, T.alpha, 1.0, smem);
      break;
    case 2:  // A ((B C) D); t1 k x o, t2 k x n
      dev_gemm(t1, o, B, lb, tB, Cm, lc, tC, k, o, l, 1.0, 0.0, smem);
      dev_gemm(t2, n, t1, o, false, D, ld, tD, k, n, o, 1.0, 0.0, smem);
      dev_gemm(M, lm, A, la, tA, t2, n, false, m, n, k, T.alpha, 1.0, smem);
      break;
    case 3:  // A (B (C D)); t1 l x n, t2 k x n
      dev_gemm(t1, n, Cm, lc, tC, D, ld, tD, l, n, o, 1.0, 0.0, smem);
      dev_gemm(t2, n, B, lb, tB, t1, n, false, k, n, l, 1.0, 0.0, smem);
      dev_gemm(M, lm, A, la, tA, t2, n, false, m, n, k, T.alpha, 1.0, smem);
      break;
    default:  // 4: (A B) (C D); t1 m x l, t2 l x n
      dev_gemm(t1, l, A, la, tA, B, lb, tB, m, l, k, 1.0, 0.0, smem);
      dev_gemm(t2, n, Cm, lc, tC, D, ld, tD, l, n, o, 1.0, 0.0, smem);
      dev_gemm(M, lm, t1, l, false, t2, n, false, m, n, l, T.alpha, 1.0, smem);
      break;
  }
}

// ------------------------------------------------------------------------- ACCUM
// U1 V1^T := Q Q^T (U1 V1^T + alpha U2 V2^T), Q spanning (U1 V1^T + alpha U2 V2^T) R:
// the reference's randomized accumulation (kernel.cu:1255-1280) with Q from shifted
// CholeskyQR3 (three Gram passes) in place of the reference's Givens sweeps.
// m = ny, n = nx, k = k1 (target rank), l = k2; k1, k2 <= PP_VM_MAX_RANK.
//   S  = R^T [V1 V2]                      (k1 x (k1 + k2), one pass over the nx rows)
//   Y  = U1 S1^T + alpha U2 S2^T          (ny x k1, a thread per row)
//   3x: G = Y^T Y (+ shift), G = C^T C, Y := Y C^-1
//   P  = Y^T [U1 U2]                      (one pass over the ny rows)
//   V1 := V1 P1^T + alpha V2 P2^T,  U1 := Y
// Y stays in shared memory when it fits (ny k1 <= the Y capacity: a 512 x 32 sketch does),
// else in the task's global scratch.  The long reductions are warp-sliced (lanes own output
// columns, warps own row slices) and the warp partials are summed in a fixed order through
// two slots, so results are deterministic.
#define ACC_LG (PP_VM_MAX_RANK + 1)

template <int KB>
struct AccumSmem {
  // a partial slot holds a KB x 2KB output (ld 2KB); the first one also holds the Jacobi
  // workspace (Z, rotations, pairs) of the adaptive truncation
  static constexpr int SLOT0 = KB * 2 * KB, JAC = KB * ACC_LG + 3 * KB + 4;
  static constexpr int SLOT = SLOT0 > JAC ? SLOT0 : (JAC + 7) & ~7;
  static constexpr int RED = 2 * SLOT;
  static constexpr int SOFF = SLOT;            // S (then P): k1 x (k1 + k2), ld 2 KB, in the second
                                               // slot (written only after the slots are summed)
  static constexpr int G = KB * ACC_LG + KB;   // Gram / Cholesky factor + reciprocals
  static constexpr int YCAP = VM_SMEM_BYTES / 8 - RED - G;
};

// whether ACCUM keeps its ny x k1 sketch in shared memory (rows padded to k1 + 1 doubles, so
// that a thread per row reads distinct banks); otherwise it lives in the task's scratch (ld k1)
__host__ __device__ constexpr bool accum_y_on_chip(long long ny, int k1, int k2) {
  return ny * (k1 + 1) <= ((k1 <= 16 && k2 <= 16) ? AccumSmem<16>::YCAP : AccumSmem<32>::YCAP);
}

// out1 = the first b1, out2 = the next b2 columns of the a x (b1 + b2) sum of the two slots
// (each read before any is written, so out may alias the slots)
template <int KB>
__device__ __forceinline__ void accum_combine(const double* red, int a, int b1, int b2, double* out1, double* out2,
                                              int ldo) {
  constexpr int SW = 2 * KB, SL = AccumSmem<KB>::SLOT, PER = (KB * 2 * KB + NT - 1) / NT;
  const int bt = b1 + b2;
  double v[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * NT;
    v[q] = 0.0;
    if (e < a * bt) {
      const int i = e / bt, j = e % bt, col = j < b1 ? j : KB + (j - b1);
      v[q] = red[i * SW + col] + red[SL + i * SW + col];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * NT;
    if (e < a * bt) {
      const int i = e / bt, j = e % bt;
      if (j < b1) out1[i * ldo + j] = v[q];
      else out2[i * ldo + (j - b1)] = v[q];
    }
  }
  __syncthreads();
}

template <bool GLOBAL>
__device__ __forceinline__ double ld_any(const double* p) {
  if constexpr (GLOBAL) return ldcg(p);
  else return *p;
}

// out1[a x b1] = X^T W1 and out2[a x b2] = X^T W2 (shared memory, ld ldo), X: L x a,
// W*: L x b* (or stored transposed when tW*).  Warp w sums rows [w L/8, (w+1) L/8); lane j
// owns column j of W1 and of W2; row l of X reaches the lanes by shuffles (XG: X in global
// memory, read once per row by lanes i < a) or as shared-memory broadcasts.
template <int KB, bool XG, bool WG>
__device__ __noinline__ void accum_tn(const double* X, int lx, int a, const double* W1, int lw1, bool tW1, int b1,
                                      const double* W2, int lw2, bool tW2, int b2, int L, double* out1,
                                      double* out2, int ldo, double* red) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double acc1[KB], acc2[KB];
#pragma unroll
  for (int i = 0; i < KB; ++i) acc1[i] = acc2[i] = 0.0;
  const int per = (L + 7) / 8, l0 = min(L, w * per), l1 = min(L, l0 + per);
  // rows in groups of RG: every load of a group is issued before the first product, so a
  // warp waits for one memory latency per group, not per row
  constexpr int RG = 8;
  for (int lb = l0; lb < l1; lb += RG) {
    double w1[RG], w2[RG], xr[RG];
#pragma unroll
    for (int t = 0; t < RG; ++t) {
      const int l = lb + t;
      const bool in = l < l1;
      w1[t] = in && lane < b1 ? ld_any<WG>(tW1 ? &W1[(size_t)lane * lw1 + l] : &W1[(size_t)l * lw1 + lane]) : 0.0;
      w2[t] = in && lane < b2 ? ld_any<WG>(tW2 ? &W2[(size_t)lane * lw2 + l] : &W2[(size_t)l * lw2 + lane]) : 0.0;
      xr[t] = 0.0;
      if constexpr (XG) xr[t] = in && lane < a ? ldcg(&X[(size_t)l * lx + lane]) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < RG; ++t) {
      const int l = lb + t;
      if (l >= l1) break;
#pragma unroll
      for (int i = 0; i < KB; ++i) {
        if (i < a) {
          double xi;
          if constexpr (XG) xi = __shfl_sync(0xffffffffu, xr[t], i);
          else xi = X[(size_t)l * lx + i];
          acc1[i] = fma(xi, w1[t], acc1[i]);
          acc2[i] = fma(xi, w2[t], acc2[i]);
        }
      }
    }
  }
  // warp partials through two slots: warps 6, 7 store theirs, then 4, 5, then 2, 3, then 0, 1
  // add theirs; the two slots are summed last
  constexpr int SW = 2 * KB, SL = AccumSmem<KB>::SLOT;
  for (int rd = 3; rd >= 0; --rd) {
    if ((w >> 1) == rd) {
      double* slot = red + (w & 1) * SL;
#pragma unroll
      for (int i = 0; i < KB; ++i)
        if (i < a) {
          if (lane < b1) slot[i * SW + lane] = rd == 3 ? acc1[i] : acc1[i] + slot[i * SW + lane];
          if (lane < b2) slot[i * SW + KB + lane] = rd == 3 ? acc2[i] : acc2[i] + slot[i * SW + KB + lane];
        }
    }
    __syncthreads();
  }
  accum_combine<KB>(red, a, b1, b2, out1, out2, ldo);
}

// FP64 tensor-core form of accum_tn for untransposed W (the usual case): per warp, its row
// slice is the k dimension of out = X^T [W1 W2] computed with mma.sync.m8n8k4.f64 (FP64 has
// no tcgen05 kind; this is the FP64 tensor path of sm_100a).  Fragment layouts of m8n8k4.f64:
// A (8 x 4) lane l holds A[l/4][l%4]; B (4 x 8) holds B[l%4][l/4]; C (8 x 8) holds
// C[l/4][2(l%4) + {0,1}].  Rows are taken four at a time (one k step), several k steps of
// loads issued before their products.  Warp partials are combined as in accum_tn (fixed order).
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int KB, bool XG, bool WG>
__device__ __noinline__ void accum_tn_mma(const double* X, int lx, int a, const double* W1, int lw1, int b1,
                                          const double* W2, int lw2, int b2, int L, double* out1, double* out2,
                                          int ldo, double* red) {
  constexpr int MT = KB / 8, NTL = KB / 8;  // m tiles of X^T; n tiles per W
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qr = lane >> 2, qc = lane & 3;
  double c1[MT][NTL][2], c2[MT][NTL][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j) c1[i][j][0] = c1[i][j][1] = c2[i][j][0] = c2[i][j][1] = 0.0;
  const int per = (((L + 7) / 8) + 3) & ~3, l0 = min(L, w * per), l1 = min(L, l0 + per);
  constexpr int KS = KB >= 32 ? 1 : 4;  // k steps (of 4 rows) whose loads go out together
  for (int lb = l0; lb < l1; lb += 4 * KS) {
    double fa[KS][MT], f1[KS][NTL], f2[KS][NTL];
#pragma unroll
    for (int s = 0; s < KS; ++s) {
      const int l = lb + 4 * s + qc;  // the row this lane feeds (A col / B row = lane % 4)
      const bool in = l < l1;
#pragma unroll
      for (int i = 0; i < MT; ++i) {
        const int col = 8 * i + qr;
        fa[s][i] = (in && col < a) ? ld_any<XG>(&X[(size_t)l * lx + col]) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < NTL; ++j) {
        const int col = 8 * j + qr;
        f1[s][j] = (in && col < b1) ? ld_any<WG>(&W1[(size_t)l * lw1 + col]) : 0.0;
        f2[s][j] = (in && col < b2) ? ld_any<WG>(&W2[(size_t)l * lw2 + col]) : 0.0;
      }
    }
#pragma unroll
    for (int s = 0; s < KS; ++s)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NTL; ++j) {
          if (8 * j < b1) dmma(c1[i][j][0], c1[i][j][1], fa[s][i], f1[s][j]);
          if (8 * j < b2) dmma(c2[i][j][0], c2[i][j][1], fa[s][i], f2[s][j]);
        }
  }
  constexpr int SW = 2 * KB, SL = AccumSmem<KB>::SLOT;
  auto deposit = [&](int slot, bool add) {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = 8 * i + qr, c = 8 * j + 2 * qc + e;
          if (r < a && c < b1) {
            double* p = &red[slot * SL + r * SW + c];
            *p = add ? c1[i][j][e] + *p : c1[i][j][e];
          }
          if (r < a && c < b2) {
            double* p = &red[slot * SL + r * SW + KB + c];
            *p = add ? c2[i][j][e] + *p : c2[i][j][e];
          }
        }
  };
  // warps 6, 7 store, then 4, 5, then 2, 3, then 0, 1 add (two slots), then the slots are summed
  for (int rd = 3; rd >= 0; --rd) {
    if ((w >> 1) == rd) deposit(w & 1, rd != 3);
    __syncthreads();
  }
  accum_combine<KB>(red, a, b1, b2, out1, out2, ldo);
}

// out = X^T [W1 W2]: the tensor-core form when both W are untransposed, else the SIMT form
template <int KB, bool XG, bool WG>
__device__ __forceinline__ void accum_tn_any(const double* X, int lx, int a, const double* W1, int lw1, bool tW1,
                                             int b1, const double* W2, int lw2, bool tW2, int b2, int L,
                                             double* out1, double* out2, int ldo, double* red) {
  if (!tW1 && !tW2) accum_tn_mma<KB, XG, WG>(X, lx, a, W1, lw1, b1, W2, lw2, b2, L, out1, out2, ldo, red);
  else accum_tn<KB, XG, WG>(X, lx, a, W1, lw1, tW1, b1, W2, lw2, tW2, b2, L, out1, out2, ldo, red);
}

// Y[l][0..k) = A1[l] S1^T + alpha A2[l] S2^T for every row l (a thread per row), S1: k x c1,
// S2: k x c2 in shared memory (ld lds).  Y may alias A1 (each row is read before written).
template <int KB, bool A1G>
__device__ __noinline__ void accum_rows(double* Y, int ly, const double* A1, int la1, int c1, const double* A2,
                                       int la2, bool tA2, int c2, double alpha, const double* S1,
                                       const double* S2, int lds, int k, int L) {
  for (int l = threadIdx.x; l < L; l += NT) {
    double y[KB], u[KB];
#pragma unroll
    for (int j = 0; j < KB; ++j) u[j] = j < c1 ? ld_any<A1G>(&A1[(size_t)l * la1 + j]) : 0.0;
#pragma unroll
    for (int i = 0; i < KB; ++i) {
      double t = 0.0;
      if (i < k) {
#pragma unroll
        for (int j = 0; j < KB; ++j)
          if (j < c1) t = fma(u[j], S1[i * lds + j], t);
      }
      y[i] = t;
    }
#pragma unroll
    for (int j = 0; j < KB; ++j)
      u[j] = j < c2 ? ldcg(tA2 ? &A2[(size_t)j * la2 + l] : &A2[(size_t)l * la2 + j]) : 0.0;
#pragma unroll
    for (int i = 0; i < KB; ++i) {
      if (i < k) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < KB; ++j)
          if (j < c2) t = fma(u[j], S2[i * lds + j], t);
        y[i] = fma(alpha, t, y[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < KB; ++i)
      if (i < k) Y[(size_t)l * ly + i] = y[i];
  }
}

// FP64 tensor-core form of accum_rows for an untransposed A2: warp w takes 8-row tiles
// r0 = 8 (w + 8 t); Y tile (8 x k) = A1 tile S1^T + alpha A2 tile S2^T with mma.m8n8k4.f64
// (A fragments from the rows, B fragments from S in shared memory).  A warp reads all of its
// tile's rows before it stores any, so Y may alias A1.
template <int KB, bool A1G>
__device__ __noinline__ void accum_rows_mma(double* Y, int ly, const double* A1, int la1, int c1, const double* A2,
                                           int la2, int c2, double alpha, const double* S1, const double* S2,
                                           int lds, int k, int L) {
  constexpr int NTL = KB / 8, KST = KB / 4;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int qr = lane >> 2, qc = lane & 3;
  for (int r0 = 8 * w; r0 < L; r0 += 8 * (NT / 32)) {
    const int row = r0 + qr;
    const bool rin = row < L;
    double fa1[KST], fa2[KST];
#pragma unroll
    for (int s = 0; s < KST; ++s) {
      const int col = 4 * s + qc;
      fa1[s] = (rin && col < c1) ? ld_any<A1G>(&A1[(size_t)row * la1 + col]) : 0.0;
      fa2[s] = (rin && col < c2) ? ldcg(&A2[(size_t)row * la2 + col]) : 0.0;
    }
    double y1[NTL][2], y2[NTL][2];
#pragma unroll
    for (int j = 0; j < NTL; ++j) y1[j][0] = y1[j][1] = y2[j][0] = y2[j][1] = 0.0;
#pragma unroll
    for (int s = 0; s < KST; ++s) {
      const int kk = 4 * s + qc;
#pragma unroll
      for (int j = 0; j < NTL; ++j) {
        const int n = 8 * j + qr;
        if (4 * s < c1) dmma(y1[j][0], y1[j][1], fa1[s], (n < k && kk < c1) ? S1[n * lds + kk] : 0.0);
        if (4 * s < c2) dmma(y2[j][0], y2[j][1], fa2[s], (n < k && kk < c2) ? S2[n * lds + kk] : 0.0);
      }
    }
    if (rin) {
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = 8 * j + 2 * qc + e;
          if (col < k) Y[(size_t)row * ly + col] = fma(alpha, y2[j][e], y1[j][e]);
        }
    }
  }
}

// Y = A1 S1^T + alpha A2 S2^T: the tensor-core form unless A2 is stored transposed
template <int KB, bool A1G>
__device__ __forceinline__ void accum_rows_any(double* Y, int ly, const double* A1, int la1, int c1, const double* A2,
                                              int la2, bool tA2, int c2, double alpha, const double* S1,
                                              const double* S2, int lds, int k, int L) {
  if (!tA2) accum_rows_mma<KB, A1G>(Y, ly, A1, la1, c1, A2, la2, c2, alpha, S1, S2, lds, k, L);
  else accum_rows<KB, A1G>(Y, ly, A1, la1, c1, A2, la2, tA2, c2, alpha, S1, S2, lds, k, L);
}

// One CholeskyQR pass on Y (m x k, ld ly): G = Y^T Y (+ shift I), G = C^T C, Y := Y C^-1.
// A non-positive pivot marks a rank-deficient column, which is zeroed.  The Cholesky and the
// substitution are rolled loops (a few hundred instructions): this code runs once per task in
// a kernel whose other instructions evict it from the instruction cache, and fully unrolled
// forms of it (thousands of instructions, each line fetched once) ran ten times longer.
template <int KB, bool YG>
__device__ __noinline__ void accum_cholqr(double* Y, int ly, int m, int k, bool shifted, double* G, double* red) {
  double* rinv = G + KB * ACC_LG;
  accum_tn_any<KB, YG, YG>(Y, ly, k, Y, ly, false, k, nullptr, 0, false, 0, m, G, nullptr, ACC_LG, red);
  if (threadIdx.x < 32) {  // right-looking Cholesky in shared memory: row j of C over row j of G
    const int lane = threadIdx.x;
    double tr = 0.0;
    for (int j = 0; j < k; ++j) tr += G[j * ACC_LG + j];
    const double tiny = 1e-28 * tr;
    if (shifted && lane < k) {
      // shift of shifted CholeskyQR3: 11 (m k + k (k + 1)) u ||Y||_F^2, u = 2^-53
      G[lane * ACC_LG + lane] += 11.0 * ((double)m * k + (double)k * (k + 1)) * 1.1102230246251565e-16 * tr;
    }
    __syncwarp();
    for (int j = 0; j < k; ++j) {
      const double d = G[j * ACC_LG + j];
      const bool live = d > tiny;
      const double ri = live ? rsqrt(d) : 0.0;  // 1 / c_jj
      __syncwarp();
      if (lane >= j && lane < k) G[j * ACC_LG + lane] = lane == j ? d * ri : G[j * ACC_LG + lane] * ri;  // C[j][lane]
      if (lane == j) rinv[j] = ri;
      __syncwarp();
      // G[c1][lane] -= C[j][c1] C[j][lane] for j < c1 <= lane
      if (lane > j && lane < k) {
        const double cjl = G[j * ACC_LG + lane];
        for (int c1 = j + 1; c1 <= lane; ++c1)
          G[c1 * ACC_LG + lane] = fma(-G[j * ACC_LG + c1], cjl, G[c1 * ACC_LG + lane]);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // Y := Y C^-1, a thread per row (two rows at a time, two independent chains), right-looking:
  // x_j = s_j / c_jj, then s_c -= x_j c_jc for c > j (each s_c receives its updates in
  // ascending j, the order of the substitution x_j = (y_j - sum_{p<j} x_p c_pj) / c_jj); x[0]
  // is always the current column.  Positions past column k - 1 take updates from entries
  // beyond C's rows (in bounds of G and its reciprocals) but are never stored and never feed
  // a column below k.
  for (int r = threadIdx.x; r < m; r += 2 * NT) {
    const int r2 = r + NT;
    const bool two = r2 < m;
    double x[KB], z[KB];
#pragma unroll
    for (int j = 0; j < KB; ++j) {
      x[j] = j < k ? ld_any<YG>(&Y[(size_t)r * ly + j]) : 0.0;
      z[j] = (two && j < k) ? ld_any<YG>(&Y[(size_t)r2 * ly + j]) : 0.0;
    }
    for (int j = 0; j < k; ++j) {
      const double rj = rinv[j];
      const double xj = x[0] * rj, zj = z[0] * rj;
      Y[(size_t)r * ly + j] = xj;
      if (two) Y[(size_t)r2 * ly + j] = zj;
      const double* crow = G + j * ACC_LG + j;
#pragma unroll
      for (int c = 1; c < KB; ++c) {
        const double g = crow[c];
        x[c - 1] = fma(-xj, g, x[c]);
        z[c - 1] = fma(-zj, g, z[c]);
      }
      x[KB - 1] = 0.0;
      z[KB - 1] = 0.0;
    }
  }
  __syncthreads();
}

// Symmetric eigen-decomposition G = Z diag(lambda) Z^T of a k x k matrix (k <= 32, shared
// memory, ld ACC_LG) by cyclic Jacobi in round-robin order: every step rotates k/2 disjoint
// index pairs at once (every pair once per sweep).  A step is one pass of independent 2 x 2
// block updates: the thread of block (pair a, pair b) reads G's entries at rows {p_a, q_a} and
// columns {p_b, q_b}, derives both pairs' rotations itself from the diagonal blocks (read before
// any entry changes), and writes J_a^T G_ab J_b; Z's columns of pair b turn with J_b in the same
// pass.  A pair is rotated only while |g_pq| > 1e-15 max_i g_ii: above the rounding noise a
// rotation of the largest entries leaves behind (a few units in the last place of max g_ii, so
// the sweeps end), and about the precision the Gram matrix has in the first place (its entries
// are rounded to about 1e-16 of the largest); sweeps stop after one without a rotation, or after
// 12.  The rotation of a pair is the symmetric Schur decomposition of its 2 x 2 block (Golub &
// Van Loan, sym.schur2), t = tan(theta) written as 2 g_pq sgn(d) / (|d| + h), d = g_qq - g_pp,
// h = sqrt(d^2 + 4 g_pq^2): cos = r / s, sin = 2 g_pq sgn(d) / s with r = |d| + h,
// s = sqrt(r^2 + 4 g_pq^2) (one square root and one reciprocal square root).
__device__ __forceinline__ void jacobi_pair(const double* G, int k, int kk, int r, int jp, double thr, int& p, int& q,
                                            double& c, double& sn) {
  // round-robin positions of pair jp in step r: 1 + (pos - 1 + r) mod (kk - 1), the sum below
  // 2 (kk - 1); position 0 stays
  const int pos_b = kk - 1 - jp;
  int ua = jp - 1 + r, ub = pos_b - 1 + r;
  if (ua >= kk - 1) ua -= kk - 1;
  if (ub >= kk - 1) ub -= kk - 1;
  p = jp == 0 ? 0 : 1 + ua;
  q = pos_b == 0 ? 0 : 1 + ub;
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
  c = 1.0;
  sn = 0.0;
  if (q < k) {
    const double app = G[p * ACC_LG + p], aqq = G[q * ACC_LG + q], apq = G[p * ACC_LG + q];
    if (fabs(apq) > thr) {
      const double d = aqq - app, g2 = 2.0 * apq * (d >= 0.0 ? 1.0 : -1.0);
      const double h = sqrt(fma(d, d, g2 * g2)), rr = fabs(d) + h;
      const double w = rsqrt(fma(rr, rr, g2 * g2));
      c = rr * w;
      sn = g2 * w;
    }
  }
}

__device__ __noinline__ void jacobi_eig(double* G, double* Z, int k, double* flag) {
  const int kk = (k + 1) & ~1, np = kk / 2;  // an odd k gets a dummy index k that never rotates
  for (int e = threadIdx.x; e < k * k; e += NT) Z[(e / k) * ACC_LG + e % k] = (e / k == e % k) ? 1.0 : 0.0;
  // this thread's block (pair a, pair b) and, for Z, rows zi and zi + 16 of pair b
  const int ta = threadIdx.x / 16, tb = threadIdx.x % 16;
  const bool blk = ta < np && tb < np;
  for (int sweep = 0; sweep < 12; ++sweep) {
    if (threadIdx.x < 32) {
      double dm = 0.0;
      for (int i = threadIdx.x; i < k; i += 32) dm = fmax(dm, fabs(G[i * ACC_LG + i]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
      if (threadIdx.x == 0) {
        flag[0] = 0.0;  // rotations in this sweep
        flag[1] = 1e-15 * dm;
      }
    }
    __syncthreads();
    const double thr = flag[1];
    for (int r = 0; r < kk - 1; ++r) {
      int pa = 0, qa = 0, pb = 0, qb = 0;
      double ca = 1.0, sa = 0.0, cb = 1.0, sb = 0.0;
      // pair b's rotation also turns Z's rows ta, ta + 16 (every ta, also beyond np)
      if (tb < np) jacobi_pair(G, k, kk, r, tb, thr, pb, qb, cb, sb);
      if (blk) jacobi_pair(G, k, kk, r, ta, thr, pa, qa, ca, sa);
      const bool ra = sa != 0.0, rb = sb != 0.0;
      double g11 = 0.0, g12 = 0.0, g21 = 0.0, g22 = 0.0;
      const bool qa_in = qa < k, qb_in = qb < k;
      if (blk && (ra || rb)) {
        g11 = G[pa * ACC_LG + pb];
        if (qb_in) g12 = G[pa * ACC_LG + qb];
        if (qa_in) g21 = G[qa * ACC_LG + pb];
        if (qa_in && qb_in) g22 = G[qa * ACC_LG + qb];
      }
      if (ta == tb && ra) flag[0] = 1.0;
      __syncthreads();  // every entry is read before any changes
      if (blk && (ra || rb)) {
        // columns: [g11 g12; g21 g22] J_b
        const double h11 = cb * g11 - sb * g12, h12 = sb * g11 + cb * g12;
        const double h21 = cb * g21 - sb * g22, h22 = sb * g21 + cb * g22;
        // rows: J_a^T [h]
        G[pa * ACC_LG + pb] = ca * h11 - sa * h21;
        if (qb_in) G[pa * ACC_LG + qb] = ca * h12 - sa * h22;
        if (qa_in) G[qa * ACC_LG + pb] = sa * h11 + ca * h21;
        if (qa_in && qb_in) G[qa * ACC_LG + qb] = sa * h12 + ca * h22;
      }
      if (tb < np && rb && qb_in) {  // Z J_b: rows ta and ta + 16 of pair b's columns
        for (int i = ta; i < k; i += 16) {
          const double zp = Z[i * ACC_LG + pb], zq = Z[i * ACC_LG + qb];
          Z[i * ACC_LG + pb] = cb * zp - sb * zq;
          Z[i * ACC_LG + qb] = sb * zp + cb * zq;
        }
      }
      __syncthreads();
    }
    const bool done = flag[0] == 0.0;
    __syncthreads();
    if (done) break;
  }
}

// Rank decision of the adaptive accumulation: eigenvalues (the diagonal of G) sorted in
// decreasing order, rank r = #{ lambda_i > tol^2 lambda_0 } (singular values above tol times
// the largest), and S[i][j] = Z[j][perm[i]] for i < r (zero rows beyond), so that a row
// times S^T is its coordinates in the kept singular directions.  Returns r.
template <int KB>
__device__ __noinline__ int accum_truncate(const double* G, const double* Z, int k, double tol, double* S, int lds,
                                           int* perm, int rmax = PP_VM_MAX_RANK) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < k; ++i) perm[i] = i;
    for (int i = 0; i < k; ++i) {
      int best = i;
      for (int j = i + 1; j < k; ++j)
        if (G[perm[j] * ACC_LG + perm[j]] > G[perm[best] * ACC_LG + perm[best]]) best = j;
      const int t = perm[i];
      perm[i] = perm[best];
      perm[best] = t;
    }
    const double l0 = G[perm[0] * ACC_LG + perm[0]];
    int r = 0;
    if (l0 > 0.0)
      while (r < k && r < rmax && G[perm[r] * ACC_LG + perm[r]] > tol * tol * l0) ++r;
    perm[KB] = r;
  }
  __syncthreads();
  const int r = perm[KB];
  for (int e = threadIdx.x; e < KB * KB; e += NT) {
    const int i = e / KB, j = e % KB;
    S[i * lds + j] = (i < r && j < k) ? Z[j * ACC_LG + perm[i]] : 0.0;
  }
  __syncthreads();
  return r;
}

template <int KB, bool YG>
__device__ __forceinline__ void accum_impl(const pp_task& T, double* smem) {
  using SM = AccumSmem<KB>;
  const int ny = T.m, nx = T.n, k1 = T.k, k2 = T.l;
  const bool tU2 = T.flags & PP_T(2), tV2 = T.flags & PP_T(3);
  double *U1 = T.p[0], *V1 = T.p[1];
  const double *U2 = T.p[2], *V2 = T.p[3], *R = T.p[4];
  const int lu1 = T.ld[0], lv1 = T.ld[1], lu2 = T.ld[2], lv2 = T.ld[3], lr = T.ld[4];
  double* red = smem;
  double* S = red + SM::SOFF;  // k1 x 2KB: S1 | S2, later P1 | P2
  double* G = red + SM::RED;
  double* Y = YG ? T.tmp : G + SM::G;
  const int ly = YG ? k1 : k1 + 1;  // on chip: rows padded (a thread per row reads distinct banks)
  const double al = T.alpha;
  constexpr int LS = 2 * KB;
  // S1 = R^T V1, S2 = R^T V2
  accum_tn_any<KB, true, true>(R, lr, k1, V1, lv1, false, k1, V2, lv2, tV2, k2, nx, S, S + KB, LS, red);
  // Y = U1 S1^T + alpha U2 S2^T
  accum_rows_any<KB, true>(Y, ly, U1, lu1, k1, U2, lu2, tU2, k2, al, S, S + KB, LS, k1, ny);
  __syncthreads();
  accum_cholqr<KB, YG>(Y, ly, ny, k1, true, G, red);
  accum_cholqr<KB, YG>(Y, ly, ny, k1, false, G, red);
  accum_cholqr<KB, YG>(Y, ly, ny, k1, false, G, red);
  // P1 = Y^T U1, P2 = Y^T U2
  accum_tn_any<KB, YG, true>(Y, ly, k1, U1, lu1, false, k1, U2, lu2, tU2, k2, ny, S, S + KB, LS, red);
  // V1 := V1 P1^T + alpha V2 P2^T (rows read before written)
  accum_rows_any<KB, true>(V1, lv1, V1, lv1, k1, V2, lv2, tV2, k2, al, S, S + KB, LS, k1, nx);
  __syncthreads();
  if ((T.flags & PP_ADAPT_RANK) && T.beta > 0.0) {
    // adaptive rank: U1 V1^T = Y V1^T with Y orthonormal, so the singular values are those of
    // V1; rotate both factors into the eigenbasis of V1^T V1 and keep the directions whose
    // singular value exceeds beta times the largest (zero columns beyond the new rank)
    accum_tn_any<KB, true, true>(V1, lv1, k1, V1, lv1, false, k1, nullptr, 0, false, 0, nx, G, nullptr, ACC_LG, red);
    double* Z = red;
    double* cs = red + KB * ACC_LG;
    double* flag = cs + 2 * KB;
    int* pq = reinterpret_cast<int*>(flag + 2);
    jacobi_eig(G, Z, k1, flag);
    const int r = accum_truncate<KB>(G, Z, k1, T.beta, S, LS, pq);
    accum_rows_any<KB, true>(V1, lv1, V1, lv1, k1, nullptr, 0, false, 0, 1.0, S, S, LS, k1, nx);
    accum_rows_any<KB, YG>(Y, ly, Y, ly, k1, nullptr, 0, false, 0, 1.0, S, S, LS, k1, ny);
    __syncthreads();
    if (threadIdx.x == 0 && T.p[5]) T.p[5][0] = (double)r;
  }
  // U1 := Y
  for (int e = threadIdx.x; e < ny * k1; e += NT) {
    const int r = e / k1, c = e % k1;
    U1[(size_t)r * lu1 + c] = ld_any<YG>(&Y[(size_t)r * ly + c]);
  }
  __syncthreads();
}

// Y (m x k, ld k, global) := an orthonormal basis of its range by shifted CholeskyQR3, the
// range finder of the sketched low-rank update (same passes as inside ACCUM); a Y of up to the
// sketch capacity is copied to shared memory for the three passes and back
template <int KB>
__device__ __forceinline__ void orth_impl(double* Y, int m, int k, double* smem) {
  using SM = AccumSmem<KB>;
  double* red = smem;
  double* G = red + SM::RED;
  const int total = m * k, ls = k + 1;
  if ((long long)m * ls <= SM::YCAP) {
    double* Ys = G + SM::G;  // rows padded to k + 1
    for (int e0 = threadIdx.x; e0 < total; e0 += 8 * NT) {
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = e0 + q * NT < total ? ldcg(&Y[e0 + q * NT]) : 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int e = e0 + q * NT;
        if (e < total) Ys[(e / k) * ls + e % k] = v[q];
      }
    }
    __syncthreads();
    accum_cholqr<KB, false>(Ys, ls, m, k, true, G, red);
    accum_cholqr<KB, false>(Ys, ls, m, k, false, G, red);
    accum_cholqr<KB, false>(Ys, ls, m, k, false, G, red);
    for (int e = threadIdx.x; e < total; e += NT) Y[e] = Ys[(e / k) * ls + e % k];
    __syncthreads();
    return;
  }
  accum_cholqr<KB, true>(Y, k, m, k, true, G, red);
  accum_cholqr<KB, true>(Y, k, m, k, false, G, red);
  accum_cholqr<KB, true>(Y, k, m, k, false, G, red);
}

// U V^T (U: m x k orthonormal columns, V: n x k, both global) := its best rank-r form: the
// singular values are those of V; rotate both factors into the eigenbasis of V^T V (Jacobi)
// and keep the directions above tol times the largest (at most rmax), as ACCUM's adaptive form
template <int KB>
__device__ __forceinline__ void lrtrunc_impl(const pp_task& T, double* smem) {
  using SM = AccumSmem<KB>;
  constexpr int LS = 2 * KB;
  double *U = T.p[0], *V = T.p[1];
  const int lu = T.ld[0], lv = T.ld[1], m = T.m, n = T.n, k = T.k;
  double* red = smem;
  double* S = red + SM::SOFF;
  double* G = red + SM::RED;
  accum_tn_any<KB, true, true>(V, lv, k, V, lv, false, k, nullptr, 0, false, 0, n, G, nullptr, ACC_LG, red);
  double* Z = red;
  double* cs = red + KB * ACC_LG;
  double* flag = cs + 2 * KB;
  int* pq = reinterpret_cast<int*>(flag + 2);
  jacobi_eig(G, Z, k, flag);
  const int r = accum_truncate<KB>(G, Z, k, T.beta, S, LS, pq, T.o > 0 ? T.o : k);
  accum_rows_any<KB, true>(V, lv, V, lv, k, nullptr, 0, false, 0, 1.0, S, S, LS, k, n);
  accum_rows_any<KB, true>(U, lu, U, lu, k, nullptr, 0, false, 0, 1.0, S, S, LS, k, m);
  __syncthreads();
  if (threadIdx.x == 0 && T.p[5]) T.p[5][0] = (double)r;
  __syncthreads();
}

__device__ __noinline__ void dev_lrtrunc(const pp_task& T, double* smem) {
  if (T.k <= 16) lrtrunc_impl<16>(T, smem);
  else lrtrunc_impl<32>(T, smem);
}

__device__ __noinline__ void dev_kmul(const pp_task& T, double* smem);

__device__ __noinline__ void dev_orth(double* Y, int m, int k, double* smem) {
  if (k <= 16) orth_impl<16>(Y, m, k, smem);
  else orth_impl<32>(Y, m, k, smem);
}

// C[m x n] := A[m x n]
__device__ __noinline__ void dev_copy(double* C, int ldc, const double* A, int lda, int m, int n) {
  for (int e = threadIdx.x; e < m * n; e += NT) {
    const int r = e / n, c = e % n;
    C[(size_t)r * ldc + c] = ldcg(&A[(size_t)r * lda + c]);
  }
  __syncthreads();
}

__device__ __noinline__ void dev_accum(const pp_task& T, double* smem) {
  const int ny = T.m, k1 = T.k, k2 = T.l;
  const bool on_chip = accum_y_on_chip(ny, k1, k2);
  if (k1 <= 16 && k2 <= 16) {
    if (on_chip) accum_impl<16, false>(T, smem);
    else accum_impl<16, true>(T, smem);
  } else {
    if (on_chip) accum_impl<32, false>(T, smem);
    else accum_impl<32, true>(T, smem);
  }
}

// C[m x n] := beta C + sum_p T_p (p ascending), T_p the p-th m x n block of T
__device__ __noinline__ void dev_sum(double* C, int ldc, const double* T, int ldt, int m, int n, int parts,
                                     double beta) {
  for (int e = threadIdx.x; e < m * n; e += NT) {
    const int r = e / n, c = e % n;
    double s = 0.0;
    for (int p = 0; p < parts; ++p) s += ldcg(&T[(size_t)(p * m + r) * ldt + c]);
    double* q = &C[(size_t)r * ldc + c];
    *q = beta != 0.0 ? ldcg(q) + s : s;
  }
  __syncthreads();
}

__device__ bool run_task(const pp_task& T, double* smem, TcCtx& tc, int& err) {
  switch (T.op) {
    case PP_OP_NOP: return true;
    case PP_OP_GETRF:
      if (T.m > TL || T.n > TL) return false;
      if (T.flags & PP_PIVOT) {
        if (!T.p[1]) return false;
        dev_getrf_piv(T.p[0], T.ld[0], T.m, T.n, T.p[1], smem);
      } else {
        dev_getrf(T.p[0], T.ld[0], T.m, T.n, smem);
      }
      return true;
    case PP_OP_TRSML:
      if (T.flags & PP_PIVOT) {  // one pivoted block per instruction
        if (T.m > TL || !T.p[2]) return false;
        dev_trsml_piv(T.p[0], T.ld[0], T.p[1], T.ld[1], T.p[2], T.m, T.n, smem);
        return true;
      }
      if (T.m > PP_VM_TRI) return false;
      if (T.m > TL) dev_trsml_big(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      else dev_trsml(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMR:
      if (T.n > PP_VM_TRI) return false;
      if (T.n > TL) dev_trsmr_big(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      else dev_trsmr(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMRT:
      if (T.m > PP_VM_TRI) return false;
      if (T.m > TL) dev_trsmrt_big(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      else dev_trsmrt(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_TRSMU:
      if (T.m > PP_VM_TRI) return false;
      if (T.m > TL) dev_trsmu_big(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      else dev_trsmu(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, smem);
      return true;
    case PP_OP_GEMM:
      if (T.prec == PP_PREC_BF16) {
        if (!tc.active || T.m < 128 || T.m % 128 || T.k < 64 || T.k % 64 || T.l < 0 || T.l % 64 ||
            (T.l > 0 && (!T.p[3] || !T.p[4])) ||
            !(T.n == 32 || T.n == 64 || T.n == 128 || (T.n >= BG_TILE_N && T.n % BG_TILE_N == 0)))
          return false;
        if (!dev_gemm_bf16(T.p[0], T.ld[0], reinterpret_cast<const uint8_t*>(T.p[1]),
                           reinterpret_cast<const uint8_t*>(T.p[2]), T.m, T.n, T.k, T.alpha, T.beta, smem, tc,
                           reinterpret_cast<const uint8_t*>(T.p[3]), reinterpret_cast<const uint8_t*>(T.p[4]), T.l))
          err = PP_VM_MMA_TIMEOUT;
        return true;
      }
      if (T.prec == PP_PREC_TF32) {
        if (!tc.active) return false;  // launched without tensor memory
        if (!dev_gemm_tc(T.p[0], T.ld[0], T.p[1], T.ld[1], T.flags & PP_T(1), T.p[2], T.ld[2], T.flags & PP_T(2),
                         T.m, T.n, T.k, T.alpha, T.beta, smem, tc))
          err = PP_VM_MMA_TIMEOUT;
        return true;
      }
      dev_gemm(T.p[0], T.ld[0], T.p[1], T.ld[1], T.flags & PP_T(1), T.p[2], T.ld[2], T.flags & PP_T(2), T.m, T.n,
               T.k, T.alpha, T.beta, smem, (T.flags & PP_FREE_ORDER) != 0);
      return true;
    case PP_OP_GEMM3: dev_gemm3(T, smem); return true;
    case PP_OP_GEMM4: dev_gemm4(T, smem); return true;
    case PP_OP_ACCUM:
      if (T.k > PP_VM_MAX_RANK || T.k < 1 || T.l > PP_VM_MAX_RANK || T.l < 0) return false;
      dev_accum(T, smem);
      return true;
    case PP_OP_SUM:
      dev_sum(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, T.k, T.beta);
      return true;
    case PP_OP_TRINV:
      if (T.m > PP_VM_INV || T.n < 1 || T.o < 0 || T.o + T.n > T.m) return false;
      dev_trinv(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n, T.o, T.ctrl, smem);
      return true;
    case PP_OP_TRMV: return dev_trmv(T, smem);
    case PP_OP_ORTH:
      if (T.n < 1 || T.n > PP_VM_MAX_RANK || T.ld[0] != T.n) return false;
      dev_orth(T.p[0], T.m, T.n, smem);
      return true;
    case PP_OP_COPY:
      dev_copy(T.p[0], T.ld[0], T.p[1], T.ld[1], T.m, T.n);
      return true;
    case PP_OP_KMUL:
      if (T.k < 1 || T.k > PP_VM_MAX_RANK || T.l < 1 || T.l > 3 || T.ctrl < 0 || T.ctrl > 3 || T.m < 0 || T.n < 0)
        return false;
      dev_kmul(T, smem);
      return true;
    case PP_OP_LRTRUNC:
      if (T.k < 1 || T.k > PP_VM_MAX_RANK || T.m < T.k || T.n < T.k) return false;
      dev_lrtrunc(T, smem);
      return true;
    case PP_OP_SHADOW:
      if (T.m < 32 || T.k < 64 || T.k % 64) return false;
      if (T.l < 0 || T.l > T.m || T.n < 0 || T.n > T.k) return false;
      if (!(T.ctrl == 0 || T.ctrl == 32 || T.ctrl == 64 || T.ctrl == 128) || T.m % (T.ctrl ? T.ctrl : 128)) return false;
      if (T.o != 0 && (T.o >> 8 != 3 || (T.o & ~0x7FF) || T.k % (64 * 3) || T.n > T.k / 3)) return false;
      dev_shadow(reinterpret_cast<uint8_t*>(T.p[0]), T.p[1], T.ld[1], T.flags & PP_T(1), T.m, T.k,
                 T.l > 0 ? T.l : T.m, T.n > 0 ? T.n : (T.o ? T.k / 3 : T.k), T.ctrl ? T.ctrl : 128, T.o, smem);
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

__device__ __forceinline__ unsigned long long globaltimer_ns() { return gtimer_ns(); }
__device__ __forceinline__ unsigned smid() {
  unsigned s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return s;
}

__global__ void __launch_bounds__(NT, 1)
    vm_kernel(const pp_task* __restrict__ tasks, int n_tasks, const int32_t* __restrict__ succ, int32_t* counters,
              int32_t* slots, pp_vm_state* st, long long wait_ns, unsigned long long* trace, int use_tc) {
  extern __shared__ double smem[];
  __shared__ __align__(16) pp_task s_task;
  __shared__ int s_id;
  __shared__ int s_keep;  // position (in the successor list) of the successor run next
  __shared__ unsigned long long s_t0;
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) unsigned long long s_mbar;
  __shared__ __align__(8) unsigned long long s_bg[2 * BG_STAGES + 4];  // BF16 pipeline mbarriers
  __shared__ int s_abort;
  TcCtx tc{0u, 0u, 0u, wait_ns, 0, 0, 0u, 0u, 0u, &s_abort};
  if (use_tc) {
    // TF32 tasks: 64 TMEM columns (128 lanes x 64 FP32 accumulators) and one mbarrier per CTA
    if ((threadIdx.x >> 5) == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                   "r"(TC_TMEM_COLS)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar)) : "memory");
      // BF16 pipeline: stage full / empty (one arrival each: the producer's expect_tx, the MMA
      // issuer's commit), accumulator full (a commit) / empty (one arrival per epilogue warp)
      for (int i = 0; i < 2 * BG_STAGES + 2; ++i) mbar_init(smem_u32(&s_bg[i]), 1);
      for (int i = 2 * BG_STAGES + 2; i < 2 * BG_STAGES + 4; ++i) mbar_init(smem_u32(&s_bg[i]), 4);
      s_abort = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tc.tmem = s_tmem;
    tc.mbar = smem_u32(&s_mbar);
    tc.bars = smem_u32(&s_bg[0]);
    tc.active = 1;
  }
  // Continuation: of the successors this CTA's task makes ready, the first in the
  // successor list (sorted by the host, longest remaining path first) is run next by the
  // same CTA without a round trip through the queue; the others are pushed.  Queue slots
  // therefore number fewer than tasks, so a CTA waiting on a slot also leaves once every
  // task is done.
  int next = -1;
  for (;;) {
    if (threadIdx.x == 0) {
      int id = next;
      if (id < 0) {
        const int idx = atomicAdd(&st->head, 1);
        if (idx < n_tasks) {
          const unsigned long long t_wait = gtimer_ns();
          for (;;) {
            id = ld_acquire(&slots[idx]);
            if (id >= 0) break;
            if (ld_relaxed(&st->error) || ld_relaxed(&st->done) >= n_tasks) { id = -1; break; }
            // the wait is bounded in time (globaltimer), not in polls: a poll's cost varies
            // with the load on L2 and with other grids sharing the SMs
            if ((long long)(gtimer_ns() - t_wait) > wait_ns) {
              if (atomicCAS(&st->error, 0, PP_VM_TIMEOUT) == 0) st->err_info = idx;
              id = -1;
              break;
            }
            __nanosleep(32);
          }
        }
      }
      s_id = id;
      if (trace) s_t0 = globaltimer_ns();
    }
    __syncthreads();
    const int id = s_id;
    if (id < 0) break;
    if (threadIdx.x < (int)(sizeof(pp_task) / 8))
      reinterpret_cast<unsigned long long*>(&s_task)[threadIdx.x] =
          __ldg(reinterpret_cast<const unsigned long long*>(&tasks[id]) + threadIdx.x);
    if (threadIdx.x == 0) s_keep = NT;
    __syncthreads();
    int err = PP_VM_OK;
    const bool ok = run_task(s_task, smem, tc, err);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      if (!ok && atomicCAS(&st->error, 0, PP_VM_BAD_TASK) == 0) st->err_info = id;
      if (err != PP_VM_OK && atomicCAS(&st->error, 0, err) == 0) st->err_info = id;
      if (trace) {
        trace[3 * (size_t)id] = s_t0;
        trace[3 * (size_t)id + 1] = globaltimer_ns();
        trace[3 * (size_t)id + 2] = smid() | ((unsigned long long)blockIdx.x << 32);
      }
    }
    // successors are released in parallel, one thread each (a serial loop costs one L2
    // round trip per successor on the critical path)
    const int nsucc = s_task.n_succ, sbeg = s_task.succ_begin;
    int mine = -1;
    for (int q = threadIdx.x; q < nsucc; q += NT) {
      const int sq = succ[sbeg + q];
      if (atom_add_acq_rel(&counters[sq], -1) == 1) {
        if (q < NT) {
          mine = sq;
          atomicMin(&s_keep, q);
        } else {
          st_release(&slots[atomicAdd(&st->tail, 1)], sq);
        }
      }
    }
    __syncthreads();
    const int keep = s_keep;
    if (mine >= 0 && (int)threadIdx.x != keep) st_release(&slots[atomicAdd(&st->tail, 1)], mine);
    if (threadIdx.x == 0) {
      next = keep < NT ? succ[sbeg + keep] : -1;
      atomicAdd(&st->done, 1);
    }
  }
  if (use_tc) {
    // an MMA group whose completion was never observed still owns the accumulators:
    // give it one more bounded wait before the columns are returned
    if (tc.pending) {
      mbar_wait(tc.mbar, tc.phase ^ 1u, tc.limit);
      // a BF16 task that gave up may still have bulk copies and MMAs in flight: they finish
      // within microseconds; give them a bounded 2 ms before the columns are returned
      const unsigned long long t0 = gtimer_ns();
      while (gtimer_ns() - t0 < 2000000ull) __nanosleep(1000);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tc.tmem), "r"(TC_TMEM_COLS)
                   : "memory");
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

// Estimates from the special-function unit: PTX rsqrt.approx.ftz.f64 / rcp.approx.ftz.f64
// (computed from the upper word of the double, about single-precision accuracy, full double
// exponent range; zero gives infinity).
__device__ __forceinline__ double rsqrt_est(double v) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
  return y;
}
__device__ __forceinline__ double rcp_est(double v) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
  return y;
}
// One third-order correction of an estimate y0 of 1/a: with e = 1 - a y0,
// 1/a = y0 (1 - e)^-1 = y0 (1 + e + e^2 + O(e^3)) (geometric series).  For |e| < 2^-19 the
// truncated terms are below 2^-57 relative: the result is within a few ulps of double, the
// accuracy of two Newton steps at 3 instead of 4 operations.
__device__ __forceinline__ double rcp_refine(double a, double y0) {
  const double e = fma(-a, y0, 1.0);
  return fma(y0, fma(e, e, e), y0);
}
// Entry K(d) of the kernel matrix at squared distance d2.  The distance: y0 estimates
// 1 / sqrt(max(d2, 1e-300)), s0 = d2 y0 and e = 1 - s0 y0 = 1 - d2 y0^2; then
// sqrt(d2) = s0 (1 - e)^(-1/2) = s0 (1 + e/2 + 3e^2/8 + O(e^3)) (binomial series, truncated
// terms below 2^-58 relative for |e| < 2^-19).  Exact zero on the diagonal and for coincident
// points, an absolute error below 1e-150 for 0 < d2 < 1e-300, a few ulps elsewhere.
template <int KIND>
__device__ __forceinline__ double kernel_eval_nr(double d2, double p0, double inv_p0) {
  constexpr double c = KIND == 1 ? 4.0 * 3.14159265358979323846 : 1.0;
  const double y0 = rsqrt_est(fmax(d2, 1e-300));
  const double s0 = d2 * y0;
  const double e = fma(-s0, y0, 1.0);
  const double d = fma(s0 * e, fma(0.375, e, 0.5), s0);
  if (KIND <= 1) {
    const double x = c * (d + p0);
    return rcp_refine(x, rcp_est(x));
  }
  if (KIND == 2) return exp(-d * inv_p0);
  const double s = 1.7320508075688772 * d * inv_p0;
  return (1.0 + s) * exp(-s);
}

// The same entry evaluated in FP32 with the hardware's approximate reciprocal square root,
// exponential and division: relative error of a few 1e-7 (the exponential's argument is
// rounded to FP32, so for the exp / Matern kernels the error grows like |argument| * 6e-8).
// Used only by the low-precision products of the Krylov steps, never by a residual that
// certifies a result.
template <int KIND>
__device__ __forceinline__ float kernel_eval_f32(float d2, float p0, float inv_p0) {
  const float d = d2 * rsqrtf(fmaxf(d2, 1e-30f));
  if (KIND <= 1) {
    constexpr float c = KIND == 1 ? 12.566370614359172f : 1.0f;
    return __fdividef(1.0f, c * (d + p0));
  }
  if (KIND == 2) return __expf(-d * inv_p0);
  const float sv = 1.7320508f * d * inv_p0;
  return (1.0f + sv) * __expf(-sv);
}

// C[m x k] = K(P_I, P_J) B (PP_OP_KMUL): a thread per row of C, the columns j of the kernel
// matrix in chunks of KM_JC whose points and B rows are staged in shared memory (read by all
// threads as broadcasts); points padded to three coordinates with zeros
#define KM_JC 128
template <int KIND>
__device__ __noinline__ void kmul_impl(const pp_task& T, double* smem) {
  const int m = T.m, n = T.n, k = T.k, dim = T.l;
  const double p0 = T.alpha, inv_p0 = KIND >= 2 ? 1.0 / p0 : 0.0;
  double* C = T.p[0];
  const double *PI = T.p[1], *PJ = T.p[2], *B = T.p[3];
  const int ldc = T.ld[0], ldi = T.ld[1], ldj = T.ld[2], ldb = T.ld[3];
  double* sp = smem;               // KM_JC x 3
  double* sb = smem + KM_JC * 3;   // KM_JC x PP_VM_MAX_RANK
  for (int r0 = 0; r0 < m; r0 += NT) {
    const int r = r0 + threadIdx.x;
    double pr[3] = {0.0, 0.0, 0.0};
    if (r < m)
      for (int d = 0; d < dim; ++d) pr[d] = ldcg(&PI[(size_t)r * ldi + d]);
    double acc[PP_VM_MAX_RANK];
#pragma unroll
    for (int c = 0; c < PP_VM_MAX_RANK; ++c) acc[c] = 0.0;
    for (int j0 = 0; j0 < n; j0 += KM_JC) {
      const int jc = min(KM_JC, n - j0);
      __syncthreads();
      for (int e = threadIdx.x; e < KM_JC * 3; e += NT) {
        const int j = e / 3, d = e % 3;
        sp[e] = (j < jc && d < dim) ? ldcg(&PJ[(size_t)(j0 + j) * ldj + d]) : 0.0;
      }
      for (int e = threadIdx.x; e < jc * PP_VM_MAX_RANK; e += NT) {
        const int j = e / PP_VM_MAX_RANK, c = e % PP_VM_MAX_RANK;
        sb[e] = c < k ? ldcg(&B[(size_t)(j0 + j) * ldb + c]) : 0.0;
      }
      __syncthreads();
      for (int j = 0; j < jc; ++j) {
        const double u0 = pr[0] - sp[3 * j], u1 = pr[1] - sp[3 * j + 1], u2 = pr[2] - sp[3 * j + 2];
        const double d2 = fma(u2, u2, fma(u1, u1, u0 * u0));
        const double a = kernel_eval_nr<KIND>(d2, p0, inv_p0);
#pragma unroll
        for (int c = 0; c < PP_VM_MAX_RANK; ++c) acc[c] = fma(a, sb[j * PP_VM_MAX_RANK + c], acc[c]);
      }
    }
    if (r < m)
      for (int c = 0; c < k; ++c) C[(size_t)r * ldc + c] = acc[c];
  }
  __syncthreads();
}

__device__ __noinline__ void dev_kmul(const pp_task& T, double* smem) {
  switch (T.ctrl) {
    case 0: kmul_impl<0>(T, smem); break;
    case 1: kmul_impl<1>(T, smem); break;
    case 2: kmul_impl<2>(T, smem); break;
    default: kmul_impl<3>(T, smem); break;
  }
}

#define KR_THREADS 128
#define KR_RPT 2                      /* rows per thread */
#define KR_ROWS (KR_THREADS * KR_RPT)  /* rows per CTA */
#define KR_COLS 256
#define KR_SEG 128   /* columns per partial sum (small: enough CTAs to fill the SMs) */
// matrix-free partial products of r = b - A x, A_ij = K(|p_i - p_j|) (+ shift on i == j):
// CTA (row block, column segment) sums its KR_SEG columns (points and x staged through smem
// in KR_COLS tiles; each thread carries KR_RPT rows, so every staged column feeds
// independent chains) into part[seg][i]; residual_reduce adds the segments in order.  The
// kernel, the dimension and the right-hand-side count are compile-time parameters.
template <int KIND, int DIM, int NR>
__global__ void __launch_bounds__(KR_THREADS) kernel_residual_part(double p0, double shift,
                                                                   const double* __restrict__ pts, int n,
                                                                   const double* __restrict__ x,
                                                                   double* __restrict__ part, int nrhs) {
  __shared__ double sp[KR_COLS * DIM];
  __shared__ double sx[KR_COLS * NR];
  const int seg = blockIdx.y, jb = seg * KR_SEG, je = min(n, jb + KR_SEG);
  const double inv_p0 = 1.0 / p0;
  int row[KR_RPT];
  double pi[KR_RPT][DIM];
  double acc[KR_RPT][NR];
#pragma unroll
  for (int t = 0; t < KR_RPT; ++t) {
    row[t] = blockIdx.x * KR_ROWS + t * KR_THREADS + threadIdx.x;
    const int i = min(row[t], n - 1);
#pragma unroll
    for (int d = 0; d < DIM; ++d) pi[t][d] = pts[(size_t)i * DIM + d];
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[t][q] = 0.0;
  }
  for (int j0 = jb; j0 < je; j0 += KR_COLS) {
    const int nj = min(KR_COLS, je - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < nj * DIM; e += KR_THREADS) sp[e] = pts[(size_t)j0 * DIM + e];
    for (int e = threadIdx.x; e < nj * NR; e += KR_THREADS) {
      const int jj = e / NR, q = e % NR;
      sx[e] = q < nrhs ? x[(size_t)(j0 + jj) * nrhs + q] : 0.0;
    }
    __syncthreads();
#pragma unroll 2
    for (int j = 0; j < nj; ++j) {
      double pj[DIM];
#pragma unroll
      for (int d = 0; d < DIM; ++d) pj[d] = sp[j * DIM + d];
#pragma unroll
      for (int t = 0; t < KR_RPT; ++t) {
        double d2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const double u = pi[t][d] - pj[d];
          d2 = fma(u, u, d2);
        }
        double a = kernel_eval_nr<KIND>(d2, p0, inv_p0);
        if (j0 + j == row[t]) a += shift;
#pragma unroll
        for (int q = 0; q < NR; ++q) acc[t][q] = fma(a, sx[j * NR + q], acc[t][q]);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < KR_RPT; ++t)
    if (row[t] < n)
      for (int q = 0; q < nrhs; ++q) part[((size_t)seg * n + row[t]) * nrhs + q] = acc[t][q];
}

// Jobs of one batched residual launch, passed by value (kernel parameter space): job j owns
// the launch's work items [first, next job's first) — tile pairs of the residual kernel,
// elements of the update and reduction kernels.
#define KR_LAUNCH_JOBS 64
struct ResidLaunch {
  struct Job {
    const double* pts;
    double* x;
    const double* dx;
    const double* b;
    double* r;
    double* part;
    double p0, shift;
    long long first;
    int n, nrhs, T, pad;
  } job[KR_LAUNCH_JOBS];
  int njobs;
};

// the job that owns work item `key` (the last job whose first <= key)
__device__ __forceinline__ int resid_job_of(const ResidLaunch& L, long long key) {
  int lo = 0, hi = L.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.job[mid].first <= key) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// KR_SEG steps of one warp over a tile pair: lane l takes column (l + s) mod KR_SEG at step s.
// COL: also accumulate a_ij x_i into the warp's column sums (off-diagonal tiles); EDGE: skip
// columns at or past jn (the caller skips rows past n).  DUP: the tile's points, x and column
// sums are stored twice over (2 KR_SEG entries), so the column is addressed as l + s without
// the wrap-around; column c's sums are then split between entries c and c + KR_SEG.
template <int KIND, int DIM, int NR, bool COL, bool EDGE, bool DUP>
__device__ __forceinline__ void residual_steps(const double* sp, const double* sx, double* colw, const double (&pi)[DIM],
                                               const double (&xi)[NR], double (&acc)[NR], int lane, int jn, double p0,
                                               double inv_p0) {
#pragma unroll 4
  for (int st = 0; st < KR_SEG; ++st) {
    const int jj = DUP ? lane + st : (lane + st) & (KR_SEG - 1);
    // past the ragged edge the entry is masked, not skipped: a lane that skipped steps could
    // run ahead of the others into a column another lane is still updating.  For the same
    // reason each step's column-sum updates end with a warp barrier: seen from one thread the
    // next step's column is another address, so without it the compiler may load it before
    // the neighbouring lane has stored its update there
    const bool live = !EDGE || ((lane + st) & (KR_SEG - 1)) < jn;
    double d2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double u = pi[d] - sp[jj * DIM + d];
      d2 = fma(u, u, d2);
    }
    const double ak = kernel_eval_nr<KIND>(d2, p0, inv_p0);
    const double a = live ? ak : 0.0;
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = fma(a, sx[jj * NR + q], acc[q]);
    if (COL) {
#pragma unroll
      for (int q = 0; q < NR; ++q) colw[jj * NR + q] = fma(a, xi[q], colw[jj * NR + q]);
      __syncwarp();
    }
  }
}

// residual_steps with the entries evaluated in FP32 from FP32 copies of the points (spf, pif);
// the products are still accumulated in FP64.  The skewed walk keeps the lanes of a warp on
// distinct columns only while they take their steps together: columns past the ragged edge are
// masked (entry 0) instead of skipped, and the column sums' read-modify-writes of one step end
// with a warp barrier, so no lane can run a step ahead of another into the same column.
template <int KIND, int DIM, int NR, bool COL, bool EDGE, bool DUP>
__device__ __forceinline__ void residual_steps_lowp(const float* spf, const double* sx, double* colw,
                                                    const float (&pif)[DIM], const double (&xi)[NR], double (&acc)[NR],
                                                    int lane, int jn, float p0, float inv_p0) {
#pragma unroll 4
  for (int st = 0; st < KR_SEG; ++st) {
    const int jj = DUP ? lane + st : (lane + st) & (KR_SEG - 1);
    const bool live = !EDGE || ((lane + st) & (KR_SEG - 1)) < jn;
    float d2 = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const float u = pif[d] - spf[jj * DIM + d];
      d2 = fmaf(u, u, d2);
    }
    const float a32 = kernel_eval_f32<KIND>(d2, p0, inv_p0);
    const double a = live ? (double)a32 : 0.0;
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = fma(a, sx[jj * NR + q], acc[q]);
    if (COL) {
#pragma unroll
      for (int q = 0; q < NR; ++q) colw[jj * NR + q] = fma(a, xi[q], colw[jj * NR + q]);
      __syncwarp();
    }
  }
}

// Symmetric form of the partial products (kernel matrices are symmetric): a CTA takes the
// tile pair (I, J), I <= J, of KR_SEG x KR_SEG tiles of one job and evaluates each entry once.
// Thread t owns row I*KR_SEG + t: a_ij x_j goes to its register sums (part[J][i]); for I < J,
// a_ij x_i goes to the column sums of row j (part[I][j]) through per-warp accumulators in
// shared memory, walked on a skewed diagonal (lane l visits column (l + s) mod KR_SEG at step
// s, so the lanes of a warp never touch the same column) and added in warp order at the end.
// Every (segment, row) partial is written once, by one CTA: deterministic, no atomics, and the
// same bits whatever the other jobs of the launch.
// LOWP: entries evaluated in FP32 (residual_steps_lowp), for the Krylov steps' products.
template <int KIND, int DIM, int NR, bool LOWP>
__global__ void __launch_bounds__(KR_SEG) kernel_residual_sym(const __grid_constant__ ResidLaunch L) {
  constexpr int W = KR_SEG / 32;
  constexpr bool DUP = NR == 1;             // one RHS: tile stored twice over (residual_steps)
  constexpr int SW = DUP ? 2 * KR_SEG : KR_SEG;
  __shared__ double sp[SW * DIM];
  __shared__ float spf[LOWP ? SW * DIM : 1];
  __shared__ double sx[SW * NR];
  __shared__ double col[W][SW * NR];
  const ResidLaunch::Job& jb = L.job[resid_job_of(L, (long long)blockIdx.x)];
  const double* __restrict__ pts = jb.pts;
  const double* __restrict__ x = jb.x;
  double* __restrict__ part = jb.part;
  const int n = jb.n, nrhs = jb.nrhs, T = jb.T;
  const double p0 = jb.p0, shift = jb.shift;
  // (I, J) of the job's pair index b over the upper triangle, row by row:
  // b = I T - I (I - 1) / 2 + (J - I)
  const long long b = (long long)blockIdx.x - jb.first;
  const double tt = 2.0 * T + 1.0;
  int I = (int)floor((tt - sqrt(tt * tt - 8.0 * (double)b)) * 0.5);
  auto row_start = [&](int r) { return (long long)r * T - (long long)r * (r - 1) / 2; };
  while (I > 0 && row_start(I) > b) --I;
  while (row_start(I + 1) <= b) ++I;
  const int J = I + (int)(b - row_start(I));
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int i = I * KR_SEG + t, j0 = J * KR_SEG;
  const double inv_p0 = 1.0 / p0;
  for (int e = t; e < SW * DIM; e += KR_SEG) {
    const int e0 = e % (KR_SEG * DIM), jj = e0 / DIM;
    sp[e] = j0 + jj < n ? pts[(size_t)j0 * DIM + e0] : 0.0;
    if (LOWP) spf[e] = (float)sp[e];
  }
  for (int e = t; e < SW * NR; e += KR_SEG) {
    const int e0 = e % (KR_SEG * NR), jj = e0 / NR, q = e0 % NR;
    sx[e] = (j0 + jj < n && q < nrhs) ? x[(size_t)(j0 + jj) * nrhs + q] : 0.0;
  }
  for (int e = t; e < W * SW * NR; e += KR_SEG) (&col[0][0])[e] = 0.0;
  const int ir = min(i, n - 1);
  double pi[DIM], xi[NR], acc[NR];
#pragma unroll
  for (int d = 0; d < DIM; ++d) pi[d] = pts[(size_t)ir * DIM + d];
#pragma unroll
  for (int q = 0; q < NR; ++q) {
    xi[q] = (i < n && q < nrhs) ? x[(size_t)ir * nrhs + q] : 0.0;
    acc[q] = 0.0;
  }
  __syncthreads();
  const bool offdiag = I != J;
  const int jn = min(KR_SEG, n - j0);
  const bool full = jn == KR_SEG && I * KR_SEG + KR_SEG <= n;  // full tiles: no per-entry predicates
  if constexpr (LOWP) {
    float pif[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) pif[d] = (float)pi[d];
    const float p0f = (float)p0, ip0f = (float)inv_p0;
    if (full) {
      if (offdiag) residual_steps_lowp<KIND, DIM, NR, true, false, DUP>(spf, sx, col[w], pif, xi, acc, lane, jn, p0f, ip0f);
      else residual_steps_lowp<KIND, DIM, NR, false, false, DUP>(spf, sx, col[w], pif, xi, acc, lane, jn, p0f, ip0f);
    } else if (i < n) {
      if (offdiag) residual_steps_lowp<KIND, DIM, NR, true, true, DUP>(spf, sx, col[w], pif, xi, acc, lane, jn, p0f, ip0f);
      else residual_steps_lowp<KIND, DIM, NR, false, true, DUP>(spf, sx, col[w], pif, xi, acc, lane, jn, p0f, ip0f);
    }
  } else if (full) {
    if (offdiag) residual_steps<KIND, DIM, NR, true, false, DUP>(sp, sx, col[w], pi, xi, acc, lane, jn, p0, inv_p0);
    else residual_steps<KIND, DIM, NR, false, false, DUP>(sp, sx, col[w], pi, xi, acc, lane, jn, p0, inv_p0);
  } else if (i < n) {  // ragged edge of the matrix
    if (offdiag) residual_steps<KIND, DIM, NR, true, true, DUP>(sp, sx, col[w], pi, xi, acc, lane, jn, p0, inv_p0);
    else residual_steps<KIND, DIM, NR, false, true, DUP>(sp, sx, col[w], pi, xi, acc, lane, jn, p0, inv_p0);
  }
  if (!offdiag && i < n) {  // the diagonal entry's shift
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = fma(shift, xi[q], acc[q]);
  }
  if (i < n)
    for (int q = 0; q < nrhs; ++q) part[((size_t)J * n + i) * nrhs + q] = acc[q];
  if (offdiag) {
    __syncthreads();
    const int jrow = j0 + t;
    if (jrow < n)
      for (int q = 0; q < nrhs; ++q) {
        double v = col[0][t * NR + q];
        if (DUP) v += col[0][(t + KR_SEG) * NR + q];
#pragma unroll
        for (int ww = 1; ww < W; ++ww) {
          v += col[ww][t * NR + q];
          if (DUP) v += col[ww][(t + KR_SEG) * NR + q];
        }
        part[((size_t)I * n + jrow) * nrhs + q] = v;
      }
  }
}

// r = b - (sum of the job's segments in order), one thread per (row, rhs) element
__global__ void residual_reduce(const __grid_constant__ ResidLaunch L) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const ResidLaunch::Job& jb = L.job[resid_job_of(L, e)];
  const long long k = e - jb.first, count = (long long)jb.n * jb.nrhs;
  if (k < 0 || k >= count) return;
  double s = 0.0;
  for (int g = 0; g < jb.T; ++g) s += jb.part[g * count + k];
  jb.r[k] = jb.b[k] - s;
}

// x += dx of every job, one thread per element
__global__ void residual_update(const __grid_constant__ ResidLaunch L) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const ResidLaunch::Job& jb = L.job[resid_job_of(L, e)];
  const long long k = e - jb.first, count = (long long)jb.n * jb.nrhs;
  if (k < 0 || k >= count) return;
  jb.x[k] += jb.dx[k];
}

template <int KIND, int DIM>
cudaError_t launch_residual_sym(const ResidLaunch& L, unsigned pairs, int nr, bool lowp, cudaStream_t s) {
  if (lowp) {
    if (nr == 1) kernel_residual_sym<KIND, DIM, 1, true><<<pairs, KR_SEG, 0, s>>>(L);
    else kernel_residual_sym<KIND, DIM, 4, true><<<pairs, KR_SEG, 0, s>>>(L);
  } else if (nr == 1) {
    kernel_residual_sym<KIND, DIM, 1, false><<<pairs, KR_SEG, 0, s>>>(L);
  } else {
    kernel_residual_sym<KIND, DIM, 4, false><<<pairs, KR_SEG, 0, s>>>(L);
  }
  return cudaGetLastError();
}

template <int KIND>
cudaError_t launch_residual_sym_dim(int dim, const ResidLaunch& L, unsigned pairs, int nr, bool lowp,
                                    cudaStream_t s) {
  if (dim == 1) return launch_residual_sym<KIND, 1>(L, pairs, nr, lowp, s);
  if (dim == 2) return launch_residual_sym<KIND, 2>(L, pairs, nr, lowp, s);
  return launch_residual_sym<KIND, 3>(L, pairs, nr, lowp, s);
}

template <int KIND, int DIM>
cudaError_t launch_residual_part(const pp_resid_job& j, cudaStream_t s) {
  const int segs = (j.n + KR_SEG - 1) / KR_SEG;
  const dim3 grid((j.n + KR_ROWS - 1) / KR_ROWS, segs);
  if (j.nrhs <= 8)
    kernel_residual_part<KIND, DIM, 8><<<grid, KR_THREADS, 0, s>>>(j.p0, j.shift, j.pts, j.n, j.x, j.part, j.nrhs);
  else
    kernel_residual_part<KIND, DIM, 16><<<grid, KR_THREADS, 0, s>>>(j.p0, j.shift, j.pts, j.n, j.x, j.part, j.nrhs);
  return cudaGetLastError();
}

template <int KIND>
cudaError_t launch_residual_part_dim(const pp_resid_job& j, cudaStream_t s) {
  if (j.dim == 1) return launch_residual_part<KIND, 1>(j, s);
  if (j.dim == 2) return launch_residual_part<KIND, 2>(j, s);
  return launch_residual_part<KIND, 3>(j, s);
}

ResidLaunch::Job resid_job(const pp_resid_job& j) {
  ResidLaunch::Job o{};
  o.pts = j.pts;
  o.x = j.x;
  o.dx = j.dx;
  o.b = j.b;
  o.r = j.r;
  o.part = j.part;
  o.p0 = j.p0;
  o.shift = j.shift;
  o.n = j.n;
  o.nrhs = j.nrhs;
  o.T = (j.n + KR_SEG - 1) / KR_SEG;
  return o;
}

// element-wise launch (update or reduction) over jobs[sel] in chunks of KR_LAUNCH_JOBS
template <typename F>
cudaError_t launch_elementwise(const pp_resid_job* jobs, const std::vector<int>& sel, F kernel, cudaStream_t s) {
  for (size_t c = 0; c < sel.size(); c += KR_LAUNCH_JOBS) {
    ResidLaunch L;
    L.njobs = (int)std::min<size_t>(KR_LAUNCH_JOBS, sel.size() - c);
    long long total = 0;
    for (int q = 0; q < L.njobs; ++q) {
      L.job[q] = resid_job(jobs[sel[c + q]]);
      L.job[q].first = total;
      total += (long long)L.job[q].n * L.job[q].nrhs;
    }
    kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(L);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Dense blocks of an H-matrix assembled in place from its points (the first step of building it
// on the device): entry (i, j) of the block at rows [r0, r0 + m), columns [c0, c0 + n) is
// K(|p_{r0+i} - p_{c0+j}|), plus the shift on the matrix diagonal, with the residual kernel's
// distance and entry evaluation (the same bits as the matrix the refinement applies).  One CTA
// per AS_ROWS rows of a block; blocks passed by value, up to AS_LAUNCH_JOBS per launch.
#define AS_LAUNCH_JOBS 64
#define AS_ROWS 16
struct AssembleLaunch {
  struct Job {
    double* a;
    long long first;  // first CTA of the block in the launch
    int ld, r0, c0, m, n, pad;
  } job[AS_LAUNCH_JOBS];
  const double* pts;
  double p0, shift;
  int njobs;
};

template <int KIND, int DIM>
__global__ void __launch_bounds__(256) assemble_dense_kernel(const __grid_constant__ AssembleLaunch L) {
  int lo = 0, hi = L.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.job[mid].first <= (long long)blockIdx.x) lo = mid; else hi = mid - 1;
  }
  const AssembleLaunch::Job& jb = L.job[lo];
  const int rb = (int)((long long)blockIdx.x - jb.first) * AS_ROWS;
  const double inv_p0 = 1.0 / L.p0;
  for (int e = threadIdx.x; e < AS_ROWS * jb.n; e += blockDim.x) {
    const int i = rb + e / jb.n, j = e % jb.n;
    if (i >= jb.m) break;  // e only grows: every later element is past the block too
    const int gi = jb.r0 + i, gj = jb.c0 + j;
    double d2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double u = L.pts[(size_t)gi * DIM + d] - L.pts[(size_t)gj * DIM + d];
      d2 = fma(u, u, d2);
    }
    double a = kernel_eval_nr<KIND>(d2, L.p0, inv_p0);
    if (gi == gj) a += L.shift;
    jb.a[(size_t)i * jb.ld + j] = a;
  }
}

template <int KIND>
cudaError_t launch_assemble_dim(int dim, const AssembleLaunch& L, unsigned ctas, cudaStream_t s) {
  if (dim == 1) assemble_dense_kernel<KIND, 1><<<ctas, 256, 0, s>>>(L);
  else if (dim == 2) assemble_dense_kernel<KIND, 2><<<ctas, 256, 0, s>>>(L);
  else assemble_dense_kernel<KIND, 3><<<ctas, 256, 0, s>>>(L);
  return cudaGetLastError();
}

// x += dx over `count` elements (the refinement update of a served request)
__global__ void axpy_kernel(double* __restrict__ x, const double* __restrict__ dx, size_t count) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
    x[e] += dx[e];
}

// out[0] = max |x|, out[1] = max |r| as the bit patterns of non-negative doubles (their
// integer order is their numeric order, so an integer atomicMax reduces them); out zeroed
// by the caller
__global__ void absmax2_kernel(const double* __restrict__ x, const double* __restrict__ r, size_t count,
                               unsigned long long* out) {
  double mx = 0.0, mr = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
    mx = fmax(mx, fabs(x[e]));
    mr = fmax(mr, fabs(r[e]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(mx));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(mr));
  }
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

long long pp_accum_scratch_doubles(long long ny, int k1, int k2) {
  // dev_accum keeps the ny x k1 sketch Y in shared memory while it fits beside the rest of the
  // 180 KB; only a larger Y goes to the task's scratch, and nothing else does
  return accum_y_on_chip(ny, k1, k2) ? 0 : ny * k1;
}

namespace {
// device address of the static scratch array, looked up once per device (std::call_once, so
// two host threads making their first calls at once do not race on the cache)
constexpr int kNoallocMaxDevices = 64;
std::once_flag g_noalloc_once[kNoallocMaxDevices];
double* g_noalloc_addr[kNoallocMaxDevices] = {nullptr};
cudaError_t g_noalloc_err[kNoallocMaxDevices] = {cudaSuccess};
}  // namespace

cudaError_t pp_accum_noalloc_launch(const pp_task& T, long long scratch_doubles, cudaStream_t s) {
  if (scratch_doubles < 0 || scratch_doubles > PP_NOALLOC_SCRATCH_DOUBLES) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
  std::call_once(g_noalloc_once[dev], [dev] {  // set-up, once per device, with that device current
    double* p = nullptr;
    g_noalloc_err[dev] = cudaGetSymbolAddress((void**)&p, g_accum_noalloc_scratch);
    g_noalloc_addr[dev] = p;
  });
  if (g_noalloc_err[dev] != cudaSuccess) return g_noalloc_err[dev];
  pp_task t = T;
  t.tmp = g_noalloc_addr[dev];
  // 160 KB of dynamic shared memory, as the VM's ACCUM has; pp_vm_prepare (run at context
  // creation on this device) raised the kernel's limit to that
  accum_noalloc_kernel<<<1, NT, VM_SMEM_BYTES, s>>>(t);
  return cudaGetLastError();
}

size_t pp_vm_smem_bytes() { return VM_SMEM_BYTES; }

int pp_vm_blocks_per_sm() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, vm_kernel, NT, pp_vm_smem_bytes());
  return nb;
}

namespace {
// Loads one kernel's code now (lazy module loading would otherwise do it at its first launch,
// in the middle of a served request).
template <typename F>
cudaError_t preload(F f) {
  cudaFuncAttributes a;
  return cudaFuncGetAttributes(&a, f);
}
template <int KIND, int DIM>
cudaError_t preload_residual() {
  cudaError_t e = preload(kernel_residual_sym<KIND, DIM, 1, false>);
  if (e == cudaSuccess) e = preload(kernel_residual_sym<KIND, DIM, 4, false>);
  if (e == cudaSuccess) e = preload(kernel_residual_sym<KIND, DIM, 1, true>);
  if (e == cudaSuccess) e = preload(kernel_residual_sym<KIND, DIM, 4, true>);
  if (e == cudaSuccess) e = preload(kernel_residual_part<KIND, DIM, 8>);
  if (e == cudaSuccess) e = preload(kernel_residual_part<KIND, DIM, 16>);
  return e;
}
template <int KIND>
cudaError_t preload_residual_dims() {
  cudaError_t e = preload_residual<KIND, 1>();
  if (e == cudaSuccess) e = preload_residual<KIND, 2>();
  if (e == cudaSuccess) e = preload_residual<KIND, 3>();
  if (e == cudaSuccess) e = preload(assemble_dense_kernel<KIND, 1>);
  if (e == cudaSuccess) e = preload(assemble_dense_kernel<KIND, 2>);
  if (e == cudaSuccess) e = preload(assemble_dense_kernel<KIND, 3>);
  return e;
}
}  // namespace

cudaError_t pp_vm_prepare() {
  cudaError_t e = cudaFuncSetAttribute(vm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pp_vm_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(accum_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pp_vm_smem_bytes());
  // every kernel of the refinement and serving paths, loaded at context creation
  for (cudaError_t r : {preload(vm_init), preload(residual_reduce), preload(residual_update), preload(axpy_kernel),
                        preload(absmax2_kernel), preload(dense_residual_kernel), preload_residual_dims<0>(),
                        preload_residual_dims<1>(), preload_residual_dims<2>(), preload_residual_dims<3>()})
    if (e == cudaSuccess) e = r;
  return e;
}

cudaError_t pp_vm_run(const pp_vm_launch& L, cudaStream_t s) {
  if (L.n_tasks <= 0) return cudaSuccess;
  const int ib = 256;
  vm_init<<<(L.n_tasks + ib - 1) / ib, ib, 0, s>>>(L.indeg, L.ready, L.n_ready, L.n_tasks, L.counters, L.slots,
                                                  L.state);
  vm_kernel<<<L.grid, NT, pp_vm_smem_bytes(), s>>>(L.tasks, L.n_tasks, L.succ, L.counters, L.slots, L.state,
                                                   L.wait_ns, L.trace, L.use_tc);
  return cudaGetLastError();
}

cudaError_t pp_dense_residual(const double* A, int lda, int n, const double* x, const double* b, double* r, int nrhs,
                              cudaStream_t s) {
  const int threads = 256, warps = threads / 32;
  dense_residual_kernel<<<(n + warps - 1) / warps, threads, 0, s>>>(A, lda, n, x, b, r, nrhs);
  return cudaGetLastError();
}

cudaError_t pp_kernel_residual_batch(const pp_resid_job* jobs, int njobs, cudaStream_t s, bool lowp) {
  if (njobs <= 0) return cudaSuccess;
  if (!jobs) return cudaErrorInvalidValue;
  std::vector<int> all, upd;
  for (int q = 0; q < njobs; ++q) {
    const pp_resid_job& j = jobs[q];
    if (j.dim < 1 || j.dim > 3 || j.nrhs < 1 || j.nrhs > 16 || j.n <= 0 || j.kernel < 0 || j.kernel > 3 || !j.pts ||
        !j.x || !j.b || !j.r || !j.part)
      return cudaErrorInvalidValue;
    if (j.kernel <= 1 && !(j.p0 >= 0.0 && std::isfinite(j.p0))) return cudaErrorInvalidValue;
    all.push_back(q);
    if (j.dx) upd.push_back(q);
  }
  cudaError_t e = launch_elementwise(jobs, upd, residual_update, s);
  if (e != cudaSuccess) return e;
  // tile-pair launches, one per (kernel, dimension, right-hand-side width) group
  for (int kern = 0; kern < 4; ++kern)
    for (int dim = 1; dim <= 3; ++dim)
      for (int nr : {1, 4}) {
        std::vector<int> sel;
        for (int q = 0; q < njobs; ++q)
          if (jobs[q].kernel == kern && jobs[q].dim == dim && (nr == 1 ? jobs[q].nrhs == 1 : (jobs[q].nrhs > 1 && jobs[q].nrhs <= 4)))
            sel.push_back(q);
        for (size_t c = 0; c < sel.size(); c += KR_LAUNCH_JOBS) {
          ResidLaunch L;
          L.njobs = (int)std::min<size_t>(KR_LAUNCH_JOBS, sel.size() - c);
          long long pairs = 0;
          for (int q = 0; q < L.njobs; ++q) {
            L.job[q] = resid_job(jobs[sel[c + q]]);
            L.job[q].first = pairs;
            pairs += (long long)L.job[q].T * (L.job[q].T + 1) / 2;
          }
          if (pairs >= (1LL << 31)) return cudaErrorInvalidValue;
          switch (kern) {
            case 0: e = launch_residual_sym_dim<0>(dim, L, (unsigned)pairs, nr, lowp, s); break;
            case 1: e = launch_residual_sym_dim<1>(dim, L, (unsigned)pairs, nr, lowp, s); break;
            case 2: e = launch_residual_sym_dim<2>(dim, L, (unsigned)pairs, nr, lowp, s); break;
            default: e = launch_residual_sym_dim<3>(dim, L, (unsigned)pairs, nr, lowp, s); break;
          }
          if (e != cudaSuccess) return e;
        }
      }
  // wider right-hand-side blocks: per-job row-block partial products
  for (int q = 0; q < njobs; ++q) {
    if (jobs[q].nrhs <= 4) continue;
    switch (jobs[q].kernel) {
      case 0: e = launch_residual_part_dim<0>(jobs[q], s); break;
      case 1: e = launch_residual_part_dim<1>(jobs[q], s); break;
      case 2: e = launch_residual_part_dim<2>(jobs[q], s); break;
      default: e = launch_residual_part_dim<3>(jobs[q], s); break;
    }
    if (e != cudaSuccess) return e;
  }
  return launch_elementwise(jobs, all, residual_reduce, s);
}

cudaError_t pp_kernel_residual(int kernel, double p0, double p1, double diag_shift, const double* pts, int dim, int n,
                               const double* x, const double* b, double* r, int nrhs, double* part,
                               cudaStream_t s) {
  (void)p1;
  pp_resid_job j{};
  j.kernel = kernel;
  j.dim = dim;
  j.n = n;
  j.nrhs = nrhs;
  j.p0 = p0;
  j.shift = diag_shift;
  j.pts = pts;
  j.x = const_cast<double*>(x);  // read only: no update without dx
  j.b = b;
  j.r = r;
  j.part = part;
  return pp_kernel_residual_batch(&j, 1, s);
}

cudaError_t pp_assemble_dense(const pp_assemble_block* blocks, int nblocks, int kernel, int dim, double p0,
                              double shift, const double* pts, cudaStream_t s) {
  if (nblocks <= 0) return cudaSuccess;
  if (!blocks || !pts || dim < 1 || dim > 3 || kernel < 0 || kernel > 3) return cudaErrorInvalidValue;
  if (kernel <= 1 && !(p0 >= 0.0 && std::isfinite(p0))) return cudaErrorInvalidValue;
  for (int c = 0; c < nblocks; c += AS_LAUNCH_JOBS) {
    AssembleLaunch L;
    L.pts = pts;
    L.p0 = p0;
    L.shift = shift;
    L.njobs = std::min(AS_LAUNCH_JOBS, nblocks - c);
    long long ctas = 0;
    for (int q = 0; q < L.njobs; ++q) {
      const pp_assemble_block& b = blocks[c + q];
      if (!b.a || b.m <= 0 || b.n <= 0 || b.ld < b.n || b.r0 < 0 || b.c0 < 0) return cudaErrorInvalidValue;
      L.job[q] = AssembleLaunch::Job{b.a, ctas, b.ld, b.r0, b.c0, b.m, b.n, 0};
      ctas += (b.m + AS_ROWS - 1) / AS_ROWS;
    }
    if (ctas >= (1LL << 31)) return cudaErrorInvalidValue;
    cudaError_t e;
    switch (kernel) {
      case 0: e = launch_assemble_dim<0>(dim, L, (unsigned)ctas, s); break;
      case 1: e = launch_assemble_dim<1>(dim, L, (unsigned)ctas, s); break;
      case 2: e = launch_assemble_dim<2>(dim, L, (unsigned)ctas, s); break;
      default: e = launch_assemble_dim<3>(dim, L, (unsigned)ctas, s); break;
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t pp_axpy(double* x, const double* dx, size_t count, cudaStream_t s) {
  const unsigned blocks = (unsigned)std::min<size_t>((count + 255) / 256, 1184);
  axpy_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(x, dx, count);
  return cudaGetLastError();
}

cudaError_t pp_absmax2(const double* x, const double* r, size_t count, unsigned long long* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  const unsigned blocks = (unsigned)std::min<size_t>((count + 255) / 256, 592);
  absmax2_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(x, r, count, out);
  return cudaGetLastError();
}

size_t pp_kernel_residual_part_elems(int n, int nrhs) {
  return (size_t)((n + KR_SEG - 1) / KR_SEG) * n * nrhs;
}
