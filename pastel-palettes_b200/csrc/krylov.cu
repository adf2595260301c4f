// krylov.cu — batched restarted GMRES around the H-LU solve (FP64), for sm_100a.
//
// Plain iterative refinement x += (LU)^-1 (b - A x) converges only while the H-LU factors are
// close enough to A that every eigenvalue of I - (LU)^-1 A lies inside the unit circle.  With
// ranks capped below what the tolerance asks for (weak admissibility on 2-D points, where
// neighbouring clusters interact with a rank that grows with the cluster size) that fails and
// the refinement stalls.  GMRES on A (LU)^-1 y = b, x = (LU)^-1 y, converges whenever the
// preconditioned operator is merely well clustered; its residual is recomputed in FP64 from
// the points at every restart (the matrix-free residual kernels of vm.cu), so the accuracy of
// the answer does not depend on the accuracy of the factors.
//
// The reference has no solve or refinement path; these kernels carry the Krylov arithmetic of
// many instances of uneven size in one launch each (one CTA per instance, the largest first):
//   gmres_start    beta = ||r||, v0 = r / beta, g = beta e1
//   gmres_arnoldi  w = A z_j (given as -w by the residual kernel), classical Gram-Schmidt with
//                  one re-orthogonalisation pass (CGS2), h_{j+1,j} = ||w||, v_{j+1} = w / h,
//                  earlier Givens rotations applied to the new column, a new rotation, g updated
//   gmres_finish   H y = g by back substitution, x += Z y
// Every reduction runs in a fixed order (per-thread sums over a fixed stride, a shuffle tree,
// warps added in index order), so results do not depend on timing.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "vm.cuh"

namespace {

constexpr int KT = 256;          // threads per instance CTA
constexpr int KW = KT / 32;      // warps
constexpr int KCH = 8;           // basis vectors per dot-product pass

struct GState {                  // views into one instance's small state (pp_gmres_state_elems)
  double* H;                     // (m + 1) x m, column-major: H[c * (m + 1) + r]
  double* cs;                    // m cosines
  double* sn;                    // m sines
  double* g;                     // m + 1: rotated right-hand side of the least-squares problem
  double* meta;                  // [0] active dimension, [1] frozen flag, [2] beta, [3] |g_k|
  __device__ GState(double* st, int m)
      : H(st), cs(st + (size_t)(m + 1) * m), sn(cs + m), g(sn + m), meta(g + m + 1) {}
};

// sum of v over the CTA (fixed order); every thread gets the result
__device__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < KW; ++w) s += red[w];
  return s;
}

__global__ void __launch_bounds__(KT) gmres_start_kernel(const pp_gmres_slot* __restrict__ slots) {
  __shared__ double red[KW];
  const pp_gmres_slot S = slots[blockIdx.x];
  GState G(S.st, S.m);
  const int n = S.n;
  double s = 0.0;
  for (int e = threadIdx.x; e < n; e += KT) s = fma(S.r[e], S.r[e], s);
  const double beta = sqrt(block_sum(s, red));
  const bool ok = beta > 0.0 && isfinite(beta);
  for (int e = threadIdx.x; e < n; e += KT) S.V[e] = ok ? S.r[e] / beta : 0.0;
  for (int i = threadIdx.x; i <= S.m; i += KT) G.g[i] = (i == 0 && ok) ? beta : 0.0;
  if (threadIdx.x == 0) {
    G.meta[0] = 0.0;
    G.meta[1] = ok ? 0.0 : 1.0;
    G.meta[2] = beta;
    G.meta[3] = ok ? beta : 0.0;
  }
}

// Step j: on entry V[j + 1] holds -A z_j (the matrix-free residual of z_j against b = 0).
__global__ void __launch_bounds__(KT) gmres_arnoldi_kernel(const pp_gmres_slot* __restrict__ slots, int j) {
  __shared__ double red[KW * KCH];
  __shared__ double hp[PP_GMRES_MAX_RESTART + 1];
  __shared__ double hsum[PP_GMRES_MAX_RESTART + 1];
  __shared__ double scale;
  const pp_gmres_slot S = slots[blockIdx.x];
  GState G(S.st, S.m);
  const int n = S.n;
  double* __restrict__ w = S.V + (size_t)(j + 1) * n;
  if (j >= S.m) return;
  if (G.meta[1] != 0.0) {  // frozen (converged exactly or broke down): keep the basis finite
    for (int e = threadIdx.x; e < n; e += KT) w[e] = 0.0;
    return;
  }
  for (int e = threadIdx.x; e < n; e += KT) w[e] = -w[e];
  for (int pass = 0; pass < 2; ++pass) {
    for (int i0 = 0; i0 <= j; i0 += KCH) {
      double acc[KCH];
#pragma unroll
      for (int q = 0; q < KCH; ++q) acc[q] = 0.0;
      const int cnt = min(KCH, j + 1 - i0);
      for (int e = threadIdx.x; e < n; e += KT) {
        const double we = w[e];
#pragma unroll
        for (int q = 0; q < KCH; ++q)
          if (q < cnt) acc[q] = fma(S.V[(size_t)(i0 + q) * n + e], we, acc[q]);
      }
#pragma unroll
      for (int q = 0; q < KCH; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      }
      if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int q = 0; q < KCH; ++q) red[q * KW + (threadIdx.x >> 5)] = acc[q];
      }
      __syncthreads();
      if (threadIdx.x < cnt) {
        double t = 0.0;
#pragma unroll
        for (int ww = 0; ww < KW; ++ww) t += red[threadIdx.x * KW + ww];
        hp[i0 + threadIdx.x] = t;
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < n; e += KT) {
      double t = w[e];
      for (int i = 0; i <= j; ++i) t = fma(-hp[i], S.V[(size_t)i * n + e], t);
      w[e] = t;
    }
    for (int i = threadIdx.x; i <= j; i += KT) hsum[i] = pass == 0 ? hp[i] : hsum[i] + hp[i];
    __syncthreads();
  }
  double s = 0.0;
  for (int e = threadIdx.x; e < n; e += KT) s = fma(w[e], w[e], s);
  const double hn = sqrt(block_sum(s, red));
  if (threadIdx.x == 0) {
    const int ld = S.m + 1;
    double* col = G.H + (size_t)j * ld;
    for (int i = 0; i <= j; ++i) col[i] = hsum[i];
    for (int i = 0; i < j; ++i) {  // earlier rotations
      const double a = col[i], b = col[i + 1];
      col[i] = G.cs[i] * a + G.sn[i] * b;
      col[i + 1] = -G.sn[i] * a + G.cs[i] * b;
    }
    const double a = col[j], r = hypot(a, hn);
    double sc = 0.0;
    if (r > 0.0 && isfinite(r)) {
      const double c = a / r, sg = hn / r;
      G.cs[j] = c;
      G.sn[j] = sg;
      col[j] = r;
      col[j + 1] = 0.0;
      G.g[j + 1] = -sg * G.g[j];
      G.g[j] = c * G.g[j];
      G.meta[0] = (double)(j + 1);
      G.meta[3] = fabs(G.g[j + 1]);
      // an exact zero (or denormal) norm: the Krylov space is invariant, the least-squares
      // solution of this cycle is exact; later steps of the cycle leave this instance alone
      if (hn > 1e-300) sc = 1.0 / hn; else G.meta[1] = 1.0;
    } else {
      G.meta[1] = 1.0;  // w = 0 and no new direction: the active dimension stays j
    }
    scale = sc;
  }
  __syncthreads();
  const double hnv = hn, sc = scale;
  for (int e = threadIdx.x; e < n; e += KT) w[e] = sc != 0.0 ? w[e] / hnv : 0.0;
}

__global__ void __launch_bounds__(KT) gmres_finish_kernel(const pp_gmres_slot* __restrict__ slots) {
  __shared__ double y[PP_GMRES_MAX_RESTART];
  const pp_gmres_slot S = slots[blockIdx.x];
  GState G(S.st, S.m);
  const int n = S.n, k = (int)G.meta[0], ld = S.m + 1;
  if (threadIdx.x == 0) {
    for (int i = k - 1; i >= 0; --i) {
      double t = G.g[i];
      for (int c = i + 1; c < k; ++c) t = fma(-G.H[(size_t)c * ld + i], y[c], t);
      y[i] = t / G.H[(size_t)i * ld + i];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += KT) {
    double t = S.x[e];
    for (int i = 0; i < k; ++i) t = fma(y[i], S.Z[(size_t)i * n + e], t);
    S.x[e] = t;
  }
}

}  // namespace

size_t pp_gmres_state_elems(int m) { return (size_t)(m + 1) * m + 2 * (size_t)m + (size_t)(m + 1) + 4; }

cudaError_t pp_gmres_start(const pp_gmres_slot* slots, int count, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  gmres_start_kernel<<<count, KT, 0, s>>>(slots);
  return cudaGetLastError();
}

cudaError_t pp_gmres_arnoldi(const pp_gmres_slot* slots, int count, int j, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  if (j < 0 || j >= PP_GMRES_MAX_RESTART) return cudaErrorInvalidValue;
  gmres_arnoldi_kernel<<<count, KT, 0, s>>>(slots, j);
  return cudaGetLastError();
}

cudaError_t pp_gmres_finish(const pp_gmres_slot* slots, int count, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  gmres_finish_kernel<<<count, KT, 0, s>>>(slots);
  return cudaGetLastError();
}
