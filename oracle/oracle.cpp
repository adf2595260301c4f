/* oracle.cpp — TEST ORACLE (CPU restatement of the reference's FP64 block routines).
 *
 * Test infrastructure only: used by tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py as the checker / CPU reference.  Nothing in the product links it.
 *
 * Each routine restates Pastel-Palettes src/kernel.cu in the reference's own arithmetic
 * order (row-major, no pivoting, one fma per update, same operand order):
 *   o_getrf       DenseGetrf            src/kernel.cu:104-147 (blockDenseGetrf :820-882 regroups
 *                                       the same per-element updates into panels)
 *   o_trsml       DenseTrsmL            :150-182  (blockDenseTrsmL :667-715)
 *   o_trsmr       DenseTrsmR            :185-226  (blockDenseTrsmR :718-766)
 *   o_trsmrt      DenseTrsmR_transposeB :229-285  (blockDenseTrsmR_transposeB :769-817)
 *   o_gemm        blockDenseGemm        :415-664  (beta == 0 zero fill, M *= beta/alpha,
 *                                       k-ascending fma, M *= alpha)
 *   o_gemm3/4     blockDenseGemm_3x/_4x :886-955
 *   o_accum       blockLowRankAccum     :1255-1280 with blockGivensRotation :1160-1204 and
 *                                       blockGivensRecoverQ :1206-1253
 * plus o_trsmu (B := U^-1 B), the solve step the reference does not have, and the engine's
 * mixed-precision pair (no reference counterpart): SHADOW (an operand rounded to BF16 in the
 * tensor core's tiled layout) and the BF16 GEMM (products of the shadows summed in FP64 here; the
 * tensor cores sum in FP32, so the two agree to a tolerance, not bitwise).
 * And the engine's opt-in partial pivoting inside GETRF blocks (PP_PIVOT): o_getrf_piv (pivot row
 * = largest magnitude, first of equal ones, as the reference's unused blockReduceMax_Index /
 * blockSwapRows at src/kernel.cu:958-1051 pick and swap; then o_getrf's elimination) and
 * o_permute_rows (a TRSML's right-hand side put in the block's pivot order before o_trsml).
 * `rhypot(1, t)` of the reference is written here from its definition, 1 / hypot(1, t).
 *
 * Parity pins: dense routines must agree bitwise with the CUDA path; the Givens-based
 * accumulation agrees with the engine's Householder variant to rounding (the span is the
 * same; column signs of Q may differ, the product U V^T does not).
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "../pastel-palettes_b200/csrc/pp_task.h"

namespace {

inline double& at(double* M, int ld, int r, int c) { return M[(int64_t)r * ld + c]; }
inline double at(const double* M, int ld, int r, int c) { return M[(int64_t)r * ld + c]; }

void o_getrf(double* M, int nx, int ny, int ld) {
  const int mn = std::min(nx, ny);
  for (int i = 0; i < mn; ++i)
    for (int row = i + 1; row < ny; ++row) {
      const double left = at(M, ld, row, i) / at(M, ld, i, i);
      at(M, ld, row, i) = left;
      for (int col = i + 1; col < nx; ++col) at(M, ld, row, col) = std::fma(at(M, ld, i, col), -left, at(M, ld, row, col));
    }
}

// GETRF with partial pivoting inside the block (the engine's PP_PIVOT): at step i the row
// r >= i of largest |a_ri| (the first of equal ones), whole rows i and r swapped, then the
// unpivoted elimination above; perm_out[i] = the original row of row i (as a double).  The
// reference's pivot helpers pick and swap rows this way (src/kernel.cu:958-1051:
// blockReduceMax_Index takes the largest magnitude, blockSwapRows exchanges whole rows) but
// the reference never calls them.
void o_getrf_piv(double* M, int nx, int ny, int ld, double* perm_out) {
  std::vector<int> perm(ny);
  for (int i = 0; i < ny; ++i) perm[i] = i;
  const int mn = std::min(nx, ny);
  for (int i = 0; i < mn; ++i) {
    int r = i;
    double best = -1.0;
    for (int row = i; row < ny; ++row) {
      const double v = std::fabs(at(M, ld, row, i));
      if (v > best) { best = v; r = row; }
    }
    if (r != i) {
      for (int col = 0; col < nx; ++col) std::swap(at(M, ld, i, col), at(M, ld, r, col));
      std::swap(perm[i], perm[r]);
    }
    for (int row = i + 1; row < ny; ++row) {
      const double left = at(M, ld, row, i) / at(M, ld, i, i);
      at(M, ld, row, i) = left;
      for (int col = i + 1; col < nx; ++col) at(M, ld, row, col) = std::fma(at(M, ld, i, col), -left, at(M, ld, row, col));
    }
  }
  for (int i = 0; i < ny; ++i) perm_out[i] = (double)perm[i];
}

// rows of B (ny_b x nx_b) put in the order of a pivoted block's permutation: row i := old row perm[i]
void o_permute_rows(double* B, const double* perm, int nx_b, int ny_b, int ld_b) {
  std::vector<double> tmp((size_t)nx_b * ny_b);
  for (int i = 0; i < ny_b; ++i)
    for (int col = 0; col < nx_b; ++col) tmp[(size_t)i * nx_b + col] = at(B, ld_b, (int)perm[i], col);
  for (int i = 0; i < ny_b; ++i)
    for (int col = 0; col < nx_b; ++col) at(B, ld_b, i, col) = tmp[(size_t)i * nx_b + col];
}

void o_trsml(double* B, const double* L, int nx_b, int ny_b, int nx_l, int ld_b, int ld_l) {
  const int mn = std::min(nx_l, ny_b);
  for (int i = 0; i < mn; ++i)
    for (int row = i + 1; row < ny_b; ++row) {
      const double left = -at(L, ld_l, row, i);
      for (int col = 0; col < nx_b; ++col) at(B, ld_b, row, col) = std::fma(at(B, ld_b, i, col), left, at(B, ld_b, row, col));
    }
}

void o_trsmr(double* B, const double* U, int nx_b, int ny_b, int ny_u, int ld_b, int ld_u) {
  const int mn = std::min(nx_b, ny_u);
  for (int i = 0; i < mn; ++i)
    for (int row = 0; row < ny_b; ++row) {
      const double x = at(B, ld_b, row, i) / at(U, ld_u, i, i);
      at(B, ld_b, row, i) = x;
      const double left = -x;
      for (int col = i + 1; col < nx_b; ++col) at(B, ld_b, row, col) = std::fma(left, at(U, ld_u, i, col), at(B, ld_b, row, col));
    }
}

// B stored transposed: nx_b storage rows, ny_b storage columns
void o_trsmrt(double* B, const double* U, int nx_b, int ny_b, int ny_u, int ld_b, int ld_u) {
  const int mn = std::min(nx_b, ny_u);
  for (int i = 0; i < mn; ++i) {
    const double diag = 1. / at(U, ld_u, i, i);
    for (int col = 0; col < ny_b; ++col) at(B, ld_b, i, col) *= diag;
    for (int row = i + 1; row < nx_b; ++row) {
      const double left = -at(U, ld_u, i, row);
      for (int col = 0; col < ny_b; ++col) at(B, ld_b, row, col) = std::fma(left, at(B, ld_b, i, col), at(B, ld_b, row, col));
    }
  }
}

// B[m x n] := U^-1 B, U upper m x m (solve; no reference counterpart): row i is scaled by
// the reciprocal of u_ii, then eliminated from the rows above
void o_trsmu64(double* B, const double* U, int m, int n, int ld_b, int ld_u) {
  for (int i = m - 1; i >= 0; --i) {
    const double rd = 1. / at(U, ld_u, i, i);
    for (int c = 0; c < n; ++c) at(B, ld_b, i, c) = at(B, ld_b, i, c) * rd;
    for (int r = 0; r < i; ++r) {
      const double left = -at(U, ld_u, r, i);
      for (int c = 0; c < n; ++c) at(B, ld_b, r, c) = std::fma(left, at(B, ld_b, i, c), at(B, ld_b, r, c));
    }
  }
}

// M (m x n) = alpha * op(A) (m x k) * op(B) (k x n) + beta * M, literally as blockDenseGemm
void o_gemm(double alpha, double beta, double* M, const double* A, const double* B, int m, int n, int k, int ld_m,
            int ld_a, int ld_b, bool a_T, bool b_T) {
  const double mult = beta / alpha;
  if (beta == 0.) {
    for (int r = 0; r < m; ++r)
      for (int c = 0; c < n; ++c) at(M, ld_m, r, c) = 0.;
  } else if (mult != 1.) {
    for (int r = 0; r < m; ++r)
      for (int c = 0; c < n; ++c) at(M, ld_m, r, c) *= mult;
  }
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < n; ++c) {
      double acc = at(M, ld_m, r, c);
      for (int i = 0; i < k; ++i) {
        const double a = a_T ? at(A, ld_a, i, r) : at(A, ld_a, r, i);
        const double b = b_T ? at(B, ld_b, c, i) : at(B, ld_b, i, c);
        acc = std::fma(a, b, acc);
      }
      at(M, ld_m, r, c) = acc;
    }
  if (alpha != 1.) {
    for (int r = 0; r < m; ++r)
      for (int c = 0; c < n; ++c) at(M, ld_m, r, c) *= alpha;
  }
}

// TRSMU on up to 256 rows: 64-row blocks from the bottom, each solved as above, the rows
// above a block updated by one ascending-k product per block (the engine's definition)
void o_trsmu(double* B, const double* U, int m, int n, int ld_b, int ld_u) {
  const int nb = (m + 63) / 64;
  for (int bi = nb - 1; bi >= 0; --bi) {
    const int d = bi * 64, md = std::min(64, m - d);
    o_trsmu64(B + (int64_t)d * ld_b, U + (int64_t)d * ld_u + d, md, n, ld_b, ld_u);
    if (d > 0) o_gemm(-1., 1., B, U + d, B + (int64_t)d * ld_b, d, n, md, ld_b, ld_u, ld_b, false, false);
  }
}

void o_gemm3(double alpha, double beta, double* M, const double* A, const double* B, const double* C, int m, int n,
             int k, int l, int ld_m, int ld_a, int ld_b, int ld_c, bool a_T, bool b_T, bool c_T, int control,
             double* tmp) {
  double* t1 = tmp;
  if (control) {
    o_gemm(1., 0., t1, A, B, m, l, k, l, ld_a, ld_b, a_T, b_T);
    o_gemm(alpha, beta, M, t1, C, m, n, l, ld_m, l, ld_c, false, c_T);
  } else {
    o_gemm(1., 0., t1, B, C, k, n, l, n, ld_b, ld_c, b_T, c_T);
    o_gemm(alpha, beta, M, A, t1, m, n, k, ld_m, ld_a, n, a_T, false);
  }
}

void o_gemm4(double alpha, double beta, double* M, const double* A, const double* B, const double* C, const double* D,
             int m, int n, int k, int l, int o, int ld_m, int ld_a, int ld_b, int ld_c, int ld_d, bool a_T, bool b_T,
             bool c_T, bool d_T, int control, int offset, double* tmp) {
  double *t1 = tmp, *t2 = tmp + offset;
  switch (control) {
    case 0:
      o_gemm(1., 0., t1, A, B, m, l, k, l, ld_a, ld_b, a_T, b_T);
      o_gemm(1., 0., t2, t1, C, m, o, l, o, l, ld_c, false, c_T);
      o_gemm(alpha, beta, M, t2, D, m, n, o, ld_m, o, ld_d, false, d_T);
      break;
    case 1:
      o_gemm(1., 0., t1, B, C, k, o, l, o, ld_b, ld_c, b_T, c_T);
      o_gemm(1., 0., t2, A, t1, m, o, k, o, ld_a, o, a_T, false);
      o_gemm(alpha, beta, M, t2, D, m, n, o, ld_m, o, ld_d, false, d_T);
      break;
    case 2:
      o_gemm(1., 0., t1, B, C, k, o, l, o, ld_b, ld_c, b_T, c_T);
      o_gemm(1., 0., t2, t1, D, k, n, o, n, o, ld_d, false, d_T);
      o_gemm(alpha, beta, M, A, t2, m, n, k, ld_m, ld_a, n, a_T, false);
      break;
    case 3:
      o_gemm(1., 0., t1, C, D, l, n, o, n, ld_c, ld_d, c_T, d_T);
      o_gemm(1., 0., t2, B, t1, k, n, l, n, ld_b, n, b_T, false);
      o_gemm(alpha, beta, M, A, t2, m, n, k, ld_m, ld_a, n, a_T, false);
      break;
    case 4:
      o_gemm(1., 0., t1, A, B, m, l, k, l, ld_a, ld_b, a_T, b_T);
      o_gemm(1., 0., t2, C, D, l, n, o, n, ld_c, ld_d, c_T, d_T);
      o_gemm(alpha, beta, M, t1, t2, m, n, l, ld_m, l, n, false, false);
      break;
    default:
      break;
  }
}

// blockGivensRotation: the reference's wavefront order (iter, then column) executed serially;
// rotations of one wavefront touch disjoint row pairs.
void o_givens(double* M, int nx, int ny, int ld) {
  const int n = nx + ny - 2;
  for (int iter = 0; iter < n; ++iter)
    for (int col = 0; col < nx; ++col) {
      const int row = ny - 2 + 2 * col - iter;
      if (!(row < ny - 1 && row >= col)) continue;
      const int row2 = row + 1;
      double* Mr = M + (int64_t)row * ld;
      double* Mr2 = M + (int64_t)row2 * ld;
      const double a = Mr[col], b = Mr2[col];
      double cosine, sine, r, p;
      if (b == 0) { cosine = std::copysign(1., a); sine = 0.; r = std::fabs(a); p = 0.; }
      else if (a == 0) { cosine = 0.; sine = std::copysign(1., b); r = std::fabs(b); p = 1.; }
      else if (std::fabs(b) > std::fabs(a)) {
        const double t = -a / b;
        sine = 1. / std::hypot(1., t);
        cosine = sine * t;
        r = -b / sine;
        p = 2. / cosine;
      } else {
        const double t = -b / a;
        cosine = 1. / std::hypot(1., t);
        sine = cosine * t;
        r = a / cosine;
        p = sine / 2.;
      }
      Mr[col] = r;
      Mr2[col] = p;
      for (int i = col + 1; i < nx; ++i) {
        const double x = Mr[i], y = Mr2[i];
        Mr[i] = std::fma(cosine, x, std::fma(-sine, y, 0.));
        Mr2[i] = std::fma(sine, x, std::fma(cosine, y, 0.));
      }
    }
}

void o_givens_q(double* Q, const double* R, int nx, int ny, int p, int ld_q, int ld_r) {
  const int n = nx + ny - 2;
  for (int row = 0; row < ny; ++row)
    for (int col = 0; col < p; ++col) Q[(int64_t)row * ld_q + col] = (double)(row == col);
  for (int iter = 0; iter < n; ++iter)
    for (int col = 0; col < nx; ++col) {
      const int row = 2 * col + 1 - nx + iter;
      if (!(row < ny - 1 && row >= col)) continue;
      const int row2 = row + 1;
      double* Qr = Q + (int64_t)row * ld_q;
      double* Qr2 = Q + (int64_t)row2 * ld_q;
      const double pv = R[(int64_t)row2 * ld_r + col];
      double cosine, sine;
      if (pv == 0) { cosine = 1.; sine = 0.; }
      else if (pv == 1) { cosine = 0.; sine = 1.; }
      else if (std::fabs(pv) > 2) { cosine = 2. / pv; sine = std::sqrt(std::fma(cosine, -cosine, 1.)); }
      else { sine = 2. * pv; cosine = std::sqrt(std::fma(sine, -sine, 1.)); }
      for (int i = col; i < p; ++i) {
        const double a = Qr[i], b = Qr2[i];
        Qr[i] = std::fma(cosine, a, std::fma(sine, b, 0.));
        Qr2[i] = std::fma(-sine, a, std::fma(cosine, b, 0.));
      }
    }
}

// blockLowRankAccum with an optional sign on the added term (the reference adds with +1)
void o_accum(double* U1, double* VT1, const double* U2, const double* VT2, int nx, int ny, int k1, int k2, int ld_u1,
             int ld_vt1, int ld_u2, int ld_vt2, bool t_u2, bool t_vt2, double sign, const double* rnd, int ld_r) {
  std::vector<double> Ub((size_t)ny * k1), Vb((size_t)nx * k1),
      Qb((size_t)std::max<int64_t>((int64_t)ny * k1, (int64_t)k1 * std::max(k1, k2)));
  double *U = Ub.data(), *V = Vb.data(), *Q = Qb.data();
  o_gemm(1., 0., Q, rnd, VT1, k1, k1, nx, k1, ld_r, ld_vt1, true, false);
  o_gemm(1., 0., U, U1, Q, ny, k1, k1, k1, ld_u1, k1, false, true);
  o_gemm(1., 0., Q, rnd, VT2, k1, k2, nx, k2, ld_r, ld_vt2, true, t_vt2);
  o_gemm(sign, 1., U, U2, Q, ny, k1, k2, k1, ld_u2, k2, t_u2, true);
  o_givens(U, k1, ny, k1);
  o_givens_q(Q, U, k1, ny, k1, k1, k1);
  o_gemm(1., 0., U, Q, U1, k1, k1, ny, k1, k1, ld_u1, true, false);
  o_gemm(1., 0., V, VT1, U, nx, k1, k1, k1, ld_vt1, k1, false, true);
  for (int r = 0; r < ny; ++r)
    for (int c = 0; c < k1; ++c) U1[(int64_t)r * ld_u1 + c] = Q[(int64_t)r * k1 + c];
  o_gemm(1., 0., U, Q, U2, k1, k2, ny, k2, k1, ld_u2, true, t_u2);
  o_gemm(sign, 1., V, VT2, U, nx, k1, k2, k1, ld_vt2, k2, t_vt2, true);
  for (int r = 0; r < nx; ++r)
    for (int c = 0; c < k1; ++c) VT1[(int64_t)r * ld_vt1 + c] = V[(int64_t)r * k1 + c];
}

// Y := Y C^-1 with G = Y^T Y (+ shift) = C^T C, three passes (the first shifted by
// 11 (m k + k (k + 1)) u ||Y||_F^2): the range finder of the engine's sketched updates
void o_cholqr3(double* Y, int m, int k) {
  std::vector<double> G((size_t)k * k);
  for (int pass = 0; pass < 3; ++pass) {
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        double s = 0.0;
        for (int r = 0; r < m; ++r) s += Y[(int64_t)r * k + i] * Y[(int64_t)r * k + j];
        G[(size_t)i * k + j] = s;
      }
    double tr = 0.0;
    for (int j = 0; j < k; ++j) tr += G[(size_t)j * k + j];
    if (pass == 0) {
      const double sh = 11.0 * ((double)m * k + (double)k * (k + 1)) * 1.1102230246251565e-16 * tr;
      for (int j = 0; j < k; ++j) G[(size_t)j * k + j] += sh;
    }
    const double tiny = 1e-28 * tr;
    std::vector<double> rinv(k);
    for (int j = 0; j < k; ++j) {  // upper Cholesky factor in place (rows j, columns >= j)
      const double d = G[(size_t)j * k + j];
      const bool live = d > tiny;
      const double rjj = live ? std::sqrt(d) : 0.0;
      G[(size_t)j * k + j] = rjj;
      rinv[j] = live ? 1.0 / rjj : 0.0;
      for (int c = j + 1; c < k; ++c) G[(size_t)j * k + c] = live ? G[(size_t)j * k + c] / rjj : 0.0;
      for (int c1 = j + 1; c1 < k; ++c1)
        for (int c = c1; c < k; ++c) G[(size_t)c1 * k + c] -= G[(size_t)j * k + c1] * G[(size_t)j * k + c];
    }
    for (int r = 0; r < m; ++r) {
      double* y = Y + (int64_t)r * k;
      for (int j = 0; j < k; ++j) {
        double s = y[j];
        for (int p = 0; p < j; ++p) s -= y[p] * G[(size_t)p * k + j];
        y[j] = s * rinv[j];
      }
    }
  }
}

// ---------------------------------------------------------------- BF16 shadows (engine only)
// Round to nearest even: FP64 -> FP32 (the hardware conversion), then FP32 -> BF16 by adding
// 0x7FFF plus the lowest kept bit to the bit pattern and truncating (finite values; NaN kept
// quiet).
uint16_t to_bf16(double x) {
  const float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)((u >> 16) | ((u & 0xFFFFu) ? 0x40u : 0u));
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
double from_bf16(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return (double)f;
}
// byte offset of element (r, c) of an R x K operand in the tiled layout (pp_task.h) with chunks of
// cr rows x 64 columns
inline int64_t tiled_at(int r, int c, int K, int cr) {
  const int64_t chunk = (int64_t)(r / cr) * (K / 64) + c / 64;
  const int rr = r % cr, cc = c % 64;
  return chunk * (int64_t)cr * 128 + ((cc / 8) * (cr / 8) + rr / 8) * 128 + (rr % 8) * 16 + (cc % 8) * 2;
}

int run_one(const pp_task& T, std::vector<double>& tmp) {
  const bool t1 = T.flags & PP_T(1), t2 = T.flags & PP_T(2), t3 = T.flags & PP_T(3), t4 = T.flags & PP_T(4);
  switch (T.op) {
    case PP_OP_NOP: return 0;
    case PP_OP_GETRF:
      if (T.flags & PP_PIVOT) {
        if (!T.p[1]) return -1;
        o_getrf_piv(T.p[0], T.n, T.m, T.ld[0], T.p[1]);
      } else {
        o_getrf(T.p[0], T.n, T.m, T.ld[0]);
      }
      return 0;
    case PP_OP_TRSML:
      if (T.flags & PP_PIVOT) {
        if (!T.p[2]) return -1;
        for (int i = 0; i < T.m; ++i)
          if (!(T.p[2][i] >= 0.0 && T.p[2][i] < T.m)) return -1;
        o_permute_rows(T.p[0], T.p[2], T.n, T.m, T.ld[0]);
      }
      o_trsml(T.p[0], T.p[1], T.n, T.m, T.m, T.ld[0], T.ld[1]);
      return 0;
    case PP_OP_TRSMR: o_trsmr(T.p[0], T.p[1], T.n, T.m, T.n, T.ld[0], T.ld[1]); return 0;
    case PP_OP_TRSMRT: o_trsmrt(T.p[0], T.p[1], T.m, T.n, T.m, T.ld[0], T.ld[1]); return 0;
    case PP_OP_TRSMU: o_trsmu(T.p[0], T.p[1], T.m, T.n, T.ld[0], T.ld[1]); return 0;
    case PP_OP_GEMM:
      if (T.prec == PP_PREC_BF16) {  // engine instruction: products of the BF16 shadows, FP64 sums
        // a second pair (p[3], p[4], inner dimension l) adds its products to the same sums
        if (T.m % 128 || T.n % 32 || T.k % 64 || T.l < 0 || T.l % 64 || (T.l > 0 && (!T.p[3] || !T.p[4]))) return -1;
        const int bcr = T.n % 256 == 0 ? 128 : (T.n < 128 ? T.n : 128);  // the B shadow's chunk rows
        const uint8_t* As = reinterpret_cast<const uint8_t*>(T.p[1]);
        const uint8_t* Bs = reinterpret_cast<const uint8_t*>(T.p[2]);
        const uint8_t* As2 = reinterpret_cast<const uint8_t*>(T.p[3]);
        const uint8_t* Bs2 = reinterpret_cast<const uint8_t*>(T.p[4]);
        for (int r = 0; r < T.m; ++r)
          for (int c = 0; c < T.n; ++c) {
            double s = 0.0;
            for (int q = 0; q < T.k; ++q) {
              uint16_t a, b;
              std::memcpy(&a, As + tiled_at(r, q, T.k, 128), 2);
              std::memcpy(&b, Bs + tiled_at(c, q, T.k, bcr), 2);
              s += from_bf16(a) * from_bf16(b);
            }
            for (int q = 0; q < T.l; ++q) {
              uint16_t a, b;
              std::memcpy(&a, As2 + tiled_at(r, q, T.l, 128), 2);
              std::memcpy(&b, Bs2 + tiled_at(c, q, T.l, bcr), 2);
              s += from_bf16(a) * from_bf16(b);
            }
            double& x = T.p[0][(int64_t)r * T.ld[0] + c];
            x = (T.beta != 0.0 ? x : 0.0) + T.alpha * s;
          }
        return 0;
      }
      o_gemm(T.alpha, T.beta, T.p[0], T.p[1], T.p[2], T.m, T.n, T.k, T.ld[0], T.ld[1], T.ld[2], t1, t2);
      return 0;
    case PP_OP_SHADOW: {  // engine instruction: BF16 copy of an operand in the tiled layout
      const int cr = T.ctrl ? T.ctrl : 128;  // chunk rows of the layout
      if (T.m % cr || T.k % 64) return -1;
      // split shadow (pp_task.h PP_SPLIT_*): nseg copies of the source columns, bf16(x) or the
      // residual bf16(x - bf16(x)) where the segment's bit of the low mask is set
      const int nseg = T.o ? T.o >> 8 : 1, lo_mask = T.o & 0xFF;
      if (T.o && (nseg != 3 || T.k % (64 * nseg))) return -1;
      const int ks = T.k / nseg;
      uint8_t* S = reinterpret_cast<uint8_t*>(T.p[0]);
      const int mr = T.l > 0 ? T.l : T.m, nc = T.n > 0 ? T.n : ks;  // source rows / columns; zeros beyond
      for (int r = 0; r < T.m; ++r)
        for (int c = 0; c < ks; ++c) {
          const double x = (r >= mr || c >= nc) ? 0.0
                           : t1 ? T.p[1][(int64_t)c * T.ld[1] + r] : T.p[1][(int64_t)r * T.ld[1] + c];
          const uint16_t h = to_bf16(x);
          const uint16_t lo = to_bf16(x - from_bf16(h));
          for (int sg = 0; sg < nseg; ++sg) {
            const uint16_t v = ((lo_mask >> sg) & 1) ? lo : h;
            std::memcpy(S + tiled_at(r, c + sg * ks, T.k, cr), &v, 2);
          }
        }
      return 0;
    }
    case PP_OP_GEMM3: {
      const int64_t need = T.ctrl ? (int64_t)T.m * T.l : (int64_t)T.k * T.n;
      if ((int64_t)tmp.size() < need) tmp.resize(need);
      o_gemm3(T.alpha, 1., T.p[0], T.p[1], T.p[2], T.p[3], T.m, T.n, T.k, T.l, T.ld[0], T.ld[1], T.ld[2], T.ld[3], t1, t2,
              t3, T.ctrl, tmp.data());
      return 0;
    }
    case PP_OP_GEMM4: {
      const int64_t big = (int64_t)std::max({T.m, T.k, T.l}) * std::max({T.n, T.l, T.o});
      if ((int64_t)tmp.size() < (int64_t)T.aux + big) tmp.resize((size_t)T.aux + big);
      o_gemm4(T.alpha, 1., T.p[0], T.p[1], T.p[2], T.p[3], T.p[4], T.m, T.n, T.k, T.l, T.o, T.ld[0], T.ld[1], T.ld[2],
              T.ld[3], T.ld[4], t1, t2, t3, t4, T.ctrl, T.aux, tmp.data());
      return 0;
    }
    case PP_OP_ACCUM:
      o_accum(T.p[0], T.p[1], T.p[2], T.p[3], T.n, T.m, T.k, T.l, T.ld[0], T.ld[1], T.ld[2], T.ld[3], t2, t3, T.alpha,
              T.p[4], T.ld[4]);
      return 0;
    case PP_OP_SUM:  // reduction of split-k partial products (engine instruction, p ascending)
      for (int r = 0; r < T.m; ++r)
        for (int c = 0; c < T.n; ++c) {
          double s = 0.0;
          for (int p = 0; p < T.k; ++p) s += T.p[1][(int64_t)(p * T.m + r) * T.ld[1] + c];
          double& q = T.p[0][(int64_t)r * T.ld[0] + c];
          q = T.beta != 0.0 ? q + s : s;
        }
      return 0;
    case PP_OP_TRINV: {  // engine instruction: identity columns, then the blocked sweep
      const int m = T.m, w = T.n, c0 = T.o, ldi = T.ld[0], lda = T.ld[1];
      double* I = T.p[0];
      for (int r = 0; r < m; ++r)
        for (int j = 0; j < w; ++j) I[(int64_t)r * ldi + j] = r == c0 + j ? 1.0 : 0.0;
      if (T.ctrl == 0)
        o_trsml(I + (int64_t)c0 * ldi, T.p[1] + (int64_t)c0 * lda + c0, w, m - c0, m - c0, ldi, lda);
      else
        o_trsmu(I, T.p[1], c0 + w, w, ldi, lda);
      return 0;
    }
    case PP_OP_TRMV: {  // engine instruction: B := M B, M triangular (ascending column sums);
                        // l > 0: rows [o, o + l) of M S (S at p[2]) into p[0]
      const int m = T.m, n = T.n, ldm = T.ld[1];
      const bool part = T.l > 0;
      const double* S = part ? T.p[2] : T.p[0];
      const int lds = part ? T.ld[2] : T.ld[0], r0 = part ? T.o : 0, r1 = part ? T.o + T.l : m;
      if (r0 < 0 || r1 > m || !S) return -1;
      std::vector<double> out((size_t)(r1 - r0) * n);
      for (int r = r0; r < r1; ++r)
        for (int q = 0; q < n; ++q) {
          double s = 0.0;
          const int c_lo = T.ctrl ? r : 0, c_hi = T.ctrl ? m : r + 1;
          for (int c = c_lo; c < c_hi; ++c) s = std::fma(T.p[1][(int64_t)r * ldm + c], S[(int64_t)c * lds + q], s);
          out[(size_t)(r - r0) * n + q] = s;
        }
      for (int r = r0; r < r1; ++r)
        for (int q = 0; q < n; ++q) T.p[0][(int64_t)(r - r0) * T.ld[0] + q] = out[(size_t)(r - r0) * n + q];
      return 0;
    }
    case PP_OP_ORTH: {  // engine instruction: shifted CholeskyQR3 of Y (m x k, ld k)
      o_cholqr3(T.p[0], T.m, T.n);
      return 0;
    }
    case PP_OP_COPY:
      for (int r = 0; r < T.m; ++r)
        for (int c = 0; c < T.n; ++c) T.p[0][(int64_t)r * T.ld[0] + c] = T.p[1][(int64_t)r * T.ld[1] + c];
      return 0;
    default: return -1;
  }
}

}  // namespace

extern "C" {

// Runs n tasks in program order (a valid topological order of their DAG).
int oracle_run_program(const pp_task* tasks, int n) {
  std::vector<double> tmp;
  for (int i = 0; i < n; ++i)
    if (run_one(tasks[i], tmp) != 0) return i + 1;
  return 0;
}

// Runs n tasks over their DAG with `threads` host threads: a task starts when its
// in-degree counter reaches zero (the CPU baseline timed beside the GPU).
int oracle_run_parallel(const pp_task* tasks, int n, const int32_t* succ, const int32_t* indeg, int threads) {
  if (threads <= 1) return oracle_run_program(tasks, n);
  std::vector<std::atomic<int>> cnt(n);
  std::deque<int> ready;
  for (int i = 0; i < n; ++i) {
    cnt[i].store(indeg[i]);
    if (indeg[i] == 0) ready.push_back(i);
  }
  std::mutex mu;
  std::condition_variable cv;
  int done = 0, bad = 0;
  auto worker = [&]() {
    std::vector<double> tmp;
    for (;;) {
      int t;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !ready.empty() || done == n || bad; });
        if (done == n || bad) return;
        t = ready.front();
        ready.pop_front();
      }
      const int rc = run_one(tasks[t], tmp);
      std::vector<int> fresh;
      for (int q = 0; q < tasks[t].n_succ; ++q) {
        const int s = succ[tasks[t].succ_begin + q];
        if (cnt[s].fetch_sub(1) == 1) fresh.push_back(s);
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        if (rc) bad = t + 1;
        for (int s : fresh) ready.push_back(s);
        ++done;
      }
      cv.notify_all();
    }
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  return bad;
}

// Whole-matrix textbook right-looking LU without pivoting (the order every blocking of
// the reference reproduces element by element).
void oracle_dense_getrf(double* A, int n, int lda) { o_getrf(A, n, n, lda); }

// One block's LU with partial pivoting (the engine's PP_PIVOT GETRF); perm: n doubles.
void oracle_getrf_piv(double* A, int n, int lda, double* perm) { o_getrf_piv(A, n, n, lda, perm); }

// Single routines, for unit tests against the CUDA path.
void oracle_gemm(double alpha, double beta, double* M, const double* A, const double* B, int m, int n, int k, int ld_m,
                 int ld_a, int ld_b, int a_T, int b_T) {
  o_gemm(alpha, beta, M, A, B, m, n, k, ld_m, ld_a, ld_b, a_T != 0, b_T != 0);
}
void oracle_accum(double* U1, double* VT1, const double* U2, const double* VT2, int nx, int ny, int k1, int k2,
                  int ld_u1, int ld_vt1, int ld_u2, int ld_vt2, double sign, const double* rnd, int ld_r) {
  o_accum(U1, VT1, U2, VT2, nx, ny, k1, k2, ld_u1, ld_vt1, ld_u2, ld_vt2, false, false, sign, rnd, ld_r);
}

}  // extern "C"
