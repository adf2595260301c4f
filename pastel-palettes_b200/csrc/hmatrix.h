// hmatrix.h — Dense blocks and the Hierarchical block tree.
//
// Mirrors Pastel-Palettes matrix/Dense.h:6-18 (Dense(m, n, lda) owning `double* a`)
// and the Hierarchical interface the reference's launcher uses
// (src/launcher.cu:126,138-139: getNy_abs / getNx_abs / getRootIndex /
// generateOps_GETRF; the class itself is an empty stub at matrix/Hierarchical.h:4-7).
//
// Storage convention: row-major, as the reference's VM kernel reads blocks
// (`M[row * ld + col]`, src/kernel.cu:42).  (matrix/Dense.cpp:10 allocates
// column-major; this engine transposes at the boundary instead.)  Every block of one
// H-matrix lives in one arena: dense leaves as m x n (ld n), low-rank blocks as
// U (m x kmax) and V (n x kmax), the block equal to U V^T.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pp {

class Dense {
 public:
  int64_t m, n, lda;
  double* a;
  Dense(int64_t m, int64_t n, int64_t lda);  // lda := max(n, lda) (row-major)
  ~Dense();
  Dense(const Dense&) = delete;
  Dense& operator=(const Dense&) = delete;
};

struct StorageObj {
  int64_t off;  // element offset in the arena
  int rows, cols, ld;
};

struct HNode {
  enum Kind : int { D = 0, LR = 1, H = 2 };
  Kind kind;
  int r0, c0, m, n;  // rows [r0, r0+m), columns [c0, c0+n) of the whole matrix
  int level;
  int obj = -1;      // D: the block; LR: U
  int objV = -1;     // LR: V
  int rank = 0;      // LR: columns the instructions use (kmax in the adaptive-rank mode)
  int rank_obj = -1; // LR: one-element object holding the block's numerical rank
  int kmax = 0;      // LR: storage capacity (columns of U and V)
  int ch[4] = {-1, -1, -1, -1};  // H: children, row-major 2 x 2
  int invL = -1, invU = -1;      // D on the diagonal: L^-1 and U^-1 of its factors (solve)
  int piv = -1;                  // D on the diagonal: m x 1 row permutations of its pivoted
                                 // factorization (one per GETRF tile, tile-local indices)
};

class Hierarchical {
 public:
  int n = 0;
  int root = -1;
  std::vector<HNode> nodes;
  std::vector<StorageObj> objs;
  int64_t arena_elems = 0;
  // adaptive-rank mode (rank_tol > 0): low-rank blocks keep kmax columns, zero beyond their
  // numerical rank; the accumulations truncate to the singular values above rank_tol times
  // the largest and record the new rank in the block's rank object
  double rank_tol = 0.0;
  // the matrix blocks (and the per-block rank words) occupy the arena prefix
  // [0, block_elems); the tail holds the explicit
  // inverses of the diagonal leaves' triangular factors, which the factorization writes and
  // the solves read (never uploaded, downloaded or restored)
  int64_t block_elems = 0;
  // dimension of the points a geometric tree was built on (0: the all-dense tree)
  int point_dim = 0;
  // host image of the arena (filled by set_dense / set_lowrank), allocated at its first use
  // (ensure_host): a matrix built on the device never needs one
  mutable std::vector<double> host;
  void ensure_host() const;

  // All-dense 2x2 partition of an n x n matrix down to blocks of <= leaf rows.
  static Hierarchical* dense_tiled(int n, int leaf);
  // Geometric block tree over points already in cluster order (e.g. Morton-sorted):
  // clusters halve index ranges down to <= leaf points; a block (t, s) is low-rank
  // when admissible — weak (adm == 0): t != s; standard (adm == 1):
  // eta * max(diam t, diam s) <= dist(t, s) over bounding boxes.
  static Hierarchical* geometric(int n, int dim, const double* points, int leaf, int adm, double eta,
                                 int kmax);

  int getNy_abs() const { return n; }
  int getNx_abs() const { return n; }
  int getRootIndex() const { return root; }
  int count(HNode::Kind k) const;
  int depth() const;

  void set_dense(int node, const double* a, int lda);  // row-major m x n
  void set_lowrank(int node, const double* U, int ldu, const double* V, int ldv, int rank);
  // dense reconstruction of the whole matrix from the host image (tests, small n)
  void to_dense(double* out) const;
  // bytes of matrix data (dense entries + rank * (m + n) for low-rank blocks)
  int64_t storage_elems() const;

 private:
  int add_obj(int rows, int cols);
  // appends the rank words of the low-rank blocks (arena prefix), then the L^-1 / U^-1
  // objects for every square diagonal dense leaf of at most kInvMax rows (arena tail)
  void add_inverses();
 public:
  // numerical rank of a low-rank block as stored in the host image
  int stored_rank(int node) const;
  void set_rank_tolerance(double tol);
};

// largest diagonal leaf whose triangular factors get explicit inverses
constexpr int kInvMax = 512;

}  // namespace pp
