// hops.h — H-LU operation generator, task program, DAG and encoders.
//
// Covers the reference's missing h_ops/* (h-op tree generation, DAG flattening) and
// instructions/* (instruction encoding) layers, whose interfaces are visible at
// Pastel-Palettes src/launcher.cu:46-90,138-139 and rts/scheduler.cpp:73-77.
//
// The generator walks the block tree the way the reference's H-LU does
// (docs: GETRF -> TRSM L / TRSM R -> GEMM -> GETRF on the trailing block, recursively)
// and emits instructions of the reference's instruction set (getrf, trsml, trsmr with
// and without transposed B, gemm, gemm_plus, accum), on blocks of at most `tile` rows
// and columns for the dense parts.  Intermediate low-rank products go to zero-filled
// work buffers, the sign folded into them exactly as a reference stream would have to
// (gemm: M -= A B, gemm_plus: M += A B, accum: U1 V1^T += U2 V2^T), so every program
// of a factorization is also a valid reference instruction stream.  Only the solve
// uses one instruction the reference lacks (TRSMU: B := U^-1 B).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "hmatrix.h"
#include "pp_task.h"
#include "rts.h"

namespace pp {

// arena kinds; arena id = instance * PP_ARENAS + kind
enum ArenaKind { AR_MATRIX = 0, AR_WORK = 1, AR_SCRATCH = 2, AR_RHS = 3, AR_RAND = 4, PP_ARENAS = 5 };

struct PObj {
  int arena;
  int64_t off;  // element offset of storage (0, 0) in the arena
  int rows, cols, ld;
  bool tracked;  // false: read-only inputs the DAG can ignore (random sketch)
};

// Dense operand: logical m x n; logical (i, j) lives at storage (r0 + i, c0 + j) of
// object `obj`, or at storage (r0 + j, c0 + i) when `t` (transposed view).
struct View {
  int obj = -1;
  int r0 = 0, c0 = 0;
  int m = 0, n = 0;
  bool t = false;
  View sub(int i, int j, int mm, int nn) const;
  View T() const;
  int srows() const { return t ? n : m; }
  int scols() const { return t ? m : n; }
};

// Operand of the recursive generator: dense view, low-rank pair, or H node.
struct Mat {
  enum Kind { D = 0, LR = 1, H = 2 } kind = D;
  int m = 0, n = 0;
  int rank_obj = -1;  // LR: program object of the block's rank word
  View d;          // D
  View u, v;       // LR: block = u v^T, u: m x k, v: n x k
  int k = 0;
  int node = -1;   // H: node of the instance's tree
  bool tr = false; // H: transposed
};

struct Region {
  int obj;
  int r0, c0, nr, nc;
  bool ro;
};

struct HTask {
  pp_task t{};           // pointers filled at encode time
  View opnd[6];
  bool has[6] = {false, false, false, false, false, false};
  int64_t scratch_elems = 0, scratch_off = 0;
  std::vector<Region> regions;
  int64_t flops = 0;
};

class Program {
 public:
  int n_instances = 0;
  std::vector<PObj> objs;
  std::vector<HTask> tasks;
  std::vector<int64_t> arena_elems;  // per arena id
  // DAG over tasks (program order is topological)
  std::vector<std::vector<int>> succ, pred;
  std::vector<std::vector<uint8_t>> pred_bits;  // dependency_t bits of each pred edge
  // the typed edges as the reference's dependency_table (rts/dependency.h), built on request
  const dependency_table& dep_table();
  std::vector<int64_t> blevel;  // FLOP-weighted longest path to an exit
  int64_t edges = 0;
 private:
  dependency_table deps_;
  bool deps_built_ = false;
 public:

  int add_instance();  // returns instance id
  int add_obj(int arena, int rows, int cols, bool tracked = true);
  int add_obj_at(int arena, int64_t off, int rows, int cols, int ld, bool tracked);
  int arena_id(int inst, int kind) const { return inst * PP_ARENAS + kind; }
  int64_t total_flops() const;
  int64_t aux_flops() const;
  int64_t count_op(int op) const;
  // Contraction precision of every GEMM instruction (PP_PREC_TF32: tensor cores with FP32
  // accumulation; GETRF, TRSM*, ACCUM and SUM stay FP64).  Returns the tasks changed.
  int64_t set_gemm_precision(int prec);
  // the mixed form's BF16 updates of one target that follow each other with nothing else
  // touching the target in between become one task with two operand pairs (one pass over the
  // target instead of two); returns the number of merges.  Call before build_dag.
  int64_t merge_bf16_updates();

  void build_dag();
  // bottom levels (and a fresh dependency table) once succ / pred / pred_bits are set
  void finish_dag();
  h_ops_dag to_dag() const;
  // Pointer binding and device-table encoding.  bases[arena id] = base address.
  void encode(const std::vector<double*>& bases, std::vector<pp_task>& out, std::vector<int32_t>& succ_out,
              std::vector<int32_t>& indeg_out, std::vector<int32_t>& ready_out) const;
  // Append all tasks of `other` (another instance's program); arenas are renumbered.
  void merge(const Program& other);

  // Reference-format per-worker streams (format of src/kernel.cu:1384-1522).
  // ptr_bases: index into the reference's `void** ptrs` for each arena id.
  bool encode_reference(int workers, std::vector<std::vector<int32_t>>& streams, std::string& err,
                        int64_t* tmp_elems_per_worker) const;
};

// The same DAG as Program::build_dag, with the dependency discovery on the current CUDA device
// (dag.cu).  Returns false with `err` set when it cannot (a CUDA error, or a dependency walk
// with more partial writes than it keeps); the caller then builds on the host.  device_ms: wall
// time of the device part (upload, walks, sort, download).
bool build_dag_device(Program& prog, std::string& err, double* device_ms);

// largest triangle of one solve-phase TRSML / TRSMU instruction (the VM's blocked
// triangular routines take up to 256 rows)
constexpr int kSolveTri = 256;
// right-hand-side columns of one TRMV instruction
constexpr int kTrmvCols = 16;
// a leaf product M B on triangles of at least kTrmvSplitMin rows is split into kTrmvParts row
// blocks of equal triangle area (one CTA each, into a work buffer) and a copy back: the solve's
// critical path then waits for a quarter of the triangle's loads instead of all of them
constexpr int kTrmvSplitMin = 128;
constexpr int kTrmvParts = 4;
constexpr int kTrmvPartRows = 64;
// rows of one product instruction of the solve with at most 16 columns: every row slice of a
// right-hand-side block is a dependency chain of its own (the updates of one slice are ordered,
// of different slices not).  Products with a leaf of kBigLeaf columns or more take 64-row
// instructions, which stream their slice of a 512-column leaf in four rounds of loads per warp,
// so the chains of a single job's critical path advance four times faster than with 256 rows;
// the others keep 256 rows (low-rank factors are short, and batched jobs of smaller leaves have
// parallelism enough, where fewer instructions cost less)
constexpr int kSolveGemmRowsBig = 64;
constexpr int kSolveGemmRows = 256;
// largest rank of the added term of one ACCUM (the VM keeps it in registers)
constexpr int kAccumMaxK2 = 32;
// smallest m, n and k of a GEMM instruction the TF32 form runs on the tensor cores
constexpr int kTcMinDim = 64;
// products of whole dense leaves of at least kBigLeaf rows and columns are one instruction
// each (a Schur update of large leaves); their triangular solves take triangles of kBigTri rows
constexpr int kBigLeaf = 512;
constexpr int kBigTri = 256;

class Generator {
 public:
  // Builds programs on one H-matrix instance.  `tile`: dense blocks larger than this
  // are split (2 x 2) before they reach an instruction.
  // `split_k`: small products over a long k become partial products on many CTAs plus a
  // SUM reduction (an engine instruction the reference's set does not have)
  Generator(Program& P, Hierarchical& H, int tile, int max_n_rand, bool split_k = true);
  int inst() const { return inst_; }
  void getrf_program();            // H-LU factorization of the whole matrix
  // explicit inverses of the diagonal leaves' triangular factors (TRINV), which the solve
  // program then applies with TRMV instead of substituting; set before building programs
  void use_inverses(bool on) { inverses_ = on && !pivot_; }
  // partial pivoting inside every GETRF block (PP_PIVOT), applied lazily by the TRSML
  // instructions against that block; the solves then substitute (no explicit inverses)
  void use_pivoting(bool on) {
    pivot_ = on;
    if (on) inverses_ = false;
  }
  // edge of the output tiles products are split into (64 or 128; larger tiles: fewer, longer
  // tasks)
  void set_gemm_tile(int t) { gemm_tile_ = t >= 128 ? 128 : 64; }
  // contraction precision of the whole-leaf Schur updates: PP_PREC_BF16 runs them on the tensor
  // cores from BF16 shadows of their operands (SHADOW instructions, one per operand block,
  // emitted at its first use); the other instructions stay FP64
  void set_precision(int prec) { prec_ = prec; }
  void solve_program(int nrhs);    // B := U^-1 L^-1 B on the RHS object (n x nrhs)
  // Device construction of the low-rank blocks from points (the RHS arena holds the n x dim
  // points): per block a randomized range finder with one power step, U = orth(K Omega),
  // V = K^T orth(K orth(K^T U)) ..., then truncation of U V^T to the singular values above
  // `tol` times the largest (at most the block's rank); kernel as PP_OP_KMUL
  void construct_program(int kernel, int dim, double p0, double tol);
  int rhs_obj() const { return rhs_obj_; }

  // building blocks (exposed for tests)
  Mat node(int id, bool tr = false) const;
  void getrf(const Mat& A);
  void trsml(const Mat& L, const Mat& B);
  void trsmr(const Mat& U, const Mat& B);
  void trsmrt(const Mat& U, const View& V);
  void trsmu(const Mat& U, const Mat& B);
  void gemm(const Mat& C, const Mat& A, const Mat& B, int alpha);

 private:
  Program& P_;
  Hierarchical& H_;
  int inst_;
  int T_;
  int rand_ld_obj_[64 + 1];
  std::vector<int> node_obj_;  // Hierarchical obj -> program obj
  int rhs_obj_ = -1;
  int max_n_rand_;
  bool split_k_;
  bool inverses_ = false;
  bool pivot_ = false;
  std::vector<int> piv_obj_;  // program object of a diagonal leaf -> its pivot object (or -1)
  View pivot_view(const View& tile) const;
  int gemm_tile_ = 64;
  bool solve_ = false;  // building a solve program
  int prec_ = PP_PREC_FP64;
  // shadow object of an operand view (obj, r0, c0, m, n, t), dropped when the object is written
  struct ShadowKey {
    int obj, r0, c0, m, n;
    bool t;
    int cr, split;
    bool operator==(const ShadowKey& o) const {
      return obj == o.obj && r0 == o.r0 && c0 == o.c0 && m == o.m && n == o.n && t == o.t && cr == o.cr &&
             split == o.split;
    }
  };
  std::vector<std::vector<std::pair<ShadowKey, int>>> shadows_;  // per program object
  // the shadow of X in the tiled layout with chunks of cr rows (128 for an A operand; for a B
  // operand 128 or its row count), columns padded with zeros to a multiple of 64; split: 0, or
  // PP_SPLIT_A / PP_SPLIT_B (three segments of the padded columns, pp_task.h)
  View shadow_of(const View& X, int cr = 128, int split = 0);
  bool bf16_product(const View& C, const View& A, const View& B, int alpha);
  // C := A B from split shadows (about 2^-16 accurate), C possibly aliasing A or B; false when
  // the shapes do not fit the BF16 GEMM
  bool split_product(const View& C, const View& A, const View& B, int64_t flops);
  // the mixed form's triangular solves of a factorization against a whole diagonal leaf of
  // kBigLeaf or more: the product with the leaf's explicit inverse (its TRINV tasks emitted
  // right after the leaf's GETRF) as one split-shadow product; returns the inverse objects
  bool mixed_inverse(const Mat& T, int& invL, int& invU) const;
  void emit_inverse(int leaf_obj, int m);
  std::vector<char> inv_done_;  // program obj of a diagonal leaf -> its TRINV tasks are emitted
  bool whole_leaf(const View& v) const;
  int tri_limit(int target_extent) const;
  void trmv(int inv, int upper, int m, const View& B);
  void kmul(const View& C, const View& PI, const View& PJ, const View& B, int kernel, double p0);
  void orth(const View& Y);
  std::vector<std::pair<int, int>> inv_obj_;  // program obj of a diagonal leaf -> (L^-1, U^-1) objs
  bool inverse_of(const Mat& T, int& invL, int& invU) const;
  void emit_inverses();

  struct LRP { View x, y; int sign; };  // x y^T * sign
  LRP lr_product(const Mat& A, const Mat& B, int alpha);
  void lr_update(const Mat& C, const View& X, const View& Y, int sign);
  void accum(const Mat& C, const View& X, const View& Y, int sign);
  // C := rank-k recompression of C + alpha A B for hierarchical / dense operands whose
  // product has no small low-rank form (standard admissibility), by a k-column sketch
  void sketch_update(const Mat& C, const Mat& A, const Mat& B, int alpha);
  void gemm_tiles(const View& C, const View& A, const View& B, int alpha);
  View tmp(int rows, int cols);
  Mat asD(const View& v) const;
  Mat child(const Mat& X, int i, int j) const;
  int hsplit_r(const Mat& X) const;
  int hsplit_c(const Mat& X) const;
  int tri_split(const Mat& X, int limit) const;
  // largest triangle of one TRSM* instruction the generator emits: T_ (measured: 256-row
  // blocked solves lengthen the factor's critical path; the device accepts up to 256 rows,
  // which reference-format streams need)
  int Ttri_;
  void partition(const Mat& X, int rs, int cs, Mat out[2][2], int& nr, int& nc) const;
  int rand_obj(int k1);

  HTask& emit(int op);
  void bind(HTask& t, int slot, const View& v, bool write);
};

}  // namespace pp
