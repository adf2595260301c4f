// hops.cpp — H-LU operation generator, DAG construction and encoders.
#include "hops.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace pp {

// ----------------------------------------------------------------------------- views
View View::sub(int i, int j, int mm, int nn) const {
  View v = *this;
  v.m = mm;
  v.n = nn;
  if (!t) { v.r0 += i; v.c0 += j; }
  else { v.r0 += j; v.c0 += i; }
  return v;
}

View View::T() const {
  View v = *this;
  v.t = !t;
  std::swap(v.m, v.n);
  return v;
}

static Mat transpose(const Mat& X) {
  Mat Y = X;
  std::swap(Y.m, Y.n);
  if (X.kind == Mat::D) Y.d = X.d.T();
  else if (X.kind == Mat::LR) { Y.u = X.v; Y.v = X.u; }
  else Y.tr = !X.tr;
  return Y;
}

// ----------------------------------------------------------------------------- flops
static int64_t flops_getrf(int64_t m, int64_t n) {
  int64_t f = 0;
  const int64_t mn = std::min(m, n);
  for (int64_t i = 0; i < mn; ++i) f += (m - i - 1) + 2 * (m - i - 1) * (n - i - 1);
  return f;
}

// ----------------------------------------------------------------------------- program
int Program::add_instance() {
  int id = n_instances++;
  arena_elems.resize((size_t)n_instances * PP_ARENAS, 0);
  return id;
}

int Program::add_obj_at(int arena, int64_t off, int rows, int cols, int ld, bool tracked) {
  objs.push_back({arena, off, rows, cols, ld, tracked});
  return (int)objs.size() - 1;
}

int Program::add_obj(int arena, int rows, int cols, bool tracked) {
  int64_t off = (arena_elems[arena] + 3) & ~int64_t(3);
  arena_elems[arena] = off + (int64_t)rows * cols;
  return add_obj_at(arena, off, rows, cols, cols, tracked);
}

int64_t Program::total_flops() const {
  // the algorithmic count of the factorization / solve; the TRINV instructions that prepare
  // the solves' explicit inverses are accounted apart (aux_flops)
  int64_t s = 0;
  for (auto& t : tasks)
    if (t.t.op != PP_OP_TRINV) s += t.flops;
  return s;
}

int64_t Program::aux_flops() const {
  int64_t s = 0;
  for (auto& t : tasks)
    if (t.t.op == PP_OP_TRINV) s += t.flops;
  return s;
}

int64_t Program::count_op(int op) const {
  int64_t c = 0;
  for (auto& t : tasks) c += t.t.op == op;
  return c;
}

int64_t Program::set_gemm_precision(int prec) {
  // the tensor-core form pays for staging the operands (FP64 -> TF32 in shared memory) and
  // reading the accumulators back from tensor memory; only contractions of at least
  // kTcMinDim in every dimension (the dense Schur updates) gain from it, the skinny low-rank
  // products stay FP64 SIMT
  int64_t c = 0;
  for (auto& t : tasks) {
    if (t.t.op != PP_OP_GEMM) continue;
    const bool big = t.t.m >= kTcMinDim && t.t.n >= kTcMinDim && t.t.k >= kTcMinDim;
    const int want = big ? prec : PP_PREC_FP64;
    if (t.t.prec != want) {
      t.t.prec = want;
      ++c;
    }
  }
  return c;
}

// Consecutive BF16 updates of the same target C (C += alpha A1 B1, then C += alpha A2 B2, the
// second the next task after the first to touch C's object, both with one pair, the same
// alpha and beta 1, the first one's inputs not rewritten in between) become one task at the
// second one's place: C += alpha (A1 B1 + A2 B2).  Program order stays a valid sequential
// execution: nothing between the two reads or writes C, and the first one's inputs hold the
// same values at the later place.  Pairs are taken in order: (1st, 2nd), (3rd, 4th), ...
int64_t Program::merge_bf16_updates() {
  const int n = (int)tasks.size();
  std::vector<int> last(objs.size(), -1), last_w(objs.size(), -1);
  std::vector<char> dead(n, 0);
  int64_t merged = 0;
  auto single = [](const HTask& h) {
    return h.t.op == PP_OP_GEMM && h.t.prec == PP_PREC_BF16 && h.t.beta == 1.0 && h.t.l == 0 && h.has[0] &&
           h.has[1] && h.has[2] && !h.has[3] && !h.has[4];
  };
  for (int t = 0; t < n; ++t) {
    HTask& h = tasks[t];
    if (single(h)) {
      const View& C = h.opnd[0];
      const int p = last[C.obj];
      if (p >= 0 && !dead[p] && single(tasks[p])) {
        HTask& g = tasks[p];
        const View& D = g.opnd[0];
        bool ok = D.obj == C.obj && D.r0 == C.r0 && D.c0 == C.c0 && D.m == C.m && D.n == C.n && D.t == C.t &&
                  g.t.alpha == h.t.alpha && g.t.m == h.t.m && g.t.n == h.t.n && !g.opnd[1].t && !g.opnd[2].t &&
                  !h.opnd[1].t && !h.opnd[2].t;
        for (int sl = 1; sl <= 2 && ok; ++sl) ok = last_w[g.opnd[sl].obj] < p;
        if (ok) {
          h.opnd[3] = h.opnd[1];
          h.opnd[4] = h.opnd[2];
          h.has[3] = h.has[4] = true;
          h.t.ld[3] = h.t.ld[1];
          h.t.ld[4] = h.t.ld[2];
          h.opnd[1] = g.opnd[1];
          h.opnd[2] = g.opnd[2];
          h.t.ld[1] = g.t.ld[1];
          h.t.ld[2] = g.t.ld[2];
          h.t.l = h.t.k;
          h.t.k = g.t.k;
          for (const Region& r : g.regions)
            if (r.ro) h.regions.push_back(r);
          h.flops += g.flops;
          dead[p] = 1;
          ++merged;
        }
      }
    }
    for (const Region& r : h.regions) {
      last[r.obj] = t;
      if (!r.ro) last_w[r.obj] = t;
    }
  }
  if (merged) {
    std::vector<HTask> kept;
    kept.reserve(n - merged);
    for (int t = 0; t < n; ++t)
      if (!dead[t]) kept.push_back(std::move(tasks[t]));
    tasks.swap(kept);
  }
  return merged;
}

static inline bool rect_overlap(const Region& a, const Region& b) {
  return a.r0 < b.r0 + b.nr && b.r0 < a.r0 + a.nr && a.c0 < b.c0 + b.nc && b.c0 < a.c0 + a.nc;
}
static inline bool rect_covers(const Region& a, const Region& b) {
  return a.r0 <= b.r0 && b.r0 + b.nr <= a.r0 + a.nr && a.c0 <= b.c0 && b.c0 + b.nc <= a.c0 + a.nc;
}

// Program order is a valid sequential execution; an edge joins every pair of tasks
// whose regions overlap with at least one write (flow / anti / out).  Scanning an
// object's earlier accesses newest-first stops at a write that covers the current
// region: anything older that overlaps it is already ordered before that write.
// Accesses fully covered by a later write are dropped for the same reason.
void Program::build_dag() {
  const int n = (int)tasks.size();
  succ.assign(n, {});
  pred.assign(n, {});
  pred_bits.assign(n, {});
  deps_.clear();
  deps_built_ = false;
  struct Acc { int task; Region r; };
  std::vector<std::vector<Acc>> acc(objs.size());
  std::vector<int> mark(n, -1), depbits(n, 0);
  std::vector<int> touched;
  edges = 0;
  for (int t = 0; t < n; ++t) {
    touched.clear();
    for (const Region& r : tasks[t].regions) {
      auto& L = acc[r.obj];
      for (int q = (int)L.size() - 1; q >= 0; --q) {
        const Acc& a = L[q];
        if (a.task == t || !rect_overlap(a.r, r)) continue;
        int d = 0;
        if (!a.r.ro && r.ro) d |= (int)dependency_t::flow;
        if (a.r.ro && !r.ro) d |= (int)dependency_t::anti;
        if (!a.r.ro && !r.ro) d |= (int)dependency_t::out;
        if (d) {
          if (mark[a.task] != t) { mark[a.task] = t; depbits[a.task] = 0; touched.push_back(a.task); }
          depbits[a.task] |= d;
        }
        if (!a.r.ro && rect_covers(a.r, r)) break;
      }
    }
    for (const Region& r : tasks[t].regions) {
      auto& L = acc[r.obj];
      if (!r.ro)
        L.erase(std::remove_if(L.begin(), L.end(), [&](const Acc& a) { return rect_covers(r, a.r); }), L.end());
      L.push_back({t, r});
    }
    std::sort(touched.begin(), touched.end());
    for (int p : touched) {
      pred[t].push_back(p);
      pred_bits[t].push_back((uint8_t)depbits[p]);
      succ[p].push_back(t);
      ++edges;
    }
  }
  finish_dag();
}

void Program::finish_dag() {
  const int n = (int)tasks.size();
  deps_.clear();
  deps_built_ = false;
  blevel.assign(n, 0);
  for (int t = n - 1; t >= 0; --t) {
    int64_t b = 0;
    for (int s : succ[t]) b = std::max(b, blevel[s]);
    blevel[t] = b + std::max<int64_t>(tasks[t].flops, 1 << 14);
  }
}

const dependency_table& Program::dep_table() {
  if (!deps_built_) {
    deps_.clear();
    for (size_t t = 0; t < pred.size(); ++t)
      for (size_t q = 0; q < pred[t].size(); ++q) deps_.update(pred[t][q], (int64_t)t, (dependency_t)pred_bits[t][q]);
    deps_built_ = true;
  }
  return deps_;
}

h_ops_dag Program::to_dag() const {
  h_ops_dag d;
  d.length = (int)tasks.size();
  d.succ = succ;
  d.pred = pred;
  d.flops.resize(tasks.size());
  for (size_t i = 0; i < tasks.size(); ++i) d.flops[i] = tasks[i].flops;
  return d;
}

void Program::encode(const std::vector<double*>& bases, std::vector<pp_task>& out, std::vector<int32_t>& succ_out,
                     std::vector<int32_t>& indeg_out, std::vector<int32_t>& ready_out) const {
  const int n = (int)tasks.size();
  out.resize(n);
  succ_out.clear();
  indeg_out.resize(n);
  ready_out.clear();
  std::vector<int> s;
  for (int t = 0; t < n; ++t) {
    const HTask& h = tasks[t];
    pp_task x = h.t;
    for (int k = 0; k < 6; ++k) {
      if (!h.has[k]) { x.p[k] = nullptr; continue; }
      const View& v = h.opnd[k];
      const PObj& o = objs[v.obj];
      double* base = bases.at(o.arena);
      x.p[k] = base ? base + o.off + (int64_t)v.r0 * o.ld + v.c0 : nullptr;
      x.ld[k] = o.ld;
    }
    if (h.scratch_elems > 0) {
      double* base = bases.at(h.t.instance * PP_ARENAS + AR_SCRATCH);
      x.tmp = base ? base + h.scratch_off : nullptr;
    } else {
      x.tmp = nullptr;
    }
    s = succ[t];
    std::stable_sort(s.begin(), s.end(), [&](int a, int b) { return blevel[a] > blevel[b]; });
    x.succ_begin = (int32_t)succ_out.size();
    x.n_succ = (int32_t)s.size();
    succ_out.insert(succ_out.end(), s.begin(), s.end());
    indeg_out[t] = (int32_t)pred[t].size();
    if (pred[t].empty()) ready_out.push_back(t);
    out[t] = x;
  }
  std::stable_sort(ready_out.begin(), ready_out.end(), [&](int a, int b) { return blevel[a] > blevel[b]; });
}

void Program::merge(const Program& o) {
  const int obj0 = (int)objs.size(), task0 = (int)tasks.size(), inst0 = n_instances;
  for (const PObj& p : o.objs) {
    PObj q = p;
    q.arena += inst0 * PP_ARENAS;
    objs.push_back(q);
  }
  n_instances += o.n_instances;
  arena_elems.insert(arena_elems.end(), o.arena_elems.begin(), o.arena_elems.end());
  for (const HTask& h : o.tasks) {
    HTask g = h;
    g.t.instance += inst0;
    for (int k = 0; k < 6; ++k)
      if (g.has[k]) g.opnd[k].obj += obj0;
    for (Region& r : g.regions) r.obj += obj0;
    tasks.push_back(std::move(g));
  }
  succ.resize(tasks.size());
  pred.resize(tasks.size());
  blevel.resize(tasks.size());
  pred_bits.resize(tasks.size());
  for (size_t t = 0; t < o.tasks.size(); ++t) {
    for (int x : o.succ[t]) succ[task0 + t].push_back(x + task0);
    for (int x : o.pred[t]) pred[task0 + t].push_back(x + task0);
    if (t < o.pred_bits.size()) pred_bits[task0 + t] = o.pred_bits[t];
    blevel[task0 + t] = o.blevel[t];
  }
  deps_built_ = false;
  edges += o.edges;
}

// ----------------------------------------------------------------------------- reference format
// Word layout of src/kernel.cu:1404-1501 (operation arguments after opcode, signal, operation).
namespace refisa {
enum { finish = 0, execute = 1, signal_wait = 2 };
enum { nop = 0, getrf = 1, trsml = 2, trsmr = 3, gemm = 4, gemm_plus = 5, gemm_3x = 6, gemm_4x = 7, accum = 8 };
}  // namespace refisa

bool Program::encode_reference(int workers, std::vector<std::vector<int32_t>>& streams, std::string& err,
                               int64_t* tmp_elems_per_worker) const {
  if (workers <= 0) { err = "workers must be positive"; return false; }
  h_ops_dag dag = to_dag();
  instructions_scheduler sched(dag, workers);
  streams.assign(workers, {});
  int64_t tmp_need = 0;
  auto ptr_off = [&](const HTask& h, int k, int32_t& ptr, int32_t& off) -> bool {
    const View& v = h.opnd[k];
    const PObj& o = objs[v.obj];
    int64_t e = o.off + (int64_t)v.r0 * o.ld + v.c0;
    if (e > INT32_MAX) { err = "element offset exceeds the reference's int32 format"; return false; }
    ptr = o.arena;
    off = (int32_t)e;
    return true;
  };
  for (int w = 0; w < workers; ++w) {
    auto& S = streams[w];
    for (const auto& en : sched.getSchedule(w)) {
      if (!en.exe) {
        S.insert(S.end(), {refisa::signal_wait, en.inst, 64});
        continue;
      }
      const HTask& h = tasks[en.inst];
      const pp_task& x = h.t;
      // the solves' inverse preparation writes only the arena tail and nothing waits on it:
      // the reference (which has no solve) gets the factorization proper
      if (x.op == PP_OP_TRINV) continue;
      if (x.flags & PP_PIVOT) { err = "pivoted programs have no reference-format stream"; return false; }
      auto T = [&](int k) { return (x.flags & PP_T(k)) ? 1 : 0; };
      int32_t p[6] = {0}, o[6] = {0};
      for (int k = 0; k < 6; ++k)
        if (h.has[k] && !ptr_off(h, k, p[k], o[k])) return false;
      S.push_back(refisa::execute);
      S.push_back(en.inst);
      switch (x.op) {
        case PP_OP_GETRF:
          S.insert(S.end(), {refisa::getrf, p[0], o[0], x.n, x.m, x.ld[0]});
          break;
        case PP_OP_TRSML:
          S.insert(S.end(), {refisa::trsml, p[0], p[1], o[0], o[1], x.n, x.m, x.m, x.ld[0], x.ld[1], 0});
          break;
        case PP_OP_TRSMR:
          S.insert(S.end(), {refisa::trsmr, p[0], p[1], o[0], o[1], x.n, x.m, x.n, x.ld[0], x.ld[1], 0});
          break;
        case PP_OP_TRSMRT:
          S.insert(S.end(), {refisa::trsmr, p[0], p[1], o[0], o[1], x.m, x.n, x.m, x.ld[0], x.ld[1], 1});
          break;
        case PP_OP_GEMM: {
          int opn;
          if (x.beta == 1.0 && x.alpha == -1.0) opn = refisa::gemm;
          else if (x.beta == 1.0 && x.alpha == 1.0) opn = refisa::gemm_plus;
          else { err = "GEMM with alpha/beta outside the reference's gemm / gemm_plus"; return false; }
          S.insert(S.end(), {opn, p[0], p[1], p[2], o[0], o[1], o[2], x.m, x.n, x.k, x.ld[0], x.ld[1], x.ld[2],
                             T(1), T(2)});
          break;
        }
        case PP_OP_GEMM3:
          if (x.alpha != -1.0) { err = "GEMM3 alpha must be -1 in the reference format"; return false; }
          S.insert(S.end(), {refisa::gemm_3x, p[0], p[1], p[2], p[3], o[0], o[1], o[2], o[3], x.m, x.n, x.k, x.l,
                             x.ld[0], x.ld[1], x.ld[2], x.ld[3], T(1), T(2), T(3), x.ctrl});
          tmp_need = std::max<int64_t>(tmp_need, h.scratch_elems);
          break;
        case PP_OP_GEMM4: {
          if (x.alpha != -1.0) { err = "GEMM4 alpha must be -1 in the reference format"; return false; }
          // the reference keeps t1 at my_tmp[0] and t2 at my_tmp[offset]
          const int32_t offset = x.aux;
          S.insert(S.end(), {refisa::gemm_4x, p[0], p[1], p[2], p[3], p[4], o[0], o[1], o[2], o[3], o[4], x.m, x.n,
                             x.k, x.l, x.o, x.ld[0], x.ld[1], x.ld[2], x.ld[3], x.ld[4], T(1), T(2), T(3), T(4),
                             x.ctrl, offset});
          tmp_need = std::max<int64_t>(tmp_need, h.scratch_elems);
          break;
        }
        case PP_OP_ACCUM: {
          if (x.alpha != 1.0 || T(2) || T(3)) { err = "accum with a sign or transposed factors has no reference form"; return false; }
          if (x.ld[4] != x.k) { err = "accum random sketch must have ld = rank"; return false; }
          // my_tmp: U (ny x k1) | V (nx x k1) | Q (max(ny x k1, k1 x k2))
          const int64_t off1 = (int64_t)x.m * x.k, off2 = off1 + (int64_t)x.n * x.k;
          const int64_t qsz = std::max<int64_t>((int64_t)x.m * x.k, (int64_t)x.k * std::max(x.k, x.l));
          tmp_need = std::max<int64_t>(tmp_need, off2 + qsz);
          S.insert(S.end(), {refisa::accum, p[0], p[1], p[2], p[3], o[0], o[1], o[2], o[3], x.n, x.m, x.k, x.l,
                             x.ld[0], x.ld[1], x.ld[2], x.ld[3], (int32_t)off1, (int32_t)off2});
          break;
        }
        default:
          err = "instruction has no reference-format counterpart (op " + std::to_string(x.op) + ")";
          return false;
      }
    }
    S.push_back(refisa::finish);
  }
  if (tmp_elems_per_worker) *tmp_elems_per_worker = tmp_need;
  return true;
}

// ----------------------------------------------------------------------------- generator
Generator::Generator(Program& P, Hierarchical& H, int tile, int max_n_rand, bool split_k)
    : P_(P), H_(H), T_(tile), max_n_rand_(max_n_rand), split_k_(split_k), Ttri_(tile) {
  if (tile < 8) throw std::invalid_argument("tile must be >= 8");
  inst_ = P.add_instance();
  const int ar = P.arena_id(inst_, AR_MATRIX);
  P.arena_elems[ar] = H.arena_elems;
  node_obj_.resize(H.objs.size());
  for (size_t i = 0; i < H.objs.size(); ++i)
    node_obj_[i] = P.add_obj_at(ar, H.objs[i].off, H.objs[i].rows, H.objs[i].cols, H.objs[i].ld, true);
  for (auto& x : rand_ld_obj_) x = -1;
  inv_obj_.assign(P.objs.size(), {-1, -1});
  for (auto& nd : H.nodes)
    if (nd.kind == HNode::D && nd.invL >= 0) inv_obj_[node_obj_[nd.obj]] = {node_obj_[nd.invL], node_obj_[nd.invU]};
  piv_obj_.assign(P.objs.size(), -1);
  for (auto& nd : H.nodes)
    if (nd.kind == HNode::D && nd.piv >= 0) piv_obj_[node_obj_[nd.obj]] = node_obj_[nd.piv];
  int kmax = 1;
  for (auto& nd : H.nodes)
    if (nd.kind == HNode::LR) kmax = std::max(kmax, nd.kmax);
  P.arena_elems[P.arena_id(inst_, AR_RAND)] = (int64_t)std::max(max_n_rand, H.n) * kmax;
}

int Generator::rand_obj(int k1) {
  if (k1 < 1 || k1 > 64) throw std::invalid_argument("rank outside 1..64");
  if (rand_ld_obj_[k1] < 0)
    rand_ld_obj_[k1] = P_.add_obj_at(P_.arena_id(inst_, AR_RAND), 0, std::max(max_n_rand_, H_.n), k1, k1, false);
  return rand_ld_obj_[k1];
}

Mat Generator::asD(const View& v) const {
  Mat M;
  M.kind = Mat::D;
  M.m = v.m;
  M.n = v.n;
  M.d = v;
  return M;
}

Mat Generator::node(int id, bool tr) const {
  const HNode& nd = H_.nodes.at(id);
  Mat M;
  M.m = tr ? nd.n : nd.m;
  M.n = tr ? nd.m : nd.n;
  if (nd.kind == HNode::D) {
    M.kind = Mat::D;
    View v;
    v.obj = node_obj_[nd.obj];
    v.m = nd.m;
    v.n = nd.n;
    M.d = tr ? v.T() : v;
  } else if (nd.kind == HNode::LR) {
    M.kind = Mat::LR;
    View u, v;
    u.obj = node_obj_[nd.obj];
    u.m = nd.m;
    u.n = nd.rank;
    v.obj = node_obj_[nd.objV];
    v.m = nd.n;
    v.n = nd.rank;
    M.k = nd.rank;
    M.u = tr ? v : u;
    M.v = tr ? u : v;
    M.rank_obj = nd.rank_obj >= 0 ? node_obj_[nd.rank_obj] : -1;
  } else {
    M.kind = Mat::H;
    M.node = id;
    M.tr = tr;
  }
  return M;
}

Mat Generator::child(const Mat& X, int i, int j) const {
  const HNode& nd = H_.nodes.at(X.node);
  return X.tr ? node(nd.ch[j * 2 + i], true) : node(nd.ch[i * 2 + j], false);
}

int Generator::hsplit_r(const Mat& X) const { return X.kind == Mat::H ? child(X, 0, 0).m : -1; }
int Generator::hsplit_c(const Mat& X) const { return X.kind == Mat::H ? child(X, 0, 0).n : -1; }

// Split point of a diagonal block: H blocks by their children; dense blocks in halves while
// larger than `limit` (T_ for GETRF; the triangular solves take blocks up to Ttri_ whole).
int Generator::tri_split(const Mat& X, int limit) const {
  if (X.kind == Mat::H) return hsplit_r(X);
  if (X.kind == Mat::D && X.m > limit) {
    int s = X.m / 2;
    if (X.m >= 32) s = (s + 7) & ~7;
    return s;
  }
  return -1;
}

void Generator::partition(const Mat& X, int rs, int cs, Mat out[2][2], int& nr, int& nc) const {
  nr = rs < 0 ? 1 : 2;
  nc = cs < 0 ? 1 : 2;
  const int roff[2] = {0, rs < 0 ? 0 : rs}, coff[2] = {0, cs < 0 ? 0 : cs};
  const int rsz[2] = {rs < 0 ? X.m : rs, rs < 0 ? 0 : X.m - rs};
  const int csz[2] = {cs < 0 ? X.n : cs, cs < 0 ? 0 : X.n - cs};
  if (X.kind == Mat::H) {
    if (rs != hsplit_r(X) || cs != hsplit_c(X))
      throw std::runtime_error("partition: block structures of the operands do not match");
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) out[i][j] = child(X, i, j);
    return;
  }
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      Mat M;
      M.kind = X.kind;
      M.m = rsz[i];
      M.n = csz[j];
      if (X.kind == Mat::D) {
        M.d = X.d.sub(roff[i], coff[j], rsz[i], csz[j]);
      } else {
        M.k = X.k;
        M.u = X.u.sub(roff[i], 0, rsz[i], X.k);
        M.v = X.v.sub(coff[j], 0, csz[j], X.k);
      }
      out[i][j] = M;
    }
}

View Generator::tmp(int rows, int cols) {
  View v;
  v.obj = P_.add_obj(P_.arena_id(inst_, AR_WORK), rows, cols, true);
  v.m = rows;
  v.n = cols;
  return v;
}

HTask& Generator::emit(int op) {
  P_.tasks.emplace_back();
  HTask& t = P_.tasks.back();
  t.t.op = op;
  t.t.instance = inst_;
  t.t.alpha = 1.0;
  t.t.beta = 1.0;
  return t;
}

void Generator::bind(HTask& t, int slot, const View& v, bool write) {
  t.opnd[slot] = v;
  t.has[slot] = true;
  const PObj& o = P_.objs[v.obj];
  t.t.ld[slot] = o.ld;
  if (v.t) t.t.flags |= PP_T(slot);
  if (v.r0 < 0 || v.c0 < 0 || v.r0 + v.srows() > o.rows || v.c0 + v.scols() > o.cols)
    throw std::logic_error("operand view outside its storage object");
  if (o.tracked) t.regions.push_back({v.obj, v.r0, v.c0, v.srows(), v.scols(), !write});
  if (write && v.obj < (int)shadows_.size()) shadows_[v.obj].clear();  // the shadows are stale now
}

// A view covering its whole storage object in the matrix arena (a dense leaf).
bool Generator::whole_leaf(const View& v) const {
  const PObj& o = P_.objs[v.obj];
  return o.arena == P_.arena_id(inst_, AR_MATRIX) && v.r0 == 0 && v.c0 == 0 && v.srows() == o.rows &&
         v.scols() == o.cols;
}

// Largest triangle of one TRSM* instruction: in a factorization, targets of kBigLeaf or more
// rows (columns) take kBigTri-row triangles whole, so that a large leaf's solve is a few long
// instructions rather than many 64-row pieces.
int Generator::tri_limit(int target_extent) const {
  return (!solve_ && target_extent >= kBigLeaf) ? std::max(Ttri_, kBigTri) : Ttri_;
}

// The BF16 shadow of an operand view (m x n logical, m a multiple of cr), columns padded to a
// multiple of 64, written by a SHADOW instruction at its first use and reused until the view's
// object is written again.
View Generator::shadow_of(const View& X, int cr, int split) {
  if ((int)shadows_.size() < (int)P_.objs.size()) shadows_.resize(P_.objs.size());
  const ShadowKey key{X.obj, X.r0, X.c0, X.m, X.n, X.t, cr, split};
  for (auto& e : shadows_[X.obj])
    if (e.first == key) {
      View s;
      s.obj = e.second;
      s.m = P_.objs[e.second].rows;
      s.n = P_.objs[e.second].cols;
      return s;
    }
  const int K = (X.n + 63) & ~63, KT = split ? (split >> 8) * K : K;
  // X.m rows of KT BF16 values: KT / 4 doubles per row (the tiled layout is opaque to the DAG)
  View s;
  s.obj = P_.add_obj(P_.arena_id(inst_, AR_SCRATCH), X.m, KT / 4, true);
  s.m = X.m;
  s.n = KT / 4;
  HTask& t = emit(PP_OP_SHADOW);
  bind(t, 0, s, true);
  bind(t, 1, X, false);
  t.t.m = X.m;
  t.t.k = KT;
  t.t.n = X.n < K ? X.n : 0;
  t.t.ctrl = cr == 128 ? 0 : cr;
  t.t.o = split;
  t.flops = 0;
  if ((int)shadows_.size() < (int)P_.objs.size()) shadows_.resize(P_.objs.size());
  shadows_[X.obj].push_back({key, s.obj});
  return s;
}

// C := C + alpha A B on the tensor cores from BF16 shadows (the mixed form), for the products of
// a factorization that the BF16 GEMM instruction takes: C's rows a multiple of 128 and its columns
// 32, 64, 128 or a multiple of 256; one of A, B a whole dense leaf of at least kBigLeaf rows and
// columns, or C a whole leaf (a Schur update, dense or low-rank); inner dimension padded to 64.
// Returns false (nothing emitted) when the product does not qualify.
bool Generator::bf16_product(const View& C, const View& A, const View& B, int alpha) {
  if (prec_ != PP_PREC_BF16 || solve_ || C.t) return false;
  const bool wide = C.n % 256 == 0;
  if (C.m % 128 != 0 || !(wide || C.n == 32 || C.n == 64 || C.n == 128)) return false;
  auto big = [&](const View& v) { return whole_leaf(v) && v.m >= kBigLeaf && v.n >= kBigLeaf; };
  const bool c_leaf = big(C);
  if (!(c_leaf || big(A) || big(B))) return false;
  if (!c_leaf && A.n % 64 != 0) return false;  // skinny products: k is a leaf's edge
  const int K = (A.n + 63) & ~63;
  const View As = shadow_of(A, 128);
  const View Bs = shadow_of(B.T(), wide ? 128 : C.n);
  HTask& t = emit(PP_OP_GEMM);
  bind(t, 0, C, true);
  bind(t, 1, As, false);
  bind(t, 2, Bs, false);
  t.t.prec = PP_PREC_BF16;
  t.t.m = C.m;
  t.t.n = C.n;
  t.t.k = K;
  t.t.alpha = (double)alpha;
  t.t.beta = 1.0;
  t.flops = 2LL * C.m * C.n * A.n;
  return true;
}

bool Generator::split_product(const View& C, const View& A, const View& B, int64_t flops) {
  const bool wide = C.n % 256 == 0;
  if (C.t || C.m % 128 != 0 || !(wide || C.n == 32 || C.n == 64 || C.n == 128) || A.n % 64 != 0) return false;
  const View As = shadow_of(A, 128, PP_SPLIT_A);
  const View Bs = shadow_of(B.T(), wide ? 128 : C.n, PP_SPLIT_B);
  HTask& t = emit(PP_OP_GEMM);
  bind(t, 0, C, true);
  bind(t, 1, As, false);
  bind(t, 2, Bs, false);
  t.t.prec = PP_PREC_BF16;
  t.t.m = C.m;
  t.t.n = C.n;
  t.t.k = 3 * A.n;
  t.t.alpha = 1.0;
  t.t.beta = 0.0;
  t.flops = flops;
  return true;
}

bool Generator::mixed_inverse(const Mat& T, int& invL, int& invU) const {
  if (prec_ != PP_PREC_BF16 || solve_ || T.m < kBigLeaf || !inverse_of(T, invL, invU)) return false;
  return T.d.obj < (int)inv_done_.size() && inv_done_[T.d.obj];
}

void Generator::getrf_program() {
  getrf(node(H_.root));
  if (inverses_) emit_inverses();
}

// A diagonal leaf used whole as the triangle of a solve step, and its inverse objects.
bool Generator::inverse_of(const Mat& T, int& invL, int& invU) const {
  if (!inverses_ || T.kind != Mat::D || T.d.t || T.d.r0 != 0 || T.d.c0 != 0) return false;
  if (T.d.obj < 0 || T.d.obj >= (int)inv_obj_.size() || inv_obj_[T.d.obj].first < 0) return false;
  const PObj& o = P_.objs[T.d.obj];
  if (T.d.m != o.rows || T.d.n != o.cols) return false;
  invL = inv_obj_[T.d.obj].first;
  invU = inv_obj_[T.d.obj].second;
  return true;
}

// TRINV tasks: after its GETRF a diagonal leaf is final; its L^-1 and U^-1 are built in
// column blocks of T_ on idle CTAs while the factorization goes on elsewhere.
// The mixed form emits a large leaf's TRINV tasks right after its GETRF instead (its panel
// solves use the inverses); the rest follow the factorization here.
void Generator::emit_inverses() {
  for (const HNode& nd : H_.nodes) {
    if (nd.kind != HNode::D || nd.invL < 0) continue;
    const int obj = node_obj_[nd.obj];
    if (obj < (int)inv_done_.size() && inv_done_[obj]) continue;
    emit_inverse(obj, nd.m);
  }
}

void Generator::emit_inverse(int leaf_obj, int m) {
  View A;
  A.obj = leaf_obj;
  A.m = m;
  A.n = m;
  for (int which = 0; which < 2; ++which) {
    View I;
    I.obj = which == 0 ? inv_obj_[leaf_obj].first : inv_obj_[leaf_obj].second;
    I.m = m;
    I.n = m;
    for (int c0 = 0; c0 < m; c0 += T_) {
      const int w = std::min(T_, m - c0);
      HTask& t = emit(PP_OP_TRINV);
      bind(t, 0, I.sub(0, c0, m, w), true);
      bind(t, 1, A, false);
      t.t.m = m;
      t.t.n = w;
      t.t.o = c0;
      t.t.ctrl = which;
      const int64_t rows = which == 0 ? m - c0 : c0 + w;  // rows the sweep touches
      t.flops = (int64_t)w * rows * rows;
    }
  }
  if ((int)inv_done_.size() <= leaf_obj) inv_done_.resize(leaf_obj + 1, 0);
  inv_done_[leaf_obj] = 1;
}

void Generator::solve_program(int nrhs) {
  // a solve sweeps each leaf triangle once with few right-hand sides: whole leaves (up to
  // kSolveTri rows) go to one blocked instruction, which saves the inter-task latency of
  // the 64-row pieces on the solve's sequential path
  Ttri_ = std::max(Ttri_, kSolveTri);
  solve_ = true;
  rhs_obj_ = P_.add_obj(P_.arena_id(inst_, AR_RHS), H_.n, nrhs, true);
  View b;
  b.obj = rhs_obj_;
  b.m = H_.n;
  b.n = nrhs;
  trsml(node(H_.root), asD(b));
  trsmu(node(H_.root), asD(b));
}

// C := K(P_I, P_J) B in row blocks of at most 256 rows (one CTA each)
void Generator::kmul(const View& C, const View& PI, const View& PJ, const View& B, int kernel, double p0) {
  constexpr int kRows = 256;
  for (int r = 0; r < C.m; r += kRows) {
    const int h = std::min(kRows, C.m - r);
    HTask& t = emit(PP_OP_KMUL);
    bind(t, 0, C.sub(r, 0, h, C.n), true);
    bind(t, 1, PI.sub(r, 0, h, PI.n), false);
    bind(t, 2, PJ, false);
    bind(t, 3, B, false);
    t.t.m = h;
    t.t.n = PJ.m;
    t.t.k = C.n;
    t.t.l = PI.n;
    t.t.ctrl = kernel;
    t.t.alpha = p0;
    t.flops = (int64_t)h * PJ.m * (2 * C.n + 20);
  }
}

void Generator::orth(const View& Y) {
  HTask& o = emit(PP_OP_ORTH);
  bind(o, 0, Y, true);
  o.t.m = Y.m;
  o.t.n = Y.n;
  o.t.k = Y.n;
  o.flops = 3 * (2LL * Y.m * Y.n * Y.n + (int64_t)Y.m * Y.n * Y.n);
}

void Generator::construct_program(int kernel, int dim, double p0, double tol) {
  if (dim < 1 || dim > 3) throw std::invalid_argument("construct: dim must be 1..3");
  rhs_obj_ = P_.add_obj(P_.arena_id(inst_, AR_RHS), H_.n, dim, false);
  View pts;
  pts.obj = rhs_obj_;
  pts.m = H_.n;
  pts.n = dim;
  for (const HNode& nd : H_.nodes) {
    if (nd.kind != HNode::LR) continue;
    const int k = nd.kmax;
    if (k > kAccumMaxK2 || k > nd.m || k > nd.n) throw std::runtime_error("construct: block rank above 32 or its size");
    View U, V, R;
    U.obj = node_obj_[nd.obj];
    U.m = nd.m;
    U.n = k;
    V.obj = node_obj_[nd.objV];
    V.m = nd.n;
    V.n = k;
    R.obj = rand_obj(k);
    R.m = nd.n;
    R.n = k;
    const View PI = pts.sub(nd.r0, 0, nd.m, dim), PJ = pts.sub(nd.c0, 0, nd.n, dim);
    kmul(U, PI, PJ, R, kernel, p0);  // U = K Omega
    orth(U);
    kmul(V, PJ, PI, U, kernel, p0);  // V = K^T U
    orth(V);
    kmul(U, PI, PJ, V, kernel, p0);  // U = K V   (one power step)
    orth(U);
    kmul(V, PJ, PI, U, kernel, p0);  // V = K^T U: U V^T = U U^T K
    HTask& t = emit(PP_OP_LRTRUNC);
    bind(t, 0, U, true);
    bind(t, 1, V, true);
    t.t.m = nd.m;
    t.t.n = nd.n;
    t.t.k = k;
    t.t.o = H_.rank_tol > 0.0 ? k : nd.rank;
    t.t.beta = tol;
    if (nd.rank_obj >= 0) {
      View rv;
      rv.obj = node_obj_[nd.rank_obj];
      rv.m = 1;
      rv.n = 1;
      bind(t, 5, rv, true);
    }
    t.flops = 2LL * (nd.m + nd.n) * k * k * 3;
  }
}

// The rows of a diagonal leaf's pivot object that belong to a diagonal block of that leaf.
View Generator::pivot_view(const View& tile) const {
  if (tile.t || tile.r0 != tile.c0 || tile.m != tile.n || tile.obj < 0 || tile.obj >= (int)piv_obj_.size() ||
      piv_obj_[tile.obj] < 0)
    throw std::logic_error("pivoting: a GETRF / TRSML block that is not a diagonal block of a diagonal leaf");
  View v;
  v.obj = piv_obj_[tile.obj];
  v.r0 = tile.r0;
  v.c0 = 0;
  v.m = tile.m;
  v.n = 1;
  return v;
}

void Generator::getrf(const Mat& A) {
  if (A.kind == Mat::LR) throw std::logic_error("getrf on a low-rank block");
  const int s = tri_split(A, T_);
  if (s < 0) {
    HTask& t = emit(PP_OP_GETRF);
    bind(t, 0, A.d, true);
    if (pivot_) {
      bind(t, 1, pivot_view(A.d), true);
      t.t.flags |= PP_PIVOT;
    }
    t.t.m = A.m;
    t.t.n = A.n;
    t.flops = flops_getrf(A.m, A.n);
  } else {
    Mat p[2][2];
    int nr, nc;
    partition(A, s, A.kind == Mat::H ? hsplit_c(A) : s, p, nr, nc);
    getrf(p[0][0]);
    trsml(p[0][0], p[0][1]);
    trsmr(p[0][0], p[1][0]);
    gemm(p[1][1], p[1][0], p[0][1], -1);
    getrf(p[1][1]);
  }
  int invL, invU;
  if (prec_ == PP_PREC_BF16 && !solve_ && A.m >= kBigLeaf && inverse_of(A, invL, invU)) emit_inverse(A.d.obj, A.m);
}

// An inverse of m x m as a view (the whole object).
static View whole(int obj, int m) {
  View v;
  v.obj = obj;
  v.m = m;
  v.n = m;
  return v;
}

void Generator::trsml(const Mat& L, const Mat& B) {
  if (B.kind == Mat::LR) { trsml(L, asD(B.u)); return; }
  int invL, invU;
  if (solve_ && B.kind == Mat::D && !B.d.t && inverse_of(L, invL, invU)) {
    trmv(invL, 0, L.m, B.d);
    return;
  }
  // mixed form: B := L^-1 B as one product with the explicit inverse
  if (B.kind == Mat::D && !B.d.t && mixed_inverse(L, invL, invU) &&
      split_product(B.d, whole(invL, L.m), B.d, (int64_t)B.n * L.m * (L.m - 1)))
    return;
  // with pivoting the triangles are the GETRF blocks themselves (T_, split as getrf splits)
  const int s = tri_split(L, pivot_ ? T_ : tri_limit(B.n));
  if (s < 0) {
    if (B.kind != Mat::D || B.d.t) throw std::logic_error("trsml: target must be a dense untransposed block");
    for (int c = 0; c < B.n; c += T_) {
      const int w = std::min(T_, B.n - c);
      HTask& t = emit(PP_OP_TRSML);
      bind(t, 0, B.d.sub(0, c, B.m, w), true);
      bind(t, 1, L.d, false);
      if (pivot_) {
        bind(t, 2, pivot_view(L.d), false);
        t.t.flags |= PP_PIVOT;
      }
      t.t.m = B.m;
      t.t.n = w;
      t.flops = (int64_t)w * B.m * (B.m - 1);
    }
    return;
  }
  Mat Lp[2][2], Bp[2][2];
  int a, b, br, bc;
  partition(L, s, L.kind == Mat::H ? hsplit_c(L) : s, Lp, a, b);
  partition(B, s, hsplit_c(B), Bp, br, bc);
  for (int j = 0; j < bc; ++j) {
    trsml(Lp[0][0], Bp[0][j]);
    gemm(Bp[1][j], Lp[1][0], Bp[0][j], -1);
    trsml(Lp[1][1], Bp[1][j]);
  }
}

void Generator::trsmr(const Mat& U, const Mat& B) {
  if (B.kind == Mat::LR) { trsmrt(U, B.v); return; }
  int invL, invU;
  // mixed form: B := B U^-1 as one product with the explicit inverse
  if (B.kind == Mat::D && !B.d.t && mixed_inverse(U, invL, invU) &&
      split_product(B.d, B.d, whole(invU, U.m), (int64_t)B.m * U.m * U.m))
    return;
  const int s = tri_split(U, tri_limit(B.m));
  if (s < 0) {
    if (B.kind != Mat::D || B.d.t) throw std::logic_error("trsmr: target must be a dense untransposed block");
    const int rows = std::max(T_, 4096 / std::max(1, B.n));
    for (int r = 0; r < B.m; r += rows) {
      const int h = std::min(rows, B.m - r);
      HTask& t = emit(PP_OP_TRSMR);
      bind(t, 0, B.d.sub(r, 0, h, B.n), true);
      bind(t, 1, U.d, false);
      t.t.m = h;
      t.t.n = B.n;
      t.flops = (int64_t)h * B.n * B.n;
    }
    return;
  }
  Mat Up[2][2], Bp[2][2];
  int a, b, br, bc;
  partition(U, s, U.kind == Mat::H ? hsplit_c(U) : s, Up, a, b);
  partition(B, hsplit_r(B), s, Bp, br, bc);
  for (int i = 0; i < br; ++i) {
    trsmr(Up[0][0], Bp[i][0]);
    gemm(Bp[i][1], Bp[i][0], Up[0][1], -1);
    trsmr(Up[1][1], Bp[i][1]);
  }
}

void Generator::trsmrt(const Mat& U, const View& V) {
  if (V.t) throw std::logic_error("trsmrt: V must be untransposed");
  int invL, invU;
  // mixed form: V := U^-T V as one product with the explicit inverse
  if (mixed_inverse(U, invL, invU) && split_product(V, whole(invU, U.m).T(), V, (int64_t)V.n * U.m * U.m)) return;
  const int s = tri_split(U, Ttri_);
  if (s < 0) {
    for (int c = 0; c < V.n; c += T_) {
      const int w = std::min(T_, V.n - c);
      HTask& t = emit(PP_OP_TRSMRT);
      bind(t, 0, V.sub(0, c, V.m, w), true);
      bind(t, 1, U.d, false);
      t.t.m = V.m;
      t.t.n = w;
      t.flops = (int64_t)w * V.m * V.m;
    }
    return;
  }
  Mat Up[2][2];
  int a, b;
  partition(U, s, U.kind == Mat::H ? hsplit_c(U) : s, Up, a, b);
  View V0 = V.sub(0, 0, s, V.n), V1 = V.sub(s, 0, V.m - s, V.n);
  trsmrt(Up[0][0], V0);
  gemm(asD(V1), transpose(Up[0][1]), asD(V0), -1);
  trsmrt(Up[1][1], V1);
}

void Generator::trsmu(const Mat& U, const Mat& B) {
  if (B.kind == Mat::LR) { trsmu(U, asD(B.u)); return; }
  int invL, invU;
  if (solve_ && B.kind == Mat::D && !B.d.t && inverse_of(U, invL, invU)) {
    trmv(invU, 1, U.m, B.d);
    return;
  }
  const int s = tri_split(U, Ttri_);
  if (s < 0) {
    if (B.kind != Mat::D || B.d.t) throw std::logic_error("trsmu: target must be a dense untransposed block");
    for (int c = 0; c < B.n; c += T_) {
      const int w = std::min(T_, B.n - c);
      HTask& t = emit(PP_OP_TRSMU);
      bind(t, 0, B.d.sub(0, c, B.m, w), true);
      bind(t, 1, U.d, false);
      t.t.m = B.m;
      t.t.n = w;
      t.flops = (int64_t)w * B.m * B.m;
    }
    return;
  }
  Mat Up[2][2], Bp[2][2];
  int a, b, br, bc;
  partition(U, s, U.kind == Mat::H ? hsplit_c(U) : s, Up, a, b);
  partition(B, s, hsplit_c(B), Bp, br, bc);
  for (int j = 0; j < bc; ++j) {
    trsmu(Up[1][1], Bp[1][j]);
    gemm(Bp[0][j], Up[0][1], Bp[1][j], -1);
    trsmu(Up[0][0], Bp[0][j]);
  }
}

void Generator::gemm_tiles(const View& C, const View& A, const View& B, int alpha) {
  if (C.t) throw std::logic_error("gemm target must be untransposed");
  if (A.m != C.m || B.n != C.n || A.n != B.m) throw std::logic_error("gemm dimension mismatch");
  const bool work_target = P_.objs[C.obj].arena == P_.arena_id(inst_, AR_WORK);
  constexpr int kSplitK = 512;
  if (split_k_ && work_target && (int64_t)C.m * C.n <= 256 && A.n > kSplitK) {
    // a small product over a long k (e.g. V_a^T U_b): independent partial products over
    // k slices on many SMs, then one reduction into C (order fixed, not ascending k)
    const int parts = (A.n + kSplitK - 1) / kSplitK;
    View Tp = tmp(parts * C.m, C.n);
    for (int p = 0; p < parts; ++p) {
      const int k0 = p * kSplitK, kk = std::min(kSplitK, A.n - k0);
      HTask& t = emit(PP_OP_GEMM);
      bind(t, 0, Tp.sub(p * C.m, 0, C.m, C.n), true);
      bind(t, 1, A.sub(0, k0, C.m, kk), false);
      bind(t, 2, B.sub(k0, 0, kk, C.n), false);
      t.t.m = C.m;
      t.t.n = C.n;
      t.t.k = kk;
      t.t.alpha = (double)alpha;
      t.t.beta = 0.0;
      t.t.flags |= PP_FREE_ORDER;
      t.flops = 2LL * C.m * C.n * kk;
    }
    HTask& s = emit(PP_OP_SUM);
    bind(s, 0, C, true);
    bind(s, 1, Tp, false);
    s.t.m = C.m;
    s.t.n = C.n;
    s.t.k = parts;
    s.t.alpha = 1.0;
    s.t.beta = 1.0;
    s.flops = (int64_t)C.m * C.n * parts;
    return;
  }
  // the mixed form: Schur updates of large leaves and products with a large dense leaf on the
  // tensor cores
  if (bf16_product(C, A, B, alpha)) return;
  if (!solve_ && !work_target && C.m >= kBigLeaf && C.n >= kBigLeaf && whole_leaf(C) && whole_leaf(A) &&
      whole_leaf(B)) {
    // a Schur update of whole large leaves: one instruction (its CTA loops over the tile)
    HTask& t = emit(PP_OP_GEMM);
    bind(t, 0, C, true);
    bind(t, 1, A, false);
    bind(t, 2, B, false);
    t.t.m = C.m;
    t.t.n = C.n;
    t.t.k = A.n;
    t.t.alpha = (double)alpha;
    t.t.beta = 1.0;
    t.flops = 2LL * C.m * C.n * A.n;
    return;
  }
  if (!solve_ && !work_target && C.m >= kBigLeaf && C.n >= kBigLeaf && A.n <= 64 && whole_leaf(C)) {
    // a low-rank update of a whole large leaf: one pass over the leaf in one instruction
    HTask& t = emit(PP_OP_GEMM);
    bind(t, 0, C, true);
    bind(t, 1, A, false);
    bind(t, 2, B, false);
    t.t.m = C.m;
    t.t.n = C.n;
    t.t.k = A.n;
    t.t.alpha = (double)alpha;
    t.t.beta = 1.0;
    t.flops = 2LL * C.m * C.n * A.n;
    return;
  }
  const int g = gemm_tile_;
  const int TN = std::min(C.n, g);
  int TM = std::min(C.m, std::max(g, g * g / std::max(TN, 1)));
  if (solve_ && C.n <= 16) TM = std::min(TM, A.n >= kBigLeaf ? kSolveGemmRowsBig : kSolveGemmRows);
  for (int i = 0; i < C.m; i += TM)
    for (int j = 0; j < C.n; j += TN) {
      const int mi = std::min(TM, C.m - i), nj = std::min(TN, C.n - j);
      HTask& t = emit(PP_OP_GEMM);
      bind(t, 0, C.sub(i, j, mi, nj), true);
      bind(t, 1, A.sub(i, 0, mi, A.n), false);
      bind(t, 2, B.sub(0, j, B.m, nj), false);
      t.t.m = mi;
      t.t.n = nj;
      t.t.k = A.n;
      t.t.alpha = (double)alpha;
      t.t.beta = 1.0;
      // intermediates of low-rank products (work buffers) and the solves' products may sum in
      // any fixed order (compared within a tolerance; the factorization's dense products keep
      // the reference's ascending order)
      if (solve_ || P_.objs[C.obj].arena == P_.arena_id(inst_, AR_WORK)) t.t.flags |= PP_FREE_ORDER;
      t.flops = 2LL * mi * nj * A.n;
    }
}

void Generator::gemm(const Mat& C, const Mat& A, const Mat& B, int alpha) {
  if (A.m != C.m || B.n != C.n || A.n != B.m) throw std::logic_error("gemm: dimension mismatch");
  if (A.kind == Mat::LR || B.kind == Mat::LR) {
    LRP p = lr_product(A, B, alpha);
    lr_update(C, p.x, p.y, p.sign);
    return;
  }
  if (C.kind == Mat::LR) {
    if (A.kind == Mat::D && B.kind == Mat::D && A.n <= kAccumMaxK2) { accum(C, A.d, B.d.T(), alpha); return; }
    sketch_update(C, A, B, alpha);
    return;
  }
  if (C.kind == Mat::D && A.kind == Mat::D && B.kind == Mat::D) {
    gemm_tiles(C.d, A.d, B.d, alpha);
    return;
  }
  int rs = hsplit_r(C);
  if (rs < 0) rs = hsplit_r(A);
  int cs = hsplit_c(C);
  if (cs < 0) cs = hsplit_c(B);
  int ks = hsplit_c(A);
  if (ks < 0) ks = hsplit_r(B);
  Mat Cp[2][2], Ap[2][2], Bp[2][2];
  int cr, cc, ar, ac, br, bc;
  partition(C, rs, cs, Cp, cr, cc);
  partition(A, rs, ks, Ap, ar, ac);
  partition(B, ks, cs, Bp, br, bc);
  for (int i = 0; i < cr; ++i)
    for (int j = 0; j < cc; ++j)
      for (int k = 0; k < ac; ++k) gemm(Cp[i][j], Ap[i][k], Bp[k][j], alpha);
}

// alpha * A * B as x y^T * sign, with the sign folded into a zero-filled work buffer
// whenever one is needed anyway.
Generator::LRP Generator::lr_product(const Mat& A, const Mat& B, int alpha) {
  if (A.kind == Mat::LR && B.kind == Mat::LR) {
    View S = tmp(A.k, B.k);  // alpha Va^T Ub
    gemm_tiles(S, A.v.T(), B.u, alpha);
    if (A.k <= B.k) {
      View Y = tmp(B.n, A.k);  // Vb S^T
      gemm_tiles(Y, B.v, S.T(), +1);
      return {A.u, Y, +1};
    }
    View X = tmp(A.m, B.k);  // Ua S
    gemm_tiles(X, A.u, S, +1);
    return {X, B.v, +1};
  }
  if (A.kind == Mat::LR) {
    View Y = tmp(B.n, A.k);  // alpha B^T Va
    gemm(asD(Y), transpose(B), asD(A.v), alpha);
    return {A.u, Y, +1};
  }
  if (B.kind == Mat::LR) {
    View X = tmp(A.m, B.k);  // alpha A Ub
    gemm(asD(X), A, asD(B.u), alpha);
    return {X, B.v, +1};
  }
  if (A.kind == Mat::D && B.kind == Mat::D) return {A.d, B.d.T(), alpha};
  throw std::runtime_error("unsupported: low-rank form of a hierarchical product");
}

void Generator::lr_update(const Mat& C, const View& X, const View& Y, int sign) {
  if (C.kind == Mat::D) { gemm_tiles(C.d, X, Y.T(), sign); return; }
  if (C.kind == Mat::LR) { accum(C, X, Y, sign); return; }
  const int rs = hsplit_r(C), cs = hsplit_c(C);
  const int roff[2] = {0, rs}, coff[2] = {0, cs};
  const int rsz[2] = {rs, C.m - rs}, csz[2] = {cs, C.n - cs};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      lr_update(child(C, i, j), X.sub(roff[i], 0, rsz[i], X.n), Y.sub(coff[j], 0, csz[j], Y.n), sign);
}

void Generator::accum(const Mat& C, const View& X, const View& Y, int sign) {
  if (C.kind != Mat::LR) throw std::logic_error("accum target must be low-rank");
  const int k1 = C.k, k2 = X.n;
  if (k1 <= 0) return;
  HTask& t = emit(PP_OP_ACCUM);
  bind(t, 0, C.u, true);
  bind(t, 1, C.v, true);
  bind(t, 2, X, false);
  bind(t, 3, Y, false);
  View R;
  R.obj = rand_obj(k1);
  R.m = C.n;
  R.n = k1;
  bind(t, 4, R, false);
  t.t.m = C.m;
  t.t.n = C.n;
  t.t.k = k1;
  t.t.l = k2;
  t.t.alpha = (double)sign;
  if (H_.rank_tol > 0.0 && C.rank_obj >= 0) {  // adaptive: truncate and record the new rank
    t.t.flags |= PP_ADAPT_RANK;
    t.t.beta = H_.rank_tol;
    View rv;
    rv.obj = C.rank_obj;
    rv.m = 1;
    rv.n = 1;
    bind(t, 5, rv, true);
  }
  const int64_t ny = C.m, nx = C.n;
  t.scratch_elems = 2 * ny * k1 + nx * k1 + (int64_t)k1 * std::max(k1, k2);
  const int ar = P_.arena_id(inst_, AR_SCRATCH);
  t.scratch_off = (P_.arena_elems[ar] + 3) & ~int64_t(3);
  P_.arena_elems[ar] = t.scratch_off + t.scratch_elems;
  const int64_t kk = k1, k22 = k2;
  t.flops = 2 * kk * nx * kk + 2 * ny * kk * kk + 2 * kk * nx * k22 + 2 * ny * k22 * kk  // sketch
            + 8 * ny * kk * kk                                                        // QR + Q
            + 2 * kk * ny * kk + 2 * nx * kk * kk + 2 * kk * ny * k22 + 2 * nx * k22 * kk;  // projection
}

// B := M B with M the explicit inverse (object inv, m x m; lower = ctrl 0, upper = 1) of a
// diagonal leaf's triangular factor; B's columns in groups of at most kTrmvCols
void Generator::trmv(int inv, int upper, int m, const View& B) {
  View M;
  M.obj = inv;
  M.m = m;
  M.n = m;
  for (int c = 0; c < B.n; c += kTrmvCols) {
    const int w = std::min(kTrmvCols, B.n - c);
    const View Bc = B.sub(0, c, B.m, w);
    if (m < kTrmvSplitMin) {
      HTask& t = emit(PP_OP_TRMV);
      bind(t, 0, Bc, true);
      bind(t, 1, M, false);
      t.t.m = m;
      t.t.n = w;
      t.t.ctrl = upper;
      t.flops = (int64_t)w * m * (m + 1);
      continue;
    }
    // row blocks of equal area: lower rows [0, b) hold b^2/2 entries, upper rows [b, m) (m-b)^2/2
    int bound[kTrmvParts + 1];
    for (int p = 0; p <= kTrmvParts; ++p) {
      const double f = (double)p / kTrmvParts;
      bound[p] = upper ? m - (int)std::lround(m * std::sqrt(1.0 - f)) : (int)std::lround(m * std::sqrt(f));
    }
    bound[0] = 0;
    bound[kTrmvParts] = m;
    // parts of more than kTrmvPartRows rows are cut further: the VM takes kTrmvPartRows rows
    // per pass of loads, and a second pass costs a second round of load latency
    std::vector<int> cuts{0};
    for (int p = 0; p < kTrmvParts; ++p)
      for (int r = bound[p]; r < bound[p + 1];) {
        r = std::min(bound[p + 1], r + kTrmvPartRows);
        cuts.push_back(r);
      }
    const View W = tmp(m, w);
    for (size_t p = 0; p + 1 < cuts.size(); ++p) {
      const int r0 = cuts[p], r1 = cuts[p + 1];
      if (r1 <= r0) continue;
      HTask& t = emit(PP_OP_TRMV);
      bind(t, 0, W.sub(r0, 0, r1 - r0, w), true);
      bind(t, 1, M, false);
      bind(t, 2, Bc, false);
      t.t.m = m;
      t.t.n = w;
      t.t.ctrl = upper;
      t.t.o = r0;
      t.t.l = r1 - r0;
      int64_t e = 0;
      for (int r = r0; r < r1; ++r) e += upper ? m - r : r + 1;
      t.flops = 2 * (int64_t)w * e;
    }
    HTask& cp = emit(PP_OP_COPY);
    bind(cp, 0, Bc, true);
    bind(cp, 1, W, false);
    cp.t.m = m;
    cp.t.n = w;
  }
}

// C (low-rank, u v^T with k columns) := Q W^T, the rank-k recompression of C + alpha A B:
//   T1 = B R                    (R: the k-column random sketch, n rows)
//   Y  = u (v^T R) + alpha A T1  (ny x k)            Q = orth(Y)
//   W  = v (u^T Q) + alpha B^T (A^T Q)               u := Q, v := W
// The same one-pass randomized range finder as ACCUM (the reference's accum, kernel.cu:
// 1255-1280), here over products of hierarchical or dense blocks, each product an ordinary
// GEMM of the generator (work buffers, DAG-tracked).
void Generator::sketch_update(const Mat& C, const Mat& A, const Mat& B, int alpha) {
  const int k = C.k, ny = C.m, nx = C.n, nm = A.n;
  if (k <= 0) return;
  if (k > kAccumMaxK2) throw std::runtime_error("sketched update: rank above 32");
  View R;
  R.obj = rand_obj(k);
  R.m = nx;
  R.n = k;
  View T1 = tmp(nm, k);
  gemm(asD(T1), B, asD(R), +1);
  View S = tmp(k, k);
  gemm_tiles(S, C.v.T(), R, +1);
  View Y = tmp(ny, k);
  gemm_tiles(Y, C.u, S, +1);
  gemm(asD(Y), A, asD(T1), alpha);
  HTask& o = emit(PP_OP_ORTH);
  bind(o, 0, Y, true);
  o.t.m = ny;
  o.t.n = k;
  o.t.k = k;
  o.flops = 3 * (2LL * ny * k * k + (int64_t)ny * k * k);
  View P = tmp(k, k);
  gemm_tiles(P, C.u.T(), Y, +1);
  View W = tmp(nx, k);
  gemm_tiles(W, C.v, P, +1);  // (Q^T u v^T)^T = v (u^T Q)
  View T2 = tmp(nm, k);
  gemm(asD(T2), transpose(A), asD(Y), +1);
  gemm(asD(W), transpose(B), asD(T2), alpha);
  for (int which = 0; which < 2; ++which) {
    const View& dst = which == 0 ? C.u : C.v;
    const View& src = which == 0 ? Y : W;
    HTask& c = emit(PP_OP_COPY);
    bind(c, 0, dst, true);
    bind(c, 1, src, false);
    c.t.m = dst.m;
    c.t.n = dst.n;
  }
}

}  // namespace pp
