// hmatrix.cpp — block-tree construction and host image of an H-matrix.
#include "hmatrix.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>

namespace pp {

Dense::Dense(int64_t m_, int64_t n_, int64_t lda_) : m(m_), n(n_), lda(std::max(n_, lda_)) {
  a = (double*)std::calloc((size_t)(m > 0 ? m : 1) * (size_t)lda, sizeof(double));
}
Dense::~Dense() { std::free(a); }

int Hierarchical::add_obj(int rows, int cols) {
  StorageObj o;
  // 32-byte aligned objects: vector loads stay aligned when ld is even
  o.off = (arena_elems + 3) & ~int64_t(3);
  o.rows = rows;
  o.cols = cols;
  o.ld = cols;
  arena_elems = o.off + (int64_t)rows * cols;
  objs.push_back(o);
  return (int)objs.size() - 1;
}

void Hierarchical::add_inverses() {
  for (auto& nd : nodes)
    if (nd.kind == HNode::LR) nd.rank_obj = add_obj(1, 1);
  block_elems = arena_elems;
  for (auto& nd : nodes)
    if (nd.kind == HNode::D && nd.r0 == nd.c0 && nd.m == nd.n && nd.m <= kInvMax) {
      nd.invL = add_obj(nd.m, nd.m);
      nd.invU = add_obj(nd.m, nd.m);
    }
  // after the inverses, so that their offsets do not depend on it
  for (auto& nd : nodes)
    if (nd.kind == HNode::D && nd.r0 == nd.c0 && nd.m == nd.n) nd.piv = add_obj(nd.m, 1);
}

Hierarchical* Hierarchical::dense_tiled(int n, int leaf) {
  if (n <= 0 || leaf <= 0) throw std::invalid_argument("dense_tiled: n and leaf must be positive");
  auto* h = new Hierarchical();
  h->n = n;
  std::function<int(int, int, int, int)> build = [&](int r0, int sz, int c0, int level) -> int {
    HNode nd;
    nd.r0 = r0; nd.c0 = c0; nd.m = sz; nd.n = sz; nd.level = level;
    if (sz <= leaf) {
      nd.kind = HNode::D;
      h->nodes.push_back(nd);
      int id = (int)h->nodes.size() - 1;
      h->nodes[id].obj = h->add_obj(sz, sz);
      return id;
    }
    nd.kind = HNode::H;
    h->nodes.push_back(nd);
    int id = (int)h->nodes.size() - 1;
    const int s0 = sz / 2;
    const int rs[2] = {r0, r0 + s0}, cs[2] = {c0, c0 + s0}, sz2[2] = {s0, sz - s0};
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        // off-diagonal quadrants of a square partition are square only when sizes match;
        // dense_tiled keeps them dense with their own shape
        HNode q;
        q.r0 = rs[i]; q.c0 = cs[j]; q.m = sz2[i]; q.n = sz2[j]; q.level = level + 1;
        int cid;
        if (i == j) {
          cid = build(rs[i], sz2[i], cs[j], level + 1);
        } else if (sz2[i] <= leaf && sz2[j] <= leaf) {
          q.kind = HNode::D;
          h->nodes.push_back(q);
          cid = (int)h->nodes.size() - 1;
          h->nodes[cid].obj = h->add_obj(q.m, q.n);
        } else {
          // rectangular off-diagonal block: partition like the diagonal ones
          std::function<int(int, int, int, int, int)> rect = [&](int r, int m, int c, int nn, int lv) -> int {
            HNode b;
            b.r0 = r; b.c0 = c; b.m = m; b.n = nn; b.level = lv;
            if (m <= leaf && nn <= leaf) {
              b.kind = HNode::D;
              h->nodes.push_back(b);
              int bid = (int)h->nodes.size() - 1;
              h->nodes[bid].obj = h->add_obj(m, nn);
              return bid;
            }
            b.kind = HNode::H;
            h->nodes.push_back(b);
            int bid = (int)h->nodes.size() - 1;
            const int m0 = m / 2, n0 = nn / 2;
            int k = 0;
            for (int a = 0; a < 2; ++a)
              for (int c2 = 0; c2 < 2; ++c2) {
                int cc = rect(a ? r + m0 : r, a ? m - m0 : m0, c2 ? c + n0 : c, c2 ? nn - n0 : n0, lv + 1);
                h->nodes[bid].ch[k++] = cc;
              }
            return bid;
          };
          cid = rect(rs[i], sz2[i], cs[j], sz2[j], level + 1);
        }
        h->nodes[id].ch[i * 2 + j] = cid;
      }
    return id;
  };
  h->root = build(0, n, 0, 0);
  h->add_inverses();
  return h;
}

namespace {
struct Cluster {
  int begin, size;
  std::vector<double> lo, hi;
  int child[2] = {-1, -1};
};
}  // namespace

Hierarchical* Hierarchical::geometric(int n, int dim, const double* pts, int leaf, int adm, double eta,
                                      int kmax) {
  if (n <= 0 || leaf <= 0 || dim <= 0 || kmax <= 0)
    throw std::invalid_argument("geometric: n, dim, leaf and kmax must be positive");
  auto* h = new Hierarchical();
  h->n = n;
  h->point_dim = dim;
  std::vector<Cluster> cl;
  std::function<int(int, int)> make = [&](int b, int sz) -> int {
    Cluster c;
    c.begin = b;
    c.size = sz;
    c.lo.assign(dim, 1e300);
    c.hi.assign(dim, -1e300);
    for (int i = b; i < b + sz; ++i)
      for (int d = 0; d < dim; ++d) {
        c.lo[d] = std::min(c.lo[d], pts[(size_t)i * dim + d]);
        c.hi[d] = std::max(c.hi[d], pts[(size_t)i * dim + d]);
      }
    cl.push_back(c);
    int id = (int)cl.size() - 1;
    if (sz > leaf) {
      int c0 = make(b, sz / 2);
      int c1 = make(b + sz / 2, sz - sz / 2);
      cl[id].child[0] = c0;
      cl[id].child[1] = c1;
    }
    return id;
  };
  make(0, n);
  auto diam = [&](const Cluster& c) {
    double s = 0;
    for (int d = 0; d < dim; ++d) s += (c.hi[d] - c.lo[d]) * (c.hi[d] - c.lo[d]);
    return std::sqrt(s);
  };
  auto dist = [&](const Cluster& a, const Cluster& b) {
    double s = 0;
    for (int d = 0; d < dim; ++d) {
      double g = std::max(0.0, std::max(a.lo[d] - b.hi[d], b.lo[d] - a.hi[d]));
      s += g * g;
    }
    return std::sqrt(s);
  };
  std::function<int(int, int, int)> block = [&](int t, int s, int level) -> int {
    const Cluster& a = cl[t];
    const Cluster& b = cl[s];
    HNode nd;
    nd.r0 = a.begin; nd.m = a.size; nd.c0 = b.begin; nd.n = b.size; nd.level = level;
    bool admissible;
    if (adm == 0) admissible = (t != s);
    else admissible = (t != s) && eta * std::max(diam(a), diam(b)) <= dist(a, b);
    if (admissible) {
      nd.kind = HNode::LR;
      nd.kmax = std::min(kmax, std::min(a.size, b.size));
      nd.rank = nd.kmax;
      h->nodes.push_back(nd);
      int id = (int)h->nodes.size() - 1;
      h->nodes[id].obj = h->add_obj(a.size, h->nodes[id].kmax);
      h->nodes[id].objV = h->add_obj(b.size, h->nodes[id].kmax);
      return id;
    }
    if (a.child[0] < 0 || b.child[0] < 0) {
      nd.kind = HNode::D;
      h->nodes.push_back(nd);
      int id = (int)h->nodes.size() - 1;
      h->nodes[id].obj = h->add_obj(a.size, b.size);
      return id;
    }
    nd.kind = HNode::H;
    h->nodes.push_back(nd);
    int id = (int)h->nodes.size() - 1;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        int c = block(cl[t].child[i], cl[s].child[j], level + 1);
        h->nodes[id].ch[i * 2 + j] = c;
      }
    return id;
  };
  h->root = block(0, 0, 0);
  h->add_inverses();
  return h;
}

void Hierarchical::ensure_host() const {
  if (!host.empty() || arena_elems == 0) return;
  host.assign((size_t)arena_elems, 0.0);
  for (auto& nd : nodes)
    if (nd.kind == HNode::LR && nd.rank_obj >= 0) host[objs[nd.rank_obj].off] = nd.rank;
}

int Hierarchical::stored_rank(int node) const {
  const HNode& nd = nodes.at(node);
  if (nd.kind != HNode::LR || nd.rank_obj < 0) return -1;
  if (host.empty()) return nd.rank;
  return (int)host[objs[nd.rank_obj].off];
}

void Hierarchical::set_rank_tolerance(double tol) {
  rank_tol = tol > 0.0 ? tol : 0.0;
  for (auto& nd : nodes)
    if (nd.kind == HNode::LR) {
      if (rank_tol > 0.0) nd.rank = nd.kmax;
      else if (!host.empty()) nd.rank = std::min(nd.kmax, std::max(0, (int)host[objs[nd.rank_obj].off]));
    }
}

int Hierarchical::count(HNode::Kind k) const {
  int c = 0;
  for (auto& nd : nodes) c += nd.kind == k;
  return c;
}

int Hierarchical::depth() const {
  int d = 0;
  for (auto& nd : nodes) d = std::max(d, nd.level);
  return d;
}

void Hierarchical::set_dense(int id, const double* a, int lda) {
  const HNode& nd = nodes.at(id);
  if (nd.kind != HNode::D) throw std::invalid_argument("set_dense: block is not dense");
  ensure_host();
  const StorageObj& o = objs[nd.obj];
  for (int i = 0; i < nd.m; ++i) std::memcpy(&host[o.off + (int64_t)i * o.ld], a + (int64_t)i * lda, sizeof(double) * nd.n);
}

void Hierarchical::set_lowrank(int id, const double* U, int ldu, const double* V, int ldv, int rank) {
  HNode& nd = nodes.at(id);
  if (nd.kind != HNode::LR) throw std::invalid_argument("set_lowrank: block is not low-rank");
  if (rank < 0 || rank > nd.kmax) throw std::invalid_argument("set_lowrank: rank exceeds kmax");
  ensure_host();
  nd.rank = rank_tol > 0.0 ? nd.kmax : rank;
  if (nd.rank_obj >= 0 && !host.empty()) host[objs[nd.rank_obj].off] = rank;
  const StorageObj& ou = objs[nd.obj];
  const StorageObj& ov = objs[nd.objV];
  for (int i = 0; i < nd.m; ++i)
    for (int r = 0; r < nd.kmax; ++r) host[ou.off + (int64_t)i * ou.ld + r] = r < rank ? U[(int64_t)i * ldu + r] : 0.0;
  for (int i = 0; i < nd.n; ++i)
    for (int r = 0; r < nd.kmax; ++r) host[ov.off + (int64_t)i * ov.ld + r] = r < rank ? V[(int64_t)i * ldv + r] : 0.0;
}

void Hierarchical::to_dense(double* out) const {
  ensure_host();
  for (const HNode& nd : nodes) {
    if (nd.kind == HNode::D) {
      const StorageObj& o = objs[nd.obj];
      for (int i = 0; i < nd.m; ++i)
        for (int j = 0; j < nd.n; ++j) out[(int64_t)(nd.r0 + i) * n + nd.c0 + j] = host[o.off + (int64_t)i * o.ld + j];
    } else if (nd.kind == HNode::LR) {
      const StorageObj& ou = objs[nd.obj];
      const StorageObj& ov = objs[nd.objV];
      for (int i = 0; i < nd.m; ++i)
        for (int j = 0; j < nd.n; ++j) {
          double s = 0;
          for (int r = 0; r < nd.rank; ++r) s += host[ou.off + (int64_t)i * ou.ld + r] * host[ov.off + (int64_t)j * ov.ld + r];
          out[(int64_t)(nd.r0 + i) * n + nd.c0 + j] = s;
        }
    }
  }
}

int64_t Hierarchical::storage_elems() const {
  int64_t s = 0;
  for (auto& nd : nodes) {
    if (nd.kind == HNode::D) s += (int64_t)nd.m * nd.n;
    else if (nd.kind == HNode::LR) s += (int64_t)nd.rank * (nd.m + nd.n);
  }
  return s;
}

}  // namespace pp
