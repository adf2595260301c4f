// rts.cpp — overlap predicate, dependency classification, typed edge table,
// static list scheduler.  See rts.h for the reference each piece mirrors.
#include "rts.h"

#include <algorithm>
#include <list>

namespace pp {

// Two pitched regions share a byte iff one row of each intersects.  Rows of the
// later-starting region b that can meet row i of a are found by arithmetic, so the
// cost is O(rows of a that lie inside b's span) (the reference walks the same rows,
// rts/ops.cpp:20-37).  Empty regions overlap nothing.
bool DataMap2D::checkOverlap(const DataMap2D& other) const {
  if (width == 0 || height == 0 || other.width == 0 || other.height == 0) return false;
  const DataMap2D& a = (ptr <= other.ptr) ? *this : other;
  const DataMap2D& b = (ptr <= other.ptr) ? other : *this;
  const int64_t pa = (int64_t)a.pitch, pb = (int64_t)b.pitch;
  const int64_t wa = (int64_t)a.width, wb = (int64_t)b.width;
  const int64_t ha = (int64_t)a.height, hb = (int64_t)b.height;
  const int64_t d = (int64_t)(b.ptr - a.ptr);  // >= 0: b's start relative to a's start
  const int64_t b_end = d + (hb - 1) * pb + wb;  // one past b's last byte (relative)
  if (pa == 0) {  // degenerate pitch: a is one row repeated
    const int64_t s = 0, e = wa;
    int64_t j = (s - d - wb < 0) ? 0 : (s - d - wb) / (pb ? pb : 1) + 1;
    return j < hb && d + j * pb < e;
  }
  for (int64_t i = d / pa; i < ha; ++i) {
    const int64_t s = i * pa, e = s + wa;  // row i of a: [s, e)
    if (s >= b_end) break;
    // first row j of b whose end lies beyond s: j*pb + wb > s - d
    int64_t j;
    if (s - d - wb < 0) j = 0;
    else j = (pb == 0) ? hb : (s - d - wb) / pb + 1;
    if (j < hb && d + j * pb < e) return true;
  }
  return false;
}

// RAW when an earlier write meets a later read, WAR when an earlier read meets a
// later write, WAW when both write (rts/ops.cpp:42-61; `first` = read-only).
dependency_t Operation::checkDependencyFrom(const Operation& op_from) const {
  dependency_t dep = dependency_t::no;
  for (const auto& f : op_from.data)
    for (const auto& t : data) {
      if (!f.second.checkOverlap(t.second)) continue;
      if (!f.first && t.first) dep = dep + dependency_t::flow;
      if (f.first && !t.first) dep = dep + dependency_t::anti;
      if (!f.first && !t.first) dep = dep + dependency_t::out;
    }
  return dep;
}

void dependency_table::update(int64_t from, int64_t to, dependency_t dep) {
  auto key = std::make_pair(from, to);
  auto it = type_.find(key);
  if (dep > dependency_t::no) {
    if (it == type_.end()) {
      type_.emplace(key, dep);
      from_.emplace(from, to);
      to_.emplace(to, from);
    } else {
      it->second = dep;
    }
    return;
  }
  if (it == type_.end()) return;
  type_.erase(it);
  for (auto r = from_.equal_range(from); r.first != r.second; ++r.first)
    if (r.first->second == to) { from_.erase(r.first); break; }
  for (auto r = to_.equal_range(to); r.first != r.second; ++r.first)
    if (r.first->second == from) { to_.erase(r.first); break; }
}

dependency_t dependency_table::lookup(int64_t from, int64_t to) const {
  auto it = type_.find(std::make_pair(from, to));
  return it == type_.end() ? dependency_t::no : it->second;
}

void dependency_table::getDepFrom(int64_t from, std::vector<int64_t>& lis) const {
  lis.clear();
  for (auto r = from_.equal_range(from); r.first != r.second; ++r.first) lis.push_back(r.first->second);
}

void dependency_table::getDepTo(int64_t to, std::vector<int64_t>& lis) const {
  lis.clear();
  for (auto r = to_.equal_range(to); r.first != r.second; ++r.first) lis.push_back(r.first->second);
}

size_t dependency_table::countDepFrom(int64_t from) const { return from_.count(from); }
size_t dependency_table::countDepTo(int64_t to) const { return to_.count(to); }

void dependency_table::clear() {
  type_.clear();
  from_.clear();
  to_.clear();
}

std::vector<int> h_ops_dag::getDepCountList_To() const {
  std::vector<int> c(length);
  for (int i = 0; i < length; ++i) c[i] = (int)pred[i].size();
  return c;
}

int64_t h_ops_dag::getFlops() const {
  int64_t s = 0;
  for (auto f : flops) s += f;
  return s;
}

double h_ops_dag::dag_density() const {
  if (length < 2) return 0.0;
  int64_t e = 0;
  for (auto& s : succ) e += (int64_t)s.size();
  return (double)e / ((double)length * (length - 1) / 2.0);
}

// ---------------------------------------------------------------------------
// Static list scheduler.  Same heuristics as the reference (rts/scheduler.cpp):
//  * ready entries are kept ordered by the FLOP time their last input finishes
//    (max_sync); new entries go after every existing entry with max_sync <= theirs;
//  * "start early / least wait": if the least loaded worker is already past the
//    head's max_sync, among the entries already startable pick the one with the
//    most successors (:163-200);
//  * the chosen worker is the one that finishes latest while still before max_sync,
//    else the earliest after it (:267-287);
//  * waits on instructions whose completion an earlier wait already implies are
//    dropped (:289-304).
instructions_scheduler::instructions_scheduler(const h_ops_dag& dag, int workers, int64_t min_inst_flops)
    : workers_(workers), queues_(workers), executed_by_(dag.length, -1) {
  struct Ready {
    int inst, num_deps;
    int64_t flops, max_sync;
    std::vector<int> sync_with;
  };
  const int n = dag.length;
  std::vector<int64_t> flops_after(n, 0), flops_worker(workers, 0);
  std::vector<int64_t> last_sync((size_t)workers * workers, 0);
  std::vector<int> indeg = dag.getDepCountList_To();

  auto make_ready = [&](int inst) {
    Ready r;
    r.inst = inst;
    r.num_deps = dag.getDepCount_From(inst);
    r.flops = dag.getFlops_Trim(inst, min_inst_flops);
    r.max_sync = 0;
    r.sync_with.assign(workers, -1);
    std::vector<int64_t> latest(workers, 0);
    for (int p : dag.pred[inst]) {
      const int w = executed_by_[p];
      const int64_t f = flops_after[p];
      if (latest[w] < f) { latest[w] = f; r.sync_with[w] = p; }
      if (r.max_sync < f) r.max_sync = f;
    }
    return r;
  };
  // insert `incoming` (ordered) after the head of `q`, each after every entry with
  // max_sync <= its own (rts/scheduler.cpp:269-288)
  auto hookup = [](std::list<Ready>& q, std::list<Ready>& incoming) {
    auto it = std::next(q.begin());
    while (!incoming.empty()) {
      const int64_t s = incoming.front().max_sync;
      while (it != q.end() && it->max_sync <= s) ++it;
      q.splice(it, incoming, incoming.begin());
    }
  };

  std::list<Ready> work;
  for (int i = 0; i < n; ++i)
    if (indeg[i] == 0) work.push_front(make_ready(i));

  int64_t flops_total = 0;
  int waits = 0;
  for (int done = 0; done < n; ++done) {
    const int64_t smallest = *std::min_element(flops_worker.begin(), flops_worker.end());
    auto target = work.begin();
    if (!(smallest < work.front().max_sync)) {
      int max_n = work.front().num_deps;
      for (auto it = std::next(work.begin()); it != work.end() && it->max_sync <= smallest; ++it)
        if (it->num_deps > max_n) { max_n = it->num_deps; target = it; }
    }
    Ready r = std::move(*target);
    work.erase(target);

    // findWorkerWithMinimalWaiting
    int before = -1, after = 0;
    int64_t latest_before = -1, earliest_after = flops_worker[0];
    for (int w = 0; w < workers; ++w) {
      const int64_t f = flops_worker[w];
      if (f <= r.max_sync && f > latest_before) { before = w; latest_before = f; }
      else if (f > r.max_sync && f < earliest_after) { after = w; earliest_after = f; }
    }
    const int wk = before >= 0 ? before : after;

    // eliminateExtraSync
    r.sync_with[wk] = -1;
    for (int w = 0; w < workers; ++w) {
      const int s = r.sync_with[w];
      if (s >= 0 && flops_after[s] <= last_sync[(size_t)wk * workers + w]) r.sync_with[w] = -1;
    }
    for (int w = 0; w < workers; ++w) {
      const int s = r.sync_with[w];
      if (s < 0) continue;
      queues_[wk].push_back({s, false});
      if (flops_worker[wk] < flops_after[s]) flops_worker[wk] = flops_after[s];
      last_sync[(size_t)wk * workers + executed_by_[s]] = flops_after[s];
      ++waits;
    }
    queues_[wk].push_back({r.inst, true});
    flops_after[r.inst] = (flops_worker[wk] += r.flops);
    executed_by_[r.inst] = wk;
    flops_total += r.flops;

    // updateDepsCounts
    std::list<Ready> fresh;
    for (int s : dag.succ[r.inst]) {
      if (--indeg[s] != 0) continue;
      Ready e = make_ready(s);
      if (fresh.empty() || e.max_sync <= fresh.front().max_sync) {
        fresh.push_front(std::move(e));
      } else {
        std::list<Ready> one;
        one.push_back(std::move(e));
        hookup(fresh, one);
      }
    }
    if (work.empty()) work.swap(fresh);
    else if (!fresh.empty()) hookup(work, fresh);
  }

  int64_t max_w = 0;
  for (auto f : flops_worker) max_w = std::max(max_w, f);
  if (n > 0 && max_w > 0) {
    heaviest_worker_pct = 100.0 * max_w / flops_total;
    utilization_pct = 100.0 * flops_total / max_w / workers;
    comm_per_inst = (double)waits / n;
  }
}

std::vector<int> instructions_scheduler::getLengths() const {
  std::vector<int> l(workers_);
  for (int w = 0; w < workers_; ++w) l[w] = (int)queues_[w].size();
  return l;
}

}  // namespace pp
