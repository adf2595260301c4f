// rts.h — DAG primitives and the static scheduler of the H-LU runtime.
//
// Mirrors the reference's runtime layer (Pastel-Palettes rts/ops.h, rts/dependency.h,
// rts/scheduler.h) with the same names and meanings:
//   DataMap2D::checkOverlap          rts/ops.h:9-20, rts/ops.cpp:7-40
//   Operation::checkDependencyFrom   rts/ops.h:22-36, rts/ops.cpp:42-64
//   dependency_t, dependency_table   rts/dependency.h:9-53, rts/dependency.cpp:7-76
//   instructions_scheduler           rts/scheduler.h:73-126, rts/scheduler.cpp:372-460
// The device side of this engine does not need the static schedule (it pulls ready
// tasks from a device queue), but the scheduler is kept: it orders the reference-format
// per-worker instruction streams (pp_refstream_*) and reports the same summary figures.
#pragma once
#include <cstddef>
#include <cstdint>
#include <map>
#include <set>
#include <utility>
#include <vector>

namespace pp {

// A pitched 2-D byte region: `height` rows of `width` bytes, rows `pitch` bytes apart.
struct DataMap2D {
  uintptr_t ptr;
  size_t pitch, width, height;
  DataMap2D() : ptr(0), pitch(0), width(0), height(0) {}
  DataMap2D(uintptr_t p, size_t pi, size_t w, size_t h) : ptr(p), pitch(pi), width(w), height(h) {}
  // true iff some byte belongs to both regions (rts/ops.cpp:7-40; defined for width <= pitch)
  bool checkOverlap(const DataMap2D& other) const;
};

enum class dependency_t : int {
  no = 0, flow = 1, anti = 2, flow_anti = 3, out = 4, flow_out = 5, anti_out = 6, flow_anti_out = 7
};
inline dependency_t operator+(dependency_t a, dependency_t b) { return (dependency_t)((int)a | (int)b); }
inline bool operator>(dependency_t a, dependency_t b) { return (int)a > (int)b; }

// The data an operation touches: (read_only, region) pairs.
struct Operation {
  std::vector<std::pair<bool, DataMap2D>> data;
  void addRead(const DataMap2D& d) { data.emplace_back(true, d); }
  void addWrite(const DataMap2D& d) { data.emplace_back(false, d); }
  // dependency of *this on an earlier op_from: flow (RAW), anti (WAR), out (WAW), OR-ed
  dependency_t checkDependencyFrom(const Operation& op_from) const;
  dependency_t checkDependencyTo(const Operation& op_to) const { return op_to.checkDependencyFrom(*this); }
};

// Typed edge set with from/to adjacency (rts/dependency.h:24-53).
class dependency_table {
 public:
  void update(int64_t from, int64_t to, dependency_t dep);  // dep == no erases the edge
  dependency_t lookup(int64_t from, int64_t to) const;
  void getDepFrom(int64_t from, std::vector<int64_t>& lis) const;  // successors of `from`
  void getDepTo(int64_t to, std::vector<int64_t>& lis) const;      // predecessors of `to`
  size_t countDepFrom(int64_t from) const;
  size_t countDepTo(int64_t to) const;
  size_t size() const { return type_.size(); }
  void clear();
 private:
  std::map<std::pair<int64_t, int64_t>, dependency_t> type_;
  std::multimap<int64_t, int64_t> from_, to_;
};

// The flattened DAG the scheduler consumes (interface of the reference's missing
// h_ops_dag, as used at rts/scheduler.cpp:73-77,240,334,433,451).
struct h_ops_dag {
  int length = 0;
  std::vector<std::vector<int>> succ, pred;  // adjacency, program order preserved
  std::vector<int64_t> flops;
  int getLength() const { return length; }
  int getDepCount_From(int i) const { return (int)succ[i].size(); }
  std::vector<int> getDepCountList_To() const;
  int64_t getFlops(int i) const { return flops[i]; }
  int64_t getFlops_Trim(int i, int64_t min_flops) const { return flops[i] > min_flops ? flops[i] : min_flops; }
  int64_t getFlops() const;
  double dag_density() const;
};

// Static FLOP-weighted list scheduler (rts/scheduler.cpp:372-460): assigns every
// instruction to one of `workers` queues and inserts waits on cross-worker
// dependencies that earlier waits do not already imply.
class instructions_scheduler {
 public:
  struct Entry { int inst; bool exe; };  // exe=false: wait for `inst` (executed elsewhere)
  instructions_scheduler(const h_ops_dag& dag, int workers, int64_t min_inst_flops = 1 << 16);
  const std::vector<Entry>& getSchedule(int worker) const { return queues_[worker]; }
  int getLength(int worker) const { return (int)queues_[worker].size(); }
  std::vector<int> getLengths() const;
  int getWorkers() const { return workers_; }
  int getExecutedBy(int inst) const { return executed_by_[inst]; }
  // summary figures of rts/scheduler.cpp:405-427
  double heaviest_worker_pct = 0, utilization_pct = 0, comm_per_inst = 0;
 private:
  int workers_;
  std::vector<std::vector<Entry>> queues_;
  std::vector<int> executed_by_;
};

}  // namespace pp
