// dag.cu — the dependency DAG of an instruction program built on the device.
//
// Replaces the host-side dependency discovery of the reference (rts/ops.cpp:42-61
// `Operation::checkDependencyFrom` over every earlier instruction, rts/dependency.cpp's table)
// and of this engine's Program::build_dag, with the same result, edge for edge and bit for bit:
//
//   every (task, region) access becomes one record; records are ordered by (object, task,
//   region index) with a stable radix sort; one thread per record walks its object's earlier
//   records newest first, exactly as the host walks an object's access list:
//     * records of the same task are skipped;
//     * a record that does not overlap this region is skipped;
//     * a record covered by a write met earlier in the walk is skipped (the host has
//       dropped it from its list when that write was inserted: anything it orders is
//       ordered through that write);
//     * otherwise the pair gets its dependency type (flow: write then read, anti: read then
//       write, out: write then write) and, when the record is a write covering this region,
//       the walk stops (everything older is ordered before that write).
//   The writes met are kept per thread (at most kWalkWrites; more sets an overflow flag and
//   the caller falls back to the host build).  Edges are emitted in two passes (count, then
//   fill at scanned offsets), sorted by (task, predecessor) and merged with a bitwise OR of
//   their types: each task's predecessor list comes out sorted, as the host's.
//
// Only the longest-path weights (bottom levels) stay on the host: one reverse sweep over the
// edges in program order.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <chrono>
#include <string>
#include <vector>

#include "hops.h"

namespace {

struct Access {
  int obj, task, r0, c0, r1, c1, ro, pad;  // rows [r0, r1), columns [c0, c1)
};

constexpr int kWalkWrites = 96;  // writes one walk keeps for the covered-record test
constexpr int kThreads = 128;

__device__ __forceinline__ bool overlaps(const Access& a, const Access& b) {
  return a.r0 < b.r1 && b.r0 < a.r1 && a.c0 < b.c1 && b.c0 < a.c1;
}

__device__ __forceinline__ bool covers(int4 w, const Access& b) {
  return w.x <= b.r0 && b.r1 <= w.z && w.y <= b.c0 && b.c1 <= w.w;
}

__global__ void gather_sorted(const Access* __restrict__ in, const int* __restrict__ idx, Access* __restrict__ out,
                              long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = in[idx[p]];
}

__global__ void mark_starts(const Access* __restrict__ acc, long long n, long long* __restrict__ obj_start) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && (p == 0 || acc[p - 1].obj != acc[p].obj)) obj_start[acc[p].obj] = p;
}

template <bool FILL>
__global__ void __launch_bounds__(kThreads) walk(const Access* __restrict__ acc, long long n,
                                                 const long long* __restrict__ obj_start,
                                                 long long* __restrict__ count, const long long* __restrict__ offs,
                                                 unsigned long long* __restrict__ keys,
                                                 unsigned char* __restrict__ types, int* __restrict__ overflow) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const Access me = acc[p];
  const long long start = obj_start[me.obj];
  int4 W[kWalkWrites];
  int nw = 0;
  long long cnt = 0, o = FILL ? offs[p] : 0;
  for (long long q = p - 1; q >= start; --q) {
    const Access e = acc[q];
    if (e.task == me.task || !overlaps(e, me)) continue;
    bool hidden = false;
    for (int i = 0; i < nw; ++i)
      if (covers(W[i], e)) { hidden = true; break; }
    if (hidden) continue;
    const int d = (!e.ro && me.ro) ? 1 : (e.ro && !me.ro) ? 2 : (!e.ro && !me.ro) ? 4 : 0;
    if (d) {
      if (FILL) {
        keys[o] = ((unsigned long long)(unsigned)me.task << 32) | (unsigned)e.task;
        types[o] = (unsigned char)d;
        ++o;
      } else {
        ++cnt;
      }
    }
    if (!e.ro) {
      if (e.r0 <= me.r0 && me.r1 <= e.r1 && e.c0 <= me.c0 && me.c1 <= e.c1) break;
      if (nw < kWalkWrites) W[nw++] = make_int4(e.r0, e.c0, e.r1, e.c1);
      else *overflow = 1;
    }
  }
  if (!FILL) count[p] = cnt;
}

struct OrOp {
  __device__ __forceinline__ unsigned char operator()(unsigned char a, unsigned char b) const { return a | b; }
};

// device buffers of one build, freed on every exit path
struct Buffers {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  ~Buffers() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    cudaError_t e = cudaMallocAsync((void**)p, sizeof(T) * (count ? count : 1), s);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

int bits_for(long long v) {
  int b = 1;
  while (b < 63 && (1LL << b) <= v) ++b;
  return b;
}

}  // namespace

namespace pp {

#define DAG_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      return false;                                                           \
    }                                                                         \
  } while (0)

// Builds succ / pred / pred_bits / edges / blevel of `prog` on the current device; the result
// equals Program::build_dag's.  Returns false (prog's DAG left empty, err set) when a CUDA call
// fails or a walk met more writes than it keeps; the caller then builds on the host.
bool build_dag_device(Program& prog, std::string& err, double* device_ms) {
  const int n = (int)prog.tasks.size();
  prog.succ.assign(n, {});
  prog.pred.assign(n, {});
  prog.pred_bits.assign(n, {});
  prog.edges = 0;
  std::vector<Access> h;
  for (int t = 0; t < n; ++t)
    for (const Region& r : prog.tasks[t].regions)
      h.push_back(Access{r.obj, t, r.r0, r.c0, r.r0 + r.nr, r.c0 + r.nc, r.ro ? 1 : 0, 0});
  const long long na = (long long)h.size();
  if (na >= (1LL << 31) - 1) {  // the sorts and scans count items in int
    err = "more than 2^31 accesses";
    return false;
  }
  auto t0 = std::chrono::steady_clock::now();
  std::vector<unsigned long long> ekeys;
  std::vector<unsigned char> etypes;
  if (na > 0) {
    Buffers B;
    DAG_CUDA(cudaStreamCreateWithFlags(&B.s, cudaStreamNonBlocking));
    cudaStream_t s = B.s;
    Access *d_in = nullptr, *d_acc = nullptr;
    int *d_obj = nullptr, *d_obj_sorted = nullptr, *d_idx = nullptr, *d_idx_sorted = nullptr, *d_over = nullptr;
    long long *d_start = nullptr, *d_count = nullptr, *d_offs = nullptr;
    DAG_CUDA(B.alloc(&d_in, na));
    DAG_CUDA(B.alloc(&d_acc, na));
    DAG_CUDA(B.alloc(&d_obj, na));
    DAG_CUDA(B.alloc(&d_obj_sorted, na));
    DAG_CUDA(B.alloc(&d_idx, na));
    DAG_CUDA(B.alloc(&d_idx_sorted, na));
    DAG_CUDA(B.alloc(&d_over, 1));
    DAG_CUDA(B.alloc(&d_start, prog.objs.size()));
    DAG_CUDA(B.alloc(&d_count, na + 1));  // one more slot, zero: its scanned offset is the total
    DAG_CUDA(B.alloc(&d_offs, na + 1));
    std::vector<int> ho(na), hi(na);
    for (long long i = 0; i < na; ++i) {
      ho[i] = h[i].obj;
      hi[i] = (int)i;
    }
    DAG_CUDA(cudaMemcpyAsync(d_in, h.data(), sizeof(Access) * na, cudaMemcpyHostToDevice, s));
    DAG_CUDA(cudaMemcpyAsync(d_obj, ho.data(), sizeof(int) * na, cudaMemcpyHostToDevice, s));
    DAG_CUDA(cudaMemcpyAsync(d_idx, hi.data(), sizeof(int) * na, cudaMemcpyHostToDevice, s));
    DAG_CUDA(cudaMemsetAsync(d_over, 0, sizeof(int), s));
    // stable sort by object: records of one object stay in (task, region) order
    size_t tmp_bytes = 0, need = 0;
    DAG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need, d_obj, d_obj_sorted, d_idx, d_idx_sorted, (int)na, 0,
                                             bits_for((long long)prog.objs.size()), s));
    tmp_bytes = std::max(tmp_bytes, need);
    DAG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, need, d_count, d_offs, (int)(na + 1), s));
    tmp_bytes = std::max(tmp_bytes, need);
    void* d_tmp = nullptr;
    DAG_CUDA(B.alloc((char**)&d_tmp, tmp_bytes));
    need = tmp_bytes;
    DAG_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, need, d_obj, d_obj_sorted, d_idx, d_idx_sorted, (int)na, 0,
                                             bits_for((long long)prog.objs.size()), s));
    const unsigned grid = (unsigned)((na + kThreads - 1) / kThreads);
    gather_sorted<<<grid, kThreads, 0, s>>>(d_in, d_idx_sorted, d_acc, na);
    mark_starts<<<grid, kThreads, 0, s>>>(d_acc, na, d_start);
    walk<false><<<grid, kThreads, 0, s>>>(d_acc, na, d_start, d_count, nullptr, nullptr, nullptr, d_over);
    DAG_CUDA(cudaGetLastError());
    DAG_CUDA(cudaMemsetAsync(d_count + na, 0, sizeof(long long), s));
    need = tmp_bytes;
    DAG_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, need, d_count, d_offs, (int)(na + 1), s));
    long long total = 0;
    int over = 0;
    DAG_CUDA(cudaMemcpyAsync(&total, d_offs + na, sizeof(long long), cudaMemcpyDeviceToHost, s));
    DAG_CUDA(cudaMemcpyAsync(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost, s));
    DAG_CUDA(cudaStreamSynchronize(s));
    if (over) {
      err = "a dependency walk met more than " + std::to_string(kWalkWrites) + " partial writes";
      return false;
    }
    if (total >= (1LL << 31) - 1) {
      err = "more than 2^31 dependency pairs before merging";
      return false;
    }
    if (total > 0) {
      unsigned long long *d_keys = nullptr, *d_keys_sorted = nullptr, *d_ukeys = nullptr;
      unsigned char *d_types = nullptr, *d_types_sorted = nullptr, *d_utypes = nullptr;
      int* d_runs = nullptr;
      DAG_CUDA(B.alloc(&d_keys, total));
      DAG_CUDA(B.alloc(&d_keys_sorted, total));
      DAG_CUDA(B.alloc(&d_ukeys, total));
      DAG_CUDA(B.alloc(&d_types, total));
      DAG_CUDA(B.alloc(&d_types_sorted, total));
      DAG_CUDA(B.alloc(&d_utypes, total));
      DAG_CUDA(B.alloc(&d_runs, 1));
      walk<true><<<grid, kThreads, 0, s>>>(d_acc, na, d_start, nullptr, d_offs, d_keys, d_types, d_over);
      DAG_CUDA(cudaGetLastError());
      const int kbits = 32 + bits_for(n);
      size_t need2 = 0, need3 = 0;
      DAG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, need2, d_keys, d_keys_sorted, d_types, d_types_sorted,
                                               (int)total, 0, kbits, s));
      DAG_CUDA(cub::DeviceReduce::ReduceByKey(nullptr, need3, d_keys_sorted, d_ukeys, d_types_sorted, d_utypes,
                                              d_runs, OrOp(), (int)total, s));
      void* d_tmp2 = nullptr;
      DAG_CUDA(B.alloc((char**)&d_tmp2, std::max(need2, need3)));
      DAG_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp2, need2, d_keys, d_keys_sorted, d_types, d_types_sorted,
                                               (int)total, 0, kbits, s));
      DAG_CUDA(cub::DeviceReduce::ReduceByKey(d_tmp2, need3, d_keys_sorted, d_ukeys, d_types_sorted, d_utypes,
                                              d_runs, OrOp(), (int)total, s));
      int runs = 0;
      DAG_CUDA(cudaMemcpyAsync(&runs, d_runs, sizeof(int), cudaMemcpyDeviceToHost, s));
      DAG_CUDA(cudaStreamSynchronize(s));
      ekeys.resize(runs);
      etypes.resize(runs);
      DAG_CUDA(cudaMemcpyAsync(ekeys.data(), d_ukeys, sizeof(unsigned long long) * runs, cudaMemcpyDeviceToHost, s));
      DAG_CUDA(cudaMemcpyAsync(etypes.data(), d_utypes, runs, cudaMemcpyDeviceToHost, s));
      DAG_CUDA(cudaStreamSynchronize(s));
    }
  }
  if (device_ms) *device_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  // per-task lists: keys are sorted by (task, predecessor), so each pred list is sorted and
  // each succ list fills in increasing task order, as on the host
  std::vector<int> npred(n, 0), nsucc(n, 0);
  for (unsigned long long k : ekeys) {
    ++npred[(int)(k >> 32)];
    ++nsucc[(int)(k & 0xffffffffu)];
  }
  for (int t = 0; t < n; ++t) {
    prog.pred[t].reserve(npred[t]);
    prog.pred_bits[t].reserve(npred[t]);
    prog.succ[t].reserve(nsucc[t]);
  }
  for (size_t i = 0; i < ekeys.size(); ++i) {
    const int t = (int)(ekeys[i] >> 32), p = (int)(ekeys[i] & 0xffffffffu);
    prog.pred[t].push_back(p);
    prog.pred_bits[t].push_back(etypes[i]);
    prog.succ[p].push_back(t);
  }
  prog.edges = (int64_t)ekeys.size();
  prog.finish_dag();
  return true;
}

}  // namespace pp
