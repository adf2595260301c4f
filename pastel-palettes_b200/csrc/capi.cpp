// capi.cpp — extern "C" boundary of the engine (include/pastel_palettes.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pastel_palettes.h"
#include "hmatrix.h"
#include "hops.h"
#include "rts.h"
#include "vm.cuh"

struct pp_context {
  int device = -1;   // -1: host-only context (planning, encoding; no compute)
  int sm_count = 0;
  int blocks_per_sm = 0;
  pp_config cfg{};
  std::string err;
  double* d_resid = nullptr;  // partial sums of the matrix-free residual (grown on demand)
  size_t resid_elems = 0;
  int dag_device = 0;         // 1: dependency discovery of new programs on the device (dag.cu)
  ~pp_context() { cudaFree(d_resid); }
};

namespace {

struct VmPlan {
  pp::Program prog;
  bool built = false;
  bool on_device = false;
  int n_tasks = 0, n_ready = 0;
  pp_task* d_tasks = nullptr;
  int32_t *d_succ = nullptr, *d_indeg = nullptr, *d_ready = nullptr, *d_counters = nullptr, *d_slots = nullptr;
  pp_vm_state* d_state = nullptr;
  double *d_work = nullptr, *d_scratch = nullptr, *d_rhs = nullptr;
  int64_t work_elems = 0, scratch_elems = 0, rhs_elems = 0;
  double build_ms = 0;
  double dag_ms = 0;       // wall time of the DAG build alone
  int dag_on_device = 0;   // 1: built by build_dag_device
  int grid = 0;
  int use_tc = 0;  // holds TF32 contractions (tensor memory per CTA)
  unsigned long long* d_trace = nullptr;  // per-task (start, end, sm | cta << 32) when tracing
  std::vector<int64_t> work_off, scratch_off, rhs_off;  // per instance (batched plans)
  // stream-ordered memory (cudaMallocAsync / cudaFreeAsync on `astream`, from `apool` when
  // set) for plans of a served request, so that allocating or freeing never waits for other
  // streams' work
  cudaStream_t astream = nullptr;
  cudaMemPool_t apool = nullptr;
  bool async_mem = false;
  void dfree(void* p) {
    if (!p) return;
    if (async_mem) cudaFreeAsync(p, astream);
    else cudaFree(p);
  }
  void release() {
    dfree(d_tasks); dfree(d_succ); dfree(d_indeg); dfree(d_ready); dfree(d_counters);
    dfree(d_slots); dfree(d_state); dfree(d_work); dfree(d_scratch); dfree(d_rhs);
    dfree(d_trace);
    d_tasks = nullptr; d_succ = d_indeg = d_ready = d_counters = d_slots = nullptr; d_state = nullptr;
    d_work = d_scratch = d_rhs = nullptr;
    d_trace = nullptr;
    on_device = false;
  }
};

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

struct pp_hmatrix {
  pp_context* ctx = nullptr;
  std::unique_ptr<pp::Hierarchical> H;
  double* d_arena = nullptr;
  double* d_orig = nullptr;
  double* d_rand = nullptr;
  bool pinned = false;
  int precision = PP_PREC_FP64;  // contraction precision of the factor's GEMM instructions
  int tile = 0;                  // dense tile of its programs (0: the context's)
  int gemm_tile = 64;            // output tile edge of its product tasks (64 or 128)
  int pivoting = 0;              // 1: partial pivoting inside the GETRF blocks (PP_PIVOT)
  std::vector<double> rand_host;
  VmPlan factor;
  std::map<int, std::unique_ptr<VmPlan>> solves;
  VmPlan construct;              // device construction of the low-rank blocks
  int c_kernel = -1, c_dim = 0;  // what the construction program was built for
  double c_p0 = 0.0;
  VmPlan* last = nullptr;
  // stream-ordered memory mode (set by the server for the requests it owns)
  cudaStream_t astream = nullptr;
  cudaMemPool_t apool = nullptr;
  bool async_mem = false;
  cudaError_t dalloc(void** p, size_t bytes) {
    bytes = bytes ? bytes : 8;
    if (!async_mem) return cudaMalloc(p, bytes);
    return apool ? cudaMallocFromPoolAsync(p, bytes, apool, astream) : cudaMallocAsync(p, bytes, astream);
  }
  void dfree(void* p) {
    if (!p) return;
    if (async_mem) cudaFreeAsync(p, astream);
    else cudaFree(p);
  }
  cudaError_t h2d(void* dst, const void* src, size_t bytes) {
    return async_mem ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, astream)
                     : cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  }
  void set_async(cudaStream_t s, cudaMemPool_t pool) {
    async_mem = true;
    astream = s;
    apool = pool;
    for (VmPlan* p : all_plans()) {
      p->async_mem = true;
      p->astream = s;
      p->apool = pool;
    }
  }
  std::vector<VmPlan*> all_plans() {
    std::vector<VmPlan*> v{&factor, &construct};
    for (auto& kv : solves) v.push_back(kv.second.get());
    return v;
  }
  ~pp_hmatrix() {
    factor.release();
    construct.release();
    for (auto& kv : solves) kv.second->release();
    if (pinned) cudaHostUnregister(H->host.data());
    dfree(d_arena);
    dfree(d_orig);
    dfree(d_rand);
  }
};

namespace {

pp_status fail(pp_context* c, pp_status s, const std::string& msg) {
  if (c) c->err = msg;
  return s;
}

pp_status cuda_fail(pp_context* c, cudaError_t e, const char* what) {
  return fail(c, e == cudaErrorMemoryAllocation ? PP_OOM : PP_CUDA_ERROR,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define PP_CUDA(call)                                          \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);   \
  } while (0)

bool has_device(const pp_context* c) { return c && c->device >= 0; }

void make_rand(pp_hmatrix* h) {
  const int64_t count = h->factor.prog.arena_elems.size() > (size_t)pp::AR_RAND
                            ? h->factor.prog.arena_elems[pp::AR_RAND]
                            : 0;
  h->rand_host.resize((size_t)count);
  uint64_t s = h->ctx->cfg.seed;
  for (int64_t i = 0; i < count; ++i) {
    const uint64_t z = splitmix64(s);
    // uniform in [-1, 1): 53 random bits
    h->rand_host[(size_t)i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// op generation + DAG for the factor (which = 0) or solve (which = 1) program
pp_status build_program(pp_hmatrix* h, int which, int nrhs, VmPlan& plan) {
  pp_context* ctx = h->ctx;
  if (plan.built) return PP_OK;
  auto t0 = std::chrono::steady_clock::now();
  try {
    pp::Generator g(plan.prog, *h->H, h->tile > 0 ? h->tile : ctx->cfg.tile, h->H->n, ctx->cfg.reference_isa == 0);
    g.use_inverses(ctx->cfg.reference_isa == 0);
    if (h->pivoting) g.use_pivoting(true);
    if (which == 0) g.set_gemm_tile(h->gemm_tile);  // the solve's products keep 64
    if (which == 0) {
      if (h->precision == PP_PREC_BF16) g.set_precision(PP_PREC_BF16);
      g.getrf_program();
      if (h->precision == PP_PREC_BF16) plan.prog.merge_bf16_updates();
      if (h->precision == PP_PREC_TF32) plan.prog.set_gemm_precision(h->precision);
    } else if (which == 2) {
      g.construct_program(h->c_kernel, h->c_dim, h->c_p0, h->H->rank_tol);
    } else {
      g.solve_program(nrhs);
    }
    auto td = std::chrono::steady_clock::now();
    bool dev = false;
    if (ctx->dag_device && has_device(ctx)) {
      std::string derr;
      int prev = -1;
      cudaGetDevice(&prev);
      if (prev != ctx->device) cudaSetDevice(ctx->device);
      dev = pp::build_dag_device(plan.prog, derr, nullptr);
      if (prev != ctx->device && prev >= 0) cudaSetDevice(prev);
      if (!dev) ctx->err = "device DAG build fell back to the host: " + derr;  // not an error
    }
    if (!dev) plan.prog.build_dag();
    plan.dag_on_device = dev ? 1 : 0;
    plan.dag_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - td).count();
  } catch (const std::exception& e) {
    plan.prog = pp::Program();
    return fail(ctx, PP_UNSUPPORTED, std::string("program generation: ") + e.what());
  }
  plan.n_tasks = (int)plan.prog.tasks.size();
  plan.work_elems = plan.prog.arena_elems[pp::AR_WORK];
  plan.scratch_elems = plan.prog.arena_elems[pp::AR_SCRATCH];
  plan.rhs_elems = plan.prog.arena_elems[pp::AR_RHS];
  plan.built = true;
  plan.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return PP_OK;
}

// Device copy of a program over one or more instances (a batch merges their programs):
// one contiguous work / scratch / rhs buffer each, instance j at offsets *_off[j].
pp_status plan_to_device_multi(pp_context* ctx, const std::vector<pp_hmatrix*>& insts, VmPlan& plan) {
  if (plan.on_device) return PP_OK;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  for (auto* h : insts)
    if (!h->d_arena || !h->d_rand) return fail(ctx, PP_INVALID_ARG, "H-matrix not uploaded");
  if ((int)insts.size() != plan.prog.n_instances) return fail(ctx, PP_INTERNAL, "instance count mismatch");
  auto t0 = std::chrono::steady_clock::now();
  const int n = plan.n_tasks;
  auto alloc = [&](void** p, size_t bytes) {
    bytes = bytes ? bytes : 8;
    if (!plan.async_mem) return cudaMalloc(p, bytes);
    return plan.apool ? cudaMallocFromPoolAsync(p, bytes, plan.apool, plan.astream)
                      : cudaMallocAsync(p, bytes, plan.astream);
  };
  auto h2d = [&](void* dst, const void* src, size_t bytes) {
    return plan.async_mem ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, plan.astream)
                          : cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  };
  const int ni = (int)insts.size();
  plan.work_off.assign(ni, 0);
  plan.scratch_off.assign(ni, 0);
  plan.rhs_off.assign(ni, 0);
  plan.work_elems = plan.scratch_elems = plan.rhs_elems = 0;
  for (int j = 0; j < ni; ++j) {
    auto grow = [](int64_t& total, int64_t add) {
      const int64_t at = (total + 31) & ~int64_t(31);
      total = at + add;
      return at;
    };
    plan.work_off[j] = grow(plan.work_elems, plan.prog.arena_elems[j * pp::PP_ARENAS + pp::AR_WORK]);
    plan.scratch_off[j] = grow(plan.scratch_elems, plan.prog.arena_elems[j * pp::PP_ARENAS + pp::AR_SCRATCH]);
    plan.rhs_off[j] = grow(plan.rhs_elems, plan.prog.arena_elems[j * pp::PP_ARENAS + pp::AR_RHS]);
  }
  PP_CUDA(alloc((void**)&plan.d_work, sizeof(double) * plan.work_elems));
  PP_CUDA(alloc((void**)&plan.d_scratch, sizeof(double) * plan.scratch_elems));
  PP_CUDA(alloc((void**)&plan.d_rhs, sizeof(double) * plan.rhs_elems));
  std::vector<double*> bases((size_t)ni * pp::PP_ARENAS);
  for (int j = 0; j < ni; ++j) {
    bases[j * pp::PP_ARENAS + pp::AR_MATRIX] = insts[j]->d_arena;
    bases[j * pp::PP_ARENAS + pp::AR_WORK] = plan.d_work + plan.work_off[j];
    bases[j * pp::PP_ARENAS + pp::AR_SCRATCH] = plan.d_scratch + plan.scratch_off[j];
    bases[j * pp::PP_ARENAS + pp::AR_RHS] = plan.d_rhs + plan.rhs_off[j];
    bases[j * pp::PP_ARENAS + pp::AR_RAND] = insts[j]->d_rand;
  }
  std::vector<pp_task> tasks;
  std::vector<int32_t> succ, indeg, ready;
  plan.prog.encode(bases, tasks, succ, indeg, ready);
  plan.n_ready = (int)ready.size();
  plan.use_tc = 0;
  for (const auto& t : tasks)
    if (t.prec == PP_PREC_TF32 || t.prec == PP_PREC_BF16) plan.use_tc = 1;
  PP_CUDA(alloc((void**)&plan.d_tasks, sizeof(pp_task) * n));
  PP_CUDA(alloc((void**)&plan.d_succ, sizeof(int32_t) * succ.size()));
  PP_CUDA(alloc((void**)&plan.d_indeg, sizeof(int32_t) * n));
  PP_CUDA(alloc((void**)&plan.d_ready, sizeof(int32_t) * ready.size()));
  PP_CUDA(alloc((void**)&plan.d_counters, sizeof(int32_t) * n));
  PP_CUDA(alloc((void**)&plan.d_slots, sizeof(int32_t) * n));
  PP_CUDA(alloc((void**)&plan.d_state, sizeof(pp_vm_state)));
  PP_CUDA(h2d(plan.d_tasks, tasks.data(), sizeof(pp_task) * n));
  if (!succ.empty()) PP_CUDA(h2d(plan.d_succ, succ.data(), sizeof(int32_t) * succ.size()));
  PP_CUDA(h2d(plan.d_indeg, indeg.data(), sizeof(int32_t) * n));
  if (!ready.empty()) PP_CUDA(h2d(plan.d_ready, ready.data(), sizeof(int32_t) * ready.size()));
  if (plan.async_mem) PP_CUDA(cudaMemsetAsync(plan.d_state, 0, sizeof(pp_vm_state), plan.astream));
  else PP_CUDA(cudaMemset(plan.d_state, 0, sizeof(pp_vm_state)));
  const int per_sm = ctx->cfg.ctas_per_sm > 0 ? std::min(ctx->cfg.ctas_per_sm, ctx->blocks_per_sm) : ctx->blocks_per_sm;
  plan.grid = std::max(1, std::min(n, ctx->sm_count * std::max(1, per_sm)));
  plan.on_device = true;
  plan.build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return PP_OK;
}

pp_status plan_to_device(pp_hmatrix* h, VmPlan& plan) { return plan_to_device_multi(h->ctx, {h}, plan); }

pp_status launch_plan(pp_context* ctx, VmPlan& plan, cudaStream_t s, int grid_cap) {
  if (plan.work_elems > 0) PP_CUDA(cudaMemsetAsync(plan.d_work, 0, sizeof(double) * plan.work_elems, s));
  pp_vm_launch L;
  L.tasks = plan.d_tasks;
  L.n_tasks = plan.n_tasks;
  L.succ = plan.d_succ;
  L.indeg = plan.d_indeg;
  L.ready = plan.d_ready;
  L.n_ready = plan.n_ready;
  L.counters = plan.d_counters;
  L.slots = plan.d_slots;
  L.state = plan.d_state;
  L.wait_ns = ctx->cfg.spin_limit * 1000;
  L.grid = grid_cap > 0 ? std::min(plan.grid, grid_cap) : plan.grid;
  L.trace = plan.d_trace;
  L.use_tc = plan.use_tc;
  PP_CUDA(pp_vm_run(L, s));
  return PP_OK;
}

pp_status launch_plan(pp_hmatrix* h, VmPlan& plan, cudaStream_t s, int grid_cap) {
  pp_status st = launch_plan(h->ctx, plan, s, grid_cap);
  if (st == PP_OK) h->last = &plan;
  return st;
}

// error record of a finished VM launch -> status and message
pp_status vm_state_status(pp_context* ctx, const pp_vm_state& s, int n_tasks) {
  if (s.error == PP_VM_TIMEOUT)
    return fail(ctx, PP_TIMEOUT, "VM: ready-queue slot " + std::to_string(s.err_info) + " never filled");
  if (s.error == PP_VM_MMA_TIMEOUT)
    return fail(ctx, PP_TIMEOUT, "VM: tensor-core completion of task " + std::to_string(s.err_info) + " not observed");
  if (s.error == PP_VM_BAD_TASK)
    return fail(ctx, PP_INTERNAL, "VM: task " + std::to_string(s.err_info) + " has unsupported shape");
  if (s.done != n_tasks)
    return fail(ctx, PP_INTERNAL, "VM: " + std::to_string(s.done) + " of " + std::to_string(n_tasks) + " tasks ran");
  return PP_OK;
}

// status of a finished launch (after the stream was synchronized)
pp_status plan_status(pp_context* ctx, VmPlan& plan) {
  pp_vm_state s;
  PP_CUDA(cudaMemcpy(&s, plan.d_state, sizeof(s), cudaMemcpyDeviceToHost));
  return vm_state_status(ctx, s, plan.n_tasks);
}

}  // namespace

extern "C" {

pp_status pp_context_create(int device, const pp_config* cfg, pp_context** out) {
  if (!out) return PP_INVALID_ARG;
  *out = nullptr;
  auto* c = new (std::nothrow) pp_context();
  if (!c) return PP_OOM;
  c->cfg.tile = 64;
  c->cfg.ctas_per_sm = 0;
  c->cfg.spin_limit = 120ll * 1000 * 1000;  // 120 s
  c->cfg.seed = 0x5eed5eedull;
  if (cfg) {
    if (cfg->tile > 0) c->cfg.tile = cfg->tile;
    c->cfg.ctas_per_sm = cfg->ctas_per_sm;
    if (cfg->spin_limit > 0) c->cfg.spin_limit = cfg->spin_limit;
    if (cfg->seed) c->cfg.seed = cfg->seed;
    c->cfg.reference_isa = cfg->reference_isa;
  }
  if (c->cfg.tile < 8 || c->cfg.tile > PP_VM_TILE) { delete c; return PP_INVALID_ARG; }
  c->device = device;
  if (device >= 0) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device >= count) { delete c; return PP_CUDA_ERROR; }
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return PP_CUDA_ERROR; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete c; return PP_CUDA_ERROR; }
    c->sm_count = prop.multiProcessorCount;
    if (pp_vm_prepare() != cudaSuccess) { delete c; return PP_CUDA_ERROR; }
    c->blocks_per_sm = pp_vm_blocks_per_sm();
    if (c->blocks_per_sm < 1) { delete c; return PP_CUDA_ERROR; }
  }
  *out = c;
  return PP_OK;
}

void pp_context_destroy(pp_context* ctx) { delete ctx; }

int pp_last_error(const pp_context* ctx, char* buf, size_t size) {
  if (!ctx) return 0;
  if (buf && size) {
    std::strncpy(buf, ctx->err.c_str(), size - 1);
    buf[size - 1] = 0;
  }
  return (int)ctx->err.size();
}

int pp_device_sm_count(const pp_context* ctx) { return ctx ? ctx->sm_count : 0; }

static pp_status wrap_hmatrix(pp_context* ctx, pp::Hierarchical* H, pp_hmatrix** out) {
  auto* h = new (std::nothrow) pp_hmatrix();
  if (!h) { delete H; return PP_OOM; }
  h->ctx = ctx;
  h->H.reset(H);
  *out = h;
  return PP_OK;
}

pp_status pp_hmatrix_create_dense(pp_context* ctx, int n, int leaf, pp_hmatrix** out) {
  if (!ctx || !out || n <= 0 || leaf <= 0) return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_create_dense: bad argument");
  try {
    return wrap_hmatrix(ctx, pp::Hierarchical::dense_tiled(n, leaf), out);
  } catch (const std::exception& e) {
    return fail(ctx, PP_INVALID_ARG, e.what());
  }
}

pp_status pp_hmatrix_create_geometric(pp_context* ctx, int n, int dim, const double* points, int leaf,
                                      int admissibility, double eta, int kmax, pp_hmatrix** out) {
  if (!ctx || !out || !points || n <= 0 || dim <= 0 || leaf <= 0 || kmax <= 0 || kmax > PP_VM_MAX_RANK ||
      (admissibility != 0 && admissibility != 1))
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_create_geometric: bad argument");
  try {
    return wrap_hmatrix(ctx, pp::Hierarchical::geometric(n, dim, points, leaf, admissibility, eta, kmax), out);
  } catch (const std::exception& e) {
    return fail(ctx, PP_INVALID_ARG, e.what());
  }
}

void pp_hmatrix_destroy(pp_hmatrix* h) { delete h; }

int pp_hmatrix_num_blocks(const pp_hmatrix* h) { return h ? (int)h->H->nodes.size() : 0; }
int pp_hmatrix_root(const pp_hmatrix* h) { return h ? h->H->root : -1; }

pp_status pp_hmatrix_block_info(const pp_hmatrix* h, int b, pp_block_info* info) {
  if (!h || !info || b < 0 || b >= (int)h->H->nodes.size()) return PP_INVALID_ARG;
  const pp::HNode& nd = h->H->nodes[b];
  info->kind = (int)nd.kind;
  info->row0 = nd.r0;
  info->col0 = nd.c0;
  info->m = nd.m;
  info->n = nd.n;
  info->rank = nd.rank;
  info->kmax = nd.kmax;
  info->level = nd.level;
  for (int i = 0; i < 4; ++i) info->children[i] = nd.ch[i];
  return PP_OK;
}

pp_status pp_hmatrix_block_storage(const pp_hmatrix* h, int b, long long* off, long long* off_v, long long* off_rank) {
  if (!h || b < 0 || b >= (int)h->H->nodes.size()) return PP_INVALID_ARG;
  const pp::HNode& nd = h->H->nodes[b];
  auto at = [&](int obj) -> long long { return obj >= 0 ? (long long)h->H->objs[obj].off : -1; };
  if (off) *off = at(nd.obj);
  if (off_v) *off_v = at(nd.objV);
  if (off_rank) *off_rank = at(nd.rank_obj);
  return PP_OK;
}

pp_status pp_hmatrix_set_dense(pp_hmatrix* h, int b, const double* a, int lda) {
  if (!h || !a) return PP_INVALID_ARG;
  try {
    if (lda < h->H->nodes.at(b).n) return fail(h->ctx, PP_INVALID_ARG, "lda smaller than the block width");
    h->H->set_dense(b, a, lda);
  } catch (const std::exception& e) {
    return fail(h->ctx, PP_INVALID_ARG, e.what());
  }
  return PP_OK;
}

pp_status pp_hmatrix_set_lowrank(pp_hmatrix* h, int b, const double* U, int ldu, const double* V, int ldv, int rank) {
  if (!h || !U || !V) return PP_INVALID_ARG;
  try {
    if (h->factor.built && rank != h->H->nodes.at(b).rank)
      return fail(h->ctx, PP_INVALID_ARG, "rank change after the factor program was built");
    h->H->set_lowrank(b, U, ldu, V, ldv, rank);
  } catch (const std::exception& e) {
    return fail(h->ctx, PP_INVALID_ARG, e.what());
  }
  return PP_OK;
}

// the random sketch of the accumulations (its size depends on the factor program's arenas)
static pp_status upload_rand(pp_hmatrix* h) {
  pp_context* ctx = h->ctx;
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st != PP_OK) return st;
  if (!h->d_rand) {
    make_rand(h);
    PP_CUDA(h->dalloc((void**)&h->d_rand, sizeof(double) * std::max<size_t>(h->rand_host.size(), 1)));
    PP_CUDA(h->h2d(h->d_rand, h->rand_host.data(), sizeof(double) * h->rand_host.size()));
  }
  return PP_OK;
}

pp_status pp_hmatrix_upload(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  const size_t bytes = sizeof(double) * (size_t)std::max<int64_t>(h->H->arena_elems, 1);
  if (!h->d_arena) PP_CUDA(h->dalloc((void**)&h->d_arena, bytes));
  h->H->ensure_host();
  PP_CUDA(cudaMemcpyAsync(h->d_arena, h->H->host.data(), sizeof(double) * h->H->block_elems, cudaMemcpyHostToDevice,
                          (cudaStream_t)stream));
  return upload_rand(h);
}

pp_status pp_hmatrix_download(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!h->d_arena) return fail(ctx, PP_INVALID_ARG, "H-matrix not uploaded");
  h->H->ensure_host();
  PP_CUDA(cudaMemcpyAsync(h->H->host.data(), h->d_arena, sizeof(double) * h->H->block_elems, cudaMemcpyDeviceToHost,
                          (cudaStream_t)stream));
  PP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_hmatrix_pin_host(pp_hmatrix* h) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (h->pinned) return PP_OK;
  h->H->ensure_host();
  if (h->H->host.empty()) return PP_OK;
  PP_CUDA(cudaHostRegister(h->H->host.data(), sizeof(double) * h->H->host.size(), cudaHostRegisterDefault));
  h->pinned = true;
  return PP_OK;
}

pp_status pp_hmatrix_keep_original(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!h->d_arena) return fail(ctx, PP_INVALID_ARG, "H-matrix not uploaded");
  const size_t bytes = sizeof(double) * (size_t)h->H->block_elems;
  if (!h->d_orig) PP_CUDA(h->dalloc((void**)&h->d_orig, std::max<size_t>(bytes, 8)));
  PP_CUDA(cudaMemcpyAsync(h->d_orig, h->d_arena, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_hmatrix_restore(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!h->d_orig) return fail(ctx, PP_INVALID_ARG, "no original kept (pp_hmatrix_keep_original)");
  PP_CUDA(cudaMemcpyAsync(h->d_arena, h->d_orig, sizeof(double) * (size_t)h->H->block_elems,
                          cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_hmatrix_set_precision(pp_hmatrix* h, int precision) {
  if (!h) return PP_INVALID_ARG;
  if (precision != PP_PREC_FP64 && precision != PP_PREC_TF32 && precision != PP_PREC_BF16)
    return fail(h->ctx, PP_INVALID_ARG, "pp_hmatrix_set_precision: unknown precision");
  if (precision == h->precision) return PP_OK;
  h->precision = precision;
  if (h->last == &h->factor) h->last = nullptr;
  h->factor.release();
  h->factor.prog = pp::Program();
  h->factor.built = false;
  return PP_OK;
}

int pp_hmatrix_get_precision(const pp_hmatrix* h) { return h ? h->precision : -1; }

pp_status pp_hmatrix_set_pivoting(pp_hmatrix* h, int on) {
  if (!h || (on != 0 && on != 1)) return PP_INVALID_ARG;
  if (on == h->pivoting) return PP_OK;
  h->pivoting = on;
  h->last = nullptr;
  h->factor.release();
  h->factor.prog = pp::Program();
  h->factor.built = false;
  for (auto& kv : h->solves) kv.second->release();
  h->solves.clear();
  return PP_OK;
}

pp_status pp_hmatrix_set_gemm_tile(pp_hmatrix* h, int edge) {
  if (!h) return PP_INVALID_ARG;
  if (edge != 64 && edge != 128) return fail(h->ctx, PP_INVALID_ARG, "pp_hmatrix_set_gemm_tile: 64 or 128");
  if (edge == h->gemm_tile) return PP_OK;
  h->gemm_tile = edge;
  if (h->last == &h->factor) h->last = nullptr;
  h->factor.release();
  h->factor.prog = pp::Program();
  h->factor.built = false;
  return PP_OK;
}

pp_status pp_hmatrix_set_rank_tolerance(pp_hmatrix* h, double tol) {
  if (!h || !(tol >= 0.0) || tol >= 1.0) return PP_INVALID_ARG;
  if (h->d_arena) return fail(h->ctx, PP_INVALID_ARG, "pp_hmatrix_set_rank_tolerance: set it before the upload");
  h->H->set_rank_tolerance(tol);
  h->factor.release();
  h->factor.prog = pp::Program();
  h->factor.built = false;
  for (auto& kv : h->solves) {
    kv.second->release();
    kv.second->prog = pp::Program();
    kv.second->built = false;
  }
  return PP_OK;
}

int pp_hmatrix_block_rank(const pp_hmatrix* h, int block) {
  if (!h || block < 0 || block >= (int)h->H->nodes.size()) return -1;
  return h->H->stored_rank(block);
}

pp_status pp_hmatrix_to_dense(const pp_hmatrix* h, double* out) {
  if (!h || !out) return PP_INVALID_ARG;
  h->H->to_dense(out);
  return PP_OK;
}

long long pp_hmatrix_storage_elems(const pp_hmatrix* h) { return h ? h->H->storage_elems() : 0; }

double* pp_hmatrix_host_arena(pp_hmatrix* h, long long* elems) {
  if (!h) return nullptr;
  if (elems) *elems = h->H->arena_elems;
  h->H->ensure_host();
  return h->H->host.data();
}
const double* pp_hmatrix_device_arena(const pp_hmatrix* h) { return h ? h->d_arena : nullptr; }
long long pp_hmatrix_block_elems(const pp_hmatrix* h) { return h ? h->H->block_elems : 0; }

pp_status pp_hlu_factor(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st != PP_OK) return st;
  st = plan_to_device(h, h->factor);
  if (st != PP_OK) return st;
  return launch_plan(h, h->factor, (cudaStream_t)stream, 0);
}

static VmPlan* solve_plan(pp_hmatrix* h, int nrhs) {
  auto it = h->solves.find(nrhs);
  if (it != h->solves.end()) return it->second.get();
  auto p = std::make_unique<VmPlan>();
  p->async_mem = h->async_mem;
  p->astream = h->astream;
  p->apool = h->apool;
  VmPlan* raw = p.get();
  h->solves.emplace(nrhs, std::move(p));
  return raw;
}

pp_status pp_hlu_solve(pp_hmatrix* h, const double* b_dev, double* x_dev, int nrhs, void* stream) {
  if (!h || !b_dev || !x_dev || nrhs <= 0) return fail(h ? h->ctx : nullptr, PP_INVALID_ARG, "pp_hlu_solve: bad argument");
  pp_context* ctx = h->ctx;
  VmPlan* plan = solve_plan(h, nrhs);
  pp_status st = build_program(h, 1, nrhs, *plan);
  if (st != PP_OK) return st;
  st = plan_to_device(h, *plan);
  if (st != PP_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = sizeof(double) * (size_t)h->H->n * nrhs;
  PP_CUDA(cudaMemcpyAsync(plan->d_rhs, b_dev, bytes, cudaMemcpyDeviceToDevice, s));
  st = launch_plan(h, *plan, s, 0);
  if (st != PP_OK) return st;
  PP_CUDA(cudaMemcpyAsync(x_dev, plan->d_rhs, bytes, cudaMemcpyDeviceToDevice, s));
  return PP_OK;
}

pp_status pp_hmatrix_sync(pp_hmatrix* h, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  PP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  if (!h->last) return PP_OK;
  return plan_status(ctx, *h->last);
}

pp_status pp_hmatrix_program_info(pp_hmatrix* h, int which, int nrhs, pp_program_info* info) {
  if (!h || !info || (which != 0 && which != 1) || (which == 1 && nrhs <= 0)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  std::memset(info, 0, sizeof(*info));
  info->n_tasks = plan->n_tasks;
  info->n_edges = plan->prog.edges;
  info->flops = plan->prog.total_flops();
  for (int op = 0; op < PP_OP_COUNT; ++op) info->op_count[op] = plan->prog.count_op(op);
  for (int a = 0; a < 5; ++a) info->arena_elems[a] = plan->prog.arena_elems[a];
  info->host_build_ms = plan->build_ms;
  return PP_OK;
}

pp_status pp_dev_hierarchical_getrf(pp_hmatrix* h, int num_blocks, int num_threads, int kernel_size) {
  (void)kernel_size;
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (num_threads != 0 && num_threads != PP_VM_THREADS)
    return fail(ctx, PP_INVALID_ARG, "num_threads must be 0 or 256");
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st != PP_OK) return st;
  if (!h->d_arena) {
    st = pp_hmatrix_upload(h, nullptr);
    if (st != PP_OK) return st;
  }
  st = plan_to_device(h, h->factor);
  if (st != PP_OK) return st;
  st = launch_plan(h, h->factor, nullptr, num_blocks > 0 ? num_blocks : 0);
  if (st != PP_OK) return st;
  return pp_hmatrix_sync(h, nullptr);
}

pp_status pp_dense_residual_dev(pp_context* ctx, const double* A, int lda, int n, const double* x, const double* b,
                                double* r, int nrhs, void* stream) {
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (!A || !x || !b || !r || n <= 0 || nrhs <= 0 || lda < n) return fail(ctx, PP_INVALID_ARG, "dense residual: bad argument");
  PP_CUDA(pp_dense_residual(A, lda, n, x, b, r, nrhs, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_kernel_residual_dev(pp_context* ctx, int kernel, double p0, double shift, const double* pts, int dim,
                                 int n, const double* x, const double* b, double* r, int nrhs, void* stream) {
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (!pts || !x || !b || !r || n <= 0 || nrhs <= 0 || nrhs > 16 || dim < 1 || dim > 3 || kernel < 0 || kernel > 3)
    return fail(ctx, PP_INVALID_ARG, "kernel residual: bad argument");
  const size_t need = pp_kernel_residual_part_elems(n, nrhs);
  if (need > ctx->resid_elems) {  // grown before any stream capture by the first (eager) call
    cudaFree(ctx->d_resid);
    ctx->d_resid = nullptr;
    ctx->resid_elems = 0;
    PP_CUDA(cudaMalloc((void**)&ctx->d_resid, sizeof(double) * need));
    ctx->resid_elems = need;
  }
  const cudaError_t e = pp_kernel_residual(kernel, p0, 0.0, shift, pts, dim, n, x, b, r, nrhs, ctx->d_resid,
                                           (cudaStream_t)stream);
  if (e == cudaErrorInvalidValue) return fail(ctx, PP_INVALID_ARG, "kernel residual: p0 negative or not finite");
  PP_CUDA(e);
  return PP_OK;
}

pp_status pp_hmatrix_assemble_dense_dev(pp_hmatrix* h, int kernel, double p0, double shift, const double* pts,
                                        int dim, void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (!pts || dim < 1 || dim > 3 || kernel < 0 || kernel > 3)
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_assemble_dense_dev: bad argument");
  if (kernel <= 1 && !(p0 >= 0.0 && std::isfinite(p0)))
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_assemble_dense_dev: p0 negative or not finite");
  if (h->H->point_dim != 0 && dim != h->H->point_dim)
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_assemble_dense_dev: dim differs from the tree's point dimension");
  if (!h->d_arena) return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_assemble_dense_dev: upload the H-matrix first");
  std::vector<pp_assemble_block> blocks;
  for (const pp::HNode& nd : h->H->nodes) {
    if (nd.kind != pp::HNode::D || nd.obj < 0) continue;
    const pp::StorageObj& o = h->H->objs[nd.obj];
    blocks.push_back(pp_assemble_block{h->d_arena + o.off, o.ld, nd.r0, nd.c0, nd.m, nd.n});
  }
  PP_CUDA(pp_assemble_dense(blocks.data(), (int)blocks.size(), kernel, dim, p0, shift, pts, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_hmatrix_construct_dev(pp_hmatrix* h, int kernel, double p0, double shift, const double* pts, int dim,
                                   void* stream) {
  if (!h) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (!pts || dim < 1 || dim > 3 || kernel < 0 || kernel > 3)
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_construct_dev: bad argument");
  if (kernel <= 1 ? !(p0 >= 0.0 && std::isfinite(p0)) : !(p0 > 0.0 && std::isfinite(p0)))
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_construct_dev: p0 out of range for the kernel");
  if (h->H->point_dim != 0 && dim != h->H->point_dim)
    return fail(ctx, PP_INVALID_ARG, "pp_hmatrix_construct_dev: dim differs from the tree's point dimension");
  cudaStream_t s = (cudaStream_t)stream;
  if (!h->d_arena) {
    const size_t bytes = sizeof(double) * (size_t)std::max<int64_t>(h->H->arena_elems, 1);
    PP_CUDA(h->dalloc((void**)&h->d_arena, bytes));
    PP_CUDA(cudaMemsetAsync(h->d_arena, 0, bytes, s));
  }
  pp_status st = upload_rand(h);
  if (st != PP_OK) return st;
  st = pp_hmatrix_assemble_dense_dev(h, kernel, p0, shift, pts, dim, stream);
  if (st != PP_OK) return st;
  if (h->construct.built && (h->c_kernel != kernel || h->c_dim != dim || h->c_p0 != p0)) {
    h->construct.release();
    h->construct = VmPlan();
  }
  h->c_kernel = kernel;
  h->c_dim = dim;
  h->c_p0 = p0;
  st = build_program(h, 2, 0, h->construct);
  if (st != PP_OK) return st;
  if (h->construct.n_tasks == 0) return PP_OK;  // no low-rank blocks
  st = plan_to_device(h, h->construct);
  if (st != PP_OK) return st;
  // the program's right-hand-side arena holds the n x dim points
  PP_CUDA(cudaMemcpyAsync(h->construct.d_rhs, pts, sizeof(double) * (size_t)h->H->n * dim, cudaMemcpyDeviceToDevice,
                          s));
  return launch_plan(h, h->construct, s, 0);
}

namespace {
pp_status residual_batch(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream, bool lowp);
}

pp_status pp_kernel_residual_batch_dev(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream) {
  return residual_batch(ctx, njobs, jobs, stream, false);
}

pp_status pp_kernel_residual_batch_lowp_dev(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream) {
  return residual_batch(ctx, njobs, jobs, stream, true);
}

namespace {
pp_status residual_batch(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream, bool lowp) {
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (njobs < 0 || (njobs > 0 && !jobs)) return fail(ctx, PP_INVALID_ARG, "kernel residual batch: bad argument");
  size_t need = 0;
  for (int q = 0; q < njobs; ++q) {
    const pp_residual_job& j = jobs[q];
    if (!j.points || !j.x || !j.b || !j.r || j.n <= 0 || j.nrhs <= 0 || j.nrhs > 16 || j.dim < 1 || j.dim > 3 ||
        j.kernel < 0 || j.kernel > 3)
      return fail(ctx, PP_INVALID_ARG, "kernel residual batch: bad job " + std::to_string(q));
    if (j.kernel <= 1 && !(j.p0 >= 0.0 && std::isfinite(j.p0)))
      return fail(ctx, PP_INVALID_ARG, "kernel residual batch: p0 negative or not finite in job " + std::to_string(q));
    need += pp_kernel_residual_part_elems(j.n, j.nrhs);
  }
  if (njobs == 0) return PP_OK;
  if (need > ctx->resid_elems) {  // grown before any stream capture by the first (eager) call
    cudaFree(ctx->d_resid);
    ctx->d_resid = nullptr;
    ctx->resid_elems = 0;
    PP_CUDA(cudaMalloc((void**)&ctx->d_resid, sizeof(double) * need));
    ctx->resid_elems = need;
  }
  std::vector<pp_resid_job> dj(njobs);
  size_t off = 0;
  for (int q = 0; q < njobs; ++q) {
    const pp_residual_job& j = jobs[q];
    pp_resid_job& o = dj[q];
    o.kernel = j.kernel;
    o.dim = j.dim;
    o.n = j.n;
    o.nrhs = j.nrhs;
    o.p0 = j.p0;
    o.shift = j.shift;
    o.pts = j.points;
    o.x = j.x;
    o.dx = j.dx;
    o.b = j.b;
    o.r = j.r;
    o.part = ctx->d_resid + off;
    off += pp_kernel_residual_part_elems(j.n, j.nrhs);
  }
  PP_CUDA(pp_kernel_residual_batch(dj.data(), njobs, (cudaStream_t)stream, lowp));
  return PP_OK;
}
}  // namespace

int pp_datamap2d_check_overlap(uintptr_t pa, size_t pitch_a, size_t width_a, size_t height_a, uintptr_t pb,
                               size_t pitch_b, size_t width_b, size_t height_b) {
  pp::DataMap2D a(pa, pitch_a, width_a, height_a), b(pb, pitch_b, width_b, height_b);
  return a.checkOverlap(b) ? 1 : 0;
}

int pp_operation_dependency(int n_from, const uint64_t* rf, const int* ro_from, int n_to, const uint64_t* rt,
                            const int* ro_to) {
  pp::Operation from, to;
  for (int i = 0; i < n_from; ++i)
    from.data.emplace_back(ro_from[i] != 0, pp::DataMap2D(rf[4 * i], rf[4 * i + 1], rf[4 * i + 2], rf[4 * i + 3]));
  for (int i = 0; i < n_to; ++i)
    to.data.emplace_back(ro_to[i] != 0, pp::DataMap2D(rt[4 * i], rt[4 * i + 1], rt[4 * i + 2], rt[4 * i + 3]));
  return (int)to.checkDependencyFrom(from);
}

pp_status pp_hmatrix_encode_program(pp_hmatrix* h, int which, int nrhs, double* const* bases, void* tasks,
                                    int32_t* succ, int32_t* indeg, int32_t* order) {
  if (!h || !bases || !tasks || !indeg || (which != 0 && which != 1)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  std::vector<double*> b(bases, bases + pp::PP_ARENAS);
  std::vector<pp_task> t;
  std::vector<int32_t> s, d, r;
  plan->prog.encode(b, t, s, d, r);
  std::memcpy(tasks, t.data(), sizeof(pp_task) * t.size());
  if (succ && !s.empty()) std::memcpy(succ, s.data(), sizeof(int32_t) * s.size());
  std::memcpy(indeg, d.data(), sizeof(int32_t) * d.size());
  if (order) {
    for (size_t i = 0; i < t.size(); ++i) order[i] = i < r.size() ? r[i] : -1;
  }
  return PP_OK;
}

pp_status pp_hmatrix_trace(pp_hmatrix* h, int which, int nrhs, int enable, uint64_t* out) {
  if (!h || (which != 0 && which != 1)) return PP_INVALID_ARG;
  pp_context* ctx = h->ctx;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  const size_t bytes = sizeof(unsigned long long) * 3 * (size_t)std::max(plan->n_tasks, 1);
  if (out) {
    if (!plan->d_trace) return fail(ctx, PP_INVALID_ARG, "tracing was not enabled for this program");
    PP_CUDA(cudaMemcpy(out, plan->d_trace, bytes, cudaMemcpyDeviceToHost));
    return PP_OK;
  }
  if (enable && !plan->d_trace) {
    PP_CUDA(cudaMalloc((void**)&plan->d_trace, bytes));
    PP_CUDA(cudaMemset(plan->d_trace, 0, bytes));
  } else if (!enable && plan->d_trace) {
    cudaFree(plan->d_trace);
    plan->d_trace = nullptr;
  }
  return PP_OK;
}

pp_status pp_hmatrix_program_edges(pp_hmatrix* h, int which, int nrhs, int64_t* from, int64_t* to, int32_t* type) {
  if (!h || !from || !to || !type || (which != 0 && which != 1)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  int64_t e = 0;
  std::vector<int64_t> lis;
  const pp::dependency_table& deps = plan->prog.dep_table();
  for (int t = 0; t < plan->n_tasks; ++t) {
    deps.getDepFrom(t, lis);
    for (int64_t s : lis) {
      from[e] = t;
      to[e] = s;
      type[e] = (int32_t)deps.lookup(t, s);
      ++e;
    }
  }
  return PP_OK;
}

pp_status pp_vm_execute(pp_context* ctx, const void* tasks, int n, const int32_t* succ, long long n_succ,
                        const int32_t* indeg, long long spin_limit, int grid, void* stream) {
  if (!ctx || !tasks || !indeg || n <= 0 || n_succ < 0 || (n_succ > 0 && !succ))
    return fail(ctx, PP_INVALID_ARG, "pp_vm_execute: bad argument");
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  const pp_task* T = static_cast<const pp_task*>(tasks);
  std::vector<int32_t> ready;
  for (int i = 0; i < n; ++i) {
    if (T[i].n_succ < 0 || T[i].succ_begin < 0 || (long long)T[i].succ_begin + T[i].n_succ > n_succ)
      return fail(ctx, PP_INVALID_ARG, "pp_vm_execute: successor range outside succ");
    if (indeg[i] == 0) ready.push_back(i);
  }
  for (long long q = 0; q < n_succ; ++q)
    if (succ[q] < 0 || succ[q] >= n) return fail(ctx, PP_INVALID_ARG, "pp_vm_execute: successor id out of range");
  VmPlan p;
  p.n_tasks = n;
  p.n_ready = (int)ready.size();
  PP_CUDA(cudaMalloc((void**)&p.d_tasks, sizeof(pp_task) * n));
  PP_CUDA(cudaMalloc((void**)&p.d_succ, sizeof(int32_t) * std::max<long long>(n_succ, 1)));
  PP_CUDA(cudaMalloc((void**)&p.d_indeg, sizeof(int32_t) * n));
  PP_CUDA(cudaMalloc((void**)&p.d_ready, sizeof(int32_t) * std::max<size_t>(ready.size(), 1)));
  PP_CUDA(cudaMalloc((void**)&p.d_counters, sizeof(int32_t) * n));
  PP_CUDA(cudaMalloc((void**)&p.d_slots, sizeof(int32_t) * n));
  PP_CUDA(cudaMalloc((void**)&p.d_state, sizeof(pp_vm_state)));
  PP_CUDA(cudaMemcpy(p.d_tasks, T, sizeof(pp_task) * n, cudaMemcpyHostToDevice));
  if (n_succ > 0) PP_CUDA(cudaMemcpy(p.d_succ, succ, sizeof(int32_t) * n_succ, cudaMemcpyHostToDevice));
  PP_CUDA(cudaMemcpy(p.d_indeg, indeg, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  if (!ready.empty()) PP_CUDA(cudaMemcpy(p.d_ready, ready.data(), sizeof(int32_t) * ready.size(), cudaMemcpyHostToDevice));
  pp_vm_launch L;
  L.tasks = p.d_tasks; L.n_tasks = n; L.succ = p.d_succ; L.indeg = p.d_indeg; L.ready = p.d_ready;
  L.n_ready = p.n_ready; L.counters = p.d_counters; L.slots = p.d_slots; L.state = p.d_state;
  L.wait_ns = (spin_limit > 0 ? spin_limit : ctx->cfg.spin_limit) * 1000;
  L.grid = grid > 0 ? grid : std::max(1, std::min(n, ctx->sm_count * ctx->blocks_per_sm));
  for (int i = 0; i < n; ++i)
    if (T[i].prec == PP_PREC_TF32 || T[i].prec == PP_PREC_BF16) L.use_tc = 1;
  cudaStream_t s = (cudaStream_t)stream;
  PP_CUDA(pp_vm_run(L, s));
  PP_CUDA(cudaStreamSynchronize(s));
  pp_vm_state st;
  PP_CUDA(cudaMemcpy(&st, p.d_state, sizeof(st), cudaMemcpyDeviceToHost));
  p.release();
  return vm_state_status(ctx, st, n);
}

pp_status pp_lowrank_accum_noalloc(pp_context* ctx, double* U1, int ld_u1, double* V1, int ld_v1, const double* U2,
                                   int ld_u2, const double* V2, int ld_v2, const double* R, int ld_r, int ny, int nx,
                                   int k1, int k2, double sign, void* stream) {
  if (!ctx) return PP_INVALID_ARG;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (!U1 || !V1 || !U2 || !V2 || !R || ny < 1 || nx < 1 || k1 < 1 || k1 > PP_VM_MAX_RANK || k1 > ny || k1 > nx ||
      k2 < 1 || k2 > PP_VM_MAX_RANK || ld_u1 < k1 || ld_v1 < k1 || ld_u2 < k2 || ld_v2 < k2 || ld_r < k1 ||
      (sign != 1.0 && sign != -1.0))
    return fail(ctx, PP_INVALID_ARG, "pp_lowrank_accum_noalloc: bad argument (1 <= k1, k2 <= 32, k1 <= ny, nx)");
  const long long need = pp_accum_scratch_doubles(ny, k1, k2);
  if (need > pp_accum_noalloc_capacity())
    return fail(ctx, PP_INVALID_ARG,
                "pp_lowrank_accum_noalloc: needs " + std::to_string(need) + " doubles of scratch, the static array holds " +
                    std::to_string(pp_accum_noalloc_capacity()));
  pp_task T{};
  T.op = PP_OP_ACCUM;
  T.m = ny;
  T.n = nx;
  T.k = k1;
  T.l = k2;
  T.alpha = sign;
  T.beta = 1.0;
  T.p[0] = U1;
  T.p[1] = V1;
  T.p[2] = const_cast<double*>(U2);
  T.p[3] = const_cast<double*>(V2);
  T.p[4] = const_cast<double*>(R);
  T.ld[0] = ld_u1;
  T.ld[1] = ld_v1;
  T.ld[2] = ld_u2;
  T.ld[3] = ld_v2;
  T.ld[4] = ld_r;
  // the context's device is current for the call (its scratch address and its launch)
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return fail(ctx, PP_CUDA_ERROR, "cudaGetDevice failed");
  if (prev != ctx->device && cudaSetDevice(ctx->device) != cudaSuccess)
    return fail(ctx, PP_CUDA_ERROR, "cudaSetDevice failed");
  const cudaError_t e = pp_accum_noalloc_launch(T, need, (cudaStream_t)stream);
  if (prev != ctx->device) cudaSetDevice(prev);
  PP_CUDA(e);
  return PP_OK;
}

pp_status pp_hmatrix_rand_host(pp_hmatrix* h, double* out, long long count) {
  if (!h || !out) return PP_INVALID_ARG;
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st != PP_OK) return st;
  if (h->rand_host.empty()) make_rand(h);
  if (count > (long long)h->rand_host.size()) return fail(h->ctx, PP_INVALID_ARG, "rand_host: count too large");
  std::memcpy(out, h->rand_host.data(), sizeof(double) * count);
  return PP_OK;
}

pp_status pp_refstream_encode(pp_hmatrix* h, int workers, int32_t* words, long long capacity, int32_t* lengths,
                              long long* tmp_elems) {
  if (!h || workers <= 0 || !lengths) return PP_INVALID_ARG;
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st != PP_OK) return st;
  std::vector<std::vector<int32_t>> streams;
  std::string err;
  int64_t tmp = 0;
  if (!h->factor.prog.encode_reference(workers, streams, err, &tmp)) return fail(h->ctx, PP_UNSUPPORTED, err);
  long long total = 0;
  for (auto& s : streams) total += (long long)s.size();
  for (int w = 0; w < workers; ++w) lengths[w] = (int32_t)streams[w].size();
  if (tmp_elems) *tmp_elems = tmp;
  if (!words) return PP_OK;  // size query
  if (total > capacity) return fail(h->ctx, PP_INVALID_ARG, "refstream: capacity too small");
  long long at = 0;
  for (auto& s : streams) {
    std::memcpy(words + at, s.data(), sizeof(int32_t) * s.size());
    at += (long long)s.size();
  }
  return PP_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------- batches
struct pp_batch {
  pp_context* ctx = nullptr;
  std::vector<pp_hmatrix*> hs;
  int grid_cap = 0;  // persistent CTAs of its launches (0: all); set by pp_batch_autotune
  VmPlan factor;
  std::map<int, std::unique_ptr<VmPlan>> solves;
  VmPlan* last = nullptr;
  ~pp_batch() {
    factor.release();
    for (auto& kv : solves) kv.second->release();
  }
};

namespace {

// merged program of all instances: instance j keeps arena ids j * PP_ARENAS + kind
pp_status batch_program(pp_batch* b, int which, int nrhs, VmPlan& plan) {
  if (plan.built) return PP_OK;
  auto t0 = std::chrono::steady_clock::now();
  for (auto* h : b->hs) {
    VmPlan* src = which == 0 ? &h->factor : solve_plan(h, nrhs);
    pp_status st = build_program(h, which, nrhs, *src);
    if (st != PP_OK) return st;
    plan.prog.merge(src->prog);
  }
  plan.n_tasks = (int)plan.prog.tasks.size();
  plan.built = true;
  plan.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return PP_OK;
}

VmPlan* batch_solve_plan(pp_batch* b, int nrhs) {
  auto it = b->solves.find(nrhs);
  if (it != b->solves.end()) return it->second.get();
  auto p = std::make_unique<VmPlan>();
  VmPlan* raw = p.get();
  b->solves.emplace(nrhs, std::move(p));
  return raw;
}

}  // namespace

extern "C" {

pp_status pp_batch_create(pp_context* ctx, pp_hmatrix* const* hs, int n, pp_batch** out) {
  if (!ctx || !hs || n <= 0 || !out) return fail(ctx, PP_INVALID_ARG, "pp_batch_create: bad argument");
  *out = nullptr;
  auto b = std::make_unique<pp_batch>();
  b->ctx = ctx;
  for (int i = 0; i < n; ++i) {
    if (!hs[i] || hs[i]->ctx != ctx) return fail(ctx, PP_INVALID_ARG, "pp_batch_create: instance from another context");
    if (!hs[i]->d_arena) return fail(ctx, PP_INVALID_ARG, "pp_batch_create: instance not uploaded");
    b->hs.push_back(hs[i]);
  }
  pp_status st = batch_program(b.get(), 0, 0, b->factor);
  if (st != PP_OK) return st;
  *out = b.release();
  return PP_OK;
}

void pp_batch_destroy(pp_batch* b) { delete b; }

pp_status pp_batch_factor(pp_batch* b, void* stream) {
  if (!b) return PP_INVALID_ARG;
  pp_status st = batch_program(b, 0, 0, b->factor);  // (re)built after an autotuner tile change
  if (st != PP_OK) return st;
  st = plan_to_device_multi(b->ctx, b->hs, b->factor);
  if (st != PP_OK) return st;
  st = launch_plan(b->ctx, b->factor, (cudaStream_t)stream, b->grid_cap);
  if (st == PP_OK) b->last = &b->factor;
  return st;
}

pp_status pp_batch_solve(pp_batch* b, const double* const* B, double* const* X, int nrhs, void* stream) {
  if (!b || !B || !X || nrhs <= 0) return fail(b ? b->ctx : nullptr, PP_INVALID_ARG, "pp_batch_solve: bad argument");
  pp_context* ctx = b->ctx;
  VmPlan* plan = batch_solve_plan(b, nrhs);
  pp_status st = batch_program(b, 1, nrhs, *plan);
  if (st != PP_OK) return st;
  st = plan_to_device_multi(ctx, b->hs, *plan);
  if (st != PP_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  for (size_t j = 0; j < b->hs.size(); ++j) {
    if (!B[j] || !X[j]) return fail(ctx, PP_INVALID_ARG, "pp_batch_solve: null right-hand side");
    PP_CUDA(cudaMemcpyAsync(plan->d_rhs + plan->rhs_off[j], B[j], sizeof(double) * (size_t)b->hs[j]->H->n * nrhs,
                            cudaMemcpyDeviceToDevice, s));
  }
  st = launch_plan(ctx, *plan, s, b->grid_cap);
  if (st != PP_OK) return st;
  b->last = plan;
  for (size_t j = 0; j < b->hs.size(); ++j)
    PP_CUDA(cudaMemcpyAsync(X[j], plan->d_rhs + plan->rhs_off[j], sizeof(double) * (size_t)b->hs[j]->H->n * nrhs,
                            cudaMemcpyDeviceToDevice, s));
  return PP_OK;
}

pp_status pp_batch_restore(pp_batch* b, void* stream) {
  if (!b) return PP_INVALID_ARG;
  for (auto* h : b->hs) {
    pp_status st = pp_hmatrix_restore(h, stream);
    if (st != PP_OK) return st;
  }
  return PP_OK;
}

pp_status pp_batch_sync(pp_batch* b, void* stream) {
  if (!b) return PP_INVALID_ARG;
  pp_context* ctx = b->ctx;
  PP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  if (!b->last) return PP_OK;
  return plan_status(ctx, *b->last);
}

pp_status pp_batch_program_info(pp_batch* b, int which, int nrhs, pp_program_info* info) {
  if (!b || !info || (which != 0 && which != 1) || (which == 1 && nrhs <= 0)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &b->factor : batch_solve_plan(b, nrhs);
  pp_status st = batch_program(b, which, nrhs, *plan);
  if (st != PP_OK) return st;
  std::memset(info, 0, sizeof(*info));
  info->n_tasks = plan->n_tasks;
  info->n_edges = plan->prog.edges;
  info->flops = plan->prog.total_flops();
  for (int op = 0; op < PP_OP_COUNT; ++op) info->op_count[op] = plan->prog.count_op(op);
  for (int a = 0; a < 5; ++a)
    for (int j = 0; j < plan->prog.n_instances; ++j) info->arena_elems[a] += plan->prog.arena_elems[j * pp::PP_ARENAS + a];
  info->host_build_ms = plan->build_ms;
  return PP_OK;
}

// Invalidates the programs of an instance and of the batch (a new tile rebuilds them).
static void batch_reset_programs(pp_batch* b) {
  auto reset = [](VmPlan& p) {
    p.release();
    p.prog = pp::Program();
    p.built = false;
  };
  for (auto* h : b->hs) {
    if (h->last) h->last = nullptr;
    reset(h->factor);
    for (auto& kv : h->solves) reset(*kv.second);
  }
  reset(b->factor);
  for (auto& kv : b->solves) reset(*kv.second);
  b->last = nullptr;
}

pp_status pp_batch_autotune(pp_batch* b, void* stream, pp_tune_result* out) {
  if (!b) return PP_INVALID_ARG;
  pp_context* ctx = b->ctx;
  for (auto* h : b->hs)
    if (!h->d_orig) return fail(ctx, PP_INVALID_ARG, "pp_batch_autotune: every instance needs pp_hmatrix_keep_original");
  cudaStream_t s = (cudaStream_t)stream;
  const int full = ctx->sm_count * std::max(1, ctx->blocks_per_sm);
  const int tiles[] = {32, 64};
  const int gemm_tiles[] = {64, 128};
  const int grids[] = {full, (3 * full) / 4, full / 2};
  cudaEvent_t e0, e1;
  PP_CUDA(cudaEventCreate(&e0));
  PP_CUDA(cudaEventCreate(&e1));
  double best = 1e300;
  int best_tile = 0, best_grid = 0, best_gt = 64, trials = 0;
  pp_status st = PP_OK;
  for (int t : tiles)
  for (int gt : gemm_tiles) {
    if (t > PP_VM_TILE) continue;
    for (auto* h : b->hs) {
      h->tile = t;
      h->gemm_tile = gt;
    }
    batch_reset_programs(b);
    for (int g : grids) {
      b->grid_cap = g;
      float ms = 0.f;
      for (int rep = 0; rep < 2 && st == PP_OK; ++rep) {  // the first run builds and warms up
        st = pp_batch_restore(b, stream);
        if (st == PP_OK && cudaEventRecord(e0, s) != cudaSuccess) st = PP_CUDA_ERROR;
        if (st == PP_OK) st = pp_batch_factor(b, stream);
        if (st == PP_OK && cudaEventRecord(e1, s) != cudaSuccess) st = PP_CUDA_ERROR;
        if (st == PP_OK && cudaEventSynchronize(e1) != cudaSuccess) st = PP_CUDA_ERROR;
        if (st == PP_OK) st = plan_status(ctx, b->factor);
        if (st == PP_OK) cudaEventElapsedTime(&ms, e0, e1);
      }
      if (st != PP_OK) break;
      ++trials;
      if (ms < best) {
        best = ms;
        best_tile = t;
        best_grid = g;
        best_gt = gt;
      }
    }
    if (st != PP_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != PP_OK) return st;
  for (auto* h : b->hs) {
    h->tile = best_tile;
    h->gemm_tile = best_gt;
  }
  batch_reset_programs(b);
  b->grid_cap = best_grid;
  st = pp_batch_restore(b, stream);
  if (st != PP_OK) return st;
  if (out) {
    out->tile = best_tile;
    out->grid = best_grid;
    out->gemm_tile = best_gt;
    out->factor_ms = best;
    out->trials = trials;
  }
  return PP_OK;
}

pp_status pp_batch_set_tuning(pp_batch* b, int tile, int gemm_tile, int grid) {
  if (!b) return PP_INVALID_ARG;
  if (tile < 8 || tile > PP_VM_TILE || (gemm_tile != 64 && gemm_tile != 128) || grid < 0)
    return fail(b->ctx, PP_INVALID_ARG, "pp_batch_set_tuning: tile 8..64, product tile 64 or 128, grid >= 0");
  for (auto* h : b->hs) {
    h->tile = tile;
    h->gemm_tile = gemm_tile;
  }
  batch_reset_programs(b);
  b->grid_cap = grid;
  return PP_OK;
}

pp_status pp_batch_trace(pp_batch* b, int which, int nrhs, int enable, uint64_t* out) {
  if (!b || (which != 0 && which != 1)) return PP_INVALID_ARG;
  pp_context* ctx = b->ctx;
  VmPlan* plan = which == 0 ? &b->factor : batch_solve_plan(b, nrhs);
  pp_status st = batch_program(b, which, nrhs, *plan);
  if (st != PP_OK) return st;
  const size_t bytes = sizeof(unsigned long long) * 3 * (size_t)std::max(plan->n_tasks, 1);
  if (out) {
    if (!plan->d_trace) return fail(ctx, PP_INVALID_ARG, "tracing was not enabled for this program");
    PP_CUDA(cudaMemcpy(out, plan->d_trace, bytes, cudaMemcpyDeviceToHost));
    return PP_OK;
  }
  if (enable && !plan->d_trace) {
    PP_CUDA(cudaMalloc((void**)&plan->d_trace, bytes));
    PP_CUDA(cudaMemset(plan->d_trace, 0, bytes));
  }
  return PP_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------- serving
// A request loop over one context: factor + solve jobs of different sizes are admitted in
// arrival order as in-flight slots and the HBM budget allow (a later, smaller job may pass a
// waiting larger one); every admitted job runs on its own stream with a persistent grid of
// a slot's share of the SMs, so the work of several jobs overlaps on the device.  A job
// keeps its factors resident for its follow-up right-hand-side sets and refines each set in
// FP64 until the normwise backward error meets its tolerance.  Its memory is stream-ordered
// (cudaMallocAsync / cudaFreeAsync), so admitting or retiring a job never waits for the
// others.  No reference counterpart (the reference factors one matrix per launch).
namespace {

enum ServeState { SRV_QUEUED = 0, SRV_RUNNING = 1, SRV_DONE = 2, SRV_FAILED = 3 };

struct ServeRequest {
  long long id = 0;
  pp_hmatrix* h = nullptr;  // owned from submission
  int n = 0, dim = 0, kernel = 0, nrhs = 0, n_sets = 0, max_iter = 0;
  double p0 = 0, shift = 0, norm_inf = 0, tol = 0;
  std::vector<double> pts, rhs;
  bool construct = false;  // the H-matrix has no host image: build it on the device at admission
  double* x_out = nullptr;  // caller's host buffer
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  double *d_pts = nullptr, *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_dx = nullptr, *d_part = nullptr;
  unsigned long long* d_norms = nullptr;
  long long bytes = 0;
  int state = SRV_QUEUED;
  int set = 0, iters_set = 0, iters_total = 0;
  double bmax = 0, worst = 0;
  double t_submit = 0, t_admit = -1, t_done = -1, t_enqueued = -1;
  std::string err;
};

}  // namespace

struct pp_server {
  pp_context* ctx = nullptr;
  // the requests' device memory: a pool of its own that keeps up to the budget mapped between
  // requests (no page mapping on the admission path, no effect on other users of the device)
  cudaMemPool_t pool = nullptr;
  long long budget = 0;
  int slots = 1, grid = 0;
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  std::deque<ServeRequest*> queue;
  std::vector<ServeRequest*> active;
  std::map<long long, std::unique_ptr<ServeRequest>> all;
  long long next_id = 1, used = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  void run();
  bool start(ServeRequest* q);
  bool iterate(ServeRequest* q);
  bool start_set(ServeRequest* q);
  bool advance(ServeRequest* q);
  void retire(ServeRequest* q, bool ok);
};

namespace {

bool srv_check(ServeRequest* q, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  q->err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

bool srv_status(ServeRequest* q, pp_status st, pp_context* ctx, const char* what) {
  if (st == PP_OK) return true;
  q->err = std::string(what) + ": " + ctx->err;
  return false;
}

}  // namespace

bool pp_server::start(ServeRequest* q) {
  pp_hmatrix* h = q->h;
  if (!srv_check(q, cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking), "stream")) return false;
  if (!srv_check(q, cudaEventCreateWithFlags(&q->ev, cudaEventDisableTiming), "event")) return false;
  h->set_async(q->stream, pool);
  const size_t vec = sizeof(double) * (size_t)q->n * q->nrhs;
  if (!srv_check(q, h->dalloc((void**)&q->d_pts, sizeof(double) * q->pts.size()), "alloc")) return false;
  for (double** p : {&q->d_b, &q->d_x, &q->d_r, &q->d_dx})
    if (!srv_check(q, h->dalloc((void**)p, vec), "alloc")) return false;
  if (!srv_check(q, h->dalloc((void**)&q->d_part, sizeof(double) * pp_kernel_residual_part_elems(q->n, q->nrhs)),
                 "alloc"))
    return false;
  if (!srv_check(q, h->dalloc((void**)&q->d_norms, 2 * sizeof(unsigned long long)), "alloc")) return false;
  if (!srv_check(q, cudaMemcpyAsync(q->d_pts, q->pts.data(), sizeof(double) * q->pts.size(), cudaMemcpyHostToDevice,
                                    q->stream), "points"))
    return false;
  if (q->construct) {  // no host image: the blocks are built on the device from the points
    if (!srv_status(q, pp_hmatrix_construct_dev(h, q->kernel, q->p0, q->shift, q->d_pts, q->dim, q->stream), ctx,
                    "construct"))
      return false;
  } else if (!srv_status(q, pp_hmatrix_upload(h, q->stream), ctx, "upload")) {
    return false;
  }
  if (!srv_status(q, plan_to_device(h, h->factor), ctx, "factor plan")) return false;
  if (!srv_status(q, launch_plan(h, h->factor, q->stream, grid), ctx, "factor")) return false;
  return start_set(q);
}

bool pp_server::start_set(ServeRequest* q) {
  const size_t cnt = (size_t)q->n * q->nrhs, vec = sizeof(double) * cnt;
  const double* b = q->rhs.data() + (size_t)q->set * cnt;
  q->bmax = 0;
  for (size_t e = 0; e < cnt; ++e) q->bmax = std::max(q->bmax, std::fabs(b[e]));
  q->iters_set = 0;
  if (!srv_check(q, cudaMemcpyAsync(q->d_b, b, vec, cudaMemcpyHostToDevice, q->stream), "rhs")) return false;
  if (!srv_check(q, cudaMemcpyAsync(q->d_r, q->d_b, vec, cudaMemcpyDeviceToDevice, q->stream), "rhs")) return false;
  if (!srv_check(q, cudaMemsetAsync(q->d_x, 0, vec, q->stream), "x")) return false;
  return iterate(q);
}

// one refinement step: dx = (LU)^-1 r, x += dx, r = b - A x (FP64, matrix-free), norms
bool pp_server::iterate(ServeRequest* q) {
  pp_hmatrix* h = q->h;
  const size_t cnt = (size_t)q->n * q->nrhs;
  VmPlan* plan = solve_plan(h, q->nrhs);
  if (!srv_status(q, build_program(h, 1, q->nrhs, *plan), ctx, "solve program")) return false;
  if (!srv_status(q, plan_to_device(h, *plan), ctx, "solve plan")) return false;
  if (!srv_check(q, cudaMemcpyAsync(plan->d_rhs, q->d_r, sizeof(double) * cnt, cudaMemcpyDeviceToDevice, q->stream),
                 "solve"))
    return false;
  if (!srv_status(q, launch_plan(h, *plan, q->stream, grid), ctx, "solve")) return false;
  if (!srv_check(q, pp_axpy(q->d_x, plan->d_rhs, cnt, q->stream), "update")) return false;
  if (!srv_check(q, pp_kernel_residual(q->kernel, q->p0, 0.0, q->shift, q->d_pts, q->dim, q->n, q->d_x, q->d_b,
                                       q->d_r, q->nrhs, q->d_part, q->stream), "residual"))
    return false;
  if (!srv_check(q, pp_absmax2(q->d_x, q->d_r, cnt, q->d_norms, q->stream), "norms")) return false;
  if (!srv_check(q, cudaEventRecord(q->ev, q->stream), "event")) return false;
  ++q->iters_set;
  ++q->iters_total;
  return true;
}

// returns true when the request made progress (its last step finished on the device)
bool pp_server::advance(ServeRequest* q) {
  if (cudaEventQuery(q->ev) != cudaSuccess) return false;
  unsigned long long nb[2];
  pp_vm_state vs, vf;
  VmPlan* plan = solve_plan(q->h, q->nrhs);
  bool ok = srv_check(q, cudaMemcpyAsync(nb, q->d_norms, sizeof(nb), cudaMemcpyDeviceToHost, q->stream), "norms") &&
            srv_check(q, cudaMemcpyAsync(&vs, plan->d_state, sizeof(vs), cudaMemcpyDeviceToHost, q->stream), "state") &&
            srv_check(q, cudaMemcpyAsync(&vf, q->h->factor.d_state, sizeof(vf), cudaMemcpyDeviceToHost, q->stream),
                      "state") &&
            srv_check(q, cudaStreamSynchronize(q->stream), "sync");
  if (ok && (vs.error || vf.error)) {
    q->err = "VM error " + std::to_string(vf.error ? vf.error : vs.error) + (vf.error ? " in the factorization" : " in a solve");
    ok = false;
  }
  if (!ok) {
    retire(q, false);
    return true;
  }
  double xmax, rmax;
  std::memcpy(&xmax, &nb[0], sizeof(double));
  std::memcpy(&rmax, &nb[1], sizeof(double));
  const double err = rmax / (q->norm_inf * xmax + q->bmax);
  if (!(err <= q->tol) && q->iters_set < q->max_iter) {
    if (!iterate(q)) retire(q, false);
    return true;
  }
  q->worst = std::max(q->worst, err);
  const size_t cnt = (size_t)q->n * q->nrhs;
  ok = srv_check(q, cudaMemcpyAsync(q->x_out + (size_t)q->set * cnt, q->d_x, sizeof(double) * cnt,
                                    cudaMemcpyDeviceToHost, q->stream), "result") &&
       srv_check(q, cudaStreamSynchronize(q->stream), "sync");
  if (!ok || !(err <= q->tol)) {
    if (ok) q->err = "refinement did not reach the tolerance";
    retire(q, false);
    return true;
  }
  if (++q->set < q->n_sets) {
    if (!start_set(q)) retire(q, false);
    return true;
  }
  retire(q, true);
  return true;
}

void pp_server::retire(ServeRequest* q, bool ok) {
  pp_hmatrix* h = q->h;
  for (void* p : {(void*)q->d_pts, (void*)q->d_b, (void*)q->d_x, (void*)q->d_r, (void*)q->d_dx, (void*)q->d_part,
                  (void*)q->d_norms})
    h->dfree(p);
  pp_hmatrix_destroy(h);  // stream-ordered frees of the arena and the plans
  q->h = nullptr;
  if (q->ev) cudaEventDestroy(q->ev);
  if (q->stream) cudaStreamDestroy(q->stream);  // resources go when the queued frees have run
  q->ev = nullptr;
  q->stream = nullptr;
  q->state = ok ? SRV_DONE : SRV_FAILED;
  q->t_done = now_ms();
  used -= q->bytes;
}

void pp_server::run() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    if (stop && queue.empty() && active.empty()) break;
    for (auto it = queue.begin(); it != queue.end() && (int)active.size() < slots;) {
      ServeRequest* q = *it;
      if (used + q->bytes > budget) {
        ++it;
        continue;
      }
      it = queue.erase(it);
      used += q->bytes;
      q->state = SRV_RUNNING;
      q->t_admit = now_ms();
      active.push_back(q);
      if (!start(q)) retire(q, false);
      else q->t_enqueued = now_ms();
    }
    bool progressed = false;
    for (ServeRequest* q : active)
      if (q->state == SRV_RUNNING) progressed |= advance(q);
    active.erase(std::remove_if(active.begin(), active.end(), [](ServeRequest* q) { return q->state != SRV_RUNNING; }),
                 active.end());
    if (!progressed) cv.wait_for(lk, std::chrono::microseconds(50));
  }
}

extern "C" {

pp_status pp_server_create(pp_context* ctx, const pp_serve_config* cfg, pp_server** out) {
  if (!ctx || !cfg || !out) return PP_INVALID_ARG;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (cfg->hbm_budget_bytes <= 0 || cfg->max_inflight <= 0)
    return fail(ctx, PP_INVALID_ARG, "pp_server_create: budget and slots must be positive");
  auto* s = new (std::nothrow) pp_server();
  if (!s) return PP_OOM;
  s->ctx = ctx;
  s->budget = cfg->hbm_budget_bytes;
  s->slots = cfg->max_inflight;
  s->grid = cfg->grid_per_request > 0 ? cfg->grid_per_request
                                      : std::max(8, ctx->sm_count * std::max(1, ctx->blocks_per_sm) / s->slots);
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
  unsigned long long keep = (unsigned long long)s->budget;
  if (e == cudaSuccess) e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (e == cudaSuccess) {
    // map the first part of the budget now (one allocation, freed at once: the pool keeps it),
    // so that admitting the first requests does not wait for the device memory to be mapped
    const size_t warm = (size_t)std::min<long long>(s->budget, 1ll << 30);
    cudaStream_t ws = nullptr;
    void* p = nullptr;
    e = cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&p, warm, s->pool, ws);
    if (e == cudaSuccess) e = cudaFreeAsync(p, ws);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ws);
    if (ws) cudaStreamDestroy(ws);
  }
  if (e != cudaSuccess) {
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return fail(ctx, PP_CUDA_ERROR, std::string("pp_server_create: memory pool: ") + cudaGetErrorString(e));
  }
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return PP_OK;
}

pp_status pp_server_submit(pp_server* s, pp_hmatrix* h, const pp_request_desc* d, long long* id) {
  if (!s || !h || !d || !id || h->ctx != s->ctx) return PP_INVALID_ARG;
  pp_context* ctx = s->ctx;
  const int n = h->H->n;
  if (!d->points || d->dim < 1 || d->dim > 3 || !d->rhs || d->nrhs < 1 || d->nrhs > 16 || d->n_sets < 1 ||
      !d->x_out || d->max_iter < 1 || !(d->tol > 0) || !(d->norm_inf > 0) || d->kernel < 0 || d->kernel > 3)
    return fail(ctx, PP_INVALID_ARG, "pp_server_submit: bad request");
  auto q = std::make_unique<ServeRequest>();
  q->h = h;
  q->n = n;
  q->dim = d->dim;
  q->kernel = d->kernel;
  q->p0 = d->p0;
  q->shift = d->shift;
  q->norm_inf = d->norm_inf;
  q->nrhs = d->nrhs;
  q->n_sets = d->n_sets;
  q->tol = d->tol;
  q->max_iter = d->max_iter;
  q->x_out = d->x_out;
  q->pts.assign(d->points, d->points + (size_t)n * d->dim);
  q->rhs.assign(d->rhs, d->rhs + (size_t)n * d->nrhs * d->n_sets);
  q->construct = h->H->host.empty();
  std::lock_guard<std::mutex> lk(s->mu);
  // programs are built here (host work) so that the device bytes are known before admission
  VmPlan* sp = solve_plan(h, d->nrhs);
  pp_status st = build_program(h, 0, 0, h->factor);
  if (st == PP_OK) st = build_program(h, 1, d->nrhs, *sp);
  if (st == PP_OK && q->construct) {
    h->c_kernel = d->kernel;
    h->c_dim = d->dim;
    h->c_p0 = d->p0;
    st = build_program(h, 2, 0, h->construct);
  }
  if (st != PP_OK) return st;
  if (h->d_arena) return fail(ctx, PP_INVALID_ARG, "pp_server_submit: the H-matrix must not be uploaded yet");
  auto plan_bytes = [](const VmPlan& p) {
    const auto& a = p.prog.arena_elems;
    return (long long)sizeof(double) * (a[pp::AR_WORK] + a[pp::AR_SCRATCH] + a[pp::AR_RHS]) +
           (long long)p.n_tasks * (long long)(sizeof(pp_task) + 4 * sizeof(int32_t)) +
           (long long)p.prog.edges * (long long)sizeof(int32_t) + 4096;
  };
  const long long vec = (long long)sizeof(double) * n * d->nrhs;
  q->bytes = (long long)sizeof(double) * (h->H->arena_elems + h->factor.prog.arena_elems[pp::AR_RAND]) +
             plan_bytes(h->factor) + plan_bytes(*sp) + (q->construct ? plan_bytes(h->construct) : 0) + 4 * vec +
             (long long)sizeof(double) * ((long long)n * d->dim + (long long)pp_kernel_residual_part_elems(n, d->nrhs)) +
             (1 << 20);
  if (q->bytes > s->budget) return fail(ctx, PP_OOM, "pp_server_submit: request exceeds the whole HBM budget");
  q->id = s->next_id++;
  q->t_submit = s->now_ms();
  *id = q->id;
  s->queue.push_back(q.get());
  s->all[q->id] = std::move(q);
  s->cv.notify_all();
  return PP_OK;
}

pp_status pp_server_poll(pp_server* s, long long id, pp_request_stats* st) {
  if (!s || !st) return PP_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return fail(s->ctx, PP_INVALID_ARG, "pp_server_poll: unknown request");
  const ServeRequest* q = it->second.get();
  std::memset(st, 0, sizeof(*st));
  st->status = q->state;
  st->iterations = q->iters_total;
  st->backward_error = q->worst;
  st->t_submit_ms = q->t_submit;
  st->t_admit_ms = q->t_admit;
  st->t_enqueued_ms = q->t_enqueued;
  st->t_done_ms = q->t_done;
  st->device_bytes = q->bytes;
  std::snprintf(st->message, sizeof(st->message), "%s", q->err.c_str());
  return PP_OK;
}

pp_status pp_server_wait_all(pp_server* s, double timeout_ms) {
  if (!s) return PP_INVALID_ARG;
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double, std::milli>(timeout_ms);
  for (;;) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->queue.empty() && s->active.empty()) return PP_OK;
    }
    if (std::chrono::steady_clock::now() > until) return fail(s->ctx, PP_TIMEOUT, "pp_server_wait_all: timed out");
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

double pp_server_clock_ms(pp_server* s) { return s ? s->now_ms() : 0.0; }

void pp_server_destroy(pp_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  for (auto& kv : s->all)
    if (kv.second->h) pp_hmatrix_destroy(kv.second->h);  // queued, never admitted
  if (s->pool) cudaMemPoolDestroy(s->pool);  // released once the queued frees have run
  delete s;
}

// ---------------------------------------------------------------- batched GMRES
struct pp_gmres {
  pp_context* ctx = nullptr;
  int count = 0, m = 0;
  pp_gmres_slot* d_slots = nullptr;  // device copy, ordered by n descending
  double* d_state = nullptr;
  std::vector<int> order;            // order[k]: creation index of device slot k
  size_t state_elems = 0;
  ~pp_gmres() {
    cudaFree(d_slots);
    cudaFree(d_state);
  }
};

pp_status pp_gmres_create(pp_context* ctx, int count, const int* n, int m, double* const* V, double* const* Z,
                          double* const* x, double* const* r, pp_gmres** out) {
  if (!out) return PP_INVALID_ARG;
  *out = nullptr;
  if (!has_device(ctx)) return fail(ctx, PP_CUDA_ERROR, "no CUDA device in this context");
  if (count <= 0 || !n || !V || !Z || !x || !r || m < 1 || m > PP_GMRES_MAX_RESTART)
    return fail(ctx, PP_INVALID_ARG, "pp_gmres_create: bad argument (1 <= m <= " +
                                         std::to_string(PP_GMRES_MAX_RESTART) + ")");
  for (int i = 0; i < count; ++i)
    if (n[i] <= 0 || !V[i] || !Z[i] || !x[i] || !r[i])
      return fail(ctx, PP_INVALID_ARG, "pp_gmres_create: bad instance " + std::to_string(i));
  auto* g = new pp_gmres;
  g->ctx = ctx;
  g->count = count;
  g->m = m;
  g->state_elems = pp_gmres_state_elems(m);
  g->order.resize(count);
  for (int i = 0; i < count; ++i) g->order[i] = i;
  // largest instances first: their CTAs start in the first wave
  std::stable_sort(g->order.begin(), g->order.end(), [&](int a, int b) { return n[a] > n[b]; });
  cudaError_t e = cudaMalloc((void**)&g->d_state, sizeof(double) * g->state_elems * count);
  if (e == cudaSuccess) e = cudaMemset(g->d_state, 0, sizeof(double) * g->state_elems * count);
  if (e == cudaSuccess) e = cudaMalloc((void**)&g->d_slots, sizeof(pp_gmres_slot) * count);
  if (e == cudaSuccess) {
    std::vector<pp_gmres_slot> hs(count);
    for (int k = 0; k < count; ++k) {
      const int i = g->order[k];
      hs[k] = pp_gmres_slot{n[i], m, V[i], Z[i], x[i], r[i], g->d_state + g->state_elems * i};
    }
    e = cudaMemcpy(g->d_slots, hs.data(), sizeof(pp_gmres_slot) * count, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    delete g;
    return cuda_fail(ctx, e, "pp_gmres_create");
  }
  *out = g;
  return PP_OK;
}

void pp_gmres_destroy(pp_gmres* g) { delete g; }

pp_status pp_gmres_start(pp_gmres* g, void* stream) {
  if (!g) return PP_INVALID_ARG;
  pp_context* ctx = g->ctx;
  PP_CUDA(pp_gmres_start(g->d_slots, g->count, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_gmres_arnoldi(pp_gmres* g, int j, void* stream) {
  if (!g) return PP_INVALID_ARG;
  pp_context* ctx = g->ctx;
  if (j < 0 || j >= g->m) return fail(ctx, PP_INVALID_ARG, "pp_gmres_arnoldi: step outside [0, m)");
  PP_CUDA(pp_gmres_arnoldi(g->d_slots, g->count, j, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_gmres_finish(pp_gmres* g, void* stream) {
  if (!g) return PP_INVALID_ARG;
  pp_context* ctx = g->ctx;
  PP_CUDA(pp_gmres_finish(g->d_slots, g->count, (cudaStream_t)stream));
  return PP_OK;
}

pp_status pp_gmres_status(pp_gmres* g, double* out) {
  if (!g || !out) return PP_INVALID_ARG;
  pp_context* ctx = g->ctx;
  std::vector<double> st(g->state_elems * g->count);
  PP_CUDA(cudaDeviceSynchronize());
  PP_CUDA(cudaMemcpy(st.data(), g->d_state, sizeof(double) * st.size(), cudaMemcpyDeviceToHost));
  const size_t meta = g->state_elems - 4;
  for (int i = 0; i < g->count; ++i) {
    out[2 * i] = st[g->state_elems * i + meta];
    out[2 * i + 1] = st[g->state_elems * i + meta + 3];
  }
  return PP_OK;
}

// ---------------------------------------------------------------- program regions
pp_status pp_hmatrix_program_regions(pp_hmatrix* h, int which, int nrhs, long long* count, int32_t* out) {
  if (!h || !count || (which != 0 && which != 1) || (which == 1 && nrhs <= 0)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  long long k = 0;
  for (size_t t = 0; t < plan->prog.tasks.size(); ++t)
    for (const pp::Region& r : plan->prog.tasks[t].regions) {
      if (out) {
        int32_t* o = out + 7 * k;
        o[0] = (int32_t)t;
        o[1] = r.obj;
        o[2] = r.r0;
        o[3] = r.c0;
        o[4] = r.nr;
        o[5] = r.nc;
        o[6] = r.ro ? 1 : 0;
      }
      ++k;
    }
  *count = k;
  return PP_OK;
}

// ---------------------------------------------------------------- DAG build placement
pp_status pp_context_set_device_dag(pp_context* ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return PP_INVALID_ARG;
  if (on && !has_device(ctx)) return fail(ctx, PP_INVALID_ARG, "device DAG build needs a device context");
  ctx->dag_device = on;
  return PP_OK;
}

pp_status pp_hmatrix_dag_info(pp_hmatrix* h, int which, int nrhs, double* dag_ms, int* on_device) {
  if (!h || (which != 0 && which != 1) || (which == 1 && nrhs <= 0)) return PP_INVALID_ARG;
  VmPlan* plan = which == 0 ? &h->factor : solve_plan(h, nrhs);
  pp_status st = build_program(h, which, nrhs, *plan);
  if (st != PP_OK) return st;
  if (dag_ms) *dag_ms = plan->dag_ms;
  if (on_device) *on_device = plan->dag_on_device;
  return PP_OK;
}

}  // extern "C"
