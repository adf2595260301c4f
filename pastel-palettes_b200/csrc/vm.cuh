// vm.cuh — host-side interface of the H-LU virtual machine kernels (vm.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pp_task.h"

#define PP_VM_THREADS 256
#define PP_VM_TILE 64          /* largest dense block GETRF / TRSM* keep in shared memory */
#define PP_VM_TRI 256          /* largest triangle of a TRSM* task (blocked by PP_VM_TILE)   */
#define PP_VM_INV 512          /* largest leaf of a TRINV / TRMV task (explicit inverses)       */
#define PP_VM_MAX_RANK 32      /* largest k1 of ACCUM (register-resident reductions)    */

enum pp_vm_error { PP_VM_OK = 0, PP_VM_TIMEOUT = 1, PP_VM_BAD_TASK = 2, PP_VM_MMA_TIMEOUT = 3 };

typedef struct pp_vm_state {
  int head;      /* next ready-slot index to pop                  */
  int tail;      /* next ready-slot index to fill                 */
  int done;      /* tasks completed                               */
  int error;     /* pp_vm_error                                   */
  int err_info;  /* slot index (timeout) or task id (bad task)    */
  int pad[3];
} pp_vm_state;

struct pp_vm_launch {
  const pp_task* tasks;
  int n_tasks;
  const int32_t* succ;
  const int32_t* indeg;
  const int32_t* ready;
  int n_ready;
  int32_t* counters;
  int32_t* slots;
  pp_vm_state* state;
  long long wait_ns;     /* nanoseconds a CTA waits on an empty ready slot (or on the tensor core)
                            before the kernel gives up */
  int grid;              /* CTAs (persistent)                                       */
  unsigned long long* trace = nullptr;  /* optional: 3 words per task (start ns, end ns, sm | cta << 32) */
  int use_tc = 0;        /* the program holds TF32 tasks: tensor memory + an mbarrier per CTA */
};

/* ACCUM on caller buffers with the library's static scratch array (no allocation);
 * returns cudaErrorInvalidValue when `scratch_doubles` exceeds the array */
cudaError_t pp_accum_noalloc_launch(const pp_task& T, long long scratch_doubles, cudaStream_t s);
long long pp_accum_noalloc_capacity();
/* scratch doubles one ACCUM of this shape needs (its ny x k1 sketch, when that does not fit the
 * task's shared memory; 0 otherwise) */
long long pp_accum_scratch_doubles(long long ny, int k1, int k2);

size_t pp_vm_smem_bytes();
int pp_vm_blocks_per_sm();
cudaError_t pp_vm_prepare();  /* sets the dynamic shared-memory attribute (once per device) */
cudaError_t pp_vm_run(const pp_vm_launch& L, cudaStream_t s);
/* dense FP64 residual r = b - A x, A row-major n x n, x/b/r n x nrhs row-major */
cudaError_t pp_dense_residual(const double* A, int lda, int n, const double* x, const double* b, double* r, int nrhs,
                              cudaStream_t s);
/* matrix-free residual r = b - A x for kernel matrices on points (see kernels in vm.cu);
 * `part` is caller scratch of pp_kernel_residual_part_elems(n, nrhs) doubles */
cudaError_t pp_kernel_residual(int kernel, double p0, double p1, double diag_shift, const double* pts, int dim, int n,
                               const double* x, const double* b, double* r, int nrhs, double* part,
                               cudaStream_t s);
size_t pp_kernel_residual_part_elems(int n, int nrhs);
/* one job of a batched matrix-free residual: x += dx first when dx is set, then r = b - A x */
struct pp_resid_job {
  int kernel, dim, n, nrhs;
  double p0, shift;
  const double* pts;
  double* x;
  const double* dx;
  const double* b;
  double* r;
  double* part; /* pp_kernel_residual_part_elems(n, nrhs) doubles of scratch, one per job */
};
/* the update, residual and reduction of every job in three or more launches (jobs grouped by
 * kernel, dimension and right-hand-side width); results equal those of one job per call */
cudaError_t pp_kernel_residual_batch(const pp_resid_job* jobs, int njobs, cudaStream_t s, bool lowp = false);
/* lowp: jobs of at most 4 right-hand sides evaluate the kernel entries in FP32 (relative error
 * of a few 1e-7 per entry, products still summed in FP64), for the products inside Krylov
 * cycles; wider jobs stay FP64 */
/* one dense block of an H-matrix to assemble from points: rows [r0, r0 + m), columns
 * [c0, c0 + n) of the matrix, stored row-major at a with leading dimension ld */
struct pp_assemble_block {
  double* a;
  int ld, r0, c0, m, n;
};
/* entries K(|p_i - p_j|) (+ shift on the diagonal) of every listed block, evaluated as the
 * matrix-free residual evaluates them */
cudaError_t pp_assemble_dense(const pp_assemble_block* blocks, int nblocks, int kernel, int dim, double p0,
                              double shift, const double* pts, cudaStream_t s);
/* x += dx (count elements) */
cudaError_t pp_axpy(double* x, const double* dx, size_t count, cudaStream_t s);
/* out[0] = max |x|, out[1] = max |r| (as double bit patterns; out is zeroed first) */
cudaError_t pp_absmax2(const double* x, const double* r, size_t count, unsigned long long* out, cudaStream_t s);

/* ---- batched restarted GMRES around the H-LU solve (krylov.cu) ---- */
#define PP_GMRES_MAX_RESTART 128 /* largest restart length (Arnoldi steps per cycle) */
/* one instance of a batched GMRES: device pointers, n rows, restart length m */
struct pp_gmres_slot {
  int n, m;
  double* V;   /* (m + 1) x n basis, vector k at V + k n              */
  double* Z;   /* m x n preconditioned basis, z_k = (LU)^-1 v_k         */
  double* x;   /* n: solution, x += Z y at the end of a cycle          */
  double* r;   /* n: residual b - A x at the start of a cycle         */
  double* st;  /* pp_gmres_state_elems(m) doubles of small state       */
};
size_t pp_gmres_state_elems(int m);
/* each launches one CTA per slot of the device array `slots` */
cudaError_t pp_gmres_start(const pp_gmres_slot* slots, int count, cudaStream_t s);
cudaError_t pp_gmres_arnoldi(const pp_gmres_slot* slots, int count, int j, cudaStream_t s);
cudaError_t pp_gmres_finish(const pp_gmres_slot* slots, int count, cudaStream_t s);
