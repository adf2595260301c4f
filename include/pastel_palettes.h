/* pastel_palettes.h — C ABI of the B200-native H-LU engine (libpastel_palettes.so).
 *
 * Drop-in boundary for the factor / solve path of Pastel-Palettes.  Every entry point
 * names the reference interface it replaces (file:line in the reference project).
 * Plain C: pointers, sizes and status codes only.  Device pointers are CUDA device
 * addresses; `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 *
 * Conventions
 *  - Matrices are row-major FP64 (the reference kernel's layout, src/kernel.cu:42).
 *  - The caller owns host buffers; the library owns device copies of H-matrices and
 *    their factors until pp_hmatrix_destroy.
 *  - A context is used from one host thread at a time.
 *  - No CPU fallback: without a usable CUDA device every compute entry point returns
 *    PP_CUDA_ERROR.
 */
#ifndef PASTEL_PALETTES_H
#define PASTEL_PALETTES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pp_status {
  PP_OK = 0,
  PP_INVALID_ARG = 1,
  PP_OOM = 2,
  PP_TIMEOUT = 3,     /* a device wait gave up (bounded spin) */
  PP_NUMERICAL = 4,   /* non-finite result / zero pivot        */
  PP_CUDA_ERROR = 5,
  PP_UNSUPPORTED = 6,
  PP_INTERNAL = 7
} pp_status;

typedef struct pp_context pp_context;
typedef struct pp_hmatrix pp_hmatrix;

typedef struct pp_config {
  int tile;              /* dense blocks above this are split before they reach an instruction (<= 64) */
  int ctas_per_sm;       /* persistent VM CTAs per SM (0 = occupancy maximum)                        */
  long long spin_limit;  /* microseconds a VM CTA waits for a ready task (or for its tensor-core
                            work) before it reports PP_TIMEOUT; 0 = 120 s.  Timed by the GPU's
                            global timer, so it does not depend on how fast a poll is            */
  unsigned long long seed;  /* seed of the random sketch used by accum                                */
  int reference_isa;     /* 1: factor programs use only the reference's instruction set (no split-k
                            reductions), so pp_refstream_encode can export them                         */
} pp_config;

typedef struct pp_block_info {
  int kind;       /* 0 dense, 1 low-rank, 2 hierarchical */
  int row0, col0, m, n;
  int rank, kmax, level;
  int children[4];
} pp_block_info;

typedef struct pp_program_info {
  int n_tasks;
  long long n_edges;
  long long flops;                  /* algorithmic FLOPs of all instructions */
  long long op_count[24];           /* instructions per pp_op (pp_task.h)   */
  long long arena_elems[5];         /* matrix, work, scratch, rhs, rand     */
  double host_build_ms;             /* op generation + DAG + encoding        */
} pp_program_info;

/* --- context ----------------------------------------------------------- */
/* replaces the device set-up of dev_hierarchical_GETRF (src/launcher.cu:119-123) */
pp_status pp_context_create(int device, const pp_config* cfg, pp_context** out);
void pp_context_destroy(pp_context* ctx);
/* copies the last error message (NUL-terminated) into buf; returns its length */
int pp_last_error(const pp_context* ctx, char* buf, size_t size);
int pp_device_sm_count(const pp_context* ctx);

/* --- matrix/Dense + matrix/Hierarchical --------------------------------- */
/* all-dense 2 x 2 partition down to `leaf` (matrix/Hierarchical.h:4-7 is an empty stub in
 * the reference; the tree interface follows its use at src/launcher.cu:126,138-139) */
pp_status pp_hmatrix_create_dense(pp_context* ctx, int n, int leaf, pp_hmatrix** out);
/* geometric block tree over points in cluster order; admissibility 0 = weak, 1 = standard */
pp_status pp_hmatrix_create_geometric(pp_context* ctx, int n, int dim, const double* points, int leaf,
                                      int admissibility, double eta, int kmax, pp_hmatrix** out);
void pp_hmatrix_destroy(pp_hmatrix* h);
int pp_hmatrix_num_blocks(const pp_hmatrix* h);
int pp_hmatrix_root(const pp_hmatrix* h);
pp_status pp_hmatrix_block_info(const pp_hmatrix* h, int block, pp_block_info* info);
/* where a block lives in the arena (element offsets): a dense block at off (m x n, ld n); a
 * low-rank block's U at off (m x kmax, ld kmax), V at off_v (n x kmax, ld kmax) and its rank word
 * at off_rank; -1 where a block has no such part (hierarchical blocks have none).  The storage
 * layout the reference's Dense / Hierarchical would own (matrix/Dense.h:6-18); lets a program
 * exported with pp_hmatrix_encode_program be run on arenas filled without this library. */
pp_status pp_hmatrix_block_storage(const pp_hmatrix* h, int block, long long* off, long long* off_v,
                                   long long* off_rank);
/* host data of one block (Dense(m, n, lda), matrix/Dense.h:6-18; row-major here) */
pp_status pp_hmatrix_set_dense(pp_hmatrix* h, int block, const double* a, int lda);
pp_status pp_hmatrix_set_lowrank(pp_hmatrix* h, int block, const double* U, int ldu, const double* V, int ldv,
                                 int rank);
pp_status pp_hmatrix_upload(pp_hmatrix* h, void* stream);
pp_status pp_hmatrix_download(pp_hmatrix* h, void* stream);
/* page-locks the host image so uploads / downloads run at full PCIe rate */
pp_status pp_hmatrix_pin_host(pp_hmatrix* h);
/* keeps a device copy of the uploaded (unfactored) matrix; pp_hmatrix_restore copies it
 * back over the factors (device to device, stream ordered) for repeated factorizations */
pp_status pp_hmatrix_keep_original(pp_hmatrix* h, void* stream);
pp_status pp_hmatrix_restore(pp_hmatrix* h, void* stream);
/* dense n x n image of the host copy (after download: the L\U factors) */
pp_status pp_hmatrix_to_dense(const pp_hmatrix* h, double* out);
long long pp_hmatrix_storage_elems(const pp_hmatrix* h);
/* host image of the block arena (row-major blocks at the offsets of the block tree);
 * writable: pp_hmatrix_to_dense and pp_hmatrix_upload read it */
double* pp_hmatrix_host_arena(pp_hmatrix* h, long long* elems);
/* device base of the matrix arena (read-only view for residual / export helpers) */
const double* pp_hmatrix_device_arena(const pp_hmatrix* h);
/* elements of the arena prefix that holds the matrix blocks — what upload, download,
 * keep_original and restore copy.  The rest of the arena holds the explicit inverses of
 * the diagonal leaves' triangular factors, written by the factorization and read by the
 * solves.  no reference counterpart */
long long pp_hmatrix_block_elems(const pp_hmatrix* h);

/* contraction precision of the factor's GEMM (Schur-complement and low-rank product)
 * instructions: PP_PRECISION_FP64 (default; matches the reference's FP64 factorization) or
 * PP_PRECISION_TF32 (5th-generation tensor cores, TF32 operands, FP32 accumulation, FP64
 * result; GETRF / TRSM / accumulation stay FP64 — pair it with iterative refinement).
 * Rebuilds the factor program on the next factorization; set it before pp_batch_create.
 * no reference counterpart (the reference is FP64 only) */
#define PP_PRECISION_FP64 0
#define PP_PRECISION_TF32 1
/* PP_PRECISION_BF16: the Schur-complement updates of whole dense leaves of 512 or more rows and
 * columns (multiples of 128 / 256, inner dimension of 64) run on the tensor cores from BF16
 * shadows of their operands (written once per operand block by SHADOW instructions), FP32
 * accumulation in tensor memory, FP64 result; the diagonal leaves' GETRF, the triangular solves,
 * the low-rank work and every other product stay FP64.  Pair it with iterative refinement. */
#define PP_PRECISION_BF16 2
pp_status pp_hmatrix_set_precision(pp_hmatrix* h, int precision);
int pp_hmatrix_get_precision(const pp_hmatrix* h);
/* Partial pivoting inside every GETRF block (on = 1; 0 is the reference's no-pivot LU, the
 * default), for matrices that are not diagonally dominant.  Uses the reference's pivot
 * helpers' idea (src/kernel.cu:958-1051: largest-magnitude row, row swaps, permutation applied
 * to the rows of the right-hand blocks), which the reference itself never calls: each GETRF
 * block (at most the tile, 64 rows) picks its pivot rows among its own rows, stores its row
 * permutation beside the leaf (arena tail), and every triangular solve against that block's
 * L — in the factorization (the blocks to its right, dense or the U factor of a low-rank block)
 * and in the solve (the right-hand sides) — permutes its right-hand side first.  The solve then
 * substitutes (no explicit inverses).  A block that needs no swap gives the unpivoted bits.
 * Drops the matrix's programs; FP64, TF32 and BF16 forms alike. */
pp_status pp_hmatrix_set_pivoting(pp_hmatrix* h, int on);
/* output tile edge (64, the default, or 128) that the factor's products are split into;
 * larger tiles give fewer, longer GEMM instructions (the autotuner tries both).  Results do not
 * depend on it: every element still accumulates its k products in ascending order.  Rebuilds
 * the programs on the next factorization; set it before pp_batch_create.  No reference
 * counterpart (the reference's blocking is compile-time). */
pp_status pp_hmatrix_set_gemm_tile(pp_hmatrix* h, int edge);
/* adaptive rank (tol > 0, before set_lowrank and upload): low-rank blocks keep kmax columns,
 * zero beyond their numerical rank, and every accumulation into them truncates to the
 * singular values above tol times the largest (Gram eigen-decomposition by Jacobi, the role of
 * blockSingleSideJacobiSVD / blockReadRank, src/kernel.cu:1084-1157, 1282-1315); tol = 0
 * restores the fixed-rank form (ranks as set, no truncation) */
pp_status pp_hmatrix_set_rank_tolerance(pp_hmatrix* h, double tol);
/* numerical rank of a low-rank block in the host image (set_lowrank; after a download, the
 * ranks the factorization's accumulations chose); -1 for other blocks */
int pp_hmatrix_block_rank(const pp_hmatrix* h, int block);

/* --- factor / solve (launcher.cuh) --------------------------------------- */
/* H-LU factorization in place on the device, stream ordered.
 * replaces dev_hierarchical_GETRF (include/launcher.cuh:18, src/launcher.cu:117-217) */
pp_status pp_hlu_factor(pp_hmatrix* h, void* stream);
/* X := A^-1 B with the device factors: B, X device, row-major n x nrhs (may alias).
 * no reference counterpart (the reference has no solve) */
pp_status pp_hlu_solve(pp_hmatrix* h, const double* b_dev, double* x_dev, int nrhs, void* stream);
/* waits for `stream`; returns PP_TIMEOUT / PP_INTERNAL if the last VM launch of h failed */
pp_status pp_hmatrix_sync(pp_hmatrix* h, void* stream);
/* introspection of the factor (which = 0) or solve (which = 1, nrhs) program */
pp_status pp_hmatrix_program_info(pp_hmatrix* h, int which, int nrhs, pp_program_info* info);
/* reference-signature driver: dev_hierarchical_GETRF(h, num_blocks, num_threads, kernel_size)
 * (include/launcher.cuh:18).  num_blocks > 0 caps the persistent grid; num_threads must be
 * 256 or 0; kernel_size is accepted and ignored (one launch covers the whole DAG). */
pp_status pp_dev_hierarchical_getrf(pp_hmatrix* h, int num_blocks, int num_threads, int kernel_size);

/* --- batches: many H-matrices in one persistent launch (no reference counterpart;
 *     the reference launches one DAG at a time, src/launcher.cu:146-167) ----------- */
typedef struct pp_batch pp_batch;
/* merges the factor programs of n uploaded H-matrices (sizes may differ) into one task
 * table; the instances stay owned by the caller and must outlive the batch */
pp_status pp_batch_create(pp_context* ctx, pp_hmatrix* const* hs, int n, pp_batch** out);
void pp_batch_destroy(pp_batch* b);
/* factor all instances: one VM launch (plus one memset of the work buffers) */
pp_status pp_batch_factor(pp_batch* b, void* stream);
/* X_i := A_i^-1 B_i for every instance i, one VM launch; B[i], X[i] device n_i x nrhs */
pp_status pp_batch_solve(pp_batch* b, const double* const* B, double* const* X, int nrhs, void* stream);
pp_status pp_batch_restore(pp_batch* b, void* stream);  /* pp_hmatrix_restore on every instance */
pp_status pp_batch_sync(pp_batch* b, void* stream);
pp_status pp_batch_program_info(pp_batch* b, int which, int nrhs, pp_program_info* info);
pp_status pp_batch_trace(pp_batch* b, int which, int nrhs, int enable, uint64_t* out);
/* Autotuner (no reference counterpart; the reference's tile sizes are compile-time constants
 * of a missing header): times the batch's factor launch for every dense tile in {32, 64}
 * (the largest block one GETRF / TRSM instruction takes), product tile in {64, 128}
 * (pp_hmatrix_set_gemm_tile) and persistent grid in {all, 3/4, 1/2 of the resident CTAs}, and
 * keeps the fastest for this batch's later launches.  Every
 * instance must hold an original (pp_hmatrix_keep_original): each trial restores it first, and
 * on return the instances hold their restored, unfactored matrices. */
typedef struct pp_tune_result {
  int tile, grid, trials;
  double factor_ms;
  int gemm_tile; /* output tile edge of the product tasks (64 or 128) */
} pp_tune_result;
pp_status pp_batch_autotune(pp_batch* b, void* stream, pp_tune_result* out);
/* applies a tuning (from pp_batch_autotune on a batch of the same shapes) without timing:
 * dense tile (8..64), product tile (64 or 128) and persistent grid (0: all CTAs) */
pp_status pp_batch_set_tuning(pp_batch* b, int tile, int gemm_tile, int grid);

/* --- serving: a request loop with continuous admission (no reference counterpart; the
 *     reference factors one matrix per launch) -------------------------------------------
 * A server owns a worker thread.  Factor + solve requests of any size are admitted in arrival
 * order while in-flight slots and the HBM budget allow (a smaller later request may pass a
 * larger waiting one); each admitted request runs on its own CUDA stream with a persistent
 * grid of a slot's share of the SMs, so requests that arrive while others are on the GPU
 * overlap with them.  A request keeps its factors on the device for all of its right-hand-side
 * sets (the first solve and its follow-ups), refines each set in FP64 (matrix-free kernel
 * residual) until the normwise backward error ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf)
 * meets `tol`, writes the solutions to the caller's host buffer and frees its device memory
 * (stream-ordered, so retiring one request never waits for the others).  The requests'
 * device memory comes from a memory pool of the server's own that keeps up to the budget
 * mapped between requests; pp_server_create maps its first GiB (or the whole budget, if
 * smaller) at once.  While a server runs, its context is used only through the server's
 * calls. */
typedef struct pp_server pp_server;
typedef struct pp_serve_config {
  long long hbm_budget_bytes;  /* device bytes the admitted requests may hold together        */
  int max_inflight;            /* requests on the device at once (slots)                      */
  int grid_per_request;        /* persistent CTAs per request launch (0: SMs / slots)          */
} pp_serve_config;
typedef struct pp_request_desc {
  int kernel;              /* matrix entries, as pp_kernel_residual_dev: 0 1/(r+p0), 1 Laplace,
                              2 exp(-r/p0), 3 Matern-3/2 (length p0)                            */
  double p0, shift;        /* kernel parameter and diagonal shift                             */
  double norm_inf;         /* ||A||_inf (backward-error normalisation)                        */
  int dim;                 /* point dimension (1..3)                                          */
  const double* points;    /* n x dim host points in the H-matrix's cluster order (copied)    */
  const double* rhs;       /* n_sets blocks of n x nrhs host right-hand sides (copied)        */
  int nrhs, n_sets;        /* 1 <= nrhs <= 16; n_sets >= 1 (the first solve + follow-ups)      */
  double tol;              /* backward-error target of every set                              */
  int max_iter;            /* refinement solves per set at most                               */
  double* x_out;           /* n_sets blocks of n x nrhs host solutions; must stay valid until
                              the request is done or failed                                   */
} pp_request_desc;
typedef struct pp_request_stats {
  int status;              /* 0 queued, 1 running, 2 done, 3 failed                            */
  int iterations;          /* refinement solves over all sets                                 */
  double backward_error;   /* worst final backward error over the finished sets               */
  double t_submit_ms, t_admit_ms, t_done_ms;  /* server clock (ms); -1 until reached          */
  double t_enqueued_ms;    /* when the upload, the factorization and the first solve were
                              queued on the device (the host work of admission ends)          */
  long long device_bytes;  /* device memory the request holds while admitted                  */
  char message[128];       /* why a request failed                                            */
} pp_request_stats;
pp_status pp_server_create(pp_context* ctx, const pp_serve_config* cfg, pp_server** out);
/* queues a request; the server takes ownership of h (built, not uploaded) and destroys it when
 * the request retires.  An H-matrix filled on the host (set_dense / set_lowrank) is uploaded at
 * admission; one that never had a host image is built on the device from the request's points
 * at admission (pp_hmatrix_construct_dev), inside the request's latency.  Returns PP_OOM when
 * the request alone exceeds the budget. */
pp_status pp_server_submit(pp_server* s, pp_hmatrix* h, const pp_request_desc* d, long long* id);
pp_status pp_server_poll(pp_server* s, long long id, pp_request_stats* st);
/* waits until no request is queued or running (PP_TIMEOUT after timeout_ms) */
pp_status pp_server_wait_all(pp_server* s, double timeout_ms);
double pp_server_clock_ms(pp_server* s);
/* lets the queued and running requests finish, then stops the worker */
void pp_server_destroy(pp_server* s);

/* --- residuals (FP64 refinement) ----------------------------------------- */
/* r := b - A x, A dense row-major (device); x, b, r device n x nrhs */
pp_status pp_dense_residual_dev(pp_context* ctx, const double* A, int lda, int n, const double* x, const double* b,
                                double* r, int nrhs, void* stream);
/* r := b - A x, A_ij = K(|p_i - p_j|) + shift * (i == j) evaluated on the fly.
 * kernel: 0 = 1/(r+p0), 1 = 1/(4 pi (r+p0)), 2 = exp(-r/p0), 3 = Matern-3/2 length p0.
 * Partial sums go through a context-owned buffer, grown on the first call of a larger size
 * (make that call before capturing a CUDA graph); calls on different streams must not
 * overlap. */
pp_status pp_kernel_residual_dev(pp_context* ctx, int kernel, double p0, double shift, const double* pts_dev,
                                 int dim, int n, const double* x, const double* b, double* r, int nrhs,
                                 void* stream);
/* The dense blocks of an uploaded H-matrix assembled on the device from its points (device,
 * n x dim, in the H-matrix's cluster order): entry (i, j) = K(|p_i - p_j|) with the kernels of
 * pp_kernel_residual_dev, plus `shift` on the matrix diagonal, with the same entry evaluation as
 * the residual.  Low-rank blocks are left as they are.  No reference counterpart (the
 * reference's matrices come from a separate Java compressor). */
pp_status pp_hmatrix_assemble_dense_dev(pp_hmatrix* h, int kernel, double p0, double shift, const double* pts_dev,
                                        int dim, void* stream);
/* Builds the whole H-matrix on the device from its points (device, n x dim, in the H-matrix's
 * cluster order), without a host image: the device arena is allocated (zero-filled) if needed,
 * the dense blocks are assembled as pp_hmatrix_assemble_dense_dev does, and every low-rank block
 * is compressed by a randomized range finder with one power step on the VM (instructions KMUL:
 * kernel matrix times a block of vectors, evaluated from the points; ORTH; LRTRUNC: truncation
 * to the singular values above the rank tolerance times the largest, at most the block's rank).
 * The kernel must be smooth on the admissible blocks (the four kernels of
 * pp_kernel_residual_dev are).  Stream ordered; pp_hmatrix_sync reports a failed launch.
 * No reference counterpart (the reference's matrices come from a separate Java compressor). */
pp_status pp_hmatrix_construct_dev(pp_hmatrix* h, int kernel, double p0, double shift, const double* pts_dev,
                                   int dim, void* stream);
/* One job of pp_kernel_residual_batch_dev (device pointers). */
typedef struct pp_residual_job {
  int kernel;           /* as pp_kernel_residual_dev */
  int dim;              /* 1..3 */
  int n;
  int nrhs;             /* 1..16 */
  double p0, shift;
  const double* points; /* n x dim */
  double* x;            /* n x nrhs; x += dx first when dx is not NULL */
  const double* dx;     /* n x nrhs or NULL */
  const double* b;      /* n x nrhs */
  double* r;            /* n x nrhs */
} pp_residual_job;
/* The refinement update and residual of many kernel problems: for every job x += dx (when dx
 * is set), then r = b - A x.  One update launch, one residual launch per group of jobs with the
 * same kernel, dimension and right-hand-side width (up to 64 jobs each), one reduction launch;
 * each job's r is bit-identical to pp_kernel_residual_dev's.  Kernels 0 and 1 need a finite
 * p0 >= 0.  Partial sums go through the context-owned buffer, sized for the sum of the
 * jobs' needs (grown on the first call of a larger total: make that call before capturing a
 * CUDA graph); calls on different streams must not overlap. */
pp_status pp_kernel_residual_batch_dev(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream);
/* The same with the kernel entries of jobs of at most 4 right-hand sides evaluated in FP32
 * (hardware reciprocal square root, exponential and division; a few 1e-7 relative per entry;
 * sums still in FP64).  No counterpart in the reference.  Meant for the products inside Krylov
 * cycles (pp_gmres_*), whose answer a FP64 residual then certifies; never for that residual. */
pp_status pp_kernel_residual_batch_lowp_dev(pp_context* ctx, int njobs, const pp_residual_job* jobs, void* stream);

/* --- batched restarted GMRES around the H-LU solve -------------------------
 * No counterpart in the reference (it has no solve or refinement path).  For a batch of
 * kernel problems whose plain refinement stalls (H-LU factors too coarse for the spectral
 * radius of I - (LU)^-1 A to stay below 1), GMRES on A (LU)^-1 with the FP64 matrix-free
 * residual converges to the same tolerance.  The caller owns every vector (device memory):
 * V[i]: (m + 1) x n[i] basis, Z[i]: m x n[i] preconditioned basis, x[i]: solution, r[i]: the
 * residual b - A x that starts a cycle.  A cycle is
 *   pp_gmres_start;  for j < m: Z_j = solve(V_j) (pp_batch_solve), V_{j+1} = 0 - A Z_j
 *   (pp_kernel_residual_batch_dev with b = 0), pp_gmres_arnoldi(j);  pp_gmres_finish;
 *   r = b - A x.
 * Each call is one launch on `stream`, one CTA per instance (largest first), no host
 * synchronization and no allocation (capturable).  1 <= m <= PP_GMRES_MAX_RESTART. */
#define PP_GMRES_MAX_RESTART 128
typedef struct pp_gmres pp_gmres;
pp_status pp_gmres_create(pp_context* ctx, int count, const int* n, int m, double* const* V, double* const* Z,
                          double* const* x, double* const* r, pp_gmres** out);
void pp_gmres_destroy(pp_gmres* g);
/* beta = ||r||_2, v_0 = r / beta (an instance with r = 0 stays frozen for the cycle) */
pp_status pp_gmres_start(pp_gmres* g, void* stream);
/* Arnoldi step j (0 <= j < m) of every instance: V_{j+1} holds -A z_j on entry; CGS2 against
 * V_0..V_j, normalised; the Hessenberg column rotated; |g_{j+1}| is the residual estimate */
pp_status pp_gmres_arnoldi(pp_gmres* g, int j, void* stream);
/* x += Z y, y the least-squares solution of the cycle's active dimension */
pp_status pp_gmres_finish(pp_gmres* g, void* stream);
/* (synchronous) per instance, in creation order: active dimension and residual estimate of
 * the current cycle, out[2 i] and out[2 i + 1] */
pp_status pp_gmres_status(pp_gmres* g, double* out);

/* --- DAG build on the device ---------------------------------------------
 * Replaces the host-side dependency discovery of the reference (rts/ops.cpp:42-61
 * Operation::checkDependencyFrom over earlier instructions, the edge table of
 * rts/dependency.cpp:7-76) for programs built after this call: every (instruction, region)
 * access walks its object's earlier accesses on the GPU (dag.cu).  The edges, their
 * flow / anti / out types and every instruction's predecessor and successor order are those of
 * the host build; when the device build cannot run (a CUDA error, or a walk with more partial
 * writes than it keeps) the host build runs instead and pp_last_error says why.  on = 1 needs
 * a device context; 0 (the default) builds on the host. */
pp_status pp_context_set_device_dag(pp_context* ctx, int on);
/* the factor (which 0) or solve (1, nrhs) program's DAG build: wall milliseconds, and 1 when it
 * ran on the device (builds the program first if needed) */
pp_status pp_hmatrix_dag_info(pp_hmatrix* h, int which, int nrhs, double* dag_ms, int* on_device);

/* The data regions of every instruction of the factor (which 0) or solve (1) program, the
 * reference's Operation data list (rts/ops.h:22-36: read-only flag and 2-D region per operand):
 * 7 int32 per region (task, storage object, first row, first column, rows, columns, read-only),
 * in program order; out == NULL only sets *count. */
pp_status pp_hmatrix_program_regions(pp_hmatrix* h, int which, int nrhs, long long* count, int32_t* out);

/* --- rts (DAG primitives, rts/ops.h, rts/dependency.h) ------------------- */
/* DataMap2D::checkOverlap (rts/ops.cpp:7-40); regions: ptr, pitch, width (bytes), height */
int pp_datamap2d_check_overlap(uintptr_t ptr_a, size_t pitch_a, size_t width_a, size_t height_a, uintptr_t ptr_b,
                               size_t pitch_b, size_t width_b, size_t height_b);
/* Operation::checkDependencyFrom (rts/ops.cpp:42-61): regions as flat arrays of
 * (ptr, pitch, width, height) with read_only flags; returns a dependency_t bit set
 * (1 flow, 2 anti, 4 out) */
int pp_operation_dependency(int n_from, const uint64_t* regions_from, const int* ro_from, int n_to,
                            const uint64_t* regions_to, const int* ro_to);

/* --- program export (tests, oracle, reference-format streams) ------------ */
/* Encodes the factor (which = 0) or solve (which = 1) program with caller-chosen arena
 * bases (host or device addresses; arena order matrix, work, scratch, rhs, rand).
 * tasks: n_tasks records of 160 bytes (pp_task.h); succ: n_edges; indeg: n_tasks.  */
pp_status pp_hmatrix_encode_program(pp_hmatrix* h, int which, int nrhs, double* const* bases, void* tasks,
                                    int32_t* succ, int32_t* indeg, int32_t* order);
/* Per-instruction trace (the reference stamps clock64 per instruction, src/kernel.cu:1389-1390,
 * and renders it with analyzeClocks, rts/scheduler.cpp:494-544): with out == NULL, enable != 0
 * makes later launches of the program record, per task, the globaltimer (ns) at start and end
 * and the SM (low 32 bits) and CTA (high 32 bits); out != NULL copies 3 * n_tasks words back. */
pp_status pp_hmatrix_trace(pp_hmatrix* h, int which, int nrhs, int enable, uint64_t* out);
/* typed DAG of the factor / solve program: edge e runs from[e] -> to[e] with dependency_t
 * bits type[e] (1 flow, 2 anti, 4 out); the dependency_table of rts/dependency.h:24-53 */
pp_status pp_hmatrix_program_edges(pp_hmatrix* h, int which, int nrhs, int64_t* from, int64_t* to, int32_t* type);
/* Runs an arbitrary task table (host array of n pp_task records with device operand
 * pointers; successor lists and in-degrees as pp_hmatrix_encode_program returns them) on
 * the VM and waits.  spin_limit (microseconds) <= 0 uses the context's.  Returns PP_TIMEOUT
 * when a ready slot is never filled (e.g. an in-degree that no predecessor can bring to zero).
 * Counterpart of launchKernelWithArgs (include/launcher.cuh:15-16) for decoded streams. */
pp_status pp_vm_execute(pp_context* ctx, const void* tasks, int n_tasks, const int32_t* succ, long long n_succ,
                        const int32_t* indeg, long long spin_limit, int grid, void* stream);
/* Low-rank accumulation without any device allocation.  No counterpart in the reference.
 *
 * Computes the same thing as one ACCUM task run through pp_vm_execute:
 *   U1 V1^T := Q Q^T (U1 V1^T + sign * U2 V2^T),  Q an orthonormal basis of that sum times R,
 * in place on U1 (ny x k1, ld_u1) and V1 (nx x k1, ld_v1); U2 (ny x k2), V2 (nx x k2) and the
 * sketch R (nx x k1) are read.  All pointers are device pointers the caller owns.
 *
 * For callers that cannot call cudaMalloc: code recorded into a CUDA graph while a stream is
 * being captured (an allocation there breaks the capture), serving loops whose device memory
 * is fully reserved by an admission budget, and host frameworks that own the device memory
 * pool.  Its scratch is one static device array of PP_ACCUM_NOALLOC_MAX_SCRATCH doubles
 * (8 MiB), held by every GPU that loads the library until the process exits.  The accumulation
 * keeps its ny x k1 sketch in shared memory while that fits (ny * k1 up to about 17 000 - 20 000
 * doubles, by rank); a larger sketch goes to the array, so ny * k1 <= 2^20 is the limit.
 * 1 <= k1, k2 <= 32 and k1 <= min(ny, nx); other requests return PP_INVALID_ARG without
 * touching the device.  The call runs on the context's device.
 *
 * The first call on each device looks up the array's device address (with that device
 * current, once per device even with several host threads); make that first call before any
 * stream capture.  Every call shares the array and overwrites all of it that it uses before
 * reading it, so nothing carries over between calls; calls whose executions overlap on the
 * GPU (different streams, or graphs replayed concurrently) race on it. */
#define PP_ACCUM_NOALLOC_MAX_SCRATCH (1 << 20)
pp_status pp_lowrank_accum_noalloc(pp_context* ctx, double* U1, int ld_u1, double* V1, int ld_v1, const double* U2,
                                   int ld_u2, const double* V2, int ld_v2, const double* R, int ld_r, int ny, int nx,
                                   int k1, int k2, double sign, void* stream);

/* random sketch the accum instructions read (arena `rand`, row-major n x kmax, ld = rank) */
pp_status pp_hmatrix_rand_host(pp_hmatrix* h, double* out, long long count);
/* Reference-format instruction streams of the factor program (src/kernel.cu:1384-1522)
 * for `workers` workers; pointer index = arena index above.  Returns the stream words
 * concatenated, lengths[workers], and the per-worker scratch the reference's accum needs.
 * operation enum: nop 0, getrf 1, trsml 2, trsmr 3, gemm 4, gemm_plus 5, gemm_3x 6,
 * gemm_4x 7, accum 8; opcodes: finish 0, execute 1, signal_wait 2. */
pp_status pp_refstream_encode(pp_hmatrix* h, int workers, int32_t* words, long long capacity, int32_t* lengths,
                              long long* tmp_elems_per_worker);

#ifdef __cplusplus
}
#endif

#endif
