/*
 * libprima_cuda.so -- B200 (sm_100a) backend for Prima's restarted-PDHG path.
 *
 * Plain C ABI: pointers, sizes, integer handles.  Every entry point returns an
 * int32 status (PRIMA_OK or a PRIMA_ERR_* code; prima_last_error() gives the
 * message).  Solver outcomes are NOT errors: they come back in
 * prima_solution_info.status, exactly as the reference reports numerical
 * trouble through SolveStatus rather than by exception.
 *
 * Reference interfaces replaced (paths relative to oluies/noaidi,
 * core = modules/prima-core/src/main/scala/org/noaidi/prima):
 *   - the kernel seam, trait Kernels          core/kernels/Kernels.scala:42-125
 *   - KernelCapabilities                      core/kernels/Kernels.scala:13-22
 *   - Pdhg.solveWith / WarmStart              core/Pdhg.scala:48-105
 *   - MixedPrecision.solve                    core/MixedPrecision.scala:104-199
 *   - PrimaZio.solveAll (batch shape)         modules/prima-zio/.../PrimaZio.scala:61-66
 *
 * Threading: a context is not thread-safe (one per thread, Kernels.scala:39-40);
 * any number of contexts may be open at once, each with its own CUDA stream.
 */
#ifndef PRIMA_CUDA_H
#define PRIMA_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------- */
#define PRIMA_OK 0
#define PRIMA_ERR_INVALID_ARGUMENT 1 /* the reference's `require` failures */
#define PRIMA_ERR_OUT_OF_MEMORY 2
#define PRIMA_ERR_CUDA 3
#define PRIMA_ERR_TIMEOUT 4 /* a bounded device-side wait gave up */
#define PRIMA_ERR_CLOSED 5  /* handle unknown or its context closed */
#define PRIMA_ERR_NO_DEVICE 6
#define PRIMA_ERR_PARSE 7 /* a malformed input file (MpsParseException) */

/* ---- SolveStatus (core/SolveResult.scala:9-18, same ordinals) ----------- */
#define PRIMA_STATUS_OPTIMAL 0
#define PRIMA_STATUS_PRIMAL_INFEASIBLE 1
#define PRIMA_STATUS_DUAL_INFEASIBLE 2
#define PRIMA_STATUS_ITERATION_LIMIT 3
#define PRIMA_STATUS_TIME_LIMIT 4
#define PRIMA_STATUS_NUMERICAL_ERROR 5
#define PRIMA_STATUS_INTERRUPTED 6

typedef int64_t prima_handle;

/* KernelCapabilities(name, device, supportsFloat64), Kernels.scala:13-22 */
typedef struct {
  char name[64];
  char device[128];
  int32_t supports_float64;
  int32_t precision_bits; /* storage precision of this context: 32 or 64 */
} prima_capabilities;

/* Message for the last failing call on this thread ("" if none). */
const char *prima_last_error(void);

/* ---- context (Kernels instance) ------------------------------------------ */
/* precision_bits = 64: IEEE double throughout (ScalaKernels semantics);
 * precision_bits = 32: binary32 storage and arithmetic per operation
 * (Float32Kernels semantics, core/kernels/Float32Kernels.scala:28-155). */
int32_t prima_open(int32_t device, int32_t precision_bits, prima_handle *ctx);
/* Kernels.close, Kernels.scala:65-66: releases every vector and matrix of the
 * context.  Idempotent: closing a closed context returns PRIMA_OK. */
int32_t prima_close(prima_handle ctx);
int32_t prima_capabilities_get(prima_handle ctx, prima_capabilities *out);
/* The number of polls a block of the persistent solver makes while waiting
 * at a team barrier for the other blocks before it gives up, raises the
 * team's abort flag and the call returns PRIMA_ERR_TIMEOUT (the reference's
 * solve loop has no such wait: Pdhg.scala:206-246 runs on one thread).
 * polls = 0 restores the default, 2^26 polls (seconds; a phase takes
 * microseconds).  A small value makes every multi-block solve of this context
 * give up at once, which is how the timeout path is exercised; the waits for
 * a block's own bulk copies keep their fixed bound.  No counterpart in the
 * reference. */
int32_t prima_set_device_wait_limit(prima_handle ctx, int64_t polls);
/* The persistent solver's layout for problems of more than 4,096 rows or
 * columns: blocks per SM and the row cap of the tiles its hot phases stream.
 * By default (both 0) the layout is chosen per problem and precision the
 * first time the problem is solved: a few candidates (the most blocks that
 * fit or one fewer; full or half tiles) each run a short bounded solve, and
 * the fastest per step-size trial is kept.  The layout decides how the team
 * groups its sums, so it can move the last bits of a result; pinning one
 * (blocks_per_sm > 0; tile_rows 512 or 256) makes results repeat exactly
 * across runs.  No counterpart in the reference, whose solve runs on one
 * thread. */
int32_t prima_set_solver_layout(prima_handle ctx, int32_t blocks_per_sm, int32_t tile_rows);

/* ---- memory (Kernels.scala:51-63) ---------------------------------------- */
/* Kernels.allocate: a zero-filled vector of length n. */
int32_t prima_vec_alloc(prima_handle ctx, int64_t n, prima_handle *vec);
/* Kernels.upload: copies host data (the caller may reuse `data` at once);
 * infinities survive the narrowing of a 32-bit context. */
int32_t prima_vec_upload(prima_handle ctx, const double *data, int64_t n, prima_handle *vec);
/* Kernels.download: writes vec into a caller-owned array of length n. */
int32_t prima_vec_download(prima_handle ctx, prima_handle vec, double *into, int64_t n);
/* Kernels.length */
int32_t prima_vec_length(prima_handle ctx, prima_handle vec, int64_t *n);
/* Releases one vector before close (no counterpart in the trait, whose
 * vectors live until close; offered for long-lived contexts). */
int32_t prima_vec_free(prima_handle ctx, prima_handle vec);
/* Kernels.uploadMatrix: canonical CSR (row_ptr[rows+1], col_idx/values[nnz]);
 * the backend chooses its device layout. */
int32_t prima_mat_upload_csr(prima_handle ctx, int32_t rows, int32_t cols, const int32_t *row_ptr,
                             const int32_t *col_idx, const double *values, prima_handle *mat);

/* ---- the eight numeric operations (Kernels.scala:70-123) ----------------- */
int32_t prima_spmv(prima_handle ctx, prima_handle mat, prima_handle x, prima_handle out);
/* out := alpha*x + beta*y; out may alias x or y (Kernels.scala:77) */
int32_t prima_axpby(prima_handle ctx, double alpha, prima_handle x, double beta, prima_handle y,
                    prima_handle out);
int32_t prima_scale(prima_handle ctx, double alpha, prima_handle x, prima_handle out);
int32_t prima_copy(prima_handle ctx, prima_handle src, prima_handle dst);
int32_t prima_dot(prima_handle ctx, prima_handle x, prima_handle y, double *out);
int32_t prima_squared_norm(prima_handle ctx, prima_handle x, double *out);
/* No counterpart in the reference.  prima_dot without a context and without
 * any allocation, for callers that own their device memory and must not see
 * a library cudaMalloc/cudaFree (cudaFree synchronises the device): *out :=
 * sum x[i]*y[i] accumulated in double, x and y arrays of n floats
 * (element_bits 32) or doubles (64), x, y and out device pointers on the
 * calling thread's current device, enqueued on `stream` (a cudaStream_t;
 * NULL is the default stream) and not waited for.  n at most 16,777,216;
 * larger n is rejected with PRIMA_ERR_INVALID_ARGUMENT.  The block partials
 * live in a fixed 16 KiB device array that every GPU loading the library
 * holds until exit; the first call on each device looks up its address and
 * should come before any stream capture.  The address is cached per CUDA
 * context: a device reset (cudaDeviceReset, a primary-context reset) moves
 * the array, and the first call after it looks the address up again.  x, y
 * and out are checked to be memory of the current device (or managed) before
 * anything is queued; a host pointer or another GPU's memory is refused with
 * PRIMA_ERR_INVALID_ARGUMENT.  Calls that overlap on the GPU race on that
 * array. */
int32_t prima_dot_no_alloc(const void *x, const void *y, int64_t n, int32_t element_bits, double *out,
                           void *stream);
/* out := clamp(x - tau*(cost - kty), lower, upper), two-comparison clamp */
int32_t prima_primal_step(prima_handle ctx, prima_handle x, prima_handle kty, prima_handle cost,
                          prima_handle lower, prima_handle upper, double tau, prima_handle out);
/* out := y + sigma*(rhs - kxbar); rows >= num_equalities clamped at 0 */
int32_t prima_dual_step(prima_handle ctx, prima_handle y, prima_handle kxbar, prima_handle rhs,
                        double sigma, int32_t num_equalities, prima_handle out);

/* ---- coarse entry points: the whole solve on the device ------------------ */

/* LpProblem in standard form (core/LpProblem.scala:22-104): minimise
 * c'x + offset s.t. Kx = q on the first num_equalities rows, Kx >= q on the
 * rest, lower <= x <= upper.  The matrix is canonical CSR, m x n. */
typedef struct {
  int32_t num_variables;   /* n */
  int32_t num_constraints; /* m */
  int32_t num_equalities;
  int32_t pad;
  const int32_t *row_ptr; /* m + 1 */
  const int32_t *col_idx; /* nnz */
  const double *values;   /* nnz */
  const double *objective;
  const double *rhs;
  const double *lower;
  const double *upper;
  double objective_offset;
} prima_lp;

/* PdhgParams (core/PdhgParams.scala:9-54) + ScalingParams (Scaling.scala:11-24) */
typedef struct {
  double eps_abs;
  double eps_rel;
  int32_t max_iterations;
  int32_t evaluation_frequency;
  double time_limit_ms; /* < 0: none */
  int32_t ruiz_iterations;
  int32_t apply_pock_chambolle;
  double pock_chambolle_alpha;
  double infeasibility_tolerance;
  double restart_sufficient_reduction;
  double restart_necessary_reduction;
  double restart_artificial_fraction;
  double primal_weight_smoothing;
} prima_params;

void prima_params_default(prima_params *p);

/* Pdhg.WarmStart (Pdhg.scala:72-105): a point in the caller's coordinates;
 * step_size / primal_weight NaN when not carried. */
typedef struct {
  const double *primal; /* n */
  const double *dual;   /* m */
  double step_size;
  double primal_weight;
} prima_warm_start;

/* LpSolution scalars (core/SolveResult.scala:33-65) plus device timing. */
typedef struct {
  int32_t status;
  int32_t iterations;
  int32_t restarts;
  int32_t device_error; /* PRIMA_OK, or PRIMA_ERR_TIMEOUT if a device wait gave up */
  int64_t solve_ms;     /* wall clock, setup included (solveTimeMillis) */
  double objective;     /* KktError.primalObjective */
  double dual_objective;
  double primal_residual;
  double dual_residual;
  double final_step_size;
  double final_primal_weight;
  double device_ms; /* time inside the solver kernels (CUDA events) */
  double setup_ms;  /* scaling, transpose and upload */
  int64_t trials;   /* step-size trials, accepted and rejected */
  double span_ms;   /* CUDA-event time from the call's first device work to its last */
  int32_t blocks;    /* blocks of the persistent kernel's team that ran the (last) pass */
  int32_t tile_rows; /* row cap of that pass's hot-phase tiles (the solver layout) */
} prima_solution_info;

/* Pdhg.solveWith(problem, params, this-context, cancelled, warmStart).
 * Runs in the context's precision.  warm_start and cancel may be NULL; cancel
 * is polled at evaluation points.  primal_out (n), dual_out (m) and
 * reduced_costs_out (n) may each be NULL. */
int32_t prima_pdhg_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                         const prima_warm_start *warm_start, const volatile int32_t *cancel,
                         double *primal_out, double *dual_out, double *reduced_costs_out,
                         prima_solution_info *info);

/* MixedPrecision.Params (MixedPrecision.scala:37-79) plus the device scheme. */
/* PRIMA_MIXED_TWO_PASS: the reference scheme -- FP32 pass, FP64 certificate
 * re-check, FP64 warm-started finish (both passes on the GPU).
 * PRIMA_MIXED_REFINEMENT: the same FP32 pass, then the finish also in FP32:
 * PDHG on the residual problem around an FP64 anchor (x*, y*) -- data
 * c - K'y*, q - Kx*, box [l - x*, u - x*], dual cone y >= -y* -- with the
 * anchor re-centred at every restart and the KKT test in FP64 on x* + x^. */
#define PRIMA_MIXED_TWO_PASS 0
#define PRIMA_MIXED_REFINEMENT 1
typedef struct {
  double reduced_tolerance;
  int32_t reduced_max_iterations;
  int32_t always_refine;
  double reduced_time_share;
  int32_t scheme;
  int32_t pad;
  double round_reduction; /* REFINEMENT: a fresh restart schedule (a new round) opens when
                             the weighted KKT error has fallen by this factor; 0: never */
} prima_mixed_params;

void prima_mixed_params_default(prima_mixed_params *p);

/* MixedPrecision.Result (MixedPrecision.scala:82-96) */
typedef struct {
  int32_t reduced_iterations;
  int32_t reduced_restarts;
  int64_t reduced_ms;
  int32_t refinement_iterations;
  int32_t refined;
  int64_t refinement_ms;
  int32_t refinement_rounds; /* REFINEMENT: rounds opened by round_reduction */
  int32_t pad;
} prima_mixed_info;

/* MixedPrecision.solve(problem, params, device, mixed, cancelled) with both
 * passes on the GPU.  The reported result is FP64-validated in every scheme. */
int32_t prima_mixed_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                          const prima_mixed_params *mixed, const volatile int32_t *cancel,
                          double *primal_out, double *dual_out, double *reduced_costs_out,
                          prima_solution_info *info, prima_mixed_info *mixed_info);

/* PrimaZio.solveAll's shape in one persistent launch: `count` independent
 * LPs, each solved as by prima_pdhg_solve (context precision).  Output arrays
 * are per instance; any pointer array (or entry) may be NULL. */
int32_t prima_pdhg_solve_batch(prima_handle ctx, int32_t count, const prima_lp *lps,
                               const prima_params *params, const volatile int32_t *cancel,
                               double *const *primal_out, double *const *dual_out,
                               double *const *reduced_costs_out, prima_solution_info *infos);

/* MixedPrecision.solve for `count` independent LPs, as by prima_mixed_solve,
 * with each pass run for all instances in one persistent launch: the reduced
 * FP32 pass, then the FP32 refinement finishes, then any FP64 finishes.
 * Output arrays are per instance; any pointer array (or entry) may be NULL. */
int32_t prima_mixed_solve_batch(prima_handle ctx, int32_t count, const prima_lp *lps, const prima_params *params,
                                const prima_mixed_params *mixed, const volatile int32_t *cancel,
                                double *const *primal_out, double *const *dual_out,
                                double *const *reduced_costs_out, prima_solution_info *infos,
                                prima_mixed_info *mixed_infos);

/* ---- device-resident problems ---------------------------------------------
 * A problem uploaded and equilibrated once, then solved any number of times
 * (warm-started passes, mixed-precision passes, repeated sweeps) without
 * re-uploading or re-scaling.  The equilibration follows the ScalingParams in
 * `params`; a solve whose params ask for a different scaling re-derives it.
 * No counterpart in the reference, where LpProblem is a host object; this is
 * the device residency the seam was designed for (Kernels.scala:33-37). */
int32_t prima_problem_create(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                             prima_handle *problem);
int32_t prima_problem_free(prima_handle ctx, prima_handle problem);
/* Replaces the resident problem's variable bounds (n each; lower <= upper,
 * infinities allowed), keeping its upload and equilibration: a
 * branch-and-bound node is its parent's LP with one bound moved
 * (BranchAndBound.scala:264-276, the node's LpProblem with new
 * variableLower/variableUpper). */
int32_t prima_problem_set_bounds(prima_handle ctx, prima_handle problem, const double *lower, const double *upper);
/* Scaling.apply's result for the resident problem (Scaling.scala:77-155), as
 * the device computed it: the equilibrated matrix values in the caller's CSR
 * order (nnz), the equilibrated objective, bounds (n) and right-hand side (m),
 * and the cumulative row and column scales that undo it.  Any output may be
 * NULL.  No counterpart in the reference (its ScaledProblem is a host
 * object); offered so a caller can inspect or verify the scaling. */
int32_t prima_problem_scaled(prima_handle ctx, prima_handle problem, double *values, double *objective,
                             double *rhs, double *lower, double *upper, double *row_scale, double *col_scale);
/* As prima_pdhg_solve / prima_mixed_solve on a resident problem. */
int32_t prima_problem_solve(prima_handle ctx, prima_handle problem, const prima_params *params,
                            const prima_warm_start *warm_start, const volatile int32_t *cancel,
                            double *primal_out, double *dual_out, double *reduced_costs_out,
                            prima_solution_info *info);
int32_t prima_problem_mixed_solve(prima_handle ctx, prima_handle problem, const prima_params *params,
                                  const prima_mixed_params *mixed, const volatile int32_t *cancel,
                                  double *primal_out, double *dual_out, double *reduced_costs_out,
                                  prima_solution_info *info, prima_mixed_info *mixed_info);

#ifdef __cplusplus
}
#endif
#endif
