/*
 * CPU restatement of Prima's restarted-PDHG path (oluies/noaidi, module
 * prima-core).  TEST INFRASTRUCTURE ONLY: this library is the parity oracle
 * for libprima_cuda.so and the timed CPU baseline.  Nothing in the product
 * links it.
 *
 * Scope of the restatement (reference file:line for each piece is given at the
 * function definitions in prima_oracle.c):
 *   SparseMatrix  canonical CSR, transpose, norms, spectral bound
 *   Scaling       Ruiz x N + Pock-Chambolle
 *   Kernels       ScalaKernels (fp64) and Float32Kernels (fp32-rounded)
 *   Kkt           evaluate / convergence / weighted
 *   Certificates  primal/dual infeasibility, classify
 *   Pdhg.Solve    initialise / step / accumulate / checkpoint / restartAt / finish
 *   MixedPrecision.solve
 *
 * Build with -O2 -ffp-contract=off (the JVM never fuses a*b+c).
 */
#ifndef PRIMA_ORACLE_H
#define PRIMA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* SolveStatus ordinal order (SolveResult.scala:9-18). */
enum {
  ORC_OPTIMAL = 0,
  ORC_PRIMAL_INFEASIBLE = 1,
  ORC_DUAL_INFEASIBLE = 2,
  ORC_ITERATION_LIMIT = 3,
  ORC_TIME_LIMIT = 4,
  ORC_NUMERICAL_ERROR = 5,
  ORC_INTERRUPTED = 6
};

/* PdhgParams.scala:9-54 plus ScalingParams (Scaling.scala:11-24). */
typedef struct {
  double eps_abs;
  double eps_rel;
  int32_t max_iterations;
  int32_t evaluation_frequency;
  double time_limit_ms; /* < 0: no limit */
  int32_t ruiz_iterations;
  int32_t apply_pock_chambolle;
  double pock_chambolle_alpha;
  double infeasibility_tolerance;
  double restart_sufficient_reduction;
  double restart_necessary_reduction;
  double restart_artificial_fraction;
  double primal_weight_smoothing;
} orc_params;

typedef struct {
  int32_t status;
  int32_t iterations;
  int32_t restarts;
  int32_t pad;
  int64_t solve_ms;
  double objective;      /* KktError.primalObjective */
  double dual_objective; /* KktError.dualObjective */
  double primal_residual;
  double dual_residual;
  double final_step_size;
  double final_primal_weight;
} orc_result;

/* MixedPrecision.Params (MixedPrecision.scala:37-79). */
typedef struct {
  double reduced_tolerance;
  int32_t reduced_max_iterations;
  int32_t always_refine;
  double reduced_time_share;
} orc_mixed_params;

typedef struct {
  int32_t reduced_iterations;
  int32_t reduced_restarts;
  int64_t reduced_ms;
  int32_t refinement_iterations;
  int32_t refined;
  int64_t refinement_ms;
} orc_mixed_info;

void orc_default_params(orc_params *p);
void orc_default_mixed_params(orc_mixed_params *p);

/* ---- SparseMatrix ---------------------------------------------------- */
/* Canonicalise triplets: stable sort by (row, col), sum duplicates, drop exact
 * zeros.  Output arrays must hold nnz_in entries (rowptr: rows + 1).
 * Returns the canonical nnz, or -1 on a bad index / non-finite value. */
int64_t orc_csr_from_triplets(int32_t rows, int32_t cols, int64_t nnz_in,
                              const int32_t *ri, const int32_t *ci, const double *vi,
                              int32_t *rowptr, int32_t *colidx, double *vals);
void orc_csr_transpose(int32_t rows, int32_t cols, const int32_t *rowptr,
                       const int32_t *colidx, const double *vals,
                       int32_t *t_rowptr, int32_t *t_colidx, double *t_vals);
void orc_csr_multiply(int32_t rows, const int32_t *rowptr, const int32_t *colidx,
                      const double *vals, const double *x, double *out);
double orc_csr_norm_inf(int32_t rows, const int32_t *rowptr, const double *vals);
double orc_csr_spectral_norm_bound(int32_t rows, int32_t cols, const int32_t *rowptr,
                                   const int32_t *colidx, const double *vals);

/* ---- Scaling --------------------------------------------------------- */
/* Writes the scaled problem and cumulative diagonals. */
void orc_scale(int32_t n, int32_t m, const int32_t *rowptr, const int32_t *colidx,
               const double *vals, const double *c, const double *q, const double *l,
               const double *u, int32_t ruiz_iterations, int32_t apply_pc, double pc_alpha,
               double *s_vals, double *s_c, double *s_q, double *s_l, double *s_u,
               double *row_scale, double *col_scale);

/* ---- Kernels (mode 0 = ScalaKernels fp64, mode 1 = Float32Kernels) ---- */
void orc_k_upload(int mode, int64_t n, const double *in, double *out);
void orc_k_spmv(int mode, int32_t rows, const int32_t *rowptr, const int32_t *colidx,
                const double *vals, const double *x, double *out);
void orc_k_axpby(int mode, int64_t n, double alpha, const double *x, double beta,
                 const double *y, double *out);
void orc_k_scale(int mode, int64_t n, double alpha, const double *x, double *out);
double orc_k_dot(int mode, int64_t n, const double *x, const double *y);
double orc_k_squared_norm(int mode, int64_t n, const double *x);
void orc_k_primal_step(int mode, int64_t n, const double *x, const double *kty,
                       const double *c, const double *l, const double *u, double tau,
                       double *out);
void orc_k_dual_step(int mode, int64_t m, const double *y, const double *kxbar,
                     const double *q, double sigma, int32_t neq, double *out);

/* ---- Kkt / Certificates (original-problem units) ---------------------- */
/* out = {primalResidualNorm, dualResidualNorm, primalObjective, dualObjective}.
 * kx / kty may be NULL (recomputed from the matrix). */
void orc_kkt_evaluate(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                      const int32_t *colidx, const double *vals, const double *c,
                      const double *q, const double *l, const double *u, double offset,
                      const double *x, const double *y, const double *kx,
                      const double *kty, double out[4]);
/* Returns 1 and writes *out when the direction is a candidate, else 0. */
int orc_primal_infeasibility(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                             const int32_t *colidx, const double *vals, const double *q,
                             const double *l, const double *u, const double *y,
                             const double *kty, double *out);
int orc_dual_infeasibility(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                           const int32_t *colidx, const double *vals, const double *c,
                           const double *l, const double *u, const double *d,
                           const double *kd, double *out);
/* Returns -1 for None, else the SolveStatus ordinal. */
int orc_classify(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                 const int32_t *colidx, const double *vals, const double *c,
                 const double *q, const double *l, const double *u, const double *x,
                 const double *y, double tolerance, const double *kx, const double *kty);

/* ---- Pdhg.solveWith ---------------------------------------------------- */
/* warm_x / warm_y may be NULL (cold start).  warm_step / warm_weight: NaN or
 * <= 0 means "not carried".  cancel may be NULL.  Returns 0, or -1 on an
 * invalid argument (mirrors the reference's `require` failures). */
int orc_pdhg_solve(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                   const int32_t *colidx, const double *vals, const double *c,
                   const double *q, const double *l, const double *u, double offset,
                   const orc_params *params, int mode, const double *warm_x,
                   const double *warm_y, double warm_step, double warm_weight,
                   const volatile int32_t *cancel, double *x_out, double *y_out,
                   double *rc_out, orc_result *res);

/* ---- MixedPrecision.solve (device = Float32Kernels) -------------------- */
int orc_mixed_solve(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                    const int32_t *colidx, const double *vals, const double *c,
                    const double *q, const double *l, const double *u, double offset,
                    const orc_params *params, const orc_mixed_params *mixed,
                    const volatile int32_t *cancel, double *x_out, double *y_out,
                    double *rc_out, orc_result *res, orc_mixed_info *info);

#ifdef __cplusplus
}
#endif
#endif
