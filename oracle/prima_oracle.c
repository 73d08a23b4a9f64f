/*
 * CPU restatement of Prima's restarted-PDHG path.  TEST INFRASTRUCTURE ONLY:
 * the parity oracle for libprima_cuda.so and the timed CPU baseline.
 *
 * Every function follows one reference function and cites it (paths are
 * relative to the oluies/noaidi repository; "core/" abbreviates
 * modules/prima-core/src/main/scala/org/noaidi/prima/).  Arithmetic keeps the
 * reference's operation order: index-order sums, no fused multiply-add
 * (compiled with -ffp-contract=off), clamps written as two comparisons.
 *
 * mode 0 restates core/kernels/ScalaKernels.scala (IEEE double throughout);
 * mode 1 restates core/kernels/Float32Kernels.scala (every kernel result
 * rounded to binary32, float32 sequential reductions, infinities preserved on
 * upload).  Everything above the kernel seam (Kkt, Certificates, restarts) is
 * double in both modes, as in the reference.
 */
#include "prima_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* defaults: core/PdhgParams.scala:9-54, core/Scaling.scala:11-24           */
/* ------------------------------------------------------------------------ */

void orc_default_params(orc_params *p) {
  p->eps_abs = 1e-8;
  p->eps_rel = 1e-8;
  p->max_iterations = 100000;
  p->evaluation_frequency = 64;
  p->time_limit_ms = -1.0;
  p->ruiz_iterations = 10;
  p->apply_pock_chambolle = 1;
  p->pock_chambolle_alpha = 1.0;
  p->infeasibility_tolerance = 1e-8;
  p->restart_sufficient_reduction = 0.2;
  p->restart_necessary_reduction = 0.8;
  p->restart_artificial_fraction = 0.36;
  p->primal_weight_smoothing = 0.5;
}

/* core/MixedPrecision.scala:37-79 */
void orc_default_mixed_params(orc_mixed_params *p) {
  p->reduced_tolerance = 1e-5;
  p->reduced_max_iterations = 20000;
  p->always_refine = 0;
  p->reduced_time_share = 0.5;
}

/* core/PdhgParams.scala:55-79 (the `require` block) */
static int params_valid(const orc_params *p) {
  if (!(p->eps_abs >= 0.0) || !(p->eps_rel >= 0.0)) return 0;
  if (p->max_iterations <= 0 || p->evaluation_frequency <= 0) return 0;
  if (!(p->primal_weight_smoothing >= 0.0 && p->primal_weight_smoothing <= 1.0)) return 0;
  if (!(p->restart_sufficient_reduction > 0.0 &&
        p->restart_sufficient_reduction <= p->restart_necessary_reduction))
    return 0;
  if (!(p->restart_artificial_fraction > 0.0 && p->restart_artificial_fraction <= 1.0)) return 0;
  if (!(p->infeasibility_tolerance >= 0.0)) return 0;
  if (p->ruiz_iterations < 0) return 0;
  if (!(p->pock_chambolle_alpha >= 0.0 && p->pock_chambolle_alpha <= 2.0)) return 0;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* SparseMatrix: core/SparseMatrix.scala                                    */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t rows, cols;
  int32_t *rowptr;
  int32_t *colidx;
  double *vals;
} csr;

static void csr_free(csr *a) {
  free(a->rowptr);
  free(a->colidx);
  free(a->vals);
  a->rowptr = NULL;
  a->colidx = NULL;
  a->vals = NULL;
}

static csr csr_alloc(int32_t rows, int32_t cols, int64_t nnz) {
  csr a;
  a.rows = rows;
  a.cols = cols;
  a.rowptr = (int32_t *)calloc((size_t)rows + 1, sizeof(int32_t));
  a.colidx = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
  a.vals = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
  return a;
}

static int64_t csr_nnz(const csr *a) { return a->rowptr[a->rows]; }

/* Stable merge sort of triplet indices by (row, col): the reference sorts with
 * java.util.Arrays.sort on objects, a stable TimSort (SparseMatrix.scala:216-222),
 * so duplicates are summed in their order of appearance. */
static void merge_sort_idx(int64_t *idx, int64_t *tmp, int64_t lo, int64_t hi,
                           const int32_t *ri, const int32_t *ci) {
  if (hi - lo < 2) return;
  int64_t mid = lo + (hi - lo) / 2;
  merge_sort_idx(idx, tmp, lo, mid, ri, ci);
  merge_sort_idx(idx, tmp, mid, hi, ri, ci);
  int64_t a = lo, b = mid, k = lo;
  while (a < mid && b < hi) {
    int64_t ia = idx[a], ib = idx[b];
    int take_b = (ri[ib] < ri[ia]) || (ri[ib] == ri[ia] && ci[ib] < ci[ia]);
    tmp[k++] = take_b ? idx[b++] : idx[a++];
  }
  while (a < mid) tmp[k++] = idx[a++];
  while (b < hi) tmp[k++] = idx[b++];
  memcpy(idx + lo, tmp + lo, (size_t)(hi - lo) * sizeof(int64_t));
}

/* SparseMatrix.fromTriplets, SparseMatrix.scala:204-260 */
int64_t orc_csr_from_triplets(int32_t rows, int32_t cols, int64_t nnz_in,
                              const int32_t *ri, const int32_t *ci, const double *vi,
                              int32_t *rowptr, int32_t *colidx, double *vals) {
  if (rows < 0 || cols < 0) return -1;
  for (int64_t k = 0; k < nnz_in; k++) {
    if (ri[k] < 0 || ri[k] >= rows || ci[k] < 0 || ci[k] >= cols) return -1;
    if (!isfinite(vi[k])) return -1;
  }
  int64_t *idx = (int64_t *)malloc((size_t)(nnz_in > 0 ? nnz_in : 1) * sizeof(int64_t));
  int64_t *tmp = (int64_t *)malloc((size_t)(nnz_in > 0 ? nnz_in : 1) * sizeof(int64_t));
  for (int64_t k = 0; k < nnz_in; k++) idx[k] = k;
  merge_sort_idx(idx, tmp, 0, nnz_in, ri, ci);
  int32_t *mrow = (int32_t *)malloc((size_t)(nnz_in > 0 ? nnz_in : 1) * sizeof(int32_t));
  int64_t m = 0, i = 0;
  while (i < nnz_in) {
    int64_t k0 = idx[i];
    int32_t r = ri[k0], c = ci[k0];
    double v = vi[k0];
    int64_t j = i + 1;
    while (j < nnz_in && ri[idx[j]] == r && ci[idx[j]] == c) {
      v += vi[idx[j]];
      j++;
    }
    if (v != 0.0) {
      mrow[m] = r;
      colidx[m] = c;
      vals[m] = v;
      m++;
    }
    i = j;
  }
  memset(rowptr, 0, ((size_t)rows + 1) * sizeof(int32_t));
  for (int64_t k = 0; k < m; k++) rowptr[mrow[k] + 1] += 1;
  for (int32_t r = 0; r < rows; r++) rowptr[r + 1] += rowptr[r];
  free(idx);
  free(tmp);
  free(mrow);
  return m;
}

/* SparseMatrix.transpose, SparseMatrix.scala:36-64 (counting sort by column,
 * rows visited in order, so every transposed row is column-sorted). */
void orc_csr_transpose(int32_t rows, int32_t cols, const int32_t *rowptr,
                       const int32_t *colidx, const double *vals,
                       int32_t *t_rowptr, int32_t *t_colidx, double *t_vals) {
  int64_t nnz = rowptr[rows];
  memset(t_rowptr, 0, ((size_t)cols + 1) * sizeof(int32_t));
  for (int64_t k = 0; k < nnz; k++) t_rowptr[colidx[k] + 1] += 1;
  for (int32_t c = 0; c < cols; c++) t_rowptr[c + 1] += t_rowptr[c];
  int32_t *cursor = (int32_t *)malloc(((size_t)cols + 1) * sizeof(int32_t));
  memcpy(cursor, t_rowptr, (size_t)cols * sizeof(int32_t));
  for (int32_t r = 0; r < rows; r++) {
    for (int32_t p = rowptr[r]; p < rowptr[r + 1]; p++) {
      int32_t col = colidx[p];
      int32_t dest = cursor[col];
      t_colidx[dest] = r;
      t_vals[dest] = vals[p];
      cursor[col] = dest + 1;
    }
  }
  free(cursor);
}

static csr csr_transpose(const csr *a) {
  csr t = csr_alloc(a->cols, a->rows, csr_nnz(a));
  orc_csr_transpose(a->rows, a->cols, a->rowptr, a->colidx, a->vals, t.rowptr, t.colidx,
                    t.vals);
  return t;
}

/* SparseMatrix.multiplyInto, SparseMatrix.scala:76-86 */
void orc_csr_multiply(int32_t rows, const int32_t *rowptr, const int32_t *colidx,
                      const double *vals, const double *x, double *out) {
  for (int32_t r = 0; r < rows; r++) {
    double acc = 0.0;
    for (int32_t p = rowptr[r]; p < rowptr[r + 1]; p++) acc += vals[p] * x[colidx[p]];
    out[r] = acc;
  }
}

/* SparseMatrix.rowMaxAbs, SparseMatrix.scala:95-103 */
static double row_max_abs(const csr *a, int32_t r) {
  double m = 0.0;
  for (int32_t p = a->rowptr[r]; p < a->rowptr[r + 1]; p++) {
    double v = fabs(a->vals[p]);
    if (v > m) m = v;
  }
  return m;
}

/* SparseMatrix.rowAbsPowSum, SparseMatrix.scala:106-113 */
static double row_abs_pow_sum(const csr *a, int32_t r, double alpha) {
  double s = 0.0;
  for (int32_t p = a->rowptr[r]; p < a->rowptr[r + 1]; p++) s += pow(fabs(a->vals[p]), alpha);
  return s;
}

/* SparseMatrix.scaledBy, SparseMatrix.scala:116-128: v * rs * cs, left to right. */
static void scaled_by_inplace(csr *a, const double *rs, const double *cs) {
  for (int32_t r = 0; r < a->rows; r++) {
    double f = rs[r];
    for (int32_t p = a->rowptr[r]; p < a->rowptr[r + 1]; p++)
      a->vals[p] = a->vals[p] * f * cs[a->colidx[p]];
  }
}

/* SparseMatrix.normInf, SparseMatrix.scala:144-156 */
double orc_csr_norm_inf(int32_t rows, const int32_t *rowptr, const double *vals) {
  double m = 0.0;
  for (int32_t r = 0; r < rows; r++) {
    double s = 0.0;
    for (int32_t p = rowptr[r]; p < rowptr[r + 1]; p++) s += fabs(vals[p]);
    if (s > m) m = s;
  }
  return m;
}

/* SparseMatrix.spectralNormBound = sqrt(norm1 * normInf), SparseMatrix.scala:141,181 */
double orc_csr_spectral_norm_bound(int32_t rows, int32_t cols, const int32_t *rowptr,
                                   const int32_t *colidx, const double *vals) {
  int64_t nnz = rowptr[rows];
  int32_t *tr = (int32_t *)malloc(((size_t)cols + 1) * sizeof(int32_t));
  int32_t *tc = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
  double *tv = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
  orc_csr_transpose(rows, cols, rowptr, colidx, vals, tr, tc, tv);
  double norm1 = orc_csr_norm_inf(cols, tr, tv);
  double norminf = orc_csr_norm_inf(rows, rowptr, vals);
  free(tr);
  free(tc);
  free(tv);
  return sqrt(norm1 * norminf);
}

/* ------------------------------------------------------------------------ */
/* Scaling.apply: core/Scaling.scala:77-155                                 */
/* ------------------------------------------------------------------------ */

void orc_scale(int32_t n, int32_t m, const int32_t *rowptr, const int32_t *colidx,
               const double *vals, const double *c, const double *q, const double *l,
               const double *u, int32_t ruiz_iterations, int32_t apply_pc, double pc_alpha,
               double *s_vals, double *s_c, double *s_q, double *s_l, double *s_u,
               double *row_scale, double *col_scale) {
  int64_t nnz = rowptr[m];
  csr a;
  a.rows = m;
  a.cols = n;
  a.rowptr = (int32_t *)rowptr;
  a.colidx = (int32_t *)colidx;
  a.vals = s_vals;
  memcpy(s_vals, vals, (size_t)nnz * sizeof(double));
  double *rf = (double *)calloc((size_t)m + 1, sizeof(double));
  double *cf = (double *)calloc((size_t)n + 1, sizeof(double));
  for (int32_t r = 0; r < m; r++) row_scale[r] = 1.0;
  for (int32_t i = 0; i < n; i++) col_scale[i] = 1.0;

  for (int32_t it = 0; it < ruiz_iterations; it++) {
    for (int32_t r = 0; r < m; r++) {
      double norm = row_max_abs(&a, r);
      rf[r] = norm > 0.0 ? 1.0 / sqrt(norm) : 1.0;
    }
    csr t = csr_transpose(&a);
    for (int32_t j = 0; j < n; j++) {
      double norm = row_max_abs(&t, j);
      cf[j] = norm > 0.0 ? 1.0 / sqrt(norm) : 1.0;
    }
    csr_free(&t);
    scaled_by_inplace(&a, rf, cf);
    for (int32_t r = 0; r < m; r++) row_scale[r] *= rf[r];
    for (int32_t j = 0; j < n; j++) col_scale[j] *= cf[j];
  }
  if (apply_pc) {
    for (int32_t r = 0; r < m; r++) {
      double s = row_abs_pow_sum(&a, r, 2.0 - pc_alpha);
      rf[r] = s > 0.0 ? 1.0 / sqrt(s) : 1.0;
    }
    csr t = csr_transpose(&a);
    for (int32_t j = 0; j < n; j++) {
      double s = row_abs_pow_sum(&t, j, pc_alpha);
      cf[j] = s > 0.0 ? 1.0 / sqrt(s) : 1.0;
    }
    csr_free(&t);
    scaled_by_inplace(&a, rf, cf);
    for (int32_t r = 0; r < m; r++) row_scale[r] *= rf[r];
    for (int32_t j = 0; j < n; j++) col_scale[j] *= cf[j];
  }
  for (int32_t j = 0; j < n; j++) {
    double d = col_scale[j];
    s_c[j] = c[j] * d;
    s_l[j] = l[j] / d;
    s_u[j] = u[j] / d;
  }
  for (int32_t r = 0; r < m; r++) s_q[r] = q[r] * row_scale[r];
  free(rf);
  free(cf);
}

/* ------------------------------------------------------------------------ */
/* Kernels: core/kernels/ScalaKernels.scala:19-120 (mode 0) and             */
/*          core/kernels/Float32Kernels.scala:28-155 (mode 1)               */
/* ------------------------------------------------------------------------ */

static inline double r32(double v) { return (double)(float)v; }

/* ScalaKernels.upload :29 (clone) / Float32Kernels.upload :43-52 */
void orc_k_upload(int mode, int64_t n, const double *in, double *out) {
  for (int64_t i = 0; i < n; i++) {
    if (mode == 0) out[i] = in[i];
    else out[i] = isinf(in[i]) ? in[i] : r32(in[i]);
  }
}

/* ScalaKernels.spmv :40-41 -> multiplyInto; Float32Kernels.spmv :70-80 */
void orc_k_spmv(int mode, int32_t rows, const int32_t *rowptr, const int32_t *colidx,
                const double *vals, const double *x, double *out) {
  if (mode == 0) {
    orc_csr_multiply(rows, rowptr, colidx, vals, x, out);
    return;
  }
  for (int32_t r = 0; r < rows; r++) {
    float acc = 0.0f;
    for (int32_t p = rowptr[r]; p < rowptr[r + 1]; p++)
      acc = acc + ((float)vals[p] * (float)x[colidx[p]]);
    out[r] = (double)acc;
  }
}

/* ScalaKernels.axpby :43-48; Float32Kernels.axpby :82-88 */
void orc_k_axpby(int mode, int64_t n, double alpha, const double *x, double beta,
                 const double *y, double *out) {
  if (mode == 0) {
    for (int64_t i = 0; i < n; i++) out[i] = alpha * x[i] + beta * y[i];
    return;
  }
  float a = (float)alpha, b = (float)beta;
  for (int64_t i = 0; i < n; i++) out[i] = (double)((a * (float)x[i]) + (b * (float)y[i]));
}

/* ScalaKernels.scale :50-55; Float32Kernels.scale :90-95 */
void orc_k_scale(int mode, int64_t n, double alpha, const double *x, double *out) {
  if (mode == 0) {
    for (int64_t i = 0; i < n; i++) out[i] = alpha * x[i];
    return;
  }
  float a = (float)alpha;
  for (int64_t i = 0; i < n; i++) out[i] = (double)(a * (float)x[i]);
}

/* ScalaKernels.dot :60-67; Float32Kernels.dot :100-106 */
double orc_k_dot(int mode, int64_t n, const double *x, const double *y) {
  if (mode == 0) {
    double s = 0.0;
    for (int64_t i = 0; i < n; i++) s += x[i] * y[i];
    return s;
  }
  float s = 0.0f;
  for (int64_t i = 0; i < n; i++) s = s + ((float)x[i] * (float)y[i]);
  return (double)s;
}

/* ScalaKernels.squaredNorm :69-76; Float32Kernels.squaredNorm :108-115 */
double orc_k_squared_norm(int mode, int64_t n, const double *x) {
  if (mode == 0) {
    double s = 0.0;
    for (int64_t i = 0; i < n; i++) s += x[i] * x[i];
    return s;
  }
  float s = 0.0f;
  for (int64_t i = 0; i < n; i++) {
    float v = (float)x[i];
    s = s + (v * v);
  }
  return (double)s;
}

/* ScalaKernels.primalStep :78-98; Float32Kernels.primalStep :117-134.  The
 * clamp is two comparisons so infinite bounds pass the candidate through. */
void orc_k_primal_step(int mode, int64_t n, const double *x, const double *kty,
                       const double *c, const double *l, const double *u, double tau,
                       double *out) {
  float t = (float)tau;
  for (int64_t i = 0; i < n; i++) {
    double step;
    if (mode == 0) step = x[i] - tau * (c[i] - kty[i]);
    else step = (double)((float)x[i] - (t * ((float)c[i] - (float)kty[i])));
    out[i] = step < l[i] ? l[i] : (step > u[i] ? u[i] : step);
  }
}

/* ScalaKernels.dualStep :100-118; Float32Kernels.dualStep :136-153 */
void orc_k_dual_step(int mode, int64_t m, const double *y, const double *kxbar,
                     const double *q, double sigma, int32_t neq, double *out) {
  float s = (float)sigma;
  for (int64_t i = 0; i < m; i++) {
    double step;
    if (mode == 0) step = y[i] + sigma * (q[i] - kxbar[i]);
    else step = (double)((float)y[i] + (s * ((float)q[i] - (float)kxbar[i])));
    if (i < neq) out[i] = step;
    else out[i] = step > 0.0 ? step : 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* Kkt: core/Kkt.scala                                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
  double pres, dres, pobj, dobj;
} kkt_t;

static int kkt_finite(kkt_t e) {
  return isfinite(e.pres) && isfinite(e.dres) && isfinite(e.pobj) && isfinite(e.dobj);
}

/* KktError.weighted, Kkt.scala:28-33 */
static double kkt_weighted(kkt_t e, double w) {
  double gap = e.pobj - e.dobj;
  return sqrt(w * e.pres * e.pres + (e.dres * e.dres) / w + gap * gap);
}

/* Kkt.norm2, Kkt.scala:181-187 */
static double norm2(const double *a, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; i++) s += a[i] * a[i];
  return sqrt(s);
}

/* Kkt.evaluate, Kkt.scala:68-125 with primalResidualSquared :164-179 */
static kkt_t kkt_evaluate(int32_t n, int32_t m, int32_t neq, const double *c, const double *q,
                          const double *l, const double *u, double offset, const double *x,
                          const double *y, const double *ax, const double *aty) {
  double psq = 0.0;
  int32_t i = 0;
  for (; i < neq; i++) {
    double r = ax[i] - q[i];
    psq += r * r;
  }
  for (; i < m; i++) {
    double sf = q[i] - ax[i];
    if (sf > 0.0) psq += sf * sf;
  }
  double pobj = offset;
  for (i = 0; i < n; i++) pobj += c[i] * x[i];
  double dobj = offset;
  for (i = 0; i < m; i++) dobj += q[i] * y[i];
  double dsq = 0.0;
  for (i = 0; i < n; i++) {
    double rc = c[i] - aty[i];
    if (rc > 0.0) {
      if (isinf(l[i]) && l[i] < 0) dsq += rc * rc;
      else dobj += l[i] * rc;
    } else if (rc < 0.0) {
      if (isinf(u[i]) && u[i] > 0) dsq += rc * rc;
      else dobj += u[i] * rc;
    }
  }
  kkt_t e = {sqrt(psq), sqrt(dsq), pobj, dobj};
  return e;
}

void orc_kkt_evaluate(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                      const int32_t *colidx, const double *vals, const double *c,
                      const double *q, const double *l, const double *u, double offset,
                      const double *x, const double *y, const double *kx,
                      const double *kty, double out[4]) {
  double *ax = NULL, *aty = NULL;
  if (!kx) {
    ax = (double *)malloc(((size_t)m + 1) * sizeof(double));
    orc_csr_multiply(m, rowptr, colidx, vals, x, ax);
    kx = ax;
  }
  if (!kty) {
    int64_t nnz = rowptr[m];
    int32_t *tr = (int32_t *)malloc(((size_t)n + 1) * sizeof(int32_t));
    int32_t *tc = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
    double *tv = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
    orc_csr_transpose(m, n, rowptr, colidx, vals, tr, tc, tv);
    aty = (double *)malloc(((size_t)n + 1) * sizeof(double));
    orc_csr_multiply(n, tr, tc, tv, y, aty);
    free(tr);
    free(tc);
    free(tv);
    kty = aty;
  }
  kkt_t e = kkt_evaluate(n, m, neq, c, q, l, u, offset, x, y, kx, kty);
  out[0] = e.pres;
  out[1] = e.dres;
  out[2] = e.pobj;
  out[3] = e.dobj;
  free(ax);
  free(aty);
}

/* Kkt.convergence, Kkt.scala:130-143 and Convergence.converged :46 */
static int kkt_converged(kkt_t e, double rhs_norm, double obj_norm, double eps_abs,
                         double eps_rel) {
  double ptol = eps_abs + eps_rel * rhs_norm;
  double dtol = eps_abs + eps_rel * obj_norm;
  double gtol = eps_abs + eps_rel * (fabs(e.pobj) + fabs(e.dobj));
  return kkt_finite(e) && e.pres <= ptol && e.dres <= dtol && fabs(e.pobj - e.dobj) <= gtol;
}

/* ------------------------------------------------------------------------ */
/* Certificates: core/Certificates.scala                                    */
/* ------------------------------------------------------------------------ */

/* Certificates.primalInfeasibility, Certificates.scala:60-123.
 * matrix_norm is the original matrix's spectralNormBound. */
static int primal_infeas(int32_t n, int32_t m, int32_t neq, const double *q, const double *l,
                         const double *u, const double *y, const double *aty,
                         double matrix_norm, double *out) {
  double nsq = 0.0;
  for (int32_t i = 0; i < m; i++) nsq += y[i] * y[i];
  if (nsq <= 0.0 || !isfinite(nsq)) return 0;
  double norm = sqrt(nsq);
  double value = 0.0;
  for (int32_t i = 0; i < m; i++) value += q[i] * y[i];
  double rsq = 0.0;
  for (int32_t i = 0; i < n; i++) {
    double rc = -aty[i];
    if (rc > 0.0) {
      if (isinf(l[i]) && l[i] < 0) rsq += rc * rc;
      else value += l[i] * rc;
    } else if (rc < 0.0) {
      if (isinf(u[i]) && u[i] > 0) rsq += rc * rc;
      else value += u[i] * rc;
    }
  }
  double csq = 0.0;
  for (int32_t i = neq; i < m; i++)
    if (y[i] < 0.0) csq += y[i] * y[i];
  if (!(value > 0.0) || !isfinite(value)) return 0;
  double reduced_term = matrix_norm > 0.0 ? sqrt(rsq) / (matrix_norm * norm) : 0.0;
  double cone_term = sqrt(csq) / norm;
  double h = hypot(reduced_term, cone_term);
  if (!isfinite(h)) return 0;
  *out = h;
  return 1;
}

/* Certificates.dualInfeasibility, Certificates.scala:137-195 */
static int dual_infeas(int32_t n, int32_t m, int32_t neq, const double *c, const double *l,
                       const double *u, const double *d, const double *kd,
                       double matrix_norm, double *out) {
  double nsq = 0.0;
  for (int32_t i = 0; i < n; i++) nsq += d[i] * d[i];
  if (nsq <= 0.0 || !isfinite(nsq)) return 0;
  double norm = sqrt(nsq);
  double value = 0.0;
  for (int32_t i = 0; i < n; i++) value += c[i] * d[i];
  if (!(value < 0.0) || !isfinite(value)) return 0;
  double rowsq = 0.0;
  int32_t i = 0;
  for (; i < neq; i++) rowsq += kd[i] * kd[i];
  for (; i < m; i++)
    if (kd[i] < 0.0) rowsq += kd[i] * kd[i];
  double bsq = 0.0;
  for (i = 0; i < n; i++) {
    double di = d[i];
    if (di > 0.0 && !(isinf(u[i]) && u[i] > 0)) bsq += di * di;
    else if (di < 0.0 && !(isinf(l[i]) && l[i] < 0)) bsq += di * di;
  }
  double row_term = matrix_norm > 0.0 ? sqrt(rowsq) / (matrix_norm * norm) : 0.0;
  double bound_term = sqrt(bsq) / norm;
  double h = hypot(row_term, bound_term);
  if (!isfinite(h)) return 0;
  *out = h;
  return 1;
}

typedef struct {
  int32_t n, m, neq;
  const int32_t *rowptr, *colidx;
  const double *vals;
  int32_t *t_rowptr, *t_colidx;
  double *t_vals;
} orig_matrix;

static void orig_matrix_init(orig_matrix *om, int32_t n, int32_t m, int32_t neq,
                             const int32_t *rowptr, const int32_t *colidx, const double *vals) {
  int64_t nnz = rowptr[m];
  om->n = n;
  om->m = m;
  om->neq = neq;
  om->rowptr = rowptr;
  om->colidx = colidx;
  om->vals = vals;
  om->t_rowptr = (int32_t *)malloc(((size_t)n + 1) * sizeof(int32_t));
  om->t_colidx = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
  om->t_vals = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
  orc_csr_transpose(m, n, rowptr, colidx, vals, om->t_rowptr, om->t_colidx, om->t_vals);
}

static void orig_matrix_free(orig_matrix *om) {
  free(om->t_rowptr);
  free(om->t_colidx);
  free(om->t_vals);
}

int orc_primal_infeasibility(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                             const int32_t *colidx, const double *vals, const double *q,
                             const double *l, const double *u, const double *y,
                             const double *kty, double *out) {
  orig_matrix om;
  orig_matrix_init(&om, n, m, neq, rowptr, colidx, vals);
  double *aty = NULL;
  if (!kty) {
    aty = (double *)malloc(((size_t)n + 1) * sizeof(double));
    orc_csr_multiply(n, om.t_rowptr, om.t_colidx, om.t_vals, y, aty);
    kty = aty;
  }
  double norm = orc_csr_spectral_norm_bound(m, n, rowptr, colidx, vals);
  int ok = primal_infeas(n, m, neq, q, l, u, y, kty, norm, out);
  free(aty);
  orig_matrix_free(&om);
  return ok;
}

int orc_dual_infeasibility(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                           const int32_t *colidx, const double *vals, const double *c,
                           const double *l, const double *u, const double *d,
                           const double *kd, double *out) {
  double *ax = NULL;
  if (!kd) {
    ax = (double *)malloc(((size_t)m + 1) * sizeof(double));
    orc_csr_multiply(m, rowptr, colidx, vals, d, ax);
    kd = ax;
  }
  double norm = orc_csr_spectral_norm_bound(m, n, rowptr, colidx, vals);
  int ok = dual_infeas(n, m, neq, c, l, u, d, kd, norm, out);
  free(ax);
  return ok;
}

/* Certificates.classify, Certificates.scala:207-219 */
static int classify_with(int32_t n, int32_t m, int32_t neq, const double *c, const double *q,
                         const double *l, const double *u, const double *x, const double *y,
                         double tol, const double *kx, const double *kty, double matrix_norm) {
  double v;
  if (primal_infeas(n, m, neq, q, l, u, y, kty, matrix_norm, &v) && v <= tol)
    return ORC_PRIMAL_INFEASIBLE;
  if (dual_infeas(n, m, neq, c, l, u, x, kx, matrix_norm, &v) && v <= tol)
    return ORC_DUAL_INFEASIBLE;
  return -1;
}

int orc_classify(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                 const int32_t *colidx, const double *vals, const double *c,
                 const double *q, const double *l, const double *u, const double *x,
                 const double *y, double tolerance, const double *kx, const double *kty) {
  orig_matrix om;
  orig_matrix_init(&om, n, m, neq, rowptr, colidx, vals);
  double *ax = NULL, *aty = NULL;
  if (!kty) {
    aty = (double *)malloc(((size_t)n + 1) * sizeof(double));
    orc_csr_multiply(n, om.t_rowptr, om.t_colidx, om.t_vals, y, aty);
    kty = aty;
  }
  if (!kx) {
    ax = (double *)malloc(((size_t)m + 1) * sizeof(double));
    orc_csr_multiply(m, rowptr, colidx, vals, x, ax);
    kx = ax;
  }
  double norm = orc_csr_spectral_norm_bound(m, n, rowptr, colidx, vals);
  int s = classify_with(n, m, neq, c, q, l, u, x, y, tolerance, kx, kty, norm);
  free(ax);
  free(aty);
  orig_matrix_free(&om);
  return s;
}

/* ------------------------------------------------------------------------ */
/* Pdhg.Solve: core/Pdhg.scala:123-534                                      */
/* ------------------------------------------------------------------------ */

static double now_ns(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec * 1e9 + (double)ts.tv_nsec;
}

typedef struct {
  /* original problem (caller's units) */
  int32_t n, m, neq;
  const int32_t *rowptr, *colidx;
  const double *vals, *c, *q, *l, *u;
  double offset;
  const orc_params *p;
  int mode;
  const volatile int32_t *cancel;
  double orig_matrix_norm;

  /* scaled problem, Pdhg.scala:135-138 */
  double *row_scale, *col_scale;
  csr K, Kt;
  double *sc, *sq, *sl, *su;
  double rhs_norm, obj_norm;

  /* device vectors, Pdhg.scala:148-186 (already "uploaded") */
  double *cost, *rhs, *lower, *upper;
  double *x, *y, *kx, *kty, *x_next, *y_next, *x_bar, *kx_bar, *dx, *dy, *kdx;
  double *sum_x, *sum_y, *sum_kx, *sum_kty, *avg_x, *avg_y, *avg_kx, *avg_kty;
  double *x_restart, *y_restart, *zero_n, *zero_m;
  /* host mirrors, Pdhg.scala:189-192 */
  double *hx, *hy, *hkx, *hkty;

  double step_size, primal_weight, weight_sum;
  int32_t iteration, restarts, last_restart_it;
  double error_at_restart, last_candidate;
  double start_ns;
} solve_t;

static double *vec(int64_t n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

static void copy_vec(const double *src, double *dst, int64_t n) {
  memcpy(dst, src, (size_t)n * sizeof(double));
}

/* Pdhg.evaluate + unscaleInPlace, Pdhg.scala:434-452 */
static kkt_t solve_evaluate(solve_t *s, const double *xv, const double *yv, const double *kxv,
                            const double *ktyv) {
  copy_vec(xv, s->hx, s->n);
  copy_vec(yv, s->hy, s->m);
  copy_vec(kxv, s->hkx, s->m);
  copy_vec(ktyv, s->hkty, s->n);
  for (int32_t i = 0; i < s->n; i++) {
    s->hx[i] *= s->col_scale[i];
    s->hkty[i] /= s->col_scale[i];
  }
  for (int32_t r = 0; r < s->m; r++) {
    s->hy[r] *= s->row_scale[r];
    s->hkx[r] /= s->row_scale[r];
  }
  return kkt_evaluate(s->n, s->m, s->neq, s->c, s->q, s->l, s->u, s->offset, s->hx, s->hy,
                      s->hkx, s->hkty);
}

static int solve_converged(solve_t *s, kkt_t e) {
  return kkt_converged(e, s->rhs_norm, s->obj_norm, s->p->eps_abs, s->p->eps_rel);
}

/* Pdhg.resetAverages, Pdhg.scala:311-316 */
static void reset_averages(solve_t *s) {
  s->weight_sum = 0.0;
  copy_vec(s->zero_n, s->sum_x, s->n);
  copy_vec(s->zero_n, s->sum_kty, s->n);
  copy_vec(s->zero_m, s->sum_y, s->m);
  copy_vec(s->zero_m, s->sum_kx, s->m);
}

/* Pdhg.accumulate, Pdhg.scala:384-389 */
static void accumulate(solve_t *s, double w) {
  int md = s->mode;
  s->weight_sum += w;
  orc_k_axpby(md, s->n, w, s->x, 1.0, s->sum_x, s->sum_x);
  orc_k_axpby(md, s->m, w, s->y, 1.0, s->sum_y, s->sum_y);
  orc_k_axpby(md, s->m, w, s->kx, 1.0, s->sum_kx, s->sum_kx);
  orc_k_axpby(md, s->n, w, s->kty, 1.0, s->sum_kty, s->sum_kty);
}

static void spmv_k(solve_t *s, const double *x, double *out) {
  orc_k_spmv(s->mode, s->K.rows, s->K.rowptr, s->K.colidx, s->K.vals, x, out);
}
static void spmv_kt(solve_t *s, const double *y, double *out) {
  orc_k_spmv(s->mode, s->Kt.rows, s->Kt.rowptr, s->Kt.colidx, s->Kt.vals, y, out);
}

/* Pdhg.step, Pdhg.scala:331-382 (MaxStepTrials = 60, :117) */
static double solve_step(solve_t *s) {
  int md = s->mode;
  double movement = 0.0;
  int accepted = 0, trials = 0;
  while (!accepted) {
    trials++;
    double tau = s->step_size / s->primal_weight;
    double sigma = s->step_size * s->primal_weight;
    orc_k_primal_step(md, s->n, s->x, s->kty, s->cost, s->lower, s->upper, tau, s->x_next);
    orc_k_axpby(md, s->n, 2.0, s->x_next, -1.0, s->x, s->x_bar);
    spmv_k(s, s->x_bar, s->kx_bar);
    orc_k_dual_step(md, s->m, s->y, s->kx_bar, s->rhs, sigma, s->neq, s->y_next);
    orc_k_axpby(md, s->n, 1.0, s->x_next, -1.0, s->x, s->dx);
    orc_k_axpby(md, s->m, 1.0, s->y_next, -1.0, s->y, s->dy);
    orc_k_axpby(md, s->m, 0.5, s->kx_bar, -0.5, s->kx, s->kdx);
    double dxsq = orc_k_squared_norm(md, s->n, s->dx);
    double dysq = orc_k_squared_norm(md, s->m, s->dy);
    movement = 0.5 * (s->primal_weight * dxsq + dysq / s->primal_weight);
    if (movement == 0.0) {
      accepted = 1;
    } else {
      double interaction = fabs(orc_k_dot(md, s->m, s->dy, s->kdx));
      double limit = interaction > 0.0 ? movement / interaction : INFINITY;
      double t = (double)(s->iteration + 1);
      double by_rule = (1.0 - pow(t, -0.3)) * limit;
      double by_cap = (1.0 + pow(t, -0.6)) * s->step_size;
      double proposed = by_rule < by_cap ? by_rule : by_cap; /* math.min */
      if (isnan(by_rule) || isnan(by_cap)) proposed = NAN;
      if (s->step_size <= limit || trials >= 60) {
        orc_k_axpby(md, s->m, 0.5, s->kx_bar, 0.5, s->kx, s->kx);
        copy_vec(s->x_next, s->x, s->n);
        copy_vec(s->y_next, s->y, s->m);
        spmv_kt(s, s->y, s->kty);
        accumulate(s, s->step_size);
        accepted = 1;
      }
      if (isfinite(proposed) && proposed > 0.0) s->step_size = proposed;
    }
  }
  return movement;
}

/* Pdhg.shouldRestart, Pdhg.scala:463-469 */
static int should_restart(solve_t *s, double candidate) {
  const orc_params *p = s->p;
  int sufficient = candidate <= p->restart_sufficient_reduction * s->error_at_restart;
  int necessary = candidate <= p->restart_necessary_reduction * s->error_at_restart &&
                  candidate > s->last_candidate;
  int artificial = (double)(s->iteration - s->last_restart_it) >=
                   p->restart_artificial_fraction * (double)s->iteration;
  return sufficient || necessary || artificial;
}

/* Pdhg.restartAt, Pdhg.scala:478-502 */
static void restart_at(solve_t *s, int use_average) {
  int md = s->mode;
  if (use_average) {
    copy_vec(s->avg_x, s->x, s->n);
    copy_vec(s->avg_y, s->y, s->m);
    copy_vec(s->avg_kx, s->kx, s->m);
    copy_vec(s->avg_kty, s->kty, s->n);
  }
  orc_k_axpby(md, s->n, 1.0, s->x, -1.0, s->x_restart, s->dx);
  orc_k_axpby(md, s->m, 1.0, s->y, -1.0, s->y_restart, s->dy);
  double pm = sqrt(orc_k_squared_norm(md, s->n, s->dx));
  double dm = sqrt(orc_k_squared_norm(md, s->m, s->dy));
  if (pm > 0.0 && dm > 0.0) {
    double th = s->p->primal_weight_smoothing;
    double next = exp(th * log(dm / pm) + (1.0 - th) * log(s->primal_weight));
    if (isfinite(next) && next > 0.0) s->primal_weight = next;
  }
  copy_vec(s->x, s->x_restart, s->n);
  copy_vec(s->y, s->y_restart, s->m);
  reset_averages(s);
  s->restarts += 1;
  s->last_restart_it = s->iteration;
  s->error_at_restart = kkt_weighted(solve_evaluate(s, s->x, s->y, s->kx, s->kty), s->primal_weight);
  s->last_candidate = INFINITY;
}

/* Pdhg.evaluateAverage, Pdhg.scala:419-425 */
static kkt_t evaluate_average(solve_t *s) {
  int md = s->mode;
  double inv = 1.0 / s->weight_sum;
  orc_k_scale(md, s->n, inv, s->sum_x, s->avg_x);
  orc_k_scale(md, s->m, inv, s->sum_y, s->avg_y);
  orc_k_scale(md, s->m, inv, s->sum_kx, s->avg_kx);
  orc_k_scale(md, s->n, inv, s->sum_kty, s->avg_kty);
  return solve_evaluate(s, s->avg_x, s->avg_y, s->avg_kx, s->avg_kty);
}

/* Pdhg.checkpoint, Pdhg.scala:396-417.  Returns -1 to keep going. */
static int checkpoint(solve_t *s, kkt_t *out) {
  spmv_k(s, s->x, s->kx);
  kkt_t current = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
  if (solve_converged(s, current)) {
    *out = current;
    return ORC_OPTIMAL;
  }
  int st = classify_with(s->n, s->m, s->neq, s->c, s->q, s->l, s->u, s->hx, s->hy,
                         s->p->infeasibility_tolerance, s->hkx, s->hkty, s->orig_matrix_norm);
  if (st >= 0) {
    *out = current;
    return st;
  }
  double current_error = kkt_weighted(current, s->primal_weight);
  int have_avg = s->weight_sum > 0.0;
  kkt_t average;
  if (have_avg) {
    average = evaluate_average(s);
    if (solve_converged(s, average)) {
      *out = average;
      return ORC_OPTIMAL;
    }
  }
  double average_error = have_avg ? kkt_weighted(average, s->primal_weight) : INFINITY;
  int use_average = average_error < current_error;
  double candidate = current_error < average_error ? current_error : average_error;
  if (isnan(current_error) || isnan(average_error)) candidate = NAN; /* math.min */
  if (should_restart(s, candidate)) restart_at(s, use_average);
  else s->last_candidate = candidate;
  return -1;
}

static void solve_free(solve_t *s) {
  double **vs[] = {&s->row_scale, &s->col_scale, &s->sc, &s->sq, &s->sl, &s->su, &s->cost,
                   &s->rhs, &s->lower, &s->upper, &s->x, &s->y, &s->kx, &s->kty,
                   &s->x_next, &s->y_next, &s->x_bar, &s->kx_bar, &s->dx, &s->dy, &s->kdx,
                   &s->sum_x, &s->sum_y, &s->sum_kx, &s->sum_kty, &s->avg_x, &s->avg_y,
                   &s->avg_kx, &s->avg_kty, &s->x_restart, &s->y_restart, &s->zero_n,
                   &s->zero_m, &s->hx, &s->hy, &s->hkx, &s->hkty};
  for (size_t i = 0; i < sizeof(vs) / sizeof(vs[0]); i++) {
    free(*vs[i]);
    *vs[i] = NULL;
  }
  free(s->K.vals);
  s->K.vals = NULL;
  csr_free(&s->Kt);
}

int orc_pdhg_solve(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                   const int32_t *colidx, const double *vals, const double *c,
                   const double *q, const double *l, const double *u, double offset,
                   const orc_params *params, int mode, const double *warm_x,
                   const double *warm_y, double warm_step, double warm_weight,
                   const volatile int32_t *cancel, double *x_out, double *y_out,
                   double *rc_out, orc_result *res) {
  if (!params_valid(params) || n < 0 || m < 0 || neq < 0 || neq > m) return -1;
  solve_t S;
  memset(&S, 0, sizeof(S));
  solve_t *s = &S;
  s->start_ns = now_ns();
  s->n = n;
  s->m = m;
  s->neq = neq;
  s->rowptr = rowptr;
  s->colidx = colidx;
  s->vals = vals;
  s->c = c;
  s->q = q;
  s->l = l;
  s->u = u;
  s->offset = offset;
  s->p = params;
  s->mode = mode;
  s->cancel = cancel;
  s->orig_matrix_norm = orc_csr_spectral_norm_bound(m, n, rowptr, colidx, vals);

  /* Scaling(problem, params.scaling), Pdhg.scala:135-138 */
  int64_t nnz = rowptr[m];
  s->row_scale = vec(m);
  s->col_scale = vec(n);
  s->sc = vec(n);
  s->sl = vec(n);
  s->su = vec(n);
  s->sq = vec(m);
  double *svals = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
  orc_scale(n, m, rowptr, colidx, vals, c, q, l, u, params->ruiz_iterations,
            params->apply_pock_chambolle, params->pock_chambolle_alpha, svals, s->sc, s->sq,
            s->sl, s->su, s->row_scale, s->col_scale);
  s->rhs_norm = norm2(q, m);
  s->obj_norm = norm2(c, n);

  /* uploadMatrix(K~), uploadMatrix(K~'), Pdhg.scala:145-146 */
  s->K.rows = m;
  s->K.cols = n;
  s->K.rowptr = (int32_t *)rowptr;
  s->K.colidx = (int32_t *)colidx;
  s->K.vals = svals;
  /* the opening step is taken from the double-precision scaled matrix
   * (sp.constraintMatrix.spectralNormBound, Pdhg.scala:255) */
  double bound = orc_csr_spectral_norm_bound(m, n, rowptr, colidx, svals);
  s->Kt = csr_transpose(&s->K);
  if (mode == 1) {
    for (int64_t k = 0; k < nnz; k++) {
      s->K.vals[k] = r32(s->K.vals[k]);
      s->Kt.vals[k] = r32(s->Kt.vals[k]);
    }
  }
  s->cost = vec(n);
  s->rhs = vec(m);
  s->lower = vec(n);
  s->upper = vec(n);
  orc_k_upload(mode, n, s->sc, s->cost);
  orc_k_upload(mode, m, s->sq, s->rhs);
  orc_k_upload(mode, n, s->sl, s->lower);
  orc_k_upload(mode, n, s->su, s->upper);
  s->x = vec(n); s->y = vec(m); s->kx = vec(m); s->kty = vec(n);
  s->x_next = vec(n); s->y_next = vec(m); s->x_bar = vec(n); s->kx_bar = vec(m);
  s->dx = vec(n); s->dy = vec(m); s->kdx = vec(m);
  s->sum_x = vec(n); s->sum_y = vec(m); s->sum_kx = vec(m); s->sum_kty = vec(n);
  s->avg_x = vec(n); s->avg_y = vec(m); s->avg_kx = vec(m); s->avg_kty = vec(n);
  s->x_restart = vec(n); s->y_restart = vec(m); s->zero_n = vec(n); s->zero_m = vec(m);
  s->hx = vec(n); s->hy = vec(m); s->hkx = vec(m); s->hkty = vec(n);
  s->primal_weight = 1.0;
  s->error_at_restart = INFINITY;
  s->last_candidate = INFINITY;

  /* initialise, Pdhg.scala:250-309 */
  s->step_size = !isnan(warm_step) ? warm_step : (bound > 0.0 ? 1.0 / bound : 1.0);
  double cnorm = norm2(s->sc, n), qnorm = norm2(s->sq, m);
  s->primal_weight = !isnan(warm_weight)
                         ? warm_weight
                         : ((cnorm > 0.0 && qnorm > 0.0) ? cnorm / qnorm : 1.0);
  double *start = vec(n);
  if (warm_x) {
    for (int32_t i = 0; i < n; i++)
      if (!isfinite(warm_x[i])) {
        free(start);
        solve_free(s);
        return -1;
      }
    for (int32_t i = 0; i < n; i++) start[i] = warm_x[i] / s->col_scale[i];
  }
  for (int32_t i = 0; i < n; i++) {
    double lo = s->sl[i], hi = s->su[i], v = start[i];
    start[i] = v < lo ? lo : (v > hi ? hi : v);
  }
  orc_k_upload(mode, n, start, s->x);
  free(start);
  if (warm_x && warm_y) {
    for (int32_t r = 0; r < m; r++)
      if (!isfinite(warm_y[r])) {
        solve_free(s);
        return -1;
      }
    double *sd = vec(m);
    for (int32_t r = 0; r < m; r++) {
      double v = warm_y[r] / s->row_scale[r];
      sd[r] = (r >= neq && v < 0.0) ? 0.0 : v;
    }
    orc_k_upload(mode, m, sd, s->y);
    free(sd);
  }
  spmv_k(s, s->x, s->kx);
  spmv_kt(s, s->y, s->kty);
  copy_vec(s->x, s->x_restart, n);
  copy_vec(s->y, s->y_restart, m);
  reset_averages(s);

  /* run, Pdhg.scala:206-246 */
  int status;
  kkt_t err;
  kkt_t initial = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
  if (solve_converged(s, initial)) {
    status = ORC_OPTIMAL;
    err = initial;
  } else {
    s->error_at_restart = kkt_weighted(initial, s->primal_weight);
    status = -1;
    while (status < 0) {
      double movement = solve_step(s);
      s->iteration += 1;
      if (movement == 0.0) {
        spmv_k(s, s->x, s->kx);
        err = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
        status = solve_converged(s, err) ? ORC_OPTIMAL : ORC_NUMERICAL_ERROR;
      } else if (s->iteration % params->evaluation_frequency == 0) {
        status = checkpoint(s, &err);
        if (status < 0) {
          if (cancel && *cancel) {
            status = ORC_INTERRUPTED;
            err = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
          } else if (params->time_limit_ms >= 0 &&
                     (double)(int64_t)((now_ns() - s->start_ns) / 1e6) >= params->time_limit_ms) {
            status = ORC_TIME_LIMIT;
            err = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
          }
        }
      }
      if (status < 0 && s->iteration >= params->max_iterations) {
        status = ORC_ITERATION_LIMIT;
        err = solve_evaluate(s, s->x, s->y, s->kx, s->kty);
      }
    }
  }

  /* finish, Pdhg.scala:510-532 */
  for (int32_t i = 0; i < n; i++) {
    if (rc_out) rc_out[i] = c[i] - s->hkty[i];
    if (x_out) x_out[i] = s->hx[i];
  }
  if (y_out) copy_vec(s->hy, y_out, m);
  res->status = status;
  res->iterations = s->iteration;
  res->restarts = s->restarts;
  res->pad = 0;
  res->solve_ms = (int64_t)((now_ns() - s->start_ns) / 1e6);
  res->objective = err.pobj;
  res->dual_objective = err.dobj;
  res->primal_residual = err.pres;
  res->dual_residual = err.dres;
  res->final_step_size = s->step_size;
  res->final_primal_weight = s->primal_weight;
  solve_free(s);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* MixedPrecision.solve: core/MixedPrecision.scala:104-199 with the device  */
/* pass on Float32Kernels (mode 1) and the refinement on ScalaKernels.      */
/* ------------------------------------------------------------------------ */

int orc_mixed_solve(int32_t n, int32_t m, int32_t neq, const int32_t *rowptr,
                    const int32_t *colidx, const double *vals, const double *c,
                    const double *q, const double *l, const double *u, double offset,
                    const orc_params *params, const orc_mixed_params *mixed,
                    const volatile int32_t *cancel, double *x_out, double *y_out,
                    double *rc_out, orc_result *res, orc_mixed_info *info) {
  if (!(mixed->reduced_tolerance > 0.0) || mixed->reduced_max_iterations <= 0 ||
      !(mixed->reduced_time_share > 0.0 && mixed->reduced_time_share < 1.0))
    return -1;
  orc_params rp = *params;
  rp.eps_abs = params->eps_abs > mixed->reduced_tolerance ? params->eps_abs : mixed->reduced_tolerance;
  rp.eps_rel = params->eps_rel > mixed->reduced_tolerance ? params->eps_rel : mixed->reduced_tolerance;
  rp.max_iterations = params->max_iterations < mixed->reduced_max_iterations
                          ? params->max_iterations
                          : mixed->reduced_max_iterations;
  if (params->time_limit_ms >= 0) {
    double lim = (double)(int64_t)(params->time_limit_ms * mixed->reduced_time_share);
    rp.time_limit_ms = lim > 1.0 ? lim : 1.0;
  }
  rp.infeasibility_tolerance = params->infeasibility_tolerance > mixed->reduced_tolerance
                                   ? params->infeasibility_tolerance
                                   : mixed->reduced_tolerance;
  double *rx = vec(n), *ry = vec(m), *rrc = vec(n);
  orc_result rr;
  if (orc_pdhg_solve(n, m, neq, rowptr, colidx, vals, c, q, l, u, offset, &rp, 1, NULL, NULL,
                     NAN, NAN, cancel, rx, ry, rrc, &rr) != 0) {
    free(rx); free(ry); free(rrc);
    return -1;
  }
  int conclusive = rr.status == ORC_OPTIMAL || rr.status == ORC_PRIMAL_INFEASIBLE ||
                   rr.status == ORC_DUAL_INFEASIBLE;
  int cert_holds = 0;
  if (conclusive && rr.status != ORC_OPTIMAL) {
    int st = orc_classify(n, m, neq, rowptr, colidx, vals, c, q, l, u, rx, ry,
                          params->infeasibility_tolerance, NULL, NULL);
    cert_holds = st == rr.status;
  }
  info->reduced_iterations = rr.iterations;
  info->reduced_restarts = rr.restarts;
  info->reduced_ms = rr.solve_ms;
  if (!mixed->always_refine && cert_holds) {
    *res = rr;
    if (x_out) copy_vec(rx, x_out, n);
    if (y_out) copy_vec(ry, y_out, m);
    if (rc_out) copy_vec(rrc, rc_out, n);
    info->refinement_iterations = 0;
    info->refinement_ms = 0;
    info->refined = 0;
    free(rx); free(ry); free(rrc);
    return 0;
  }
  orc_params fp = *params;
  if (params->time_limit_ms >= 0) {
    double lim = params->time_limit_ms - (double)rr.solve_ms;
    fp.time_limit_ms = lim > 1.0 ? lim : 1.0;
  }
  int usable = 1;
  for (int32_t i = 0; i < n; i++) usable &= isfinite(rx[i]);
  for (int32_t r = 0; r < m; r++) usable &= isfinite(ry[r]);
  /* Pdhg.WarmStart(solution): carry step and weight when finite and positive */
  double ws = (isfinite(rr.final_step_size) && rr.final_step_size > 0.0) ? rr.final_step_size : NAN;
  double ww = (isfinite(rr.final_primal_weight) && rr.final_primal_weight > 0.0)
                  ? rr.final_primal_weight
                  : NAN;
  int rc = orc_pdhg_solve(n, m, neq, rowptr, colidx, vals, c, q, l, u, offset, &fp, 0,
                          usable ? rx : NULL, usable ? ry : NULL, usable ? ws : NAN,
                          usable ? ww : NAN, cancel, x_out, y_out, rc_out, res);
  info->refinement_iterations = res->iterations;
  info->refinement_ms = res->solve_ms;
  info->refined = 1;
  free(rx); free(ry); free(rrc);
  return rc;
}
