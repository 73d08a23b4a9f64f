// Host-side problem preparation: validation, diagonal equilibration and the
// materialised transpose.  Runs once per solve, in IEEE double, in the same
// operation order as the reference so the equilibrated problem is bit-for-bit
// the one the reference iterates (compiled with -ffp-contract=off).
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>

#include "prima_internal.h"

namespace prima {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

}  // namespace prima

extern "C" const char *prima_last_error(void) { return prima::g_last_error.c_str(); }

extern "C" void prima_params_default(prima_params *p) {
  // PdhgParams.scala:9-54 and ScalingParams.default (Scaling.scala:11-14)
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

extern "C" void prima_mixed_params_default(prima_mixed_params *p) {
  // MixedPrecision.Params (MixedPrecision.scala:37-79) + refinement defaults
  p->reduced_tolerance = 1e-5;
  p->reduced_max_iterations = 20000;
  p->always_refine = 0;
  p->reduced_time_share = 0.5;
  p->scheme = PRIMA_MIXED_REFINEMENT;
  p->pad = 0;
  p->round_reduction = 0.0;
}

namespace prima {

static int32_t fail(const std::string &m) {
  set_error("requirement failed: " + m);
  return PRIMA_ERR_INVALID_ARGUMENT;
}

int32_t validate_params(const prima_params *p) {
  if (!p) return fail("params is NULL");
  if (!(p->eps_abs >= 0.0)) return fail("epsAbs must be non-negative");
  if (!(p->eps_rel >= 0.0)) return fail("epsRel must be non-negative");
  if (p->max_iterations <= 0) return fail("maxIterations must be positive");
  if (p->evaluation_frequency <= 0) return fail("evaluationFrequency must be positive");
  if (!(p->primal_weight_smoothing >= 0.0 && p->primal_weight_smoothing <= 1.0))
    return fail("primalWeightSmoothing must lie in [0, 1]");
  if (!(p->restart_sufficient_reduction > 0.0 &&
        p->restart_sufficient_reduction <= p->restart_necessary_reduction))
    return fail("restartSufficientReduction must be positive and no greater than restartNecessaryReduction");
  if (!(p->restart_artificial_fraction > 0.0 && p->restart_artificial_fraction <= 1.0))
    return fail("restartArtificialFraction must lie in (0, 1]");
  if (!(p->infeasibility_tolerance >= 0.0)) return fail("infeasibilityTolerance must be non-negative");
  if (p->ruiz_iterations < 0) return fail("ruizIterations must be non-negative");
  if (!(p->pock_chambolle_alpha >= 0.0 && p->pock_chambolle_alpha <= 2.0))
    return fail("pockChambolleAlpha must lie in [0, 2]");
  return PRIMA_OK;
}

int32_t validate_lp(const prima_lp *lp) {
  if (!lp) return fail("problem is NULL");
  const int32_t n = lp->num_variables, m = lp->num_constraints;
  if (n < 0 || m < 0) return fail("dimensions must be non-negative");
  if (lp->num_equalities < 0 || lp->num_equalities > m)
    return fail("numEqualities out of range [0, m]");
  if (!lp->row_ptr || (n > 0 && (!lp->objective || !lp->lower || !lp->upper)) || (m > 0 && !lp->rhs))
    return fail("missing problem array");
  if (lp->row_ptr[0] != 0) return fail("row_ptr[0] must be 0");
  for (int32_t r = 0; r < m; r++)
    if (lp->row_ptr[r + 1] < lp->row_ptr[r]) return fail("row_ptr must be non-decreasing");
  const int64_t nnz = lp->row_ptr[m];
  if (nnz > 0 && (!lp->col_idx || !lp->values)) return fail("missing matrix entries");
  for (int32_t r = 0; r < m; r++) {
    for (int32_t p = lp->row_ptr[r]; p < lp->row_ptr[r + 1]; p++) {
      const int32_t c = lp->col_idx[p];
      if (c < 0 || c >= n) {
        std::ostringstream os;
        os << "column index " << c << " out of range [0, " << n << ")";
        return fail(os.str());
      }
      if (p > lp->row_ptr[r] && lp->col_idx[p - 1] >= c)
        return fail("column indices must ascend within a row (canonical CSR)");
      if (!std::isfinite(lp->values[p])) return fail("matrix entry is not finite");
    }
  }
  for (int32_t i = 0; i < n; i++) {
    if (!(lp->lower[i] <= lp->upper[i])) {
      std::ostringstream os;
      os << "variable " << i << " has empty bound interval [" << lp->lower[i] << ", " << lp->upper[i]
         << "]";
      return fail(os.str());
    }
    if (!std::isfinite(lp->objective[i])) return fail("objective coefficient is not finite");
  }
  for (int32_t r = 0; r < m; r++)
    if (!std::isfinite(lp->rhs[r])) return fail("right-hand side is not finite");
  return PRIMA_OK;
}

// Counting sort by column; rows visited in order keep each transposed row
// column-sorted (SparseMatrix.transpose, SparseMatrix.scala:36-64).
void csr_transpose(const Csr &a, Csr *t) {
  const int64_t nnz = a.nnz();
  t->rows = a.cols;
  t->cols = a.rows;
  t->row_ptr.assign((size_t)a.cols + 1, 0);
  t->col_idx.resize((size_t)nnz);
  t->vals.resize((size_t)nnz);
  for (int64_t k = 0; k < nnz; k++) t->row_ptr[a.col_idx[k] + 1] += 1;
  for (int32_t c = 0; c < a.cols; c++) t->row_ptr[c + 1] += t->row_ptr[c];
  std::vector<int32_t> cursor(t->row_ptr.begin(), t->row_ptr.end() - 1);
  for (int32_t r = 0; r < a.rows; r++) {
    for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) {
      const int32_t dest = cursor[a.col_idx[p]]++;
      t->col_idx[dest] = r;
      t->vals[dest] = a.vals[p];
    }
  }
}

// SparseMatrix.normInf, SparseMatrix.scala:144-156 (index-order row sums)
double csr_norm_inf(const Csr &a) {
  double mx = 0.0;
  for (int32_t r = 0; r < a.rows; r++) {
    double s = 0.0;
    for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) s += std::fabs(a.vals[p]);
    if (s > mx) mx = s;
  }
  return mx;
}

// sqrt(||A||_1 ||A||_inf), SparseMatrix.scala:181
double spectral_norm_bound(const Csr &a, const Csr &at) {
  return std::sqrt(csr_norm_inf(at) * csr_norm_inf(a));
}

static double norm2(const double *v, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; i++) s += v[i] * v[i];
  return std::sqrt(s);
}

static void row_max_abs(const Csr &a, std::vector<double> &out) {
  for (int32_t r = 0; r < a.rows; r++) {
    double mx = 0.0;
    for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) {
      const double v = std::fabs(a.vals[p]);
      if (v > mx) mx = v;
    }
    out[r] = mx;
  }
}

static void row_abs_pow_sum(const Csr &a, double alpha, std::vector<double> &out) {
  for (int32_t r = 0; r < a.rows; r++) {
    double s = 0.0;
    for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) s += std::pow(std::fabs(a.vals[p]), alpha);
    out[r] = s;
  }
}

// diag(rs) A diag(cs), evaluated as v * rs * cs left to right (SparseMatrix.scala:116-128)
static void scale_in_place(Csr &a, const std::vector<double> &rs, const std::vector<double> &cs) {
  for (int32_t r = 0; r < a.rows; r++) {
    const double f = rs[r];
    for (int32_t p = a.row_ptr[r]; p < a.row_ptr[r + 1]; p++) a.vals[p] = a.vals[p] * f * cs[a.col_idx[p]];
  }
}

// Scaling.apply (Scaling.scala:77-155): Ruiz passes (1/sqrt of the row and
// column infinity norms, both taken before the pass is applied), then one
// Pock-Chambolle pass; empty rows and columns keep scale one.
void prepare_scaled(const prima_lp *lp, const prima_params *p, ScaledLp *s) {
  const int32_t n = lp->num_variables, m = lp->num_constraints;
  s->n = n;
  s->m = m;
  s->neq = lp->num_equalities;
  Csr &K = s->K;
  K.rows = m;
  K.cols = n;
  K.row_ptr.assign(lp->row_ptr, lp->row_ptr + m + 1);
  const int64_t nnz = K.row_ptr[m];
  K.col_idx.assign(lp->col_idx, lp->col_idx + nnz);
  K.vals.assign(lp->values, lp->values + nnz);

  {  // certificates are normalised by the ORIGINAL matrix's bound
    Csr t;
    csr_transpose(K, &t);
    s->orig_spectral_bound = spectral_norm_bound(K, t);
  }
  s->row_scale.assign((size_t)m, 1.0);
  s->col_scale.assign((size_t)n, 1.0);
  std::vector<double> rf((size_t)m), cf((size_t)n), tmp;
  Csr t;
  for (int32_t it = 0; it < p->ruiz_iterations; it++) {
    row_max_abs(K, rf);
    for (int32_t r = 0; r < m; r++) rf[r] = rf[r] > 0.0 ? 1.0 / std::sqrt(rf[r]) : 1.0;
    csr_transpose(K, &t);
    row_max_abs(t, cf);
    for (int32_t j = 0; j < n; j++) cf[j] = cf[j] > 0.0 ? 1.0 / std::sqrt(cf[j]) : 1.0;
    scale_in_place(K, rf, cf);
    for (int32_t r = 0; r < m; r++) s->row_scale[r] *= rf[r];
    for (int32_t j = 0; j < n; j++) s->col_scale[j] *= cf[j];
  }
  if (p->apply_pock_chambolle) {
    const double alpha = p->pock_chambolle_alpha;
    row_abs_pow_sum(K, 2.0 - alpha, rf);
    for (int32_t r = 0; r < m; r++) rf[r] = rf[r] > 0.0 ? 1.0 / std::sqrt(rf[r]) : 1.0;
    csr_transpose(K, &t);
    row_abs_pow_sum(t, alpha, cf);
    for (int32_t j = 0; j < n; j++) cf[j] = cf[j] > 0.0 ? 1.0 / std::sqrt(cf[j]) : 1.0;
    scale_in_place(K, rf, cf);
    for (int32_t r = 0; r < m; r++) s->row_scale[r] *= rf[r];
    for (int32_t j = 0; j < n; j++) s->col_scale[j] *= cf[j];
  }
  s->c.resize((size_t)n);
  s->l.resize((size_t)n);
  s->u.resize((size_t)n);
  s->q.resize((size_t)m);
  for (int32_t j = 0; j < n; j++) {
    const double d = s->col_scale[j];
    s->c[j] = lp->objective[j] * d;
    s->l[j] = lp->lower[j] / d;
    s->u[j] = lp->upper[j] / d;
  }
  for (int32_t r = 0; r < m; r++) s->q[r] = lp->rhs[r] * s->row_scale[r];
  csr_transpose(K, &s->Kt);
  s->scaled_spectral_bound = spectral_norm_bound(K, s->Kt);
  s->rhs_norm = norm2(lp->rhs, m);
  s->obj_norm = norm2(lp->objective, n);
  s->scaled_c_norm = norm2(s->c.data(), n);
  s->scaled_q_norm = norm2(s->q.data(), m);
}

// Certificates.primalInfeasibility (Certificates.scala:60-123) and
// dualInfeasibility (:137-195), classify (:207-219).
int classify_fp64(const prima_lp *lp, const double *x, const double *y, double tol) {
  const int32_t n = lp->num_variables, m = lp->num_constraints, neq = lp->num_equalities;
  Csr K;
  K.rows = m;
  K.cols = n;
  K.row_ptr.assign(lp->row_ptr, lp->row_ptr + m + 1);
  K.col_idx.assign(lp->col_idx, lp->col_idx + K.row_ptr[m]);
  K.vals.assign(lp->values, lp->values + K.row_ptr[m]);
  Csr Kt;
  csr_transpose(K, &Kt);
  const double mn = spectral_norm_bound(K, Kt);
  std::vector<double> kx((size_t)m), kty((size_t)n);
  for (int32_t r = 0; r < m; r++) {
    double acc = 0.0;
    for (int32_t p = K.row_ptr[r]; p < K.row_ptr[r + 1]; p++) acc += K.vals[p] * x[K.col_idx[p]];
    kx[r] = acc;
  }
  for (int32_t j = 0; j < n; j++) {
    double acc = 0.0;
    for (int32_t p = Kt.row_ptr[j]; p < Kt.row_ptr[j + 1]; p++) acc += Kt.vals[p] * y[Kt.col_idx[p]];
    kty[j] = acc;
  }
  const double *q = lp->rhs, *c = lp->objective, *l = lp->lower, *u = lp->upper;
  {  // primal infeasibility from y
    double nsq = 0.0;
    for (int32_t r = 0; r < m; r++) nsq += y[r] * y[r];
    if (nsq > 0.0 && std::isfinite(nsq)) {
      const double norm = std::sqrt(nsq);
      double value = 0.0, rsq = 0.0, csq = 0.0;
      for (int32_t r = 0; r < m; r++) value += q[r] * y[r];
      for (int32_t j = 0; j < n; j++) {
        const double rc = -kty[j];
        if (rc > 0.0) {
          if (std::isinf(l[j]) && l[j] < 0) rsq += rc * rc;
          else value += l[j] * rc;
        } else if (rc < 0.0) {
          if (std::isinf(u[j]) && u[j] > 0) rsq += rc * rc;
          else value += u[j] * rc;
        }
      }
      for (int32_t r = neq; r < m; r++)
        if (y[r] < 0.0) csq += y[r] * y[r];
      if (value > 0.0 && std::isfinite(value)) {
        const double rt = mn > 0.0 ? std::sqrt(rsq) / (mn * norm) : 0.0;
        const double h = std::hypot(rt, std::sqrt(csq) / norm);
        if (std::isfinite(h) && h <= tol) return PRIMA_STATUS_PRIMAL_INFEASIBLE;
      }
    }
  }
  {  // dual infeasibility from x
    double nsq = 0.0;
    for (int32_t j = 0; j < n; j++) nsq += x[j] * x[j];
    if (nsq > 0.0 && std::isfinite(nsq)) {
      const double norm = std::sqrt(nsq);
      double value = 0.0;
      for (int32_t j = 0; j < n; j++) value += c[j] * x[j];
      if (value < 0.0 && std::isfinite(value)) {
        double rowsq = 0.0, bsq = 0.0;
        for (int32_t r = 0; r < m; r++)
          if (r < neq || kx[r] < 0.0) rowsq += kx[r] * kx[r];
        for (int32_t j = 0; j < n; j++) {
          const double d = x[j];
          if (d > 0.0 && !(std::isinf(u[j]) && u[j] > 0)) bsq += d * d;
          else if (d < 0.0 && !(std::isinf(l[j]) && l[j] < 0)) bsq += d * d;
        }
        const double rt = mn > 0.0 ? std::sqrt(rowsq) / (mn * norm) : 0.0;
        const double h = std::hypot(rt, std::sqrt(bsq) / norm);
        if (std::isfinite(h) && h <= tol) return PRIMA_STATUS_DUAL_INFEASIBLE;
      }
    }
  }
  return -1;
}

}  // namespace prima
