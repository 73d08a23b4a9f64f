// Device-side problem preparation: the materialised transpose and the
// diagonal equilibration (Scaling.apply, core/Scaling.scala:77-155) on the
// GPU, so a solve's setup costs a few passes over HBM instead of eleven host
// transposes.
//
// The transpose is a stable radix sort of the entries by column (CUB), which
// yields exactly SparseMatrix.transpose's order (SparseMatrix.scala:36-64):
// within a transposed row, entries ascend by original row.  The sort gives a
// permutation perm[t] = position in K of transposed entry t, so K' values are
// always a gather of the current K values and the two never drift apart.
//
// Every reduction the reference performs per row is done by one thread in
// the reference's index order (max for Ruiz, a left-to-right sum for
// Pock-Chambolle and the norms), and scaledBy's v * rs * cs is evaluated left
// to right without FMA: the equilibrated matrix and diagonals are bit-for-bit
// the host computation's.  (Pock-Chambolle with alpha != 1 calls CUDA's pow,
// which may differ from the host libm in the last bit.)
#include <cub/cub.cuh>

#include <cmath>

#include "prima_internal.h"
#include "prima_nvtx.h"

namespace prima {
namespace {

constexpr int kT = 256;

unsigned blocks_for(int64_t n) {
  int64_t b = (n + kT - 1) / kT;
  if (b > 65535 * 16) b = 65535 * 16;
  return (unsigned)std::max<int64_t>(b, 1);
}

__global__ void k_row_of(int32_t rows, const int32_t *__restrict__ rp, int32_t *__restrict__ row_of) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
    for (int32_t k = rp[r]; k < rp[r + 1]; k++) row_of[k] = r;
}

__global__ void k_iota(int32_t n, int32_t *__restrict__ out) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = i;
}

// t_rowptr[c] = first position of column c among the sorted keys
__global__ void k_bounds(int32_t nnz, int32_t cols, const int32_t *__restrict__ sorted_cols,
                         int32_t *__restrict__ t_rp) {
  for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= cols; c += gridDim.x * blockDim.x) {
    int32_t lo = 0, hi = nnz;
    while (lo < hi) {
      const int32_t mid = lo + (hi - lo) / 2;
      if (sorted_cols[mid] < c) lo = mid + 1;
      else hi = mid;
    }
    t_rp[c] = lo;
  }
}

__global__ void k_gather_rows(int32_t nnz, const int32_t *__restrict__ perm, const int32_t *__restrict__ row_of,
                              int32_t *__restrict__ t_ci) {
  for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nnz; t += gridDim.x * blockDim.x)
    t_ci[t] = row_of[perm[t]];
}

// per-row max |a| (Ruiz) or sum |a| (Pock-Chambolle, alpha = 1) or sum |a|^e.
// Row r of K' reads K's values through perm.  Writes the scale factor.
template <int kMode>  // 0: max, 1: sum |a|, 2: sum |a|^e
__global__ void k_row_factor(int32_t rows, const int32_t *__restrict__ rp, const int32_t *__restrict__ perm,
                             const double *__restrict__ v, double e, double *__restrict__ factor) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int32_t k = rp[r]; k < rp[r + 1]; k++) {
      const double a = fabs(v[perm ? perm[k] : k]);
      if (kMode == 0) {
        if (a > acc) acc = a;
      } else if (kMode == 1) {
        acc += a;
      } else {
        acc += pow(a, e);
      }
    }
    factor[r] = acc > 0.0 ? 1.0 / sqrt(acc) : 1.0;
  }
}

__global__ void k_scale_values(int64_t nnz, const int32_t *__restrict__ row_of, const int32_t *__restrict__ ci,
                               const double *__restrict__ rf, const double *__restrict__ cf, double *__restrict__ v) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    v[k] = v[k] * rf[row_of[k]] * cf[ci[k]];
}

__global__ void k_accumulate(int32_t n, const double *__restrict__ f, double *__restrict__ cum) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) cum[i] *= f[i];
}

__global__ void k_fill(int32_t n, double v, double *__restrict__ out) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

// per-row sum |a| (index order), for the induced norms
__global__ void k_row_abs_sum(int32_t rows, const int32_t *__restrict__ rp, const int32_t *__restrict__ perm,
                              const double *__restrict__ v, double *__restrict__ out) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int32_t k = rp[r]; k < rp[r + 1]; k++) acc += fabs(v[perm ? perm[k] : k]);
    out[r] = acc;
  }
}

__global__ void k_scaled_vectors(int32_t n, int32_t m, const double *__restrict__ c, const double *__restrict__ l,
                                 const double *__restrict__ u, const double *__restrict__ q,
                                 const double *__restrict__ cs, const double *__restrict__ rs, double *__restrict__ sc,
                                 double *__restrict__ sl, double *__restrict__ su, double *__restrict__ sq) {
  const int32_t i0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
  for (int32_t j = i0; j < n; j += st) {
    const double d = cs[j];
    sc[j] = c[j] * d;
    sl[j] = l[j] / d;
    su[j] = u[j] / d;
  }
  for (int32_t r = i0; r < m; r += st) sq[r] = q[r] * rs[r];
}

// the bounds' part of k_scaled_vectors
__global__ void k_scaled_bounds(int32_t n, const double *__restrict__ l, const double *__restrict__ u,
                                const double *__restrict__ cs, double *__restrict__ sl, double *__restrict__ su) {
  for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double d = cs[j];
    sl[j] = l[j] / d;
    su[j] = u[j] / d;
  }
}

template <typename T>
__global__ void k_gather_cast(int64_t nnz, const int32_t *__restrict__ perm, const double *__restrict__ v,
                              T *__restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnz; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = (T)v[perm ? perm[t] : t];
}

template <typename T>
__global__ void k_cast(int64_t n, const double *__restrict__ v, T *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)v[i];
}

double host_max(const DeviceBuffer &b, int64_t n, cudaStream_t s, int32_t *rc) {
  std::vector<double> h((size_t)std::max<int64_t>(n, 1));
  if (n == 0) return 0.0;
  if (cudaMemcpyAsync(h.data(), b.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    *rc = PRIMA_ERR_CUDA;
    return 0.0;
  }
  double mx = 0.0;
  for (int64_t i = 0; i < n; i++)
    if (h[i] > mx) mx = h[i];
  return mx;
}

}  // namespace

// sqrt(||A||_1 ||A||_inf) of the device matrix (row sums on the device, the
// max over rows on the host: the same values the host computes).
static double device_spectral_bound(const PreparedLp &P, const double *vals, cudaStream_t s, int32_t *rc) {
  DeviceBuffer rows_sum, cols_sum;
  if ((*rc = rows_sum.reserve((size_t)std::max(P.m, 1) * 8)) || (*rc = cols_sum.reserve((size_t)std::max(P.n, 1) * 8)))
    return 0.0;
  if (P.m) k_row_abs_sum<<<blocks_for(P.m), kT, 0, s>>>(P.m, P.kp(), nullptr, vals, (double *)rows_sum.ptr);
  if (P.n) k_row_abs_sum<<<blocks_for(P.n), kT, 0, s>>>(P.n, P.tp(), P.perm(), vals, (double *)cols_sum.ptr);
  const double ninf = host_max(rows_sum, P.m, s, rc);
  const double n1 = host_max(cols_sum, P.n, s, rc);
  return std::sqrt(n1 * ninf);
}

int32_t PreparedLp::prepare(const prima_lp *lp, const prima_params *p, cudaStream_t s) {
  NvtxRange range("prima: equilibrate and transpose");
  int32_t rc;
  n = lp->num_variables;
  m = lp->num_constraints;
  neq = lp->num_equalities;
  nnz = lp->row_ptr[m];
  ruiz = p->ruiz_iterations;
  pc = p->apply_pock_chambolle;
  alpha = p->pock_chambolle_alpha;
  precision_ready[0] = precision_ready[1] = false;
  const size_t N = (size_t)std::max(n, 1), M = (size_t)std::max(m, 1), Z = (size_t)std::max<int64_t>(nnz, 1);
  if ((rc = b_kp.reserve((M + 1) * 4)) || (rc = b_kci.reserve(Z * 4)) || (rc = b_kv0.reserve(Z * 8)) ||
      (rc = b_kv.reserve(Z * 8)) || (rc = b_tp.reserve((N + 1) * 4)) || (rc = b_tci.reserve(Z * 4)) ||
      (rc = b_perm.reserve(Z * 4)) || (rc = b_c0.reserve(N * 8)) || (rc = b_l0.reserve(N * 8)) ||
      (rc = b_u0.reserve(N * 8)) || (rc = b_q0.reserve(M * 8)) || (rc = b_cs.reserve(N * 8)) ||
      (rc = b_rs.reserve(M * 8)) || (rc = b_sc.reserve(N * 8)) || (rc = b_sl.reserve(N * 8)) ||
      (rc = b_su.reserve(N * 8)) || (rc = b_sq.reserve(M * 8)))
    return rc;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(b_kp.ptr, lp->row_ptr, ((size_t)m + 1) * 4, cudaMemcpyHostToDevice, s));
  if (nnz) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(b_kci.ptr, lp->col_idx, (size_t)nnz * 4, cudaMemcpyHostToDevice, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(b_kv0.ptr, lp->values, (size_t)nnz * 8, cudaMemcpyHostToDevice, s));
  }
  if (n) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(b_c0.ptr, lp->objective, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(b_l0.ptr, lp->lower, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(b_u0.ptr, lp->upper, (size_t)n * 8, cudaMemcpyHostToDevice, s));
  }
  if (m) PRIMA_CUDA_TRY(cudaMemcpyAsync(b_q0.ptr, lp->rhs, (size_t)m * 8, cudaMemcpyHostToDevice, s));

  // transpose structure: stable sort of entry positions by column
  DeviceBuffer row_of, keys_in, keys_out, idx_in, temp;
  if ((rc = row_of.reserve(Z * 4)) || (rc = keys_out.reserve(Z * 4)) || (rc = idx_in.reserve(Z * 4))) return rc;
  if (m) k_row_of<<<blocks_for(m), kT, 0, s>>>(m, kp(), (int32_t *)row_of.ptr);
  if (nnz) {
    k_iota<<<blocks_for(nnz), kT, 0, s>>>((int32_t)nnz, (int32_t *)idx_in.ptr);
    size_t temp_bytes = 0;
    int bits = 1;
    while (bits < 31 && (1 << bits) <= n) bits++;
    cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, (const int32_t *)b_kci.ptr, (int32_t *)keys_out.ptr,
                                    (const int32_t *)idx_in.ptr, (int32_t *)b_perm.ptr, (int)nnz, 0, bits, s);
    if ((rc = temp.reserve(temp_bytes))) return rc;
    PRIMA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.ptr, temp_bytes, (const int32_t *)b_kci.ptr,
                                                   (int32_t *)keys_out.ptr, (const int32_t *)idx_in.ptr,
                                                   (int32_t *)b_perm.ptr, (int)nnz, 0, bits, s));
    k_gather_rows<<<blocks_for(nnz), kT, 0, s>>>((int32_t)nnz, perm(), (const int32_t *)row_of.ptr,
                                                 (int32_t *)b_tci.ptr);
  }
  k_bounds<<<blocks_for((int64_t)n + 1), kT, 0, s>>>((int32_t)nnz, n, (const int32_t *)keys_out.ptr,
                                                     (int32_t *)b_tp.ptr);
  PRIMA_CUDA_TRY(cudaGetLastError());

  orig_spectral_bound = device_spectral_bound(*this, kv0(), s, &rc);
  if (rc) return rc;

  // Scaling.apply
  PRIMA_CUDA_TRY(cudaMemcpyAsync(b_kv.ptr, b_kv0.ptr, (size_t)nnz * 8, cudaMemcpyDeviceToDevice, s));
  k_fill<<<blocks_for(m), kT, 0, s>>>(m, 1.0, rs_());
  k_fill<<<blocks_for(n), kT, 0, s>>>(n, 1.0, cs_());
  DeviceBuffer rf, cf;
  if ((rc = rf.reserve(M * 8)) || (rc = cf.reserve(N * 8))) return rc;
  double *RF = (double *)rf.ptr, *CF = (double *)cf.ptr;
  const int32_t *ROW = (const int32_t *)row_of.ptr;
  for (int32_t it = 0; it < ruiz; it++) {
    if (m) k_row_factor<0><<<blocks_for(m), kT, 0, s>>>(m, kp(), nullptr, kv(), 0.0, RF);
    if (n) k_row_factor<0><<<blocks_for(n), kT, 0, s>>>(n, tp(), perm(), kv(), 0.0, CF);
    if (nnz) k_scale_values<<<blocks_for(nnz), kT, 0, s>>>(nnz, ROW, kci(), RF, CF, kv());
    if (m) k_accumulate<<<blocks_for(m), kT, 0, s>>>(m, RF, rs_());
    if (n) k_accumulate<<<blocks_for(n), kT, 0, s>>>(n, CF, cs_());
  }
  if (pc) {
    if (alpha == 1.0) {  // |a|^1 = |a| exactly, as pow(|a|, 1.0) is on the host
      if (m) k_row_factor<1><<<blocks_for(m), kT, 0, s>>>(m, kp(), nullptr, kv(), 0.0, RF);
      if (n) k_row_factor<1><<<blocks_for(n), kT, 0, s>>>(n, tp(), perm(), kv(), 0.0, CF);
    } else {
      if (m) k_row_factor<2><<<blocks_for(m), kT, 0, s>>>(m, kp(), nullptr, kv(), 2.0 - alpha, RF);
      if (n) k_row_factor<2><<<blocks_for(n), kT, 0, s>>>(n, tp(), perm(), kv(), alpha, CF);
    }
    if (nnz) k_scale_values<<<blocks_for(nnz), kT, 0, s>>>(nnz, ROW, kci(), RF, CF, kv());
    if (m) k_accumulate<<<blocks_for(m), kT, 0, s>>>(m, RF, rs_());
    if (n) k_accumulate<<<blocks_for(n), kT, 0, s>>>(n, CF, cs_());
  }
  k_scaled_vectors<<<blocks_for(std::max(n, m)), kT, 0, s>>>(n, m, c0(), l0(), u0(), q0(), cs(), rs(), sc_(), sl_(),
                                                             su_(), sq_());
  PRIMA_CUDA_TRY(cudaGetLastError());
  scaled_spectral_bound = device_spectral_bound(*this, kv(), s, &rc);
  if (rc) return rc;

  // norms in the reference's index order, on the host (O(n + m))
  auto norm2 = [](const double *v, int64_t k) {
    double acc = 0.0;
    for (int64_t i = 0; i < k; i++) acc += v[i] * v[i];
    return std::sqrt(acc);
  };
  rhs_norm = norm2(lp->rhs, m);
  obj_norm = norm2(lp->objective, n);
  h_sc.resize((size_t)n);
  h_sq.resize((size_t)m);
  h_sl.resize((size_t)n);
  h_su.resize((size_t)n);
  h_cs.resize((size_t)n);
  h_rs.resize((size_t)m);
  if (n) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_sc.data(), b_sc.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_sl.data(), b_sl.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_su.data(), b_su.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_cs.data(), b_cs.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  }
  if (m) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_sq.data(), b_sq.ptr, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(h_rs.data(), b_rs.ptr, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
  }
  h_kp.assign(lp->row_ptr, lp->row_ptr + m + 1);
  h_tp.resize((size_t)n + 1);
  PRIMA_CUDA_TRY(cudaMemcpyAsync(h_tp.data(), b_tp.ptr, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost, s));
  for (int w = 0; w < 2; w++)
    for (int v = 0; v < 2; v++) {
      tiles_nb[w][v] = 0;
      for (int k = 0; k < 2; k++) {
        ntiles[w][v][k] = 0;
        h_tiles[w][v][k].clear();
        h_tile_cost[w][v][k].clear();
      }
    }
  layout_bps[0] = layout_bps[1] = layout_rows[0] = layout_rows[1] = 0;
  PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  scaled_c_norm = norm2(h_sc.data(), n);
  scaled_q_norm = norm2(h_sq.data(), m);
  return PRIMA_OK;
}

// Matrix values and scaled vectors in the storage type T (K' gathered through
// perm), made once per precision and kept.
template <typename T>
int32_t PreparedLp::materialise(cudaStream_t s) {
  const int w = sizeof(T) == 8 ? 1 : 0;
  if (precision_ready[w]) return PRIMA_OK;
  const size_t N = (size_t)std::max(n, 1), M = (size_t)std::max(m, 1), Z = (size_t)std::max<int64_t>(nnz, 1);
  int32_t rc;
  PrecisionCopy &pcpy = copies[w];
  if ((rc = pcpy.kv.reserve(Z * sizeof(T))) || (rc = pcpy.tv.reserve(Z * sizeof(T))) ||
      (rc = pcpy.c.reserve(N * sizeof(T))) || (rc = pcpy.l.reserve(N * sizeof(T))) ||
      (rc = pcpy.u.reserve(N * sizeof(T))) || (rc = pcpy.q.reserve(M * sizeof(T))))
    return rc;
  if (nnz) {
    k_gather_cast<T><<<blocks_for(nnz), kT, 0, s>>>(nnz, nullptr, kv(), (T *)pcpy.kv.ptr);
    k_gather_cast<T><<<blocks_for(nnz), kT, 0, s>>>(nnz, perm(), kv(), (T *)pcpy.tv.ptr);
  }
  if (n) {
    k_cast<T><<<blocks_for(n), kT, 0, s>>>(n, sc(), (T *)pcpy.c.ptr);
    k_cast<T><<<blocks_for(n), kT, 0, s>>>(n, sl(), (T *)pcpy.l.ptr);
    k_cast<T><<<blocks_for(n), kT, 0, s>>>(n, su(), (T *)pcpy.u.ptr);
  }
  if (m) k_cast<T><<<blocks_for(m), kT, 0, s>>>(m, sq(), (T *)pcpy.q.ptr);
  PRIMA_CUDA_TRY(cudaGetLastError());
  precision_ready[w] = true;
  return PRIMA_OK;
}

int32_t PreparedLp::set_bounds(const double *lower, const double *upper, cudaStream_t s) {
  if (n == 0) return PRIMA_OK;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(b_l0.ptr, lower, (size_t)n * 8, cudaMemcpyHostToDevice, s));
  PRIMA_CUDA_TRY(cudaMemcpyAsync(b_u0.ptr, upper, (size_t)n * 8, cudaMemcpyHostToDevice, s));
  k_scaled_bounds<<<blocks_for(n), kT, 0, s>>>(n, l0(), u0(), cs(), sl_(), su_());
  if (precision_ready[0]) {
    k_cast<float><<<blocks_for(n), kT, 0, s>>>(n, sl(), (float *)copies[0].l.ptr);
    k_cast<float><<<blocks_for(n), kT, 0, s>>>(n, su(), (float *)copies[0].u.ptr);
  }
  if (precision_ready[1]) {
    k_cast<double><<<blocks_for(n), kT, 0, s>>>(n, sl(), (double *)copies[1].l.ptr);
    k_cast<double><<<blocks_for(n), kT, 0, s>>>(n, su(), (double *)copies[1].u.ptr);
  }
  PRIMA_CUDA_TRY(cudaGetLastError());
  PRIMA_CUDA_TRY(cudaMemcpyAsync(h_sl.data(), b_sl.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  PRIMA_CUDA_TRY(cudaMemcpyAsync(h_su.data(), b_su.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  return PRIMA_OK;
}

template int32_t PreparedLp::materialise<float>(cudaStream_t);
template int32_t PreparedLp::materialise<double>(cudaStream_t);

}  // namespace prima
