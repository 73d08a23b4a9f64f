// Fused persistent restarted-PDHG kernel and the coarse solve entry points.
// Design notes are in prima_solver.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

#include <math_constants.h>

#include "prima_internal.h"
#include "prima_solver.cuh"

namespace prima {
namespace dev {

// ---- memory-model helpers -------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Data written inside this launch by other blocks is read through L2 only
// (ld.global.cg), so no stale L1 line can be observed across a barrier.
template <typename T>
__device__ __forceinline__ T ldv(const T *p) {
  return __ldcg(p);
}

// Each block owns one contiguous chunk of rows (resp. columns).
__device__ __forceinline__ void chunk(int32_t total, int nb, int rank, int32_t &lo, int32_t &hi) {
  const int64_t per = ((int64_t)total + nb - 1) / nb;
  int64_t a = (int64_t)rank * per, b = a + per;
  if (a > total) a = total;
  if (b > total) b = total;
  lo = (int32_t)a;
  hi = (int32_t)b;
}

// Row r of a CSR matrix against a vector written in this launch, summed in
// index order from zero (SparseMatrix.multiplyInto order).
template <typename T>
__device__ __forceinline__ T row_dot(const int32_t *__restrict__ p, const int32_t *__restrict__ ci,
                                     const T *__restrict__ v, const T *x, int32_t r) {
  T acc = T(0);
  const int32_t e = __ldg(p + r + 1);
  for (int32_t k = __ldg(p + r); k < e; k++) acc = acc + (__ldg(v + k) * ldv(x + __ldg(ci + k)));
  return acc;
}

// Block-wide sum of Q per-thread values in a fixed order; thread 0 stores the
// block's partials at partials[q * stride + rank].
template <int Q>
__device__ __forceinline__ void block_partials(double (&v)[Q], double *partials, int stride, int rank) {
  __shared__ double sh[kMaxQ][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < Q; q++) {
    double s = v[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sh[q][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < Q) {
    double s = 0.0;
    for (int w = 0; w < kWarps; w++) s += sh[threadIdx.x][w];
    partials[threadIdx.x * stride + rank] = s;
  }
  __syncthreads();
}

// Deciding block: total of slots [q0, q0+Q) over nb block partials, fixed order.
template <int Q>
__device__ __forceinline__ void reduce_partials(const double *partials, int stride, int nb, int q0,
                                                double *out /* shared, Q */) {
  __shared__ double sh[kMaxQ][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += kThreads) s += ldv(partials + (q0 + q) * stride + b);
    v[q] = s;
  }
#pragma unroll
  for (int q = 0; q < Q; q++) {
    double s = v[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sh[q][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < Q) {
    double s = 0.0;
    for (int w = 0; w < kWarps; w++) s += sh[threadIdx.x][w];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// ---- scalar tail (runs on one thread of the deciding block) ---------------

__device__ __forceinline__ bool kkt_finite(const Kkt &e) {
  return isfinite(e.pres) && isfinite(e.dres) && isfinite(e.pobj) && isfinite(e.dobj);
}

// KktError.weighted, Kkt.scala:28-33
__device__ __forceinline__ double weighted(const Kkt &e, double w) {
  const double gap = e.pobj - e.dobj;
  return sqrt(w * e.pres * e.pres + (e.dres * e.dres) / w + gap * gap);
}

// Kkt.convergence + Convergence.converged, Kkt.scala:130-143, :46
__device__ __forceinline__ bool converged(const Kkt &e, const Params &P) {
  const double pt = P.eps_abs + P.eps_rel * P.rhs_norm;
  const double dt = P.eps_abs + P.eps_rel * P.obj_norm;
  const double gt = P.eps_abs + P.eps_rel * (fabs(e.pobj) + fabs(e.dobj));
  return kkt_finite(e) && e.pres <= pt && e.dres <= dt && fabs(e.pobj - e.dobj) <= gt;
}

__device__ __forceinline__ double dmin(double a, double b) {  // java.lang.Math.min
  if (isnan(a) || isnan(b)) return CUDART_NAN;
  return a < b ? a : b;
}

__device__ Kkt kkt_current(const double *s, const Params &P) {
  Kkt e;
  e.pres = sqrt(s[Q_PSQ]);
  e.dres = sqrt(s[Q_DSQ]);
  e.pobj = P.offset + s[Q_CX];
  e.dobj = (P.offset + s[Q_QY]) + s[Q_DTERM];
  return e;
}

__device__ Kkt kkt_average(const double *s, const Params &P) {
  Kkt e;
  e.pres = sqrt(s[Q_A_PSQ]);
  e.dres = sqrt(s[Q_A_DSQ]);
  e.pobj = P.offset + s[Q_A_CX];
  e.dobj = (P.offset + s[Q_A_QY]) + s[Q_A_DTERM];
  return e;
}

// Certificates.classify (Certificates.scala:207-219) on reduced terms:
// primalInfeasibility (:60-123) from y, dualInfeasibility (:137-195) from x.
__device__ int classify(const double *s, const Params &P) {
  const double mn = P.matrix_norm;
  {
    const double nsq = s[Q_YSQ];
    if (nsq > 0.0 && isfinite(nsq)) {
      const double norm = sqrt(nsq);
      const double value = s[Q_QY] + s[Q_PVAL];
      if (value > 0.0 && isfinite(value)) {
        const double rt = mn > 0.0 ? sqrt(s[Q_PRSQ]) / (mn * norm) : 0.0;
        const double ct = sqrt(s[Q_CONE]) / norm;
        const double h = hypot(rt, ct);
        if (isfinite(h) && h <= P.infeas_tol) return PRIMA_STATUS_PRIMAL_INFEASIBLE;
      }
    }
  }
  {
    const double nsq = s[Q_XSQ];
    if (nsq > 0.0 && isfinite(nsq)) {
      const double norm = sqrt(nsq);
      const double value = s[Q_CX];
      if (value < 0.0 && isfinite(value)) {
        const double rt = mn > 0.0 ? sqrt(s[Q_ROWSQ]) / (mn * norm) : 0.0;
        const double bt = sqrt(s[Q_BSQ]) / norm;
        const double h = hypot(rt, bt);
        if (isfinite(h) && h <= P.infeas_tol) return PRIMA_STATUS_DUAL_INFEASIBLE;
      }
    }
  }
  return -1;
}

__device__ __forceinline__ void set_trial_scalars(Control &c) {
  c.tau = c.step / c.weight;
  c.sigma = c.step * c.weight;
}

// After a checkpoint that did not terminate: cancellation, wall clock and
// the iteration limit, in the order Pdhg.run checks them (Pdhg.scala:233-243).
__device__ void after_checkpoint(Control &c, const Kkt &point, const Params &P, const volatile int32_t *cancel) {
  if (cancel && *cancel) {
    c.status = PRIMA_STATUS_INTERRUPTED;
  } else if (P.time_limit_ms >= 0.0) {
    const double ms = P.setup_ms + (double)(global_timer_ns() - c.t0) * 1e-6;
    if (floor(ms) >= P.time_limit_ms) c.status = PRIMA_STATUS_TIME_LIMIT;
  }
  if (c.status < 0 && c.iteration >= P.max_iterations) c.status = PRIMA_STATUS_ITERATION_LIMIT;
  if (c.status >= 0) {
    c.final_kkt = point;
    c.w_avg = 0;
    c.phase = PH_W;
  } else {
    c.pend = 0;
    c.phase = PH_A;
  }
}

// ---- the team barrier -------------------------------------------------------

constexpr unsigned long long kSpinLimit = 1ull << 26;  // ~seconds; a phase takes microseconds

template <typename T>
__device__ void decide(const Args<T> &a, Control &c, int phase, int nb, double *red);

// All blocks arrive; the last one reduces and decides, then releases.  Every
// wait is bounded: on timeout the team's abort flag is raised, the kernel
// records PRIMA_ERR_TIMEOUT and every block leaves.
template <typename T>
__device__ bool barrier_decide(const Args<T> &a, Control &snap, int phase, int nb) {
  __shared__ unsigned s_gen;
  __shared__ int s_last, s_ok;
  __shared__ double s_red[kMaxQ];
  __syncthreads();
  if (threadIdx.x == 0) {
    s_gen = ld_acquire(&a.sync->gen);
    __threadfence();
    const unsigned old = atom_add_acq_rel(&a.sync->count, 1u);
    s_last = old == (unsigned)(nb - 1);
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    decide<T>(a, snap, phase, nb, s_red);  // block-wide; thread 0 updates snap
    __syncthreads();
    if (threadIdx.x == 0) {
      if (*((volatile int32_t *)&a.sync->abort)) {
        snap.error = PRIMA_ERR_TIMEOUT;
        snap.phase = PH_DONE;
      }
      // publish the new control record, then release the team
      const unsigned *src = (const unsigned *)&snap;
      unsigned *dst = (unsigned *)a.ctl;
      for (int i = 0; i < (int)(sizeof(Control) / 4); i++) dst[i] = src[i];
      a.sync->count = 0;
      __threadfence();
      st_release(&a.sync->gen, s_gen + 1);
    }
  } else if (threadIdx.x == 0) {
    unsigned long long spins = 0;
    while (ld_acquire(&a.sync->gen) == s_gen) {
      if (*((volatile int32_t *)&a.sync->abort)) {
        s_ok = 0;
        break;
      }
      if (++spins > kSpinLimit) {
        atomicExch(&a.sync->abort, 1);
        a.ctl->error = PRIMA_ERR_TIMEOUT;
        s_ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
  }
  __syncthreads();
  return s_ok;
}

template <typename T>
__device__ __forceinline__ void load_control(const Args<T> &a, Control &snap) {
  const unsigned *src = (const unsigned *)a.ctl;
  unsigned *dst = (unsigned *)&snap;
  for (int i = threadIdx.x; i < (int)(sizeof(Control) / 4); i += blockDim.x) dst[i] = __ldcg(src + i);
  __syncthreads();
}

// ---- evaluation terms --------------------------------------------------------

// Row r: current point terms (Kkt.evaluate rows, certificate rows).
__device__ __forceinline__ void eval_row(double yv, double kxv, double rs, double q0, bool eq, double *v) {
  const double yo = yv * rs, kxo = kxv / rs;
  if (eq) {
    const double d = kxo - q0;
    v[Q_PSQ] += d * d;
    v[Q_ROWSQ] += kxo * kxo;
  } else {
    const double sf = q0 - kxo;
    if (sf > 0.0) v[Q_PSQ] += sf * sf;
    if (yo < 0.0) v[Q_CONE] += yo * yo;
    if (kxo < 0.0) v[Q_ROWSQ] += kxo * kxo;
  }
  v[Q_QY] += q0 * yo;
  v[Q_YSQ] += yo * yo;
}

__device__ __forceinline__ void eval_row_avg(double yv, double kxv, double rs, double q0, bool eq, double *v) {
  const double yo = yv * rs, kxo = kxv / rs;
  if (eq) {
    const double d = kxo - q0;
    v[Q_A_PSQ] += d * d;
  } else {
    const double sf = q0 - kxo;
    if (sf > 0.0) v[Q_A_PSQ] += sf * sf;
  }
  v[Q_A_QY] += q0 * yo;
}

// Column j: current point terms (Kkt.evaluate columns, certificate columns).
__device__ __forceinline__ void eval_col(double xv, double ktv, double cs, double c0, double l0, double u0,
                                         double *v) {
  const double xo = xv * cs, kto = ktv / cs;
  const bool lfin = !(isinf(l0) && l0 < 0.0), ufin = !(isinf(u0) && u0 > 0.0);
  v[Q_CX] += c0 * xo;
  const double rc = c0 - kto;
  if (rc > 0.0) {
    if (!lfin) v[Q_DSQ] += rc * rc;
    else v[Q_DTERM] += l0 * rc;
  } else if (rc < 0.0) {
    if (!ufin) v[Q_DSQ] += rc * rc;
    else v[Q_DTERM] += u0 * rc;
  }
  const double pr = -kto;
  if (pr > 0.0) {
    if (!lfin) v[Q_PRSQ] += pr * pr;
    else v[Q_PVAL] += l0 * pr;
  } else if (pr < 0.0) {
    if (!ufin) v[Q_PRSQ] += pr * pr;
    else v[Q_PVAL] += u0 * pr;
  }
  v[Q_XSQ] += xo * xo;
  if ((xo > 0.0 && ufin) || (xo < 0.0 && lfin)) v[Q_BSQ] += xo * xo;
}

__device__ __forceinline__ void eval_col_avg(double xv, double ktv, double cs, double c0, double l0, double u0,
                                             double *v) {
  const double xo = xv * cs, kto = ktv / cs;
  v[Q_A_CX] += c0 * xo;
  const double rc = c0 - kto;
  if (rc > 0.0) {
    if (isinf(l0) && l0 < 0.0) v[Q_A_DSQ] += rc * rc;
    else v[Q_A_DTERM] += l0 * rc;
  } else if (rc < 0.0) {
    if (isinf(u0) && u0 > 0.0) v[Q_A_DSQ] += rc * rc;
    else v[Q_A_DTERM] += u0 * rc;
  }
}

// ---- phases --------------------------------------------------------------------

template <typename T>
__device__ void phase_init(const Args<T> &a, const Control &s, int nb, int rank) {
  double v[kMaxQ];
#pragma unroll
  for (int q = 0; q < kMaxQ; q++) v[q] = 0.0;
  int32_t lo, hi;
  chunk(a.n, nb, rank, lo, hi);
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    const T xj = ldv(a.x[0] + j);
    const T kt = row_dot(a.tp, a.tci, a.tv, (const T *)a.y[0], j);
    a.kty[j] = kt;
    a.xr[j] = xj;
    a.sx[j] = T(0);
    a.skty[j] = T(0);
    eval_col((double)xj, (double)kt, __ldg(a.cs + j), __ldg(a.c0 + j), __ldg(a.l0 + j), __ldg(a.u0 + j), v);
  }
  chunk(a.m, nb, rank, lo, hi);
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    const T yv = ldv(a.y[0] + r);
    const T kxv = row_dot(a.kp, a.kci, a.kv, (const T *)a.x[0], r);
    a.kx[0][r] = kxv;
    a.yr[r] = yv;
    a.sy[r] = T(0);
    a.skx[r] = T(0);
    eval_row((double)yv, (double)kxv, __ldg(a.rs + r), __ldg(a.q0 + r), r < a.neq, v);
  }
  block_partials<kMaxQ>(v, a.partials, a.max_blocks, rank);
}

// Primal half of a trial, fused with the pending commit's K'y.
template <typename T>
__device__ void phase_a(const Args<T> &a, const Control &s, int nb, int rank) {
  double v[1] = {0.0};
  int32_t lo, hi;
  chunk(a.n, nb, rank, lo, hi);
  const T tau = (T)s.tau, w = (T)s.pend_w;
  const T *x = a.x[s.xc];
  T *xn_out = a.x[s.xc ^ 1];
  const T *y = a.y[s.yc];
  const bool pend = s.pend != 0;
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    const T xj = ldv(x + j);
    T kt;
    if (pend) {
      kt = row_dot(a.tp, a.tci, a.tv, y, j);
      a.kty[j] = kt;
      a.sx[j] = (w * xj) + (T(1) * ldv(a.sx + j));
      a.skty[j] = (w * kt) + (T(1) * ldv(a.skty + j));
    } else {
      kt = ldv(a.kty + j);
    }
    // primalStep (ScalaKernels.scala:78-98), two-comparison clamp
    const T step = xj - (tau * (__ldg(a.c + j) - kt));
    const T lj = __ldg(a.l + j), uj = __ldg(a.u + j);
    const T xn = step < lj ? lj : (step > uj ? uj : step);
    xn_out[j] = xn;
    a.xbar[j] = (T(2) * xn) + (T(-1) * xj);
    const T d = (T(1) * xn) + (T(-1) * xj);
    v[0] += (double)d * (double)d;
  }
  block_partials<1>(v, a.partials + Q_DX * a.max_blocks, a.max_blocks, rank);
}

// Dual half of a trial: K xbar, dual step, speculative kx commit value.
template <typename T>
__device__ void phase_b(const Args<T> &a, const Control &s, int nb, int rank) {
  double v[2] = {0.0, 0.0};
  int32_t lo, hi;
  chunk(a.m, nb, rank, lo, hi);
  const T sigma = (T)s.sigma, w = (T)s.pend_w;
  const T *y = a.y[s.yc];
  const T *kx = a.kx[s.kxc];
  T *y_out = a.y[s.yc ^ 1];
  T *kx_out = a.kx[s.kxc ^ 1];
  const bool pend = s.pend != 0;
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    const T yr = ldv(y + r), kxr = ldv(kx + r);
    if (pend) {
      a.sy[r] = (w * yr) + (T(1) * ldv(a.sy + r));
      a.skx[r] = (w * kxr) + (T(1) * ldv(a.skx + r));
    }
    const T kb = row_dot(a.kp, a.kci, a.kv, (const T *)a.xbar, r);
    // dualStep (ScalaKernels.scala:100-118)
    T yn = yr + (sigma * (__ldg(a.q + r) - kb));
    if (r >= a.neq) yn = yn > T(0) ? yn : T(0);
    y_out[r] = yn;
    kx_out[r] = (T(0.5) * kb) + (T(0.5) * kxr);
    const T dy = (T(1) * yn) + (T(-1) * yr);
    const T kdx = (T(0.5) * kb) + (T(-0.5) * kxr);
    v[0] += (double)dy * (double)dy;
    v[1] += (double)dy * (double)kdx;
  }
  block_partials<2>(v, a.partials + Q_DY * a.max_blocks, a.max_blocks, rank);
}

// Flush the pending commit, optionally refresh kx = K x, evaluate.
template <typename T>
__device__ void phase_f(const Args<T> &a, const Control &s, int nb, int rank) {
  double v[kMaxQ];
#pragma unroll
  for (int q = 0; q < kMaxQ; q++) v[q] = 0.0;
  const T w = (T)s.pend_w, inv = (T)s.inv_w;
  const bool pend = s.pend != 0, fresh = s.f_mode != F_ITERLIMIT, avg = s.f_avg != 0;
  const T *x = a.x[s.xc];
  const T *y = a.y[s.yc];
  T *kx = a.kx[s.kxc];
  int32_t lo, hi;
  chunk(a.n, nb, rank, lo, hi);
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    const T xj = ldv(x + j);
    T kt;
    if (pend) {
      kt = row_dot(a.tp, a.tci, a.tv, y, j);
      a.kty[j] = kt;
      a.sx[j] = (w * xj) + (T(1) * ldv(a.sx + j));
      a.skty[j] = (w * kt) + (T(1) * ldv(a.skty + j));
    } else {
      kt = ldv(a.kty + j);
    }
    const double cs = __ldg(a.cs + j), c0 = __ldg(a.c0 + j), l0 = __ldg(a.l0 + j), u0 = __ldg(a.u0 + j);
    eval_col((double)xj, (double)kt, cs, c0, l0, u0, v);
    if (avg) {
      const T ax = inv * ldv(a.sx + j), akt = inv * ldv(a.skty + j);
      eval_col_avg((double)ax, (double)akt, cs, c0, l0, u0, v);
    }
  }
  chunk(a.m, nb, rank, lo, hi);
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    const T yr = ldv(y + r);
    T kxr = ldv(kx + r);
    if (pend) {
      a.sy[r] = (w * yr) + (T(1) * ldv(a.sy + r));
      a.skx[r] = (w * kxr) + (T(1) * ldv(a.skx + r));
    }
    if (fresh) {
      kxr = row_dot(a.kp, a.kci, a.kv, x, r);
      kx[r] = kxr;
    }
    const double rs = __ldg(a.rs + r), q0 = __ldg(a.q0 + r);
    eval_row((double)yr, (double)kxr, rs, q0, r < a.neq, v);
    if (avg) {
      const T ay = inv * ldv(a.sy + r), akx = inv * ldv(a.skx + r);
      eval_row_avg((double)ay, (double)akx, rs, q0, r < a.neq, v);
    }
  }
  block_partials<kMaxQ>(v, a.partials, a.max_blocks, rank);
}

// restartAt (Pdhg.scala:478-502): adopt the average if chosen, measure the
// distance travelled since the last restart, re-centre, reset the sums.
template <typename T>
__device__ void phase_r(const Args<T> &a, const Control &s, int nb, int rank) {
  double v[2] = {0.0, 0.0};
  const T inv = (T)s.inv_w;
  const bool avg = s.r_avg != 0;
  T *x = a.x[s.xc];
  T *y = a.y[s.yc];
  T *kx = a.kx[s.kxc];
  int32_t lo, hi;
  chunk(a.n, nb, rank, lo, hi);
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    T xj;
    if (avg) {
      xj = inv * ldv(a.sx + j);
      x[j] = xj;
      a.kty[j] = inv * ldv(a.skty + j);
    } else {
      xj = ldv(x + j);
    }
    const T d = (T(1) * xj) + (T(-1) * ldv(a.xr + j));
    v[0] += (double)d * (double)d;
    a.xr[j] = xj;
    a.sx[j] = T(0);
    a.skty[j] = T(0);
  }
  chunk(a.m, nb, rank, lo, hi);
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    T yr;
    if (avg) {
      yr = inv * ldv(a.sy + r);
      y[r] = yr;
      kx[r] = inv * ldv(a.skx + r);
    } else {
      yr = ldv(y + r);
    }
    const T d = (T(1) * yr) + (T(-1) * ldv(a.yr + r));
    v[1] += (double)d * (double)d;
    a.yr[r] = yr;
    a.sy[r] = T(0);
    a.skx[r] = T(0);
  }
  block_partials<2>(v, a.partials, a.max_blocks, rank);
}

// finish (Pdhg.scala:510-532): the evaluated point in the caller's units and
// the reduced costs c - K'y.
template <typename T>
__device__ void phase_w(const Args<T> &a, const Control &s, int nb, int rank) {
  const T inv = (T)s.inv_w;
  const bool avg = s.w_avg != 0;
  const T *x = a.x[s.xc];
  const T *y = a.y[s.yc];
  int32_t lo, hi;
  chunk(a.n, nb, rank, lo, hi);
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    const T xj = avg ? inv * ldv(a.sx + j) : ldv(x + j);
    const T kt = avg ? inv * ldv(a.skty + j) : ldv(a.kty + j);
    const double cs = __ldg(a.cs + j);
    a.xo[j] = (double)xj * cs;
    a.rco[j] = __ldg(a.c0 + j) - (double)kt / cs;
  }
  chunk(a.m, nb, rank, lo, hi);
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    const T yr = avg ? inv * ldv(a.sy + r) : ldv(y + r);
    a.yo[r] = (double)yr * __ldg(a.rs + r);
  }
}

// ---- decisions (deciding block; `red` is shared) ------------------------------

template <typename T>
__device__ void decide(const Args<T> &a, Control &c, int phase, int nb, double *red) {
  const Params &P = a.P;
  switch (phase) {
    case PH_INIT: {
      reduce_partials<kMaxQ>(a.partials, a.max_blocks, nb, 0, red);
      if (threadIdx.x == 0) {
        c.t0 = global_timer_ns();
        const Kkt e = kkt_current(red, P);
        if (converged(e, P)) {  // Pdhg.scala:211-212
          c.status = PRIMA_STATUS_OPTIMAL;
          c.final_kkt = e;
          c.current = e;
          c.w_avg = 0;
          c.phase = PH_W;
        } else {
          c.current = e;
          c.error_at_restart = weighted(e, c.weight);
          c.pend = 0;
          c.trials = 0;
          set_trial_scalars(c);
          c.phase = PH_A;
        }
      }
      break;
    }
    case PH_A: {
      if (threadIdx.x == 0) c.phase = PH_B;
      break;
    }
    case PH_B: {  // Solve.step's trial decision, Pdhg.scala:336-380
      reduce_partials<3>(a.partials, a.max_blocks, nb, 0, red);
      if (threadIdx.x == 0) {
        c.trials += 1;
        c.total_trials += 1;
        c.pend = 0;  // this trial's A/B consumed any pending commit
        const double dxsq = red[Q_DX], dysq = red[Q_DY];
        const double movement = 0.5 * (c.weight * dxsq + dysq / c.weight);
        if (movement == 0.0) {  // fixed point, Pdhg.scala:221-231
          c.iteration += 1;
          c.trials = 0;
          c.f_mode = F_FIXPOINT;
          c.f_avg = 0;
          c.phase = PH_F;
        } else {
          const double interaction = fabs(red[Q_INTER]);
          const double limit = interaction > 0.0 ? movement / interaction : CUDART_INF;
          const double t = (double)(c.iteration + 1);
          const double by_rule = (1.0 - pow(t, -0.3)) * limit;
          const double by_cap = (1.0 + pow(t, -0.6)) * c.step;
          const double proposed = dmin(by_rule, by_cap);
          const bool accept = c.step <= limit || c.trials >= 60;
          if (accept) {
            c.xc ^= 1;
            c.yc ^= 1;
            c.kxc ^= 1;
            c.pend = 1;
            c.pend_w = c.step;  // accumulate(stepSize) before the update
            c.weight_sum += c.step;
            c.iteration += 1;
            c.trials = 0;
          }
          if (isfinite(proposed) && proposed > 0.0) c.step = proposed;
          set_trial_scalars(c);
          c.phase = PH_A;
          if (accept) {
            if (c.iteration % P.eval_freq == 0) {
              c.f_mode = F_CHECKPOINT;
              c.f_avg = c.weight_sum > 0.0;
              c.inv_w = 1.0 / c.weight_sum;
              c.phase = PH_F;
            } else if (c.iteration >= P.max_iterations) {
              c.f_mode = F_ITERLIMIT;
              c.f_avg = 0;
              c.phase = PH_F;
            }
          }
        }
      }
      break;
    }
    case PH_F: {  // checkpoint (Pdhg.scala:396-417) and the terminal evaluations
      reduce_partials<kMaxQ>(a.partials, a.max_blocks, nb, 0, red);
      if (threadIdx.x == 0) {
        const Kkt cur = kkt_current(red, P);
        c.current = cur;
        c.pend = 0;
        if (c.f_mode == F_FIXPOINT) {
          c.status = converged(cur, P) ? PRIMA_STATUS_OPTIMAL : PRIMA_STATUS_NUMERICAL_ERROR;
          c.final_kkt = cur;
          c.w_avg = 0;
          c.phase = PH_W;
        } else if (c.f_mode == F_ITERLIMIT) {
          c.status = PRIMA_STATUS_ITERATION_LIMIT;
          c.final_kkt = cur;
          c.w_avg = 0;
          c.phase = PH_W;
        } else if (converged(cur, P)) {
          c.status = PRIMA_STATUS_OPTIMAL;
          c.final_kkt = cur;
          c.w_avg = 0;
          c.phase = PH_W;
        } else {
          const int cls = classify(red, P);
          if (cls >= 0) {
            c.status = cls;
            c.final_kkt = cur;
            c.w_avg = 0;
            c.phase = PH_W;
          } else {
            const double cur_err = weighted(cur, c.weight);
            double avg_err = CUDART_INF;
            bool done = false;
            if (c.f_avg) {
              const Kkt av = kkt_average(red, P);
              c.average = av;
              if (converged(av, P)) {
                c.status = PRIMA_STATUS_OPTIMAL;
                c.final_kkt = av;
                c.w_avg = 1;
                c.phase = PH_W;
                done = true;
              } else {
                avg_err = weighted(av, c.weight);
              }
            }
            if (!done) {
              const bool use_avg = avg_err < cur_err;
              const double cand = dmin(cur_err, avg_err);
              // shouldRestart, Pdhg.scala:463-469
              const bool sufficient = cand <= P.r_suff * c.error_at_restart;
              const bool necessary = cand <= P.r_nec * c.error_at_restart && cand > c.last_candidate;
              const bool artificial =
                  (double)(c.iteration - c.last_restart_it) >= P.r_art * (double)c.iteration;
              if (sufficient || necessary || artificial) {
                c.r_avg = use_avg;
                c.phase = PH_R;
              } else {
                c.last_candidate = cand;
                after_checkpoint(c, cur, P, a.cancel);
              }
            }
          }
        }
      }
      break;
    }
    case PH_R: {
      reduce_partials<2>(a.partials, a.max_blocks, nb, 0, red);
      if (threadIdx.x == 0) {
        const double pm = sqrt(red[Q_DXR]), dm = sqrt(red[Q_DYR]);
        if (pm > 0.0 && dm > 0.0) {
          const double th = P.smoothing;
          const double next = exp(th * log(dm / pm) + (1.0 - th) * log(c.weight));
          if (isfinite(next) && next > 0.0) c.weight = next;
        }
        c.weight_sum = 0.0;
        c.restarts += 1;
        c.last_restart_it = c.iteration;
        const Kkt point = c.r_avg ? c.average : c.current;
        c.current = point;
        c.error_at_restart = weighted(point, c.weight);
        c.last_candidate = CUDART_INF;
        set_trial_scalars(c);
        after_checkpoint(c, point, P, a.cancel);
      }
      break;
    }
    case PH_W: {
      if (threadIdx.x == 0) c.phase = PH_DONE;
      break;
    }
    default:
      if (threadIdx.x == 0) c.phase = PH_DONE;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) pdhg_kernel(Args<T> a) {
  __shared__ Control snap;
  const int nb = gridDim.x, rank = blockIdx.x;
  load_control(a, snap);
  for (;;) {
    const int ph = snap.phase;
    if (ph == PH_DONE) break;
    switch (ph) {
      case PH_INIT: phase_init(a, snap, nb, rank); break;
      case PH_A: phase_a(a, snap, nb, rank); break;
      case PH_B: phase_b(a, snap, nb, rank); break;
      case PH_F: phase_f(a, snap, nb, rank); break;
      case PH_R: phase_r(a, snap, nb, rank); break;
      case PH_W: phase_w(a, snap, nb, rank); break;
      default: break;
    }
    if (!barrier_decide(a, snap, ph, nb)) break;
    load_control(a, snap);
  }
}

}  // namespace dev

// ============================================================================
// host side
// ============================================================================

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

// Bump allocator over the context's solver arena.
struct Layout {
  size_t off = 0;
  template <typename U>
  size_t take(int64_t count) {
    const size_t at = off;
    off += ((size_t)std::max<int64_t>(count, 1) * sizeof(U) + 255) & ~(size_t)255;
    return at;
  }
};

template <typename T>
struct SolveBuffers {
  dev::Args<T> args;
  size_t bytes = 0;
  // offsets
  size_t o_kp, o_kci, o_kv, o_tp, o_tci, o_tv, o_c, o_q, o_l, o_u, o_c0, o_q0, o_l0, o_u0, o_cs, o_rs;
  size_t o_x[2], o_y[2], o_kx[2], o_xbar, o_kty, o_sx, o_sy, o_skx, o_skty, o_xr, o_yr, o_xo, o_yo, o_rco;
  size_t o_part, o_ctl, o_sync;
};

template <typename T>
void plan(SolveBuffers<T> &b, int32_t n, int32_t m, int64_t nnz, int max_blocks) {
  Layout L;
  b.o_kp = L.take<int32_t>((int64_t)m + 1);
  b.o_kci = L.take<int32_t>(nnz);
  b.o_kv = L.take<T>(nnz);
  b.o_tp = L.take<int32_t>((int64_t)n + 1);
  b.o_tci = L.take<int32_t>(nnz);
  b.o_tv = L.take<T>(nnz);
  b.o_c = L.take<T>(n);
  b.o_l = L.take<T>(n);
  b.o_u = L.take<T>(n);
  b.o_q = L.take<T>(m);
  b.o_c0 = L.take<double>(n);
  b.o_l0 = L.take<double>(n);
  b.o_u0 = L.take<double>(n);
  b.o_cs = L.take<double>(n);
  b.o_q0 = L.take<double>(m);
  b.o_rs = L.take<double>(m);
  for (int i = 0; i < 2; i++) {
    b.o_x[i] = L.take<T>(n);
    b.o_y[i] = L.take<T>(m);
    b.o_kx[i] = L.take<T>(m);
  }
  b.o_xbar = L.take<T>(n);
  b.o_kty = L.take<T>(n);
  b.o_sx = L.take<T>(n);
  b.o_skty = L.take<T>(n);
  b.o_xr = L.take<T>(n);
  b.o_sy = L.take<T>(m);
  b.o_skx = L.take<T>(m);
  b.o_yr = L.take<T>(m);
  b.o_xo = L.take<double>(n);
  b.o_rco = L.take<double>(n);
  b.o_yo = L.take<double>(m);
  b.o_part = L.take<double>((int64_t)dev::kMaxQ * max_blocks);
  b.o_ctl = L.take<dev::Control>(1);
  b.o_sync = L.take<dev::Sync>(1);
  b.bytes = L.off;
}

template <typename T>
void bind(SolveBuffers<T> &b, char *base, int32_t n, int32_t m, int32_t neq, int max_blocks) {
  dev::Args<T> &a = b.args;
  std::memset(&a, 0, sizeof(a));
  a.n = n;
  a.m = m;
  a.neq = neq;
  a.kp = (const int32_t *)(base + b.o_kp);
  a.kci = (const int32_t *)(base + b.o_kci);
  a.kv = (const T *)(base + b.o_kv);
  a.tp = (const int32_t *)(base + b.o_tp);
  a.tci = (const int32_t *)(base + b.o_tci);
  a.tv = (const T *)(base + b.o_tv);
  a.c = (const T *)(base + b.o_c);
  a.q = (const T *)(base + b.o_q);
  a.l = (const T *)(base + b.o_l);
  a.u = (const T *)(base + b.o_u);
  a.c0 = (const double *)(base + b.o_c0);
  a.q0 = (const double *)(base + b.o_q0);
  a.l0 = (const double *)(base + b.o_l0);
  a.u0 = (const double *)(base + b.o_u0);
  a.cs = (const double *)(base + b.o_cs);
  a.rs = (const double *)(base + b.o_rs);
  for (int i = 0; i < 2; i++) {
    a.x[i] = (T *)(base + b.o_x[i]);
    a.y[i] = (T *)(base + b.o_y[i]);
    a.kx[i] = (T *)(base + b.o_kx[i]);
  }
  a.xbar = (T *)(base + b.o_xbar);
  a.kty = (T *)(base + b.o_kty);
  a.sx = (T *)(base + b.o_sx);
  a.sy = (T *)(base + b.o_sy);
  a.skx = (T *)(base + b.o_skx);
  a.skty = (T *)(base + b.o_skty);
  a.xr = (T *)(base + b.o_xr);
  a.yr = (T *)(base + b.o_yr);
  a.xo = (double *)(base + b.o_xo);
  a.yo = (double *)(base + b.o_yo);
  a.rco = (double *)(base + b.o_rco);
  a.partials = (double *)(base + b.o_part);
  a.max_blocks = max_blocks;
  a.ctl = (dev::Control *)(base + b.o_ctl);
  a.sync = (dev::Sync *)(base + b.o_sync);
}

template <typename T>
std::vector<T> narrow(const std::vector<double> &v) {
  std::vector<T> out(v.size());
  for (size_t i = 0; i < v.size(); i++) out[i] = (T)v[i];
  return out;
}

template <typename T>
int32_t h2d(void *dst, const T *src, size_t count, cudaStream_t s) {
  if (count == 0) return PRIMA_OK;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
  return PRIMA_OK;
}

struct SolveRequest {
  const prima_lp *lp;
  const prima_params *params;
  const prima_warm_start *warm;
  const volatile int32_t *cancel;
  double *x_out, *y_out, *rc_out;
  prima_solution_info *info;
};

template <typename T>
int32_t max_coresident_blocks(Ctx *c, int *out) {
  int per_sm = 0;
  PRIMA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::pdhg_kernel<T>, dev::kThreads, 0));
  if (per_sm < 1) {
    set_error("solver kernel cannot be resident on an SM");
    return PRIMA_ERR_CUDA;
  }
  *out = per_sm * c->num_sms;
  return PRIMA_OK;
}

// Pdhg.Solve: setup (Solve.<init> + initialise, Pdhg.scala:131-309) on the
// host, then the whole iteration in one cooperative launch.
template <typename T>
int32_t solve_on_device(Ctx *c, const SolveRequest &req) {
  const auto t_start = Clock::now();
  const prima_lp *lp = req.lp;
  const prima_params *p = req.params;
  int32_t rc;
  if ((rc = validate_params(p)) || (rc = validate_lp(lp))) return rc;
  const int32_t n = lp->num_variables, m = lp->num_constraints, neq = lp->num_equalities;
  if (req.warm) {
    if (!req.warm->primal) return (set_error("requirement failed: warm start primal is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
    for (int32_t i = 0; i < n; i++)
      if (!std::isfinite(req.warm->primal[i]))
        return (set_error("requirement failed: warm start primal vector is not finite"), PRIMA_ERR_INVALID_ARGUMENT);
    if (m > 0 && !req.warm->dual) return (set_error("requirement failed: warm start dual is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
    for (int32_t r = 0; r < m; r++)
      if (!std::isfinite(req.warm->dual[r]))
        return (set_error("requirement failed: warm start dual vector is not finite"), PRIMA_ERR_INVALID_ARGUMENT);
  }
  ScaledLp S;
  prepare_scaled(lp, p, &S);
  const int64_t nnz = S.K.nnz();

  // initialise (Pdhg.scala:250-309)
  const double bound = S.scaled_spectral_bound;
  double step = bound > 0.0 ? 1.0 / bound : 1.0;
  double weight = (S.scaled_c_norm > 0.0 && S.scaled_q_norm > 0.0) ? S.scaled_c_norm / S.scaled_q_norm : 1.0;
  if (req.warm && !std::isnan(req.warm->step_size)) step = req.warm->step_size;
  if (req.warm && !std::isnan(req.warm->primal_weight)) weight = req.warm->primal_weight;
  std::vector<double> x0((size_t)n, 0.0), y0((size_t)m, 0.0);
  if (req.warm)
    for (int32_t i = 0; i < n; i++) x0[i] = req.warm->primal[i] / S.col_scale[i];
  for (int32_t i = 0; i < n; i++) {
    const double lo = S.l[i], hi = S.u[i], v = x0[i];
    x0[i] = v < lo ? lo : (v > hi ? hi : v);
  }
  if (req.warm)
    for (int32_t r = 0; r < m; r++) {
      const double v = req.warm->dual[r] / S.row_scale[r];
      y0[r] = (r >= neq && v < 0.0) ? 0.0 : v;
    }

  int max_blocks = 0;
  if ((rc = max_coresident_blocks<T>(c, &max_blocks))) return rc;
  const int64_t work = std::max<int64_t>(std::max(n, m), 1);
  const int blocks = (int)std::min<int64_t>(max_blocks, std::max<int64_t>(1, (work + dev::kThreads - 1) / dev::kThreads));

  SolveBuffers<T> B;
  plan<T>(B, n, m, nnz, blocks);
  if ((rc = c->solver_arena.reserve(B.bytes))) return rc;
  char *base = (char *)c->solver_arena.ptr;
  bind<T>(B, base, n, m, neq, blocks);
  cudaStream_t s = c->stream;

  const std::vector<T> kv = narrow<T>(S.K.vals), tv = narrow<T>(S.Kt.vals);
  const std::vector<T> cc = narrow<T>(S.c), qq = narrow<T>(S.q), ll = narrow<T>(S.l), uu = narrow<T>(S.u);
  const std::vector<T> xx = narrow<T>(x0), yy = narrow<T>(y0);
  if ((rc = h2d(base + B.o_kp, S.K.row_ptr.data(), (size_t)m + 1, s)) || (rc = h2d(base + B.o_kci, S.K.col_idx.data(), nnz, s)) ||
      (rc = h2d(base + B.o_kv, kv.data(), nnz, s)) || (rc = h2d(base + B.o_tp, S.Kt.row_ptr.data(), (size_t)n + 1, s)) ||
      (rc = h2d(base + B.o_tci, S.Kt.col_idx.data(), nnz, s)) || (rc = h2d(base + B.o_tv, tv.data(), nnz, s)) ||
      (rc = h2d(base + B.o_c, cc.data(), n, s)) || (rc = h2d(base + B.o_q, qq.data(), m, s)) ||
      (rc = h2d(base + B.o_l, ll.data(), n, s)) || (rc = h2d(base + B.o_u, uu.data(), n, s)) ||
      (rc = h2d(base + B.o_c0, lp->objective, n, s)) || (rc = h2d(base + B.o_q0, lp->rhs, m, s)) ||
      (rc = h2d(base + B.o_l0, lp->lower, n, s)) || (rc = h2d(base + B.o_u0, lp->upper, n, s)) ||
      (rc = h2d(base + B.o_cs, S.col_scale.data(), n, s)) || (rc = h2d(base + B.o_rs, S.row_scale.data(), m, s)) ||
      (rc = h2d(base + B.o_x[0], xx.data(), n, s)) || (rc = h2d(base + B.o_y[0], yy.data(), m, s)))
    return rc;

  dev::Control ctl;
  std::memset(&ctl, 0, sizeof(ctl));
  ctl.phase = dev::PH_INIT;
  ctl.status = -1;
  ctl.step = step;
  ctl.weight = weight;
  ctl.error_at_restart = std::numeric_limits<double>::infinity();
  ctl.last_candidate = std::numeric_limits<double>::infinity();
  ctl.tau = step / weight;
  ctl.sigma = step * weight;
  dev::Sync sync;
  std::memset(&sync, 0, sizeof(sync));
  if ((rc = h2d(base + B.o_ctl, &ctl, 1, s)) || (rc = h2d(base + B.o_sync, &sync, 1, s))) return rc;

  dev::Params &P = B.args.P;
  P.eps_abs = p->eps_abs;
  P.eps_rel = p->eps_rel;
  P.rhs_norm = S.rhs_norm;
  P.obj_norm = S.obj_norm;
  P.max_iterations = p->max_iterations;
  P.eval_freq = p->evaluation_frequency;
  P.time_limit_ms = p->time_limit_ms;
  P.infeas_tol = p->infeasibility_tolerance;
  P.r_suff = p->restart_sufficient_reduction;
  P.r_nec = p->restart_necessary_reduction;
  P.r_art = p->restart_artificial_fraction;
  P.smoothing = p->primal_weight_smoothing;
  P.matrix_norm = S.orig_spectral_bound;
  P.offset = lp->objective_offset;
  *c->cancel_mapped = (req.cancel && *req.cancel) ? 1 : 0;
  B.args.cancel = c->cancel_mapped_dev;
  PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  const double setup_ms = ms_since(t_start);
  P.setup_ms = setup_ms;

  cudaEvent_t e0, e1;
  PRIMA_CUDA_TRY(cudaEventCreate(&e0));
  PRIMA_CUDA_TRY(cudaEventCreate(&e1));
  void *kargs[] = {(void *)&B.args};
  PRIMA_CUDA_TRY(cudaEventRecord(e0, s));
  cudaError_t le = cudaLaunchCooperativeKernel((const void *)dev::pdhg_kernel<T>, dim3(blocks), dim3(dev::kThreads),
                                               kargs, 0, s);
  if (le != cudaSuccess) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    set_error(std::string("cooperative launch: ") + cudaGetErrorString(le));
    return PRIMA_ERR_CUDA;
  }
  PRIMA_CUDA_TRY(cudaEventRecord(e1, s));
  // Wait; while waiting, forward the caller's cancel flag to the mapped flag
  // the device polls at evaluation points.
  for (;;) {
    const cudaError_t q = cudaEventQuery(e1);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) {
      set_error(std::string("solver kernel: ") + cudaGetErrorString(q));
      return PRIMA_ERR_CUDA;
    }
    if (req.cancel && *req.cancel) *(volatile int32_t *)c->cancel_mapped = 1;
    std::this_thread::sleep_for(std::chrono::microseconds(req.cancel ? 50 : 10));
  }
  float kms = 0.f;
  cudaEventElapsedTime(&kms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PRIMA_CUDA_TRY(cudaMemcpy(&ctl, base + B.o_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  PRIMA_CUDA_TRY(cudaMemcpy(&sync, base + B.o_sync, sizeof(sync), cudaMemcpyDeviceToHost));
  if (sync.abort) ctl.error = PRIMA_ERR_TIMEOUT;
  if (req.x_out && n) PRIMA_CUDA_TRY(cudaMemcpy(req.x_out, base + B.o_xo, (size_t)n * 8, cudaMemcpyDeviceToHost));
  if (req.y_out && m) PRIMA_CUDA_TRY(cudaMemcpy(req.y_out, base + B.o_yo, (size_t)m * 8, cudaMemcpyDeviceToHost));
  if (req.rc_out && n) PRIMA_CUDA_TRY(cudaMemcpy(req.rc_out, base + B.o_rco, (size_t)n * 8, cudaMemcpyDeviceToHost));
  prima_solution_info *info = req.info;
  std::memset(info, 0, sizeof(*info));
  info->status = ctl.status;
  info->iterations = ctl.iteration;
  info->restarts = ctl.restarts;
  info->device_error = ctl.error;
  info->objective = ctl.final_kkt.pobj;
  info->dual_objective = ctl.final_kkt.dobj;
  info->primal_residual = ctl.final_kkt.pres;
  info->dual_residual = ctl.final_kkt.dres;
  info->final_step_size = ctl.step;
  info->final_primal_weight = ctl.weight;
  info->device_ms = kms;
  info->setup_ms = setup_ms;
  info->trials = ctl.total_trials;
  info->solve_ms = (int64_t)ms_since(t_start);
  if (ctl.error) {
    set_error("a bounded device-side wait gave up; the solve was abandoned");
    return PRIMA_ERR_TIMEOUT;
  }
  return PRIMA_OK;
}

int32_t dispatch_solve(Ctx *c, const SolveRequest &req, int bits) {
  if (!req.info) return (set_error("requirement failed: info is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  return bits == 64 ? solve_on_device<double>(c, req) : solve_on_device<float>(c, req);
}

}  // namespace
}  // namespace prima

using namespace prima;

extern "C" int32_t prima_pdhg_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                                    const prima_warm_start *warm, const volatile int32_t *cancel, double *x_out,
                                    double *y_out, double *rc_out, prima_solution_info *info) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(ctx, &rc);
  if (!c) return rc;
  cudaSetDevice(c->device);
  SolveRequest req{lp, params, warm, cancel, x_out, y_out, rc_out, info};
  return dispatch_solve(c, req, c->bits);
}

extern "C" int32_t prima_mixed_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                                     const prima_mixed_params *mixed, const volatile int32_t *cancel,
                                     double *x_out, double *y_out, double *rc_out, prima_solution_info *info,
                                     prima_mixed_info *minfo) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(ctx, &rc);
  if (!c) return rc;
  cudaSetDevice(c->device);
  set_error("prima_mixed_solve: not built yet");
  return PRIMA_ERR_INVALID_ARGUMENT;
}

extern "C" int32_t prima_pdhg_solve_batch(prima_handle ctx, int32_t count, const prima_lp *lps,
                                          const prima_params *params, const volatile int32_t *cancel,
                                          double *const *x_out, double *const *y_out, double *const *rc_out,
                                          prima_solution_info *infos) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(ctx, &rc);
  if (!c) return rc;
  cudaSetDevice(c->device);
  set_error("prima_pdhg_solve_batch: not built yet");
  return PRIMA_ERR_INVALID_ARGUMENT;
}
