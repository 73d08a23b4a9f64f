// Internal declarations shared by the translation units of libprima_cuda.so.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "prima_cuda.h"
#include "prima_tiles.h"

namespace prima {

// ---- errors -----------------------------------------------------------------
void set_error(const std::string &msg);
void clear_error();

struct Error {
  int32_t code;
  std::string msg;
};

#define PRIMA_CUDA_TRY(expr)                                                            \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) {                                                            \
      ::prima::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));           \
      return _e == cudaErrorMemoryAllocation ? PRIMA_ERR_OUT_OF_MEMORY : PRIMA_ERR_CUDA; \
    }                                                                                   \
  } while (0)

// ---- device buffers ---------------------------------------------------------
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer();
  int32_t reserve(size_t b);  // grows, never shrinks; contents not preserved
  void release();
};

// A seam vector: n elements of the context's storage precision.
struct Vec {
  int64_t n = 0;
  DeviceBuffer buf;
};

// A seam matrix: CSR with values in the context's precision.
struct Mat {
  int32_t rows = 0, cols = 0;
  int64_t nnz = 0;
  DeviceBuffer row_ptr, col_idx, vals;
  int32_t lanes = 0;  // SpMV kernel picked by the autotuner (0: CSR-stream tiles, 1: thread per row)
};

struct LpHostCopy;

// A problem resident on the device: the original CSR and data, the
// materialised transpose (as a permutation), the equilibrated matrix and
// vectors in FP64, and per-precision copies for the solver.  Built once per
// problem (prima_scaling.cu) and reused by every pass over it.
struct PreparedLp {
  int32_t n = 0, m = 0, neq = 0;
  int64_t nnz = 0;
  int32_t ruiz = -1, pc = -1;
  double alpha = -1.0;
  DeviceBuffer b_kp, b_kci, b_kv0, b_kv, b_tp, b_tci, b_perm;
  DeviceBuffer b_c0, b_l0, b_u0, b_q0, b_cs, b_rs, b_sc, b_sl, b_su, b_sq;
  struct PrecisionCopy {
    DeviceBuffer kv, tv, c, l, u, q;
  } copies[2];  // [0]: float, [1]: double
  bool precision_ready[2] = {false, false};
  double orig_spectral_bound = 0, scaled_spectral_bound = 0, rhs_norm = 0, obj_norm = 0;
  double scaled_c_norm = 0, scaled_q_norm = 0;
  std::vector<double> h_sc, h_sq, h_sl, h_su, h_cs, h_rs;  // host copies for warm starts
  std::vector<int32_t> h_kp, h_tp;                       // row pointers of K and K'
  // hot-phase tiles per [precision][row cap: 512, 256][K, K']: the host
  // table (first row, first nonzero; closed by rows, nnz), each tile's cost
  // estimate, and on the device the tiles as (start, end) pairs in the order
  // that hands them to a team of tiles_nb blocks (slot rank + k*nb is block
  // rank's k-th tile)
  std::vector<TileEdge> h_tiles[2][2][2];
  std::vector<float> h_tile_cost[2][2][2];
  DeviceBuffer b_tiles[2][2][2];
  int32_t ntiles[2][2][2] = {};
  int32_t tiles_nb[2][2] = {};
  // the solver layout chosen for this problem per precision (0: not yet):
  // blocks per SM, and the tile table's row cap (index into b_tiles)
  int32_t layout_bps[2] = {0, 0}, layout_rows[2] = {0, 0};
  std::unique_ptr<LpHostCopy> owned;  // the caller's problem, when held by a handle
  const prima_lp *host = nullptr;     // the caller's problem (valid while in use)

  const int32_t *kp() const { return (const int32_t *)b_kp.ptr; }
  const int32_t *kci() const { return (const int32_t *)b_kci.ptr; }
  const double *kv0() const { return (const double *)b_kv0.ptr; }
  double *kv() const { return (double *)b_kv.ptr; }
  const int32_t *tp() const { return (const int32_t *)b_tp.ptr; }
  const int32_t *tci() const { return (const int32_t *)b_tci.ptr; }
  const int32_t *perm() const { return (const int32_t *)b_perm.ptr; }
  const double *c0() const { return (const double *)b_c0.ptr; }
  const double *l0() const { return (const double *)b_l0.ptr; }
  const double *u0() const { return (const double *)b_u0.ptr; }
  const double *q0() const { return (const double *)b_q0.ptr; }
  const double *cs() const { return (const double *)b_cs.ptr; }
  const double *rs() const { return (const double *)b_rs.ptr; }
  double *cs_() const { return (double *)b_cs.ptr; }
  double *rs_() const { return (double *)b_rs.ptr; }
  const double *sc() const { return (const double *)b_sc.ptr; }
  const double *sl() const { return (const double *)b_sl.ptr; }
  const double *su() const { return (const double *)b_su.ptr; }
  const double *sq() const { return (const double *)b_sq.ptr; }
  double *sc_() const { return (double *)b_sc.ptr; }
  double *sl_() const { return (double *)b_sl.ptr; }
  double *su_() const { return (double *)b_su.ptr; }
  double *sq_() const { return (double *)b_sq.ptr; }
  bool scaled_like(const prima_params *p) const {
    return ruiz == p->ruiz_iterations && pc == p->apply_pock_chambolle && alpha == p->pock_chambolle_alpha;
  }
  int32_t prepare(const prima_lp *lp, const prima_params *p, cudaStream_t s);
  template <typename T>
  int32_t materialise(cudaStream_t s);
  // New variable bounds for the prepared problem: the scaling depends on the
  // matrix alone, so only the bounds' scaled and storage-type copies change.
  int32_t set_bounds(const double *lower, const double *upper, cudaStream_t s);
};

// Owned host copy of a problem (for problem handles).
struct LpHostCopy {
  std::vector<int32_t> row_ptr, col_idx;
  std::vector<double> values, objective, rhs, lower, upper;
  prima_lp lp;
};

struct Ctx {
  int32_t device = 0;
  int32_t bits = 64;
  bool closed = false;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  std::string device_name;
  int64_t next_id = 1;
  std::unordered_map<int64_t, std::unique_ptr<Vec>> vecs;
  std::unordered_map<int64_t, std::unique_ptr<Mat>> mats;
  DeviceBuffer scratch;        // reduction partials and staging for the seam ops
  double *host_scalar = nullptr;  // pinned: reduction results
  int32_t *cancel_mapped = nullptr;  // pinned + mapped: cancel flag seen by the device
  int32_t *cancel_mapped_dev = nullptr;
  int64_t wait_limit = 0;      // team-barrier polls before a block gives up (0: the default)
  int32_t pin_bps = 0, pin_rows = 0;  // a solver layout the caller pinned (0: chosen by timing)
  DeviceBuffer solver_arena;   // buffers of the coarse solvers, reused across solves
  DeviceBuffer batch_arena;    // state, arguments and queue of a batch launch
  PreparedLp scratch_lp;       // the problem of a one-shot solve call
  std::unordered_map<int64_t, std::unique_ptr<PreparedLp>> problems;
};

// Registry lookup (thread-safe); returns nullptr and sets the error on failure.
Ctx *lookup_ctx(prima_handle h, int32_t *code);

// ---- host-side problem preparation (prima_host.cpp) -----------------------
struct Csr {
  int32_t rows = 0, cols = 0;
  std::vector<int32_t> row_ptr;
  std::vector<int32_t> col_idx;
  std::vector<double> vals;
  int64_t nnz() const { return rows ? row_ptr[rows] : 0; }
};

// The equilibrated problem and the diagonals that undo it (Scaling.scala:32-61).
struct ScaledLp {
  int32_t n = 0, m = 0, neq = 0;
  Csr K, Kt;  // scaled matrix and its materialised transpose
  std::vector<double> c, q, l, u;
  std::vector<double> row_scale, col_scale;
  double scaled_spectral_bound = 0.0;  // opening step: 1 / bound
  double orig_spectral_bound = 0.0;    // certificate normalisation
  double rhs_norm = 0.0, obj_norm = 0.0;  // norms of the original q and c
  double scaled_c_norm = 0.0, scaled_q_norm = 0.0;
};

// LpProblem.apply's requirements (LpProblem.scala:62-104) plus CSR sanity.
int32_t validate_lp(const prima_lp *lp);
// PdhgParams / ScalingParams requirements (PdhgParams.scala:55-79).
int32_t validate_params(const prima_params *p);
// Scaling.apply (Scaling.scala:77-155) + transpose + norms, on the host.
void prepare_scaled(const prima_lp *lp, const prima_params *p, ScaledLp *out);
void csr_transpose(const Csr &a, Csr *t);
double csr_norm_inf(const Csr &a);
double spectral_norm_bound(const Csr &a, const Csr &at);

// Certificates.classify (Certificates.scala:207-219) in FP64 on the host,
// recomputing Kx and K'y from the original matrix (the re-check
// MixedPrecision.scala:143-152 performs).  Returns a PRIMA_STATUS_* or -1.
int classify_fp64(const prima_lp *lp, const double *x, const double *y, double tolerance);

// ---- SpMV helpers for the seam (prima_ops.cu) ------------------------------
int32_t seam_spmv(Ctx *ctx, const Mat *a, const void *x, void *out);

}  // namespace prima
