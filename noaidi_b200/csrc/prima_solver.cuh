// Fused, persistent restarted-PDHG solver (device side).
//
// One cooperative launch runs a whole solve: the iteration, the adaptive
// step-size rule, the checkpoint evaluation (FP64 KKT + Farkas certificates),
// restarts and termination -- Pdhg.Solve (core/Pdhg.scala:123-534) with the
// host loop moved onto the GPU.  Blocks of a team step through phases
// separated by team barriers; at each barrier the LAST block to arrive reduces
// the phase's per-block partial sums (a fixed tree: deterministic) and runs
// the scalar tail of the algorithm, then publishes the next phase in a
// Control record every block reads.  No host round trip per iteration.
//
// Phases and what each fuses (rows r of K over m, columns j over n):
//   INIT  kx = K x0, kty = K'y0, restart points, zero sums, KKT of the start
//   A     [pending commit: kty = K'y_new, sumX/sumKtY += w*(x, kty)]
//         x' = clamp(x - tau(c - kty)), xbar = 2x' - x, sum (x'-x)^2
//   B     [pending commit: sumY/sumKx += w*(y, kx)]
//         kxbar = K xbar, y' = proj(y + sigma(q - kxbar)), kx' = (kxbar+kx)/2,
//         sum (y'-y)^2, sum (y'-y).(kxbar-kx)/2
//   F     flush pending commit, optional fresh kx = K x, FP64 KKT of the
//         current point and of the running average, certificate terms
//   R     restart: optionally adopt the average, |x - xr|, |y - yr|, reset
//   W     write the solution in the caller's units (FP64)
// A/B form one step-size trial; an accepted trial commits by flipping the
// double-buffered x, y, kx (no copies) and leaves the K'y product and the
// running-sum updates pending for the next A/B (or F) pass, which reads the
// same vectors anyway.
//
// Element arithmetic is exactly the reference kernel expressions in the
// storage type T (double: ScalaKernels; float: Float32Kernels), built with
// --fmad=false; every row of K and K' is summed in index order from zero, so
// a double-precision team reproduces the reference's SpMV bit for bit.
// Reductions are in double, in a fixed tree order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace prima {
namespace dev {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Blocks per SM the solver kernel is compiled for (its register budget):
// three in FP32 (80 registers), two in FP64 (128), each thread owning two
// rows of a tile -- measured faster than four blocks at 64 registers, where
// the cold phases spilled and each thread had one row's gathers in flight.
#ifndef PRIMA_MIN_BLOCKS_F32
#define PRIMA_MIN_BLOCKS_F32 3
#endif
#ifndef PRIMA_MIN_BLOCKS_F64
#define PRIMA_MIN_BLOCKS_F64 2
#endif
template <typename T>
constexpr int kMinBlocksPerSm = sizeof(T) == 4 ? PRIMA_MIN_BLOCKS_F32 : PRIMA_MIN_BLOCKS_F64;
constexpr int kTileRows = 512;      // rows of one CSR-stream tile (2 per thread)
constexpr int kRowsPerThread = kTileRows / kThreads;
constexpr int kTileCap = 4096;      // staged products per tile (dynamic shared memory)
constexpr int kMaxQ = 17;
// Global block partials: slots [0, kMaxQ) for the cold phases, then two
// banks of kHotQ slots for the trial (phase A: DX, phase B: DY, INTER), used
// by alternate trials so that a block still reading one trial's partials is
// never overwritten by a faster block already in the next trial.
constexpr int kHotQ = 3;
constexpr int kSlots = kMaxQ + 2 * kHotQ;
__host__ __device__ constexpr int hot_bank(int64_t trial) { return kMaxQ + (int)(trial & 1) * kHotQ; }

enum : int { PH_INIT = 0, PH_A = 1, PH_B = 2, PH_F = 3, PH_R = 4, PH_W = 5, PH_DONE = 6, PH_R2 = 7 };
enum : int { F_FIXPOINT = 0, F_CHECKPOINT = 1, F_ITERLIMIT = 2 };

// Reduction slots.  Trial: A writes DX, B writes DY and INTER.  Evaluation:
// the row terms (slots 0-6) and the column terms (slots 7-16), each reduced
// right after its loop so at most ten accumulators are live.  Restart: DXR, DYR.
enum : int { Q_DX = 0, Q_DY = 1, Q_INTER = 2 };
enum : int {
  Q_PSQ = 0,   // primal residual^2                                (rows)
  Q_QY,        // q'y                                               (rows)
  Q_YSQ,       // |y|^2, primal certificate                         (rows)
  Q_CONE,      // dual-cone violation^2, primal certificate         (rows)
  Q_ROWSQ,     // Kx row violation^2, dual certificate              (rows)
  Q_A_PSQ,     // primal residual^2 of the running average          (rows)
  Q_A_QY,      // q'y of the running average                        (rows)
  Q_CX,        // c'x                                               (cols)
  Q_DTERM,     // bound terms of the dual objective                 (cols)
  Q_DSQ,       // dual residual^2                                   (cols)
  Q_PVAL,      // bound terms of the primal certificate value       (cols)
  Q_PRSQ,      // unabsorbed reduced cost^2, primal certificate     (cols)
  Q_XSQ,       // |x|^2, dual certificate                           (cols)
  Q_BSQ,       // bound violation^2, dual certificate               (cols)
  Q_A_CX,      // the same KKT terms for the running average        (cols)
  Q_A_DTERM,
  Q_A_DSQ,
  Q_EVAL_N
};
constexpr int kRowQ = Q_CX;             // slots [0, 7)
constexpr int kColQ = Q_EVAL_N - Q_CX;  // slots [7, 17)
enum : int { Q_DXR = 0, Q_DYR = 1 };
static_assert(Q_EVAL_N == kMaxQ, "slot count");

struct Kkt {
  double pres, dres, pobj, dobj;
};

struct Params {
  double eps_abs, eps_rel, rhs_norm, obj_norm;
  int32_t max_iterations, eval_freq;
  double time_limit_ms, setup_ms;
  double infeas_tol, r_suff, r_nec, r_art, smoothing;
  double matrix_norm;  // spectral bound of the ORIGINAL matrix (certificates)
  double offset;
  double round_rho;  // anchored mode: a checkpoint this far below the round's start error opens a new round
  long long spin_limit;  // team-barrier polls before a block gives up and raises the abort flag
};

// Published by the deciding block at every barrier.
struct Control {
  int32_t phase, f_mode, f_avg, r_avg;
  int32_t w_avg, pend, xc, yc;
  int32_t kxc, status, iteration, restarts;
  int32_t last_restart_it, trials, error, period_base;
  int64_t total_trials;
  uint64_t t0;
  double step, weight, weight_sum, pend_w;
  double inv_w, tau, sigma, error_at_restart;
  double last_candidate, round_err;
  int32_t rounds, pad3;
  uint64_t t_end;  // global timer when the solve finished (with t0: its device time)
  Kkt current, average, final_kkt;
};

// Hot barriers count arrivals in two levels, so that no one address takes
// every block's atomic: block `rank` counts itself in on group rank % G's
// counter, and the last block of each group on the team's counter.
constexpr int kArriveGroups = 32;     // G, at most
constexpr int kArriveStride = 16;     // counters 128 bytes apart (u64 words)

struct Sync {
  unsigned int count;   // cold barriers: arrivals so far (reset by the deciding block)
  unsigned int gen;     // cold barriers: released generations
  int32_t abort;
  int32_t pad;
  unsigned long long arrive;  // hot barriers: groups complete so far in the solve, never reset
  int32_t diag[8];            // where a bounded stage wait gave up (zero: none did)
};

constexpr int kProfBlocks = 1024;  // blocks whose own arrival times the phase record keeps

// Phase timing, kept by whichever block decides (one at a time): time from a
// barrier's release to the last block's arrival at the next one, per phase
// kind, and the deciding block's own time.  Only kept when asked for
// (PRIMA_PHASE_TIMES): its read-modify-writes sit on the deciding thread's
// path, and each one costs an L2 round trip while the team waits.
struct Prof {
  uint64_t t_release;
  uint64_t decide_ns;
  uint64_t phase_ns[8];
  int64_t phase_count[8];
  // the trial decision after phase B: all of it, and its partial reduction
  uint64_t decide_b_ns, reduce_b_ns;
  int64_t decide_b_count;
  uint64_t arrive_ns[8];  // every block's arrival after the release, summed
  // per block: arrival after the release in phases A and B, summed over the
  // trials, and the SM the block runs on (is the spread systematic?)
  uint64_t block_arrive[2][kProfBlocks];
  int32_t block_sm[kProfBlocks];
  // per block, summed over the trials: the phase's own work (its start to its
  // arrival), the wait at the barrier (arrival to seeing the team complete)
  // and, after phase B, the decision (seeing the team complete to starting A)
  uint64_t block_work[2][kProfBlocks], block_wait[2][kProfBlocks], block_decide[kProfBlocks];
};

template <typename T>
struct Args {
  int32_t n, m, neq, pad;
  // equilibrated matrix and its transpose, CSR
  const int32_t *kp, *kci;
  const T *kv;
  const int32_t *tp, *tci;
  const T *tv;
  // equilibrated data in the storage type
  const T *c, *q, *l, *u;
  // original data and the diagonals (FP64)
  const double *c0, *q0, *l0, *u0, *cs, *rs;
  // iterate state; x, y, kx are double-buffered
  T *x[2], *y[2], *kx[2];
  T *xbar, *kty, *sx, *sy, *skx, *skty, *xr, *yr;
  // solution in the caller's units
  double *xo, *yo, *rco;
  double *partials;  // [kSlots][max_blocks]
  int32_t max_blocks, anchored;
  const int2 *tiles_k, *tiles_t;  // tile tables of K and K': (first row, first nonzero), + a sentinel
  int32_t ntiles_k, ntiles_t;
  Prof *prof;
  // Anchored (refinement) mode: the iterate is a correction (x^, y^) to an
  // FP64 anchor (xa, ya) whose exact products kxa = K xa, ktya = K'ya are
  // kept; the working data c, q, l, u, ylo are the residual problem
  // (c - K'ya, q - K xa, l - xa, u - xa, -ya) in T, rebuilt at every
  // re-anchoring.  nullptr in the plain mode.
  double *xa, *ya, *kxa, *ktya;
  const double *sc, *sq, *sl, *su;  // FP64 equilibrated data
  const double *kv64, *tv64;        // FP64 equilibrated matrix values
  T *cw, *qw, *lw, *uw, *ylo;       // the residual problem's data
  Control *ctl;
  Sync *sync;
  const volatile int32_t *cancel;
  // batch launches: the shared queue of instance indices, and per team the
  // index its deciding block took when this instance finished.  nullptr for
  // a single solve.
  int32_t *queue, *team_next;
  int32_t team, pad2;
  // PRIMA_DEBUG_PROGRESS: host-mapped progress record, 16 words per block
  // (phase, trial, producer fill / own / state, consumer stage / state,
  // barrier state, iteration), readable while the kernel runs; else nullptr
  volatile int32_t *progress;
  unsigned long long *arrive_groups;  // hot barriers: per-group arrival counters [G * kArriveStride]
  Params P;
};

}  // namespace dev
}  // namespace prima
