// Fused persistent restarted-PDHG kernel and the coarse solve entry points.
// Design notes are in prima_solver.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>

#include <math_constants.h>

#include "prima_internal.h"
#include "prima_nvtx.h"
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
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
// An increment with release semantics that returns nothing: the thread does
// not wait for the round trip.
__device__ __forceinline__ void red_add_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// Waiting blocks poll the team's counter with relaxed loads and acquire once
// when it completes (1), or poll with acquire loads (0).
#ifndef PRIMA_POLL_RELAXED
#define PRIMA_POLL_RELAXED 0
#endif
// The trial's two barriers count arrivals on the team's counter with one
// fire-and-forget release increment per block (1), or in two levels -- a
// group counter, then the group's last block on the team's -- with
// round-trip atomics (0).
#ifndef PRIMA_HOT_RED
#define PRIMA_HOT_RED 1
#endif
// Phase A's first tiles are staged during the barrier after phase B on the
// guess that the trial is accepted (see barrier_decide); 0 stages its tile
// list only.
#ifndef PRIMA_SPEC_A
#define PRIMA_SPEC_A 1
#endif
// A block waiting at a trial's barrier reads the team's abort flag (and
// counts against its poll limit) on every PRIMA_ABORT_EVERY-th poll.
#ifndef PRIMA_ABORT_EVERY
#define PRIMA_ABORT_EVERY 8
#endif
#ifndef PRIMA_POLL_SLEEP_NS
#define PRIMA_POLL_SLEEP_NS 32
#endif
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Data written inside this launch by other blocks is read through L2 only
// (ld.global.cg), so no stale L1 line can be observed across a barrier;
// data that never changes during the launch goes through the read-only path.
template <typename T>
__device__ __forceinline__ T ldv(const T *p) {
  return __ldcg(p);
}

// Each block owns one contiguous chunk of rows (resp. columns); chunks start
// at multiples of 4 so every bulk copy of a vector slice is 16-byte aligned.
__device__ __forceinline__ void chunk(int32_t total, int nb, int rank, int32_t &lo, int32_t &hi) {
  const int64_t per = ((((int64_t)total + nb - 1) / nb) + 3) & ~(int64_t)3;
  int64_t a = (int64_t)rank * per, b = a + per;
  if (a > total) a = total;
  if (b > total) b = total;
  lo = (int32_t)a;
  hi = (int32_t)b;
}

// CSR-stream SpMV over the block's rows [lo, hi), one tile of kTileRows rows
// at a time.  Stage 1: the tile's products v[k] * x[col[k]] (rounded to T)
// are formed with coalesced matrix loads and fully parallel gathers into
// shared memory.  Stage 2: each thread sums its rows' products in index
// order starting from zero -- the reference's per-row order, bit for bit --
// and hands (row, acc, prefetched operands) to the epilogue.  The epilogue's
// own operands are loaded by `pre` before stage 1, so their latency overlaps
// the gathers.  A tile with more than kTileCap entries is summed straight
// from global memory in the same order.
template <typename T, int Cap = kTileCap, typename Pre, typename Epi>
__device__ __forceinline__ void csr_tiles(int32_t lo, int32_t hi, const int32_t *__restrict__ p,
                                          const int32_t *__restrict__ ci, const T *__restrict__ v, const T *x,
                                          T *s_prod, Pre &&pre, Epi &&epi) {
  using Ops = decltype(pre(0));
  int32_t k0 = lo < hi ? __ldg(p + lo) : 0;
  for (int32_t r0 = lo; r0 < hi; r0 += kTileRows) {
    const int32_t r1 = min(hi, r0 + kTileRows);
    Ops ops[kRowsPerThread];
    int32_t ra[kRowsPerThread], rb[kRowsPerThread];
#pragma unroll
    for (int i = 0; i < kRowsPerThread; i++) {
      const int32_t r = r0 + threadIdx.x + i * kThreads;
      if (r < r1) {
        ops[i] = pre(r);
        ra[i] = __ldg(p + r);
        rb[i] = __ldg(p + r + 1);
      }
    }
    const int32_t k1 = __ldg(p + r1);
    const bool staged = (k1 - k0) <= Cap;
    if (staged) {
#pragma unroll 4
      for (int32_t k = k0 + threadIdx.x; k < k1; k += kThreads) s_prod[k - k0] = __ldg(v + k) * ldv(x + __ldg(ci + k));
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kRowsPerThread; i++) {
      const int32_t r = r0 + threadIdx.x + i * kThreads;
      if (r < r1) {
        T acc = T(0);
        if (staged) {
          for (int32_t k = ra[i]; k < rb[i]; k++) acc = acc + s_prod[k - k0];
        } else {
          for (int32_t k = ra[i]; k < rb[i]; k++) acc = acc + (__ldg(v + k) * ldv(x + __ldg(ci + k)));
        }
        epi(r, acc, ops[i]);
      }
    }
    k0 = k1;
    __syncthreads();
  }
}

struct None {};

// ---- TMA-staged tiles for the hot phases ----------------------------------
//
// Phases A and B cut the rows of K' (A) and K (B) into tiles of at most
// kRows rows, starting at a multiple of 4, whose nonzeros (rounded out to
// 16-byte granules) fit one stage -- a table built once per matrix on the
// host and dealt to the team's blocks by estimated cost: the device table
// holds (start, end) pairs, slot rank + k*nb being block `rank`'s k-th
// tile.  A tile's row pointers, column
// indices, values and up to six vector slices arrive in one of kStages
// shared-memory stages by one-dimensional bulk copies (cp.async.bulk,
// completion on the stage's mbarrier).  Each warp then works on its own 32
// rows of the tile with no block-wide synchronisation; the last warp to
// finish with a stage refills it with the tile kStages further on.  A fast
// warp thus runs ahead into the next stage while a slow one finishes, and
// the copies for later tiles are in flight meanwhile.  Every wait is bounded.

#ifndef PRIMA_HOT_F32_CAP
#define PRIMA_HOT_F32_CAP 2048
#define PRIMA_HOT_F32_STAGES 2
#define PRIMA_HOT_F32_RPT 2
#endif
#ifndef PRIMA_HOT_F64_CAP
#define PRIMA_HOT_F64_CAP 1536
#define PRIMA_HOT_F64_STAGES 2
#define PRIMA_HOT_F64_RPT 2
#endif
template <int C, int S, int R>
struct HotShape {
  static_assert(C % 4 == 0 && C / 4 >= 32, "an unstaged tile splits the value area among its up to 4 rows");
  static constexpr int kCap = C, kStages = S, kRowsPerThread = R;
};
template <typename T>
struct Hot;
template <>
struct Hot<float> : HotShape<PRIMA_HOT_F32_CAP, PRIMA_HOT_F32_STAGES, PRIMA_HOT_F32_RPT> {};
template <>
struct Hot<double> : HotShape<PRIMA_HOT_F64_CAP, PRIMA_HOT_F64_STAGES, PRIMA_HOT_F64_RPT> {};
template <typename T>
constexpr int kHotRows = kThreads * Hot<T>::kRowsPerThread;  // rows per tile, at most
constexpr int kHotVec = 6;          // vector operands per row, at most

constexpr int kHotBatch = 128;      // tiles whose table entries a block stages at once
constexpr int kMaxStages = Hot<float>::kStages > Hot<double>::kStages ? Hot<float>::kStages : Hot<double>::kStages;

template <typename T>
struct HotLayout {
  static constexpr int kCap = Hot<T>::kCap;  // staged nonzeros (16-byte rounded span)
  static constexpr int kStages = Hot<T>::kStages;
  static constexpr size_t rp_bytes = ((size_t)(kHotRows<T> + 1) * 4 + 15) / 16 * 16;
  static constexpr size_t ci_off = rp_bytes;
  static constexpr size_t v_off = ci_off + (size_t)kCap * 4;
  static constexpr size_t vec_off = (v_off + (size_t)kCap * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t vec_stride = (size_t)kHotRows<T> * sizeof(T);
  static constexpr size_t stage_bytes = (vec_off + kHotVec * vec_stride + 127) / 128 * 128;
  static constexpr size_t total = kStages * stage_bytes;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// One poll of an mbarrier phase: the thread may be suspended until the phase
// completes, but for no more than kSuspendNs.
constexpr unsigned kSuspendNs = 10000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, uint64_t *b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// A stage's bytes land within microseconds; a wait that has lasted this long
// has failed.
constexpr unsigned long long kStageWaitNs = 2000000000ull;

__device__ __forceinline__ uint64_t stage_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for a buffer's bulk copies, by the clock (a poll may suspend
// the thread, so counting polls would bound nothing).  False: gave up, or
// the team's abort flag went up (when given); the caller raises the team's
// abort flag and leaves.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity, const int32_t *abort_flag = nullptr) {
  if (mbar_try_wait(b, parity)) return true;
  const uint64_t t0 = stage_timer_ns();
  for (unsigned i = 1;; i++) {
    if (mbar_try_wait(b, parity)) return true;
    if ((i & 15) == 0) {
      if (abort_flag && *((const volatile int32_t *)abort_flag)) return false;
      if (stage_timer_ns() - t0 > kStageWaitNs) return false;
    }
  }
}

// A word of the block's progress record (PRIMA_DEBUG_PROGRESS), if any.
__device__ __forceinline__ void progress(volatile int32_t *rec, int word, int32_t v) {
  if (rec && blockIdx.x < 256) rec[blockIdx.x * 16 + word] = v;
}

// Where a stage wait gave up, for the error the host reports: the first
// failure of a launch fills diag[0..7] = {1, tag (1: phase A, 2: phase B),
// 0, stage, parity, tile of the batch, tiles of this block, block}.
__device__ __forceinline__ void note_stage_failure(int32_t *diag, int tag, int stage, unsigned parity, int j,
                                                   int mine, int block) {
  if (diag && atomicCAS(diag, 0, 1) == 0) {
    diag[1] = tag;
    diag[2] = 0;
    diag[3] = stage;
    diag[4] = (int32_t)parity;
    diag[5] = j;
    diag[6] = mine;
    diag[7] = block;
    __threadfence();
  }
}

struct HotShared {
  uint64_t bars[kMaxStages];       // stage full: the tile's bytes have landed
  unsigned done[kMaxStages];       // warps finished with the stage's tile
  int2 tiles[2 * kHotBatch];       // per tile of the batch: (first row, first nonzero) of it and of the next
  int issued;                      // tiles of the batch issued so far
  int flag;
  int primed;                      // the next hot phase's first stages are already issued
  const int2 *listed;              // the table whose first batch hs.tiles holds, else nullptr
  int tag;                         // unused slot kept for the failure record's layout
  int32_t *diag;                   // the launch's failure record, or nullptr
  volatile int32_t *prog;          // the launch's progress record, or nullptr
};

// The tile engine over a table of ntiles tiles (see above).  rp == nullptr:
// no SpMV, vectors only.  epi(r, i, acc, vals) runs on the thread of row i
// of the tile (row r of the matrix): acc is the row's product (an
// index-order sum from zero, as csr_tiles), vals the row's vector operands
// (vecs[k][r] for k < nv).  Returns false, uniformly over the block, when the
// team's abort flag is up.
// Issue tile j of the batch staged in hs.tiles into stage j % kStages: its
// vector slices and, for an SpMV, its row pointers, column indices and
// values, all completing on the stage's mbarrier.  One thread.
template <typename T>
__device__ __forceinline__ void issue_tile(int j, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                           const T *__restrict__ v, const T *const *vecs, int nv, unsigned char *smem,
                                           HotShared &hs) {
  using L = HotLayout<T>;
  constexpr int S = L::kStages;
  const int b = j % S;
  unsigned char *buf = smem + b * L::stage_bytes;
  const int2 e0 = hs.tiles[2 * j], e1 = hs.tiles[2 * j + 1];
  const int32_t r0 = e0.x, rows = e1.x - e0.x;
  const unsigned vb = ((unsigned)rows * (unsigned)sizeof(T) + 15u) & ~15u;
  unsigned total = (unsigned)nv * vb, rpb = 0, cb = 0, vvb = 0;
  int32_t ka = 0;
  if (rp) {
    rpb = ((unsigned)(rows + 1) * 4u + 15u) & ~15u;
    ka = e0.y & ~3;
    const int32_t kbnd = (e1.y + 3) & ~3;
    if (kbnd - ka <= L::kCap && kbnd > ka) {
      cb = (unsigned)(kbnd - ka) * 4u;
      vvb = (unsigned)(kbnd - ka) * (unsigned)sizeof(T);
    }
    total += rpb + cb + vvb;
  }
  fence_proxy_async();
  hs.issued = j + 1;
  mbar_expect_tx(&hs.bars[b], total);
  for (int i = 0; i < nv; i++) bulk_copy(buf + L::vec_off + i * L::vec_stride, vecs[i] + r0, vb, &hs.bars[b]);
  if (rp) {
    bulk_copy(buf, rp + r0, rpb, &hs.bars[b]);
    if (cb) {
      bulk_copy(buf + L::ci_off, ci + ka, cb, &hs.bars[b]);
      bulk_copy(buf + L::v_off, v + ka, vvb, &hs.bars[b]);
    }
  }
}

// One warp stages this block's first batch of tiles and issues its first
// stages, ahead of the hot phase that will consume them (hs.primed tells it
// to start from there).  The stages and the tile list must be free.
template <typename T>
__device__ __forceinline__ void prime_tiles(int32_t ntiles, int nb, int rank, const int2 *__restrict__ table,
                                            const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                            const T *__restrict__ v, const T *const *vecs, int nv,
                                            unsigned char *smem, HotShared &hs) {
  constexpr int S = HotLayout<T>::kStages;
  const int lane = threadIdx.x & 31;
  const int32_t mine = rank < ntiles ? (ntiles - rank + nb - 1) / nb : 0;
  if (mine == 0) return;
  const int nj = min(kHotBatch, mine);
  for (int e = lane; e < 2 * nj; e += 32) hs.tiles[e] = __ldg(table + 2 * (rank + (int64_t)(e >> 1) * nb) + (e & 1));
  __syncwarp();
  if (lane == 0) {
    hs.listed = table;
    for (int b = 0; b < S; b++) hs.done[b] = 0;
    hs.issued = 0;
    for (int j = 0; j < S && j < nj; j++) issue_tile<T>(j, rp, ci, v, vecs, nv, smem, hs);
    hs.primed = 1;
  }
  __syncwarp();
}

// One warp stages this block's first batch of tiles of a table in hs.tiles
// (no copies issued), for the next hot phase over it to skip that load.
__device__ __forceinline__ void list_tiles(int32_t ntiles, int nb, int rank, const int2 *__restrict__ table,
                                           HotShared &hs) {
  const int lane = threadIdx.x & 31;
  const int32_t mine = rank < ntiles ? (ntiles - rank + nb - 1) / nb : 0;
  const int nj = min(kHotBatch, mine);
  for (int e = lane; e < 2 * nj; e += 32) hs.tiles[e] = __ldg(table + 2 * (rank + (int64_t)(e >> 1) * nb) + (e & 1));
  __syncwarp();
  if (lane == 0) hs.listed = table;
  __syncwarp();
}

template <typename T, typename Epi>
__device__ __forceinline__ bool hot_tiles(int32_t ntiles, int nb, int rank, const int2 *__restrict__ table,
                                          const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                          const T *__restrict__ v, const T *xg, const T *const *vecs, int nv,
                                          unsigned char *smem, HotShared &hs, unsigned &par, int32_t *abort_flag,
                                          int tag, Epi &&epi) {
  using L = HotLayout<T>;
  constexpr int S = L::kStages;
  const bool spmv = rp != nullptr;
  const int lane = threadIdx.x & 31;
  const int32_t mine = rank < ntiles ? (ntiles - rank + nb - 1) / nb : 0;  // this block's tiles
  const bool primed = hs.primed != 0;  // the first batch is staged and its first stages issued
  for (int32_t jb = 0; jb < mine; jb += kHotBatch) {
    const int nj = min(kHotBatch, mine - jb);
    const bool pre = primed && jb == 0;
    if (!pre) {
      if (!(jb == 0 && hs.listed == table))  // the first batch may already be staged
        for (int e = threadIdx.x; e < 2 * nj; e += kThreads) {
          const int64_t t = 2 * (rank + (int64_t)(jb + (e >> 1)) * nb) + (e & 1);
          hs.tiles[e] = __ldg(table + t);
        }
      __syncthreads();  // every thread has read hs.listed
      if (threadIdx.x < S) hs.done[threadIdx.x] = 0;
      if (threadIdx.x == 0) {
        hs.issued = 0;
        hs.listed = jb == 0 ? table : nullptr;
      }
      __syncthreads();
    }
    auto issue = [&](int j) {  // one thread
      issue_tile<T>(j, rp, ci, v, vecs, nv, smem, hs);
    };
    if (!pre) {
      if (threadIdx.x == 0)
        for (int j = 0; j < S && j < nj; j++) issue(j);
      __syncthreads();
    }
    int j = 0;
    for (; j < nj; j++) {
      const int b = j % S;
      if (!__all_sync(0xffffffffu, mbar_wait(&hs.bars[b], (par >> b) & 1u, abort_flag))) {
        if (lane == 0) {
          if (!*((const volatile int32_t *)abort_flag))
            note_stage_failure(hs.diag, tag, b, (par >> b) & 1u, jb + j, mine, (int)blockIdx.x);
          atomicExch(abort_flag, 1);
        }
        break;
      }
      par ^= 1u << b;
      const int2 e0 = hs.tiles[2 * j], e1 = hs.tiles[2 * j + 1];
      const int32_t r0 = e0.x, rows = e1.x - e0.x;
      const unsigned char *buf = smem + b * L::stage_bytes;
      const int32_t *rp_s = reinterpret_cast<const int32_t *>(buf);
      const int32_t *ci_s = reinterpret_cast<const int32_t *>(buf + L::ci_off);
      const T *v_s = reinterpret_cast<const T *>(buf + L::v_off);
      const T *slices = reinterpret_cast<const T *>(buf + L::vec_off);
      const int32_t ka = e0.y & ~3;
      const bool staged = spmv && ((e1.y + 3) & ~3) - ka <= L::kCap;
      // each thread takes rows threadIdx.x + r * kThreads of the tile; the
      // first four gathers of all its rows are issued together
      constexpr int RPT = Hot<T>::kRowsPerThread;
      // the vector operands of the thread's rows, from the stage
      T vv[RPT][kHotVec];
#pragma unroll
      for (int q = 0; q < RPT; q++) {
        const int i = threadIdx.x + q * kThreads;
#pragma unroll
        for (int k = 0; k < kHotVec; k++) vv[q][k] = (k < nv && i < rows) ? slices[k * kHotRows<T> + i] : T(0);
      }
      T acc[RPT];
      int32_t a0[RPT], a1[RPT];
#pragma unroll
      for (int q = 0; q < RPT; q++) {
        const int i = threadIdx.x + q * kThreads;
        acc[q] = T(0);
        a0[q] = a1[q] = 0;
        if (spmv && i < rows) {
          if (staged) {
            a0[q] = rp_s[i];
            a1[q] = rp_s[i + 1];
          }
        }
      }
      const bool dense = staged && (int64_t)(e1.y - e0.y) > 8 * (int64_t)rows;
      if (dense) {
        // Long rows: the warp first forms the products of its rows' nonzeros
        // in place in the stage (lanes side by side, four gathers each in
        // flight), then each thread sums its rows from shared memory in
        // index order.  A thread walking a 400-nonzero row four gathers at a
        // time would wait a hundred round trips.
        T *vw = const_cast<T *>(v_s);
#pragma unroll
        for (int q = 0; q < RPT; q++) {
          const int rlo = q * kThreads + (threadIdx.x & ~31);
          if (rlo < rows) {
            const int32_t k0 = rp_s[rlo], k1 = rp_s[min(rows, rlo + 32)];
            for (int32_t k = k0 + lane; k < k1; k += 4 * 32) {
              int32_t cc[4];
              T xx[4];
#pragma unroll
              for (int u = 0; u < 4; u++) cc[u] = k + u * 32 < k1 ? ci_s[k + u * 32 - ka] : -1;
#pragma unroll
              for (int u = 0; u < 4; u++) xx[u] = cc[u] >= 0 ? ldv(xg + cc[u]) : T(0);
#pragma unroll
              for (int u = 0; u < 4; u++)
                if (cc[u] >= 0) vw[k + u * 32 - ka] = vw[k + u * 32 - ka] * xx[u];
            }
          }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < RPT; q++)
          for (int32_t k = a0[q]; k < a1[q]; k++) acc[q] = acc[q] + vw[k - ka];
      } else if (staged) {  // index-order sums: the first four products of every row, then the rest four at a time
        int32_t col[RPT][4];
        T x[RPT][4];
#pragma unroll
        for (int q = 0; q < RPT; q++)
#pragma unroll
          for (int u = 0; u < 4; u++) col[q][u] = a0[q] + u < a1[q] ? ci_s[a0[q] + u - ka] : -1;
#pragma unroll
        for (int q = 0; q < RPT; q++)
#pragma unroll
          for (int u = 0; u < 4; u++) x[q][u] = col[q][u] >= 0 ? ldv(xg + col[q][u]) : T(0);
#pragma unroll
        for (int q = 0; q < RPT; q++) {
#pragma unroll
          for (int u = 0; u < 4; u++)
            if (a0[q] + u < a1[q]) acc[q] = acc[q] + (v_s[a0[q] + u - ka] * x[q][u]);
          int32_t k = a0[q] + 4;
          for (; k + 4 <= a1[q]; k += 4) {
            const int32_t c0 = ci_s[k - ka], c1 = ci_s[k + 1 - ka], c2 = ci_s[k + 2 - ka], c3 = ci_s[k + 3 - ka];
            const T x0 = ldv(xg + c0), x1 = ldv(xg + c1), x2 = ldv(xg + c2), x3 = ldv(xg + c3);
            acc[q] = acc[q] + (v_s[k - ka] * x0);
            acc[q] = acc[q] + (v_s[k + 1 - ka] * x1);
            acc[q] = acc[q] + (v_s[k + 2 - ka] * x2);
            acc[q] = acc[q] + (v_s[k + 3 - ka] * x3);
          }
          for (; k < a1[q]; k++) acc[q] = acc[q] + (v_s[k - ka] * ldv(xg + ci_s[k - ka]));
        }
      }
      if (spmv && !staged) {
        // A tile whose nonzeros do not fit a stage is one group of at most 4
        // long rows (a dense column of K, say).  Warp w takes row w: its
        // lanes form the products in chunks into the stage's value area,
        // which this tile leaves unused, and lane 0 sums each chunk in index
        // order -- the same sum as everywhere else, without one thread
        // walking thousands of dependent loads.
        constexpr int kChunk = L::kCap / 4;
        const int w = threadIdx.x >> 5;
        T accw = T(0);
        if (w < rows) {
          T *scratch = reinterpret_cast<T *>(const_cast<unsigned char *>(buf) + L::v_off) + w * kChunk;
          const int32_t b0 = __ldg(rp + r0 + w), b1 = __ldg(rp + r0 + w + 1);
          for (int32_t base = b0; base < b1; base += kChunk) {
            const int32_t cnt = min(kChunk, b1 - base);
            for (int32_t k = lane; k < cnt; k += 32) scratch[k] = __ldg(v + base + k) * ldv(xg + __ldg(ci + base + k));
            __syncwarp();
            if (lane == 0)
              for (int32_t k = 0; k < cnt; k++) accw = accw + scratch[k];
            __syncwarp();
          }
          if (lane == 0) {
            T vw[kHotVec];
#pragma unroll
            for (int k = 0; k < kHotVec; k++)
              vw[k] = k < nv ? slices[k * kHotRows<T> + w] : T(0);
            epi(r0 + w, w, accw, vw);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < RPT; q++) {
          const int i = threadIdx.x + q * kThreads;
          if (i < rows) epi(r0 + i, i, acc[q], vv[q]);
        }
      }
      // the last warp done with this stage refills it with the tile S further on
      __syncwarp();
      if (lane == 0) {
        __threadfence_block();
        if (atomicAdd(&hs.done[b], 1u) == (unsigned)(kWarps - 1)) {
          __threadfence_block();
          hs.done[b] = 0;
          if (j + S < nj) issue(j + S);
        }
      }
    }
    // leave the batch: every warp is past the loop; then let any copies still
    // in flight land (bounded) before the stages or the table are reused
    __syncthreads();
    if (threadIdx.x == 0) {
      hs.flag = *((volatile int32_t *)abort_flag);
      for (int u = j; u < hs.issued; u++) {  // only after an abort: tiles issued but never consumed
        mbar_wait(&hs.bars[u % S], (par >> (u % S)) & 1u);
        par ^= 1u << (u % S);
      }
    }
    __syncthreads();
    if (hs.flag) return false;
  }
  if (primed) {
    __syncthreads();  // every thread has read the flag
    if (threadIdx.x == 0) hs.primed = 0;
  }
  return true;
}

// One shared staging area for every block reduction (a single allocation
// per block, whatever the number of template instances).
__device__ __forceinline__ double (&reduction_scratch())[kMaxQ][kWarps] {
  __shared__ double sh[kMaxQ][kWarps];
  return sh;
}

// Block-wide totals of Q per-thread values in a fixed order.  The block's
// totals go to shared s_part[base..base+Q) and, in a multi-block team, to the
// global partials[(gbase + q) * stride + rank] (gbase = base unless given).
template <int Q>
__device__ __forceinline__ void block_partials(const double (&v)[Q], double *partials, int stride, int rank, int nb,
                                               int base, double *s_part, int gbase = -1) {
  if (gbase < 0) gbase = base;
  double(&sh)[kMaxQ][kWarps] = reduction_scratch();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < Q; q++) {
    double s = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sh[q][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < Q) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) s += sh[threadIdx.x][w];
    s_part[base + threadIdx.x] = s;
    if (nb > 1) partials[(gbase + threadIdx.x) * stride + rank] = s;
  }
  __syncthreads();
}

// Totals of slots [0, Q) over the nb block partials, in a fixed order (the
// block's own shared totals when nb == 1); global slots start at gbase.
template <int Q>
__device__ __forceinline__ void reduce_partials(const double *partials, int stride, int nb, const double *s_part,
                                                double *out, int gbase = 0) {
  if (nb == 1) {
    if (threadIdx.x < Q) out[threadIdx.x] = s_part[threadIdx.x];
    __syncthreads();
    return;
  }
  partials += (int64_t)gbase * stride;
  double(&sh)[kMaxQ][kWarps] = reduction_scratch();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[Q];
  // Every thread first issues its loads for up to kGroup slots x kWin
  // partials at once (one L2 round trip instead of one per load), then sums
  // each slot in block order.
  constexpr int kGroup = 4, kWin = 4;
#pragma unroll
  for (int q0 = 0; q0 < Q; q0 += kGroup) {
    double val[kGroup][kWin];
#pragma unroll
    for (int g = 0; g < kGroup; g++)
#pragma unroll
      for (int k = 0; k < kWin; k++) {
        const int b = threadIdx.x + k * kThreads;
        val[g][k] = (q0 + g < Q && b < nb) ? ldv(partials + (q0 + g) * stride + b) : 0.0;
      }
#pragma unroll
    for (int g = 0; g < kGroup; g++) {
      if (q0 + g < Q) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kWin; k++)
          if (threadIdx.x + k * kThreads < nb) s += val[g][k];
        for (int b = threadIdx.x + kWin * kThreads; b < nb; b += kThreads) s += ldv(partials + (q0 + g) * stride + b);
        v[q0 + g] = s;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < Q; q++) {
    double s = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sh[q][warp] = s;
  }
  __syncthreads();
  if (threadIdx.x < Q) {
    double s = 0.0;
#pragma unroll
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

// ---- evaluation terms --------------------------------------------------------

// Row r: Kkt.evaluate's primal residual and q'y; the certificates' row terms.
__device__ __forceinline__ void eval_row(double yv, double kxv, double rs, double q0, bool eq, double (&v)[kRowQ]) {
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

__device__ __forceinline__ void eval_row_avg(double yv, double kxv, double rs, double q0, bool eq,
                                             double (&v)[kRowQ]) {
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

// Column j: Kkt.evaluate's objective and dual terms; the certificates'
// column terms.  Indices are slot - Q_CX.
__device__ __forceinline__ void eval_col(double xv, double ktv, double cs, double c0, double l0, double u0,
                                         double (&v)[kColQ]) {
  const double xo = xv * cs, kto = ktv / cs;
  const bool lfin = !(isinf(l0) && l0 < 0.0), ufin = !(isinf(u0) && u0 > 0.0);
  v[Q_CX - Q_CX] += c0 * xo;
  const double rc = c0 - kto;
  if (rc > 0.0) {
    if (!lfin) v[Q_DSQ - Q_CX] += rc * rc;
    else v[Q_DTERM - Q_CX] += l0 * rc;
  } else if (rc < 0.0) {
    if (!ufin) v[Q_DSQ - Q_CX] += rc * rc;
    else v[Q_DTERM - Q_CX] += u0 * rc;
  }
  const double pr = -kto;
  if (pr > 0.0) {
    if (!lfin) v[Q_PRSQ - Q_CX] += pr * pr;
    else v[Q_PVAL - Q_CX] += l0 * pr;
  } else if (pr < 0.0) {
    if (!ufin) v[Q_PRSQ - Q_CX] += pr * pr;
    else v[Q_PVAL - Q_CX] += u0 * pr;
  }
  v[Q_XSQ - Q_CX] += xo * xo;
  if ((xo > 0.0 && ufin) || (xo < 0.0 && lfin)) v[Q_BSQ - Q_CX] += xo * xo;
}

__device__ __forceinline__ void eval_col_avg(double xv, double ktv, double cs, double c0, double l0, double u0,
                                             double (&v)[kColQ]) {
  const double xo = xv * cs, kto = ktv / cs;
  v[Q_A_CX - Q_CX] += c0 * xo;
  const double rc = c0 - kto;
  if (rc > 0.0) {
    if (isinf(l0) && l0 < 0.0) v[Q_A_DSQ - Q_CX] += rc * rc;
    else v[Q_A_DTERM - Q_CX] += l0 * rc;
  } else if (rc < 0.0) {
    if (isinf(u0) && u0 > 0.0) v[Q_A_DSQ - Q_CX] += rc * rc;
    else v[Q_A_DTERM - Q_CX] += u0 * rc;
  }
}

// ---- phases --------------------------------------------------------------------

struct Team {
  int nb, rank;
  double *s_part;  // shared: this block's totals, by slot
};

// Round-to-+inf / -inf narrowing for the residual problem's bounds, so that
// anchor + correction never leaves the box or the cone in exact arithmetic.
template <typename T>
__device__ __forceinline__ T narrow_up(double v);
template <typename T>
__device__ __forceinline__ T narrow_down(double v);
template <>
__device__ __forceinline__ float narrow_up<float>(double v) {
  return __double2float_ru(v);
}
template <>
__device__ __forceinline__ float narrow_down<float>(double v) {
  return __double2float_rd(v);
}
template <>
__device__ __forceinline__ double narrow_up<double>(double v) {
  return v;
}
template <>
__device__ __forceinline__ double narrow_down<double>(double v) {
  return v;
}

// The anchor's exact products and the residual problem's data (anchored
// mode): kxa = K xa and ktya = K'ya in FP64, then c - K'ya, q - K xa,
// l - xa (rounded up), u - xa (rounded down), -ya (rounded up) in T.
template <typename T>
__device__ void rebuild_residual_problem(const Args<T> &a, const Team &tm, T *s_prod) {
  double *s_prod64 = reinterpret_cast<double *>(s_prod);
  constexpr int kCap64 = (int)(kTileCap * sizeof(T) / sizeof(double));
  int32_t lo, hi;
  chunk(a.n, tm.nb, tm.rank, lo, hi);
  csr_tiles<double, kCap64>(lo, hi, a.tp, a.tci, a.tv64, (const double *)a.ya, s_prod64,
                            [&](int32_t) { return None{}; }, [&](int32_t j, double kt, None) {
    a.ktya[j] = kt;
    const double xa = ldv(a.xa + j);
    a.cw[j] = (T)(__ldg(a.sc + j) - kt);
    a.lw[j] = narrow_up<T>(__ldg(a.sl + j) - xa);
    a.uw[j] = narrow_down<T>(__ldg(a.su + j) - xa);
  });
  chunk(a.m, tm.nb, tm.rank, lo, hi);
  csr_tiles<double, kCap64>(lo, hi, a.kp, a.kci, a.kv64, (const double *)a.xa, s_prod64,
                            [&](int32_t) { return None{}; }, [&](int32_t r, double kxv, None) {
    a.kxa[r] = kxv;
    a.qw[r] = (T)(__ldg(a.sq + r) - kxv);
    a.ylo[r] = r < a.neq ? T(-CUDART_INF) : narrow_up<T>(-ldv(a.ya + r));
  });
}

// The point a (correction) value stands for: anchor + correction in FP64.
template <typename T>
__device__ __forceinline__ double at(const double *anchor, int32_t i, T v) {
  return anchor ? ldv(anchor + i) + (double)v : (double)v;
}

template <typename T>
__device__ void phase_init(const Args<T> &a, const Control &s, const Team &tm, T *s_prod) {
  int32_t lo, hi;
  if (a.anchored) {
    // the start point is the anchor; the correction starts at zero
    rebuild_residual_problem(a, tm, s_prod);
    __syncthreads();
  }
  {
    double v[kColQ];
#pragma unroll
    for (int q = 0; q < kColQ; q++) v[q] = 0.0;
    chunk(a.n, tm.nb, tm.rank, lo, hi);
    csr_tiles<T>(lo, hi, a.tp, a.tci, a.tv, (const T *)a.y[0], s_prod, [&](int32_t) { return None{}; },
                 [&](int32_t j, T kt, None) {
      const T xj = ldv(a.x[0] + j);
      a.kty[j] = kt;
      a.xr[j] = xj;
      a.sx[j] = T(0);
      a.skty[j] = T(0);
      eval_col(at(a.xa, j, xj), at(a.ktya, j, kt), __ldg(a.cs + j), __ldg(a.c0 + j), __ldg(a.l0 + j),
               __ldg(a.u0 + j), v);
    });
    block_partials<kColQ>(v, a.partials, a.max_blocks, tm.rank, tm.nb, Q_CX, tm.s_part);
  }
  {
    double v[kRowQ];
#pragma unroll
    for (int q = 0; q < kRowQ; q++) v[q] = 0.0;
    chunk(a.m, tm.nb, tm.rank, lo, hi);
    csr_tiles<T>(lo, hi, a.kp, a.kci, a.kv, (const T *)a.x[0], s_prod, [&](int32_t) { return None{}; },
                 [&](int32_t r, T kxv, None) {
      const T yv = ldv(a.y[0] + r);
      a.kx[0][r] = kxv;
      a.yr[r] = yv;
      a.sy[r] = T(0);
      a.skx[r] = T(0);
      eval_row(at(a.ya, r, yv), at(a.kxa, r, kxv), __ldg(a.rs + r), __ldg(a.q0 + r), r < a.neq, v);
    });
    block_partials<kRowQ>(v, a.partials, a.max_blocks, tm.rank, tm.nb, 0, tm.s_part);
  }
}

// Primal half of a trial (primalStep + extrapolation), fused with the
// pending commit's K'y and running sums; operands streamed by TMA.
template <typename T>
__device__ bool phase_a(const Args<T> &a, const Control &s, const Team &tm, unsigned char *smem, HotShared &hs,
                        unsigned &par) {
  double v[1] = {0.0};
  const T tau = (T)s.tau, w = (T)s.pend_w;
  const T *x = a.x[s.xc];
  T *xn_out = a.x[s.xc ^ 1];
  auto step = [&](int32_t j, T xj, T kt, T cj, T lj, T uj) {
    // ScalaKernels.primalStep (:78-98): two-comparison clamp
    const T st = xj - (tau * (cj - kt));
    const T xn = st < lj ? lj : (st > uj ? uj : st);
    xn_out[j] = xn;
    a.xbar[j] = (T(2) * xn) + (T(-1) * xj);
    const T d = (T(1) * xn) + (T(-1) * xj);
    v[0] += (double)d * (double)d;
  };
  bool ok;
  if (s.pend) {
    const T *vecs[6] = {x, a.sx, a.skty, a.c, a.l, a.u};
    ok = hot_tiles<T>(a.ntiles_t, tm.nb, tm.rank, a.tiles_t, a.tp, a.tci, a.tv, (const T *)a.y[s.yc], vecs, 6, smem, hs, par,
                      &a.sync->abort, 1, [&](int32_t j, int, T kt, const T *vv) {
                        const T xj = vv[0], sx = vv[1], skt = vv[2], cj = vv[3], lj = vv[4], uj = vv[5];
                        a.kty[j] = kt;
                        a.sx[j] = (w * xj) + (T(1) * sx);
                        a.skty[j] = (w * kt) + (T(1) * skt);
                        step(j, xj, kt, cj, lj, uj);
                      });
  } else {
    const T *vecs[5] = {x, a.kty, a.c, a.l, a.u};
    ok = hot_tiles<T>(a.ntiles_t, tm.nb, tm.rank, a.tiles_t, nullptr, nullptr, nullptr, nullptr, vecs, 5, smem, hs, par,
                      &a.sync->abort, 1, [&](int32_t j, int, T, const T *vv) {
                        step(j, vv[0], vv[1], vv[2], vv[3], vv[4]);
                      });
  }
  block_partials<1>(v, a.partials, a.max_blocks, tm.rank, tm.nb, Q_DX, tm.s_part, hot_bank(s.total_trials) + Q_DX);
  return ok;
}

// The vectors phase B stages per tile, in slice order: y, kx, q, then the
// running sums when a commit is pending, then the anchored lower bound.
// None of them changes during phase A, so they can be staged before it ends.
template <typename T>
__device__ __forceinline__ int b_operands(const Args<T> &a, const Control &s, const T *(&vecs)[6]) {
  vecs[0] = a.y[s.yc];
  vecs[1] = a.kx[s.kxc];
  vecs[2] = a.q;
  vecs[3] = a.sy;
  vecs[4] = a.skx;
  vecs[5] = a.ylo;
  int nv = s.pend ? 5 : 3;
  if (a.ylo) vecs[nv++] = a.ylo;
  return nv;
}

// Dual half of a trial: K xbar, dualStep, the speculative kx commit value;
// operands streamed by TMA.
template <typename T>
__device__ bool phase_b(const Args<T> &a, const Control &s, const Team &tm, unsigned char *smem, HotShared &hs,
                        unsigned &par) {
  double v[2] = {0.0, 0.0};
  const T sigma = (T)s.sigma, w = (T)s.pend_w;
  T *y_out = a.y[s.yc ^ 1];
  T *kx_out = a.kx[s.kxc ^ 1];
  const bool pend = s.pend != 0;
  const T *vecs[6];
  const int nv = b_operands(a, s, vecs);
  const int iylo = pend ? 5 : 3;
  const bool has_lo = a.ylo != nullptr;
  const bool ok = hot_tiles<T>(a.ntiles_k, tm.nb, tm.rank, a.tiles_k, a.kp, a.kci, a.kv, (const T *)a.xbar, vecs, nv, smem, hs, par,
                               &a.sync->abort, 2, [&](int32_t r, int, T kb, const T *vv) {
    const T yr = vv[0], kxr = vv[1], qr = vv[2];
    const T syr = pend ? vv[3] : T(0), skxr = pend ? vv[4] : T(0);
    const T lb = has_lo ? vv[iylo] : T(0);
    if (pend) {
      a.sy[r] = (w * yr) + (T(1) * syr);
      a.skx[r] = (w * kxr) + (T(1) * skxr);
    }
    // ScalaKernels.dualStep (:100-118); around an anchor the cone is y >= -ya
    T yn = yr + (sigma * (qr - kb));
    if (r >= a.neq) yn = yn > lb ? yn : lb;
    y_out[r] = yn;
    kx_out[r] = (T(0.5) * kb) + (T(0.5) * kxr);
    const T dy = (T(1) * yn) + (T(-1) * yr);
    const T kdx = (T(0.5) * kb) + (T(-0.5) * kxr);
    v[0] += (double)dy * (double)dy;
    v[1] += (double)dy * (double)kdx;
  });
  block_partials<2>(v, a.partials, a.max_blocks, tm.rank, tm.nb, Q_DY, tm.s_part, hot_bank(s.total_trials) + Q_DY);
  return ok;
}

// Flush the pending commit, optionally refresh kx = K x, evaluate the
// current point and the running average (anchor + correction in anchored mode).
template <typename T>
__device__ void phase_f(const Args<T> &a, const Control &s, const Team &tm, T *s_prod) {
  const T w = (T)s.pend_w, inv = (T)s.inv_w;
  const bool pend = s.pend != 0, fresh = s.f_mode != F_ITERLIMIT, avg = s.f_avg != 0;
  const T *x = a.x[s.xc];
  const T *y = a.y[s.yc];
  T *kx = a.kx[s.kxc];
  int32_t lo, hi;
  {
    double v[kColQ];
#pragma unroll
    for (int q = 0; q < kColQ; q++) v[q] = 0.0;
    chunk(a.n, tm.nb, tm.rank, lo, hi);
    auto col = [&](int32_t j, T kt) {
      const T xj = ldv(x + j);
      const double cs = __ldg(a.cs + j), c0 = __ldg(a.c0 + j), l0 = __ldg(a.l0 + j), u0 = __ldg(a.u0 + j);
      eval_col(at(a.xa, j, xj), at(a.ktya, j, kt), cs, c0, l0, u0, v);
      if (avg)
        eval_col_avg(at(a.xa, j, inv * ldv(a.sx + j)), at(a.ktya, j, inv * ldv(a.skty + j)), cs, c0, l0, u0, v);
    };
    if (pend) {
      csr_tiles<T>(lo, hi, a.tp, a.tci, a.tv, y, s_prod, [&](int32_t) { return None{}; }, [&](int32_t j, T kt, None) {
        const T xj = ldv(x + j);
        a.kty[j] = kt;
        a.sx[j] = (w * xj) + (T(1) * ldv(a.sx + j));
        a.skty[j] = (w * kt) + (T(1) * ldv(a.skty + j));
        col(j, kt);
      });
    } else {
      for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) col(j, ldv(a.kty + j));
    }
    block_partials<kColQ>(v, a.partials, a.max_blocks, tm.rank, tm.nb, Q_CX, tm.s_part);
  }
  {
    double v[kRowQ];
#pragma unroll
    for (int q = 0; q < kRowQ; q++) v[q] = 0.0;
    chunk(a.m, tm.nb, tm.rank, lo, hi);
    auto row = [&](int32_t r, T kxr) {
      const T yr = ldv(y + r);
      const double rs = __ldg(a.rs + r), q0 = __ldg(a.q0 + r);
      eval_row(at(a.ya, r, yr), at(a.kxa, r, kxr), rs, q0, r < a.neq, v);
      if (avg)
        eval_row_avg(at(a.ya, r, inv * ldv(a.sy + r)), at(a.kxa, r, inv * ldv(a.skx + r)), rs, q0, r < a.neq, v);
    };
    auto flush = [&](int32_t r) {
      if (pend) {
        a.sy[r] = (w * ldv(y + r)) + (T(1) * ldv(a.sy + r));
        a.skx[r] = (w * ldv(kx + r)) + (T(1) * ldv(a.skx + r));
      }
    };
    if (fresh) {
      csr_tiles<T>(lo, hi, a.kp, a.kci, a.kv, x, s_prod, [&](int32_t) { return None{}; }, [&](int32_t r, T kxr, None) {
        flush(r);  // the running sum takes the incremental kx, then the fresh one replaces it
        kx[r] = kxr;
        row(r, kxr);
      });
    } else {
      for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
        flush(r);
        row(r, ldv(kx + r));
      }
    }
    block_partials<kRowQ>(v, a.partials, a.max_blocks, tm.rank, tm.nb, 0, tm.s_part);
  }
}

// restartAt (Pdhg.scala:478-502): adopt the average if chosen, measure the
// distance travelled since the last restart, re-centre, reset the sums.  In
// anchored mode the restart point is folded into the FP64 anchor (clamped
// into the box and the cone) and the correction restarts from zero; the
// distances are the correction's own norms, the last restart point being the
// anchor itself.
template <typename T>
__device__ void phase_r(const Args<T> &a, const Control &s, const Team &tm) {
  double v[2] = {0.0, 0.0};
  const T inv = (T)s.inv_w;
  const bool avg = s.r_avg != 0;
  T *x = a.x[s.xc];
  T *y = a.y[s.yc];
  T *kx = a.kx[s.kxc];
  int32_t lo, hi;
  chunk(a.n, tm.nb, tm.rank, lo, hi);
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
    if (a.anchored) {
      const double xn = ldv(a.xa + j) + (double)xj, lb = __ldg(a.sl + j), ub = __ldg(a.su + j);
      a.xa[j] = xn < lb ? lb : (xn > ub ? ub : xn);
      x[j] = T(0);
      a.kty[j] = T(0);
      xj = T(0);
    }
    a.xr[j] = xj;
    a.sx[j] = T(0);
    a.skty[j] = T(0);
  }
  chunk(a.m, tm.nb, tm.rank, lo, hi);
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
    if (a.anchored) {
      const double yn = ldv(a.ya + r) + (double)yr;
      a.ya[r] = (r >= a.neq && yn < 0.0) ? 0.0 : yn;
      y[r] = T(0);
      kx[r] = T(0);
      yr = T(0);
    }
    a.yr[r] = yr;
    a.sy[r] = T(0);
    a.skx[r] = T(0);
  }
  block_partials<2>(v, a.partials, a.max_blocks, tm.rank, tm.nb, Q_DXR, tm.s_part);
}

// Anchored mode, after a re-anchoring: the anchor's exact products and the
// new residual problem.
template <typename T>
__device__ void phase_r2(const Args<T> &a, const Control &s, const Team &tm, T *s_prod) {
  rebuild_residual_problem(a, tm, s_prod);
}

// finish (Pdhg.scala:510-532): the evaluated point in the caller's units and
// the reduced costs c - K'y.
template <typename T>
__device__ void phase_w(const Args<T> &a, const Control &s, const Team &tm) {
  const T inv = (T)s.inv_w;
  const bool avg = s.w_avg != 0;
  const T *x = a.x[s.xc];
  const T *y = a.y[s.yc];
  int32_t lo, hi;
  chunk(a.n, tm.nb, tm.rank, lo, hi);
  for (int32_t j = lo + threadIdx.x; j < hi; j += kThreads) {
    const T xj = avg ? inv * ldv(a.sx + j) : ldv(x + j);
    const T kt = avg ? inv * ldv(a.skty + j) : ldv(a.kty + j);
    const double cs = __ldg(a.cs + j);
    a.xo[j] = at(a.xa, j, xj) * cs;
    a.rco[j] = __ldg(a.c0 + j) - at(a.ktya, j, kt) / cs;
  }
  chunk(a.m, tm.nb, tm.rank, lo, hi);
  for (int32_t r = lo + threadIdx.x; r < hi; r += kThreads) {
    const T yr = avg ? inv * ldv(a.sy + r) : ldv(y + r);
    a.yo[r] = at(a.ya, r, yr) * __ldg(a.rs + r);
  }
}

// ---- decisions (the whole deciding block; thread 0 updates the record) -------

template <typename T>
__device__ void decide(const Args<T> &a, Control &c, int phase, const Team &tm, double *red) {
  const Params &P = a.P;
  switch (phase) {
    case PH_INIT: {
      reduce_partials<kMaxQ>(a.partials, a.max_blocks, tm.nb, tm.s_part, red);
      if (threadIdx.x == 0) {
        c.t0 = global_timer_ns();
        const Kkt e = kkt_current(red, P);
        c.current = e;
        if (converged(e, P)) {  // the start is already optimal, Pdhg.scala:211-212
          c.status = PRIMA_STATUS_OPTIMAL;
          c.final_kkt = e;
          c.w_avg = 0;
          c.phase = PH_W;
        } else {
          c.error_at_restart = weighted(e, c.weight);
          c.round_err = c.error_at_restart;
          c.pend = 0;
          c.trials = 0;
          set_trial_scalars(c);
          c.phase = PH_A;
        }
      }
      break;
    }
    case PH_B: {  // Solve.step's trial decision, Pdhg.scala:336-380
      // the step rule's two powers depend only on the iteration count: two
      // other warps evaluate them while the partials are being reduced
      __shared__ double s_pow[2];
      const uint64_t t_in = (a.prof && threadIdx.x == 0 && tm.rank == 0) ? global_timer_ns() : 0;
      {
        const double t = (double)(c.iteration - c.period_base + 1);
        if (threadIdx.x == 32) s_pow[0] = pow(t, -0.3);
        if (threadIdx.x == 64) s_pow[1] = pow(t, -0.6);
      }
      reduce_partials<3>(a.partials, a.max_blocks, tm.nb, tm.s_part, red, hot_bank(c.total_trials));
      if (a.prof && threadIdx.x == 0 && tm.rank == 0) a.prof->reduce_b_ns += global_timer_ns() - t_in;
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
          const double by_rule = (1.0 - s_pow[0]) * limit;
          const double by_cap = (1.0 + s_pow[1]) * c.step;
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
      reduce_partials<kMaxQ>(a.partials, a.max_blocks, tm.nb, tm.s_part, red);
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
              const bool artificial = (double)(c.iteration - c.last_restart_it) >=
                                      P.r_art * (double)(c.iteration - c.period_base);
              const bool new_round = P.round_rho > 0.0 && cand <= P.round_rho * c.round_err;
              if (sufficient || necessary || artificial || new_round) {
                c.r_avg = use_avg;
                c.phase = PH_R;
                if (new_round) {  // fresh restart schedule and step-size ramp
                  c.period_base = c.iteration;
                  c.round_err = cand;
                  c.rounds += 1;
                }
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
      reduce_partials<2>(a.partials, a.max_blocks, tm.nb, tm.s_part, red);
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
        if (a.anchored) {
          c.phase = PH_R2;  // rebuild the residual problem around the new anchor
        } else {
          after_checkpoint(c, point, P, a.cancel);
        }
      }
      break;
    }
    case PH_R2: {
      if (threadIdx.x == 0) after_checkpoint(c, c.current, P, a.cancel);
      break;
    }
    default:  // PH_W
      if (threadIdx.x == 0) {
        c.phase = PH_DONE;
        c.t_end = global_timer_ns();
      }
  }
}

// ---- the team barrier -------------------------------------------------------

constexpr long long kDefaultSpinLimit = 1ll << 26;  // ~seconds; a phase takes microseconds

// The team barrier's generation as this block last saw it.  Read from the
// Sync record once when a solve starts -- no barrier of that solve can have
// released before every block of the team arrived at it -- and counted up at
// each barrier after, so that arriving costs one atomic rather than a load of
// the generation followed by the atomic.
__device__ __forceinline__ unsigned &barrier_generation() {
  __shared__ unsigned s_gen;
  return s_gen;
}

// Hot barriers (after phases A and B) this block has passed in this solve:
// the team's arrival counter reads nb times that when the last one released.
__device__ __forceinline__ unsigned long long &hot_epoch() {
  __shared__ unsigned long long s_ep;
  return s_ep;
}

// Phase timing (PRIMA_PHASE_TIMES): when this block started its current hot
// phase, and when it arrived at that phase's barrier.
__device__ __forceinline__ uint64_t (&block_clock())[2] {
  __shared__ uint64_t s_clock[2];
  return s_clock;
}

template <typename T>
__device__ __forceinline__ void publish_control(const Args<T> &a, const Control &snap) {
  const unsigned *src = (const unsigned *)&snap;
  unsigned *dst = (unsigned *)a.ctl;
  for (int i = threadIdx.x; i < (int)(sizeof(Control) / 4); i += kThreads) dst[i] = src[i];
}

template <typename T>
__device__ __forceinline__ void load_control(const Args<T> &a, Control &snap) {
  const unsigned *src = (const unsigned *)a.ctl;
  unsigned *dst = (unsigned *)&snap;
  for (int i = threadIdx.x; i < (int)(sizeof(Control) / 4); i += kThreads) dst[i] = __ldcg(src + i);
  __syncthreads();
}

// All blocks arrive; the last one reduces, decides and publishes the next
// Control record, then releases the team.  After phase A nothing needs
// deciding (B always follows), so that barrier only synchronises.  Every wait
// is bounded: on timeout the team's abort flag is raised and every block
// leaves; the host reports PRIMA_ERR_TIMEOUT.  A one-block team synchronises
// with __syncthreads and keeps its Control in shared memory.
template <typename T>
__device__ bool barrier_decide(const Args<T> &a, Control &snap, int phase, const Team &tm, unsigned char *smem,
                               HotShared &hs, unsigned &par) {
  // After phase A comes phase B, whose tiles and vectors are already final:
  // one warp stages its first tiles while the block waits for the release
  // (the last block, right after releasing the others).
  const bool prime = phase == PH_A && tm.nb > 1;
  // After phase B comes phase A (or a checkpoint first, which leaves the
  // list alone): its tile list is static, so stage that too while waiting.
  const bool list_a = phase == PH_B && tm.nb > 1;
  auto prime_b = [&] {
    const T *vecs[6];
    const int nv = b_operands(a, snap, vecs);
    prime_tiles<T>(a.ntiles_k, tm.nb, tm.rank, a.tiles_k, a.kp, a.kci, a.kv, vecs, nv, smem, hs);
  };
  auto list_a_tiles = [&] {
#if PRIMA_SPEC_A
    // nearly every trial is accepted: stage A's first tiles as an accepted
    // trial's phase A reads them (the new x, the pending commit's sums and
    // K'); a decision that goes elsewhere lets them land and drops them
    const T *vecs[6] = {a.x[snap.xc ^ 1], a.sx, a.skty, a.c, a.l, a.u};
    prime_tiles<T>(a.ntiles_t, tm.nb, tm.rank, a.tiles_t, a.tp, a.tci, a.tv, vecs, 6, smem, hs);
#else
    list_tiles(a.ntiles_t, tm.nb, tm.rank, a.tiles_t, hs);
#endif
  };
  __shared__ int s_last, s_ok;
  __shared__ double s_red[kMaxQ];
  if (tm.nb == 1) {
    __syncthreads();
    if (*((volatile int32_t *)&a.sync->abort)) return false;
    uint64_t t0 = 0;
    if (a.prof && threadIdx.x == 0) {
      t0 = global_timer_ns();
      if (a.prof->t_release) {
        a.prof->phase_ns[phase & 7] += t0 - a.prof->t_release;
        a.prof->phase_count[phase & 7] += 1;
      }
    }
    if (phase == PH_A) {
      if (threadIdx.x == 0) snap.phase = PH_B;
    } else {
      decide<T>(a, snap, phase, tm, s_red);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (a.prof) {
        const uint64_t t1 = global_timer_ns();
        a.prof->decide_ns += t1 - t0;
        a.prof->t_release = t1;
      }
      if (snap.phase == PH_DONE && a.queue) a.team_next[a.team] = atomicAdd(a.queue, 1);
    }
    __syncthreads();
    return true;
  }
  if (phase == PH_A || phase == PH_B) {
    // The trial's barriers.  Every block counts itself in on the team's
    // arrival counter with a release increment it does not wait for (or, with
    // PRIMA_HOT_RED 0, on its group's counter, the last of each group then on
    // the team's); no counter is ever reset: the k-th barrier completes when
    // the team's counter reads k * G (G the blocks, or the groups), and every
    // block waits for the whole team.  After phase B every block then reduces the
    // trial's partials itself, in the same fixed order, and takes the same
    // step-size decision on its own copy of the Control record.  Nothing is
    // published and no block waits for a deciding block: the decision inputs
    // (partials, iteration counts, step, weight) are the same everywhere, and
    // the decision reads no clock and no flag.
    unsigned long long &s_ep = hot_epoch();
    const int groups = PRIMA_HOT_RED ? tm.nb : (tm.nb < kArriveGroups ? tm.nb : kArriveGroups);
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned long long target = (s_ep + 1) * (unsigned long long)groups;
      if (a.prof) {
        const uint64_t now = global_timer_ns(), tr = ldv(&a.prof->t_release);
        if (tr) {
          const unsigned long long d = now - tr;
          atomicAdd((unsigned long long *)&a.prof->arrive_ns[phase & 7], d);
          if (tm.rank < kProfBlocks) {
            a.prof->block_arrive[phase == PH_B][tm.rank] += d;  // this block's own slot
            unsigned sm;
            asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
            a.prof->block_sm[tm.rank] = (int32_t)sm;
            if (block_clock()[0]) a.prof->block_work[phase == PH_B][tm.rank] += now - block_clock()[0];
          }
        }
        block_clock()[1] = now;
      }
      s_last = 0;
#if PRIMA_HOT_RED
      (void)target;
      red_add_release_u64(&a.sync->arrive, 1ull);
#else
      // count in on the group's counter; the group's last block counts the
      // group in on the team's
      const int g = tm.rank % groups;
      const unsigned long long gsize = (unsigned long long)((tm.nb - g + groups - 1) / groups);
      const unsigned long long gold = atom_add_acq_rel_u64(a.arrive_groups + (size_t)g * kArriveStride, 1ull);
      if (gold + 1 == (s_ep + 1) * gsize) {
        const unsigned long long old = atom_add_acq_rel_u64(&a.sync->arrive, 1ull);
        s_last = old + 1 == target;
      }
#endif
      s_ok = 1;
    }
    __syncthreads();
    if (prime && threadIdx.x >> 5 == 1) {
      prime_b();
    } else if (list_a && threadIdx.x >> 5 == 1) {
      list_a_tiles();
    } else if (threadIdx.x == 0) {
      const unsigned long long target = (s_ep + 1) * (unsigned long long)groups;
      if (!s_last) {
        // A poll is one load; the abort flag and the poll limit are read
        // every PRIMA_ABORT_EVERY polls only, and not at all once the team
        // is in: a block that gave up after arriving is missed here, and
        // the others meet its abort at the next barrier, which it never
        // reaches.
        long long spins = 0;
#if PRIMA_POLL_RELAXED
        while (ld_relaxed_u64(&a.sync->arrive) < target) {
#else
        while (ld_acquire_u64(&a.sync->arrive) < target) {
#endif
          if (++spins % PRIMA_ABORT_EVERY == 0) {
            if (*((volatile int32_t *)&a.sync->abort)) {
              s_ok = 0;
              break;
            }
            if (spins > a.P.spin_limit) {
              atomicExch(&a.sync->abort, 1);
              s_ok = 0;
              break;
            }
          }
#if PRIMA_POLL_SLEEP_NS > 0
          __nanosleep(PRIMA_POLL_SLEEP_NS);
#endif
        }
#if PRIMA_POLL_RELAXED
        fence_acq_rel_gpu();  // the polls were relaxed: acquire once, on leaving
#endif
      } else if (*((volatile int32_t *)&a.sync->abort)) {
        s_ok = 0;
      }
      s_ep += 1;
      if (a.prof) {
        const uint64_t now = global_timer_ns();
        if (tm.rank < kProfBlocks && block_clock()[1]) a.prof->block_wait[phase == PH_B][tm.rank] += now - block_clock()[1];
        block_clock()[0] = now;  // the next phase starts (after B: once decided)
      }
      // the last arrival (with one-level counting: rank 0 seeing the
      // release) stands for the release
      if (a.prof && (PRIMA_HOT_RED ? tm.rank == 0 : s_last)) {
        const uint64_t now = global_timer_ns(), tr = ldv(&a.prof->t_release);
        if (tr) {
          a.prof->phase_ns[phase & 7] += now - tr;
          a.prof->phase_count[phase & 7] += 1;
        }
        a.prof->t_release = now;
      }
      if (phase == PH_A) snap.phase = PH_B;
    }
    __syncthreads();
    if (!s_ok) {
      if (hs.primed && threadIdx.x == 0) {  // leaving: let the staged copies land first (bounded)
        constexpr int S = HotLayout<T>::kStages;
        for (int u = 0; u < hs.issued; u++) {
          mbar_wait(&hs.bars[u % S], (par >> (u % S)) & 1u);
          par ^= 1u << (u % S);
        }
        hs.primed = 0;
      }
      return false;
    }
    if (phase == PH_B) {
      const uint64_t t0 = (a.prof && tm.rank == 0 && threadIdx.x == 0) ? global_timer_ns() : 0;
      decide<T>(a, snap, PH_B, tm, s_red);
      __syncthreads();
#if PRIMA_SPEC_A
      if (hs.primed && !(snap.phase == PH_A && snap.pend)) {
        // the staged tiles were for an accepted trial's phase A: let their
        // bytes land (bounded), then drop them
        constexpr int S = HotLayout<T>::kStages;
        const int issued = hs.issued;
        if (threadIdx.x == 0)
          for (int u = 0; u < issued; u++) mbar_wait(&hs.bars[u % S], (par >> (u % S)) & 1u);
        __syncthreads();
        for (int u = 0; u < issued; u++) par ^= 1u << (u % S);
        if (threadIdx.x == 0) hs.primed = 0;
        __syncthreads();
      }
#endif
      if (t0) {
        a.prof->decide_b_ns += global_timer_ns() - t0;
        a.prof->decide_b_count += 1;
        a.prof->decide_ns += global_timer_ns() - t0;
      }
      if (a.prof && threadIdx.x == 0) {
        const uint64_t now = global_timer_ns();
        if (tm.rank < kProfBlocks) a.prof->block_decide[tm.rank] += now - block_clock()[0];
        block_clock()[0] = now;
      }
    }
    return true;
  }
  unsigned &s_gen = barrier_generation();
  __syncthreads();
  if (threadIdx.x == 0) {
    if (a.prof) {
      const uint64_t tr = ldv(&a.prof->t_release);
      if (tr) {
        const unsigned long long d = global_timer_ns() - tr;
        atomicAdd((unsigned long long *)&a.prof->arrive_ns[phase & 7], d);
        if ((phase == PH_A || phase == PH_B) && tm.rank < kProfBlocks) {
          a.prof->block_arrive[phase == PH_B][tm.rank] += d;  // this block's own slot
          unsigned sm;
          asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
          a.prof->block_sm[tm.rank] = (int32_t)sm;
        }
      }
    }
    const unsigned old = atom_add_acq_rel(&a.sync->count, 1u);
    s_last = old == (unsigned)(tm.nb - 1);
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    __shared__ uint64_t s_t0;
    if (a.prof && threadIdx.x == 0) {
      s_t0 = global_timer_ns();
      const uint64_t tr = ldv(&a.prof->t_release);
      if (tr) {
        a.prof->phase_ns[phase & 7] += s_t0 - tr;
        a.prof->phase_count[phase & 7] += 1;
      }
    }
    if (phase == PH_A) {
      if (threadIdx.x == 0) snap.phase = PH_B;
    } else {
      decide<T>(a, snap, phase, tm, s_red);
    }
    __syncthreads();
    if (phase != PH_A) publish_control(a, snap);
    if (threadIdx.x == 0 && snap.phase == PH_DONE && a.queue) a.team_next[a.team] = atomicAdd(a.queue, 1);
    if (a.prof && threadIdx.x == 0) {
      const uint64_t t1 = global_timer_ns();
      a.prof->decide_ns += t1 - s_t0;
      a.prof->t_release = t1;
      if (phase == PH_B) {
        a.prof->decide_b_ns += t1 - s_t0;
        a.prof->decide_b_count += 1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (*((volatile int32_t *)&a.sync->abort)) s_ok = 0;
      a.sync->count = 0;
      __threadfence();
      st_release(&a.sync->gen, s_gen + 1);
      s_gen += 1;
    }
  } else if (threadIdx.x == 0) {
    long long spins = 0;
    while (ld_acquire(&a.sync->gen) == s_gen) {
      if (*((volatile int32_t *)&a.sync->abort)) {
        s_ok = 0;
        break;
      }
      if (++spins > a.P.spin_limit) {
        atomicExch(&a.sync->abort, 1);
        s_ok = 0;
        break;
      }
      __nanosleep(32);
    }
    s_gen += 1;
    if (phase == PH_A) snap.phase = PH_B;
  }
  __syncthreads();
  if (s_ok) load_control(a, snap);
  return s_ok;
}

// One whole solve by one team: the phase machine from the Control record the
// host prepared to PH_DONE.  False: the team's abort flag went up.
template <typename T>
__device__ __forceinline__ bool run_solve(const Args<T> &a, const Team &tm, Control &snap, HotShared &hs,
                                          unsigned &par, unsigned char *s_dyn) {
  T *s_prod = reinterpret_cast<T *>(s_dyn);
  if (threadIdx.x == 0) {
    hs.diag = a.sync->diag;
    hs.prog = a.progress;
  }
  if (threadIdx.x == 0 && tm.nb > 1) {
    barrier_generation() = ld_acquire(&a.sync->gen);
    hot_epoch() = 0;  // the host zeroes the arrival counter before every solve
    block_clock()[0] = block_clock()[1] = 0;
  }
  load_control(a, snap);  // (syncs the block)
  bool alive = true;
  for (;;) {
    const int ph = snap.phase;
    if (ph == PH_DONE) break;
    if (threadIdx.x == 0) {
      progress(a.progress, 0, ph);
      progress(a.progress, 1, (int32_t)snap.total_trials);
      progress(a.progress, 9, snap.iteration);
    }
    bool ok = true;
    switch (ph) {
      case PH_INIT: phase_init(a, snap, tm, s_prod); break;
      case PH_A: ok = phase_a(a, snap, tm, s_dyn, hs, par); break;
      case PH_B: ok = phase_b(a, snap, tm, s_dyn, hs, par); break;
      case PH_F: phase_f(a, snap, tm, s_prod); break;
      case PH_R: phase_r(a, snap, tm); break;
      case PH_W: phase_w(a, snap, tm); break;
      case PH_R2: phase_r2(a, snap, tm, s_prod); break;
      default: break;
    }
    (void)ok;  // a failed tile wait has raised the team's abort flag; the barrier sees it
    if (!barrier_decide(a, snap, ph, tm, s_dyn, hs, par)) {
      alive = false;
      break;
    }
  }
  if (tm.nb == 1) publish_control(a, snap);  // the host reads the final record
  return alive;
}

__device__ __forceinline__ void init_stages(HotShared &hs) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < kMaxStages; i++) mbar_init(&hs.bars[i], 1);
    fence_mbar_init();
    hs.primed = 0;
    hs.listed = nullptr;
    hs.tag = 0;
    hs.diag = nullptr;
    hs.prog = nullptr;
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kThreads, kMinBlocksPerSm<T>) pdhg_kernel(Args<T> a) {
  __shared__ Control snap;
  __shared__ double s_part[kMaxQ];
  __shared__ HotShared hs;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  const Team tm{(int)gridDim.x, (int)blockIdx.x, s_part};
  unsigned par = 0;  // mbarrier phase parity of the tile stages
  init_stages(hs);
  run_solve(a, tm, snap, hs, par, s_dyn);
}

// Many independent LPs in one launch: the grid is cut into teams of tb
// blocks; team k starts with instance k (instances come largest first) and,
// whenever it finishes one, takes the next index from a shared queue (the
// deciding block of the finishing barrier takes it for the whole team).  Each
// instance has its own Control, Sync and state; a team runs exactly the
// single-solve phase machine on it.
template <typename T>
__global__ void __launch_bounds__(kThreads, kMinBlocksPerSm<T>)
    pdhg_batch_kernel(const Args<T> *__restrict__ args, int count, int tb, int32_t *queue, int32_t *team_next) {
  __shared__ Control snap;
  __shared__ double s_part[kMaxQ];
  __shared__ HotShared hs;
  __shared__ Args<T> s_a;
  __shared__ int s_inst;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  const int team = (int)blockIdx.x / tb;
  const Team tm{tb, (int)blockIdx.x % tb, s_part};
  unsigned par = 0;
  init_stages(hs);
  int inst = team;
  while (inst < count) {
    const unsigned *src = reinterpret_cast<const unsigned *>(args + inst);
    unsigned *dst = reinterpret_cast<unsigned *>(&s_a);
    for (int i = threadIdx.x; i < (int)(sizeof(Args<T>) / 4); i += kThreads) dst[i] = __ldg(src + i);
    __syncthreads();
    if (threadIdx.x == 0) {
      s_a.queue = queue;
      s_a.team_next = team_next;
      s_a.team = team;
    }
    __syncthreads();
    if (!run_solve(s_a, tm, snap, hs, par, s_dyn)) break;
    if (threadIdx.x == 0) s_inst = __ldcg(team_next + team);
    __syncthreads();
    inst = s_inst;
    __syncthreads();
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

// Bump allocator over the context's solver arena (iterate state only; the
// problem itself lives in a PreparedLp).
struct Layout {
  size_t off = 0;
  template <typename U>
  size_t take(int64_t count) {
    const size_t at = off;
    // 64 bytes of slack per buffer: bulk copies move whole 16-byte granules
    off += ((size_t)std::max<int64_t>(count, 1) * sizeof(U) + 64 + 255) & ~(size_t)255;
    return at;
  }
};

template <typename T>
struct StateLayout {
  size_t x[2], y[2], kx[2], xbar, kty, sx, sy, skx, skty, xr, yr, xo, yo, rco, part, ctl, sync, groups, prof, bytes;
  size_t xa = 0, ya = 0, kxa = 0, ktya = 0, cw = 0, lw = 0, uw = 0, qw = 0, ylo = 0;
  StateLayout(int32_t n, int32_t m, int blocks, bool anchored) {
    Layout L;
    if (anchored) {
      xa = L.take<double>(n);
      ktya = L.take<double>(n);
      ya = L.take<double>(m);
      kxa = L.take<double>(m);
      cw = L.take<T>(n);
      lw = L.take<T>(n);
      uw = L.take<T>(n);
      qw = L.take<T>(m);
      ylo = L.take<T>(m);
    }
    for (int i = 0; i < 2; i++) {
      x[i] = L.take<T>(n);
      y[i] = L.take<T>(m);
      kx[i] = L.take<T>(m);
    }
    xbar = L.take<T>(n);
    kty = L.take<T>(n);
    sx = L.take<T>(n);
    skty = L.take<T>(n);
    xr = L.take<T>(n);
    sy = L.take<T>(m);
    skx = L.take<T>(m);
    yr = L.take<T>(m);
    xo = L.take<double>(n);
    rco = L.take<double>(n);
    yo = L.take<double>(m);
    part = L.take<double>((int64_t)dev::kSlots * blocks);
    ctl = L.take<dev::Control>(1);
    sync = L.take<dev::Sync>(1);
    groups = L.take<unsigned long long>((int64_t)dev::kArriveGroups * dev::kArriveStride);
    prof = L.take<dev::Prof>(1);
    bytes = L.off;
  }
};

template <typename T>
constexpr size_t dyn_smem() {
  return std::max((size_t)dev::kTileCap * sizeof(T), dev::HotLayout<T>::total);
}

template <typename T>
int32_t max_coresident_blocks(Ctx *c, int *out) {
  int per_sm = 0;
  PRIMA_CUDA_TRY(cudaFuncSetAttribute(dev::pdhg_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem<T>()));
  PRIMA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::pdhg_kernel<T>, dev::kThreads, dyn_smem<T>()));
  if (per_sm < 1) {
    set_error("solver kernel cannot be resident on an SM");
    return PRIMA_ERR_CUDA;
  }
  *out = per_sm * c->num_sms;
  return PRIMA_OK;
}

// Blocks for a solve: small problems (<= 4096 rows and columns) run as one
// block, whose barriers never leave the SM; anything larger spreads over as
// many co-resident blocks as have a tile of work (the latency of a tile is
// hidden by the other blocks on the SM, not by the tile itself).
inline int team_blocks(int64_t n, int64_t m, int max_blocks) {
  const int64_t work = std::max<int64_t>(std::max(n, m), 1);
  if (work <= 4096) return 1;
  return (int)std::min<int64_t>(max_blocks, (work + dev::kTileRows - 1) / dev::kTileRows);
}

// The row caps of the two tile tables a problem keeps per precision: full
// tiles (two rows per thread) and half tiles.
constexpr int kTableRows[2] = {dev::kHotRows<float> == dev::kHotRows<double> ? dev::kHotRows<float> : 0,
                               dev::kHotRows<float> / 2};
static_assert(kTableRows[0] > 0, "both precisions cut tiles of the same rows");

// Builds (once per prepared problem and precision) both tile tables of K
// and K' with every tile's cost; the device copies are dealt per team size
// by ensure_deal.
template <typename T>
int32_t ensure_tile_tables(PreparedLp &L, cudaStream_t s) {
  const int w = sizeof(T) == 8;
  if (L.ntiles[w][0][0] || L.ntiles[w][0][1] || (L.m == 0 && L.n == 0)) return PRIMA_OK;
  std::vector<int32_t> kci((size_t)L.nnz), tci((size_t)L.nnz);
  if (L.nnz) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(kci.data(), L.kci(), (size_t)L.nnz * 4, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaMemcpyAsync(tci.data(), L.tci(), (size_t)L.nnz * 4, cudaMemcpyDeviceToHost, s));
    PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  }
  const std::vector<int32_t> *rps[2] = {&L.h_kp, &L.h_tp};
  const int32_t *cis[2] = {kci.data(), tci.data()};
  const int64_t cols[2] = {L.n, L.m};
  for (int v = 0; v < 2; v++) {
    L.tiles_nb[w][v] = 0;
    for (int k = 0; k < 2; k++) {
      L.h_tiles[w][v][k] = tile_table(rps[k]->data(), (int64_t)rps[k]->size() - 1, dev::HotLayout<T>::kCap,
                                      kTableRows[v]);
      L.h_tile_cost[w][v][k] = tile_costs(L.h_tiles[w][v][k], rps[k]->data(), cis[k], cols[k], (int)sizeof(T));
      L.ntiles[w][v][k] = (int32_t)L.h_tiles[w][v][k].size() - 1;
    }
  }
  return PRIMA_OK;
}

// The device copies of tile table v dealt to a team of nb blocks.
template <typename T>
int32_t ensure_deal(PreparedLp &L, int v, int nb, cudaStream_t s) {
  const int w = sizeof(T) == 8;
  if (L.tiles_nb[w][v] == nb) return PRIMA_OK;
  for (int k = 0; k < 2; k++) {
    static_assert(sizeof(TileEdge) == sizeof(int2), "the device reads the table as int2");
    const std::vector<TileEdge> pairs = deal_tiles(L.h_tiles[w][v][k], L.h_tile_cost[w][v][k], nb);
    int32_t rc;
    if ((rc = L.b_tiles[w][v][k].reserve(std::max<size_t>(1, pairs.size()) * sizeof(int2)))) return rc;
    if (!pairs.empty())
      PRIMA_CUDA_TRY(cudaMemcpyAsync(L.b_tiles[w][v][k].ptr, pairs.data(), pairs.size() * sizeof(int2),
                                     cudaMemcpyHostToDevice, s));
  }
  PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  L.tiles_nb[w][v] = nb;
  return PRIMA_OK;
}

template <typename T>
std::vector<T> narrow(const std::vector<double> &v) {
  std::vector<T> out(v.size());
  for (size_t i = 0; i < v.size(); i++) out[i] = (T)v[i];
  return out;
}

struct SolveRequest {
  const prima_params *params;
  const prima_warm_start *warm;
  const volatile int32_t *cancel;
  double *x_out, *y_out, *rc_out;
  prima_solution_info *info;
  bool anchored = false;    // iterate on the residual problem around an FP64 anchor
  double round_rho = 0.0;   // anchored: error reduction that opens a new round (0: never)
  int32_t *rounds = nullptr;
  int table = 0;            // hot-phase tile table: 0 full tiles, 1 half tiles
};

int32_t check_warm(const PreparedLp &L, const prima_warm_start *w) {
  if (!w) return PRIMA_OK;
  if (L.n > 0 && !w->primal) return (set_error("requirement failed: warm start primal is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  for (int32_t i = 0; i < L.n; i++)
    if (!std::isfinite(w->primal[i]))
      return (set_error("requirement failed: warm start primal vector is not finite"), PRIMA_ERR_INVALID_ARGUMENT);
  if (L.m > 0 && !w->dual) return (set_error("requirement failed: warm start dual is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  for (int32_t r = 0; r < L.m; r++)
    if (!std::isfinite(w->dual[r]))
      return (set_error("requirement failed: warm start dual vector is not finite"), PRIMA_ERR_INVALID_ARGUMENT);
  return PRIMA_OK;
}

// One solve in flight: the prepared problem, the caller's request and the
// device-side arguments built for it.
template <typename T>
struct Job {
  PreparedLp *L = nullptr;
  SolveRequest req{};
  Clock::time_point t0;
  dev::Args<T> a{};
  double setup_ms = 0.0;
};

// Everything a solve needs on the device before its launch that does not
// depend on where its state lives: the precision copies, the FP64 copies for
// anchored mode, the tile tables.
template <typename T>
int32_t prepare_job(Ctx *c, Job<T> &j) {
  NvtxRange range("prima: prepare solve");
  int32_t rc;
  if ((rc = check_warm(*j.L, j.req.warm))) return rc;
  PreparedLp &L = *j.L;
  if ((rc = L.materialise<T>(c->stream))) return rc;
  if (j.req.anchored && (rc = L.materialise<double>(c->stream))) return rc;
  return ensure_tile_tables<T>(L, c->stream);
}

// Per-phase device timing, printed to stderr after each solve, when the
// environment sets PRIMA_PHASE_TIMES.
bool phase_times() {
  static const bool on = std::getenv("PRIMA_PHASE_TIMES") != nullptr;
  return on;
}

// The progress record the kernel keeps when PRIMA_DEBUG_PROGRESS is set:
// host-mapped memory the host reads while the kernel runs.
volatile int32_t *progress_record(bool device_side) {
  static int32_t *host = nullptr, *dev = nullptr;
  static const bool on = std::getenv("PRIMA_DEBUG_PROGRESS") != nullptr;
  if (!on) return nullptr;
  if (!host) {
    if (cudaHostAlloc((void **)&host, 256 * 16 * 4, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&dev, host, 0) != cudaSuccess) {
      cudaGetLastError();
      host = dev = nullptr;
      return nullptr;
    }
    std::memset(host, 0, 256 * 16 * 4);
  }
  return device_side ? dev : host;
}

// Pdhg.Solve's initialise (Pdhg.scala:250-309) on the host -- the opening
// step, primal weight and the projected start point -- and the Args, Control
// and Sync records, with the iterate state at `base` laid out as S.
template <typename T>
int32_t setup_job(Ctx *c, Job<T> &j, char *base, const StateLayout<T> &S, int blocks) {
  PreparedLp &L = *j.L;
  const SolveRequest &req = j.req;
  const prima_params *p = req.params;
  cudaStream_t s = c->stream;
  const int32_t n = L.n, m = L.m, neq = L.neq;
  const bool anchored = req.anchored;

  if (L.n || L.m) {
    const int32_t rc = ensure_deal<T>(L, req.table, blocks, s);
    if (rc) return rc;
  }

  const double bound = L.scaled_spectral_bound;
  double step = bound > 0.0 ? 1.0 / bound : 1.0;
  double weight = (L.scaled_c_norm > 0.0 && L.scaled_q_norm > 0.0) ? L.scaled_c_norm / L.scaled_q_norm : 1.0;
  if (req.warm && !std::isnan(req.warm->step_size)) step = req.warm->step_size;
  if (req.warm && !std::isnan(req.warm->primal_weight)) weight = req.warm->primal_weight;

  // start point: zero (or the warm start scaled in), projected into the box;
  // in anchored mode it becomes the FP64 anchor and the correction is zero
  {
    std::vector<double> x0((size_t)n, 0.0), y0((size_t)m, 0.0);
    for (int32_t i = 0; i < n; i++) {
      const double v = req.warm ? req.warm->primal[i] / L.h_cs[i] : 0.0, lo = L.h_sl[i], hi = L.h_su[i];
      x0[i] = v < lo ? lo : (v > hi ? hi : v);
    }
    if (req.warm)
      for (int32_t r = 0; r < m; r++) {
        const double v = req.warm->dual[r] / L.h_rs[r];
        y0[r] = (r >= neq && v < 0.0) ? 0.0 : v;
      }
    if (anchored) {
      if (n) {
        PRIMA_CUDA_TRY(cudaMemcpyAsync(base + S.xa, x0.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
        PRIMA_CUDA_TRY(cudaMemsetAsync(base + S.x[0], 0, (size_t)n * sizeof(T), s));
      }
      if (m) {
        PRIMA_CUDA_TRY(cudaMemcpyAsync(base + S.ya, y0.data(), (size_t)m * 8, cudaMemcpyHostToDevice, s));
        PRIMA_CUDA_TRY(cudaMemsetAsync(base + S.y[0], 0, (size_t)m * sizeof(T), s));
      }
    } else {
      const std::vector<T> xx = narrow<T>(x0), yy = narrow<T>(y0);
      if (n) PRIMA_CUDA_TRY(cudaMemcpyAsync(base + S.x[0], xx.data(), (size_t)n * sizeof(T), cudaMemcpyHostToDevice, s));
      if (m) PRIMA_CUDA_TRY(cudaMemcpyAsync(base + S.y[0], yy.data(), (size_t)m * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  }

  dev::Args<T> &a = j.a;
  std::memset(&a, 0, sizeof(a));
  a.n = n;
  a.m = m;
  a.neq = neq;
  const int w = sizeof(T) == 8 ? 1 : 0;
  a.kp = L.kp();
  a.kci = L.kci();
  a.kv = (const T *)L.copies[w].kv.ptr;
  a.tp = L.tp();
  a.tci = L.tci();
  a.tv = (const T *)L.copies[w].tv.ptr;
  a.c = (const T *)L.copies[w].c.ptr;
  a.l = (const T *)L.copies[w].l.ptr;
  a.u = (const T *)L.copies[w].u.ptr;
  a.q = (const T *)L.copies[w].q.ptr;
  a.c0 = L.c0();
  a.l0 = L.l0();
  a.u0 = L.u0();
  a.q0 = L.q0();
  a.cs = L.cs();
  a.rs = L.rs();
  for (int i = 0; i < 2; i++) {
    a.x[i] = (T *)(base + S.x[i]);
    a.y[i] = (T *)(base + S.y[i]);
    a.kx[i] = (T *)(base + S.kx[i]);
  }
  a.xbar = (T *)(base + S.xbar);
  a.kty = (T *)(base + S.kty);
  a.sx = (T *)(base + S.sx);
  a.sy = (T *)(base + S.sy);
  a.skx = (T *)(base + S.skx);
  a.skty = (T *)(base + S.skty);
  a.xr = (T *)(base + S.xr);
  a.yr = (T *)(base + S.yr);
  a.xo = (double *)(base + S.xo);
  a.yo = (double *)(base + S.yo);
  a.rco = (double *)(base + S.rco);
  a.partials = (double *)(base + S.part);
  a.max_blocks = blocks;
  a.ctl = (dev::Control *)(base + S.ctl);
  a.sync = (dev::Sync *)(base + S.sync);
  a.prof = phase_times() ? (dev::Prof *)(base + S.prof) : nullptr;
  const int tv = j.req.table;  // tile table: full or half tiles
  a.tiles_k = (const int2 *)L.b_tiles[w][tv][0].ptr;
  a.tiles_t = (const int2 *)L.b_tiles[w][tv][1].ptr;
  a.ntiles_k = L.ntiles[w][tv][0];
  a.ntiles_t = L.ntiles[w][tv][1];

  if (anchored) {
    a.anchored = 1;
    a.xa = (double *)(base + S.xa);
    a.ya = (double *)(base + S.ya);
    a.kxa = (double *)(base + S.kxa);
    a.ktya = (double *)(base + S.ktya);
    a.sc = L.sc();
    a.sq = L.sq();
    a.sl = L.sl();
    a.su = L.su();
    a.kv64 = (const double *)L.copies[1].kv.ptr;
    a.tv64 = (const double *)L.copies[1].tv.ptr;
    a.cw = (T *)(base + S.cw);
    a.lw = (T *)(base + S.lw);
    a.uw = (T *)(base + S.uw);
    a.qw = (T *)(base + S.qw);
    a.ylo = (T *)(base + S.ylo);
    a.c = a.cw;
    a.l = a.lw;
    a.u = a.uw;
    a.q = a.qw;
  }

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
  PRIMA_CUDA_TRY(cudaMemcpyAsync(a.ctl, &ctl, sizeof(ctl), cudaMemcpyHostToDevice, s));
  PRIMA_CUDA_TRY(cudaMemcpyAsync(a.sync, &sync, sizeof(sync), cudaMemcpyHostToDevice, s));
  a.arrive_groups = (unsigned long long *)(base + S.groups);
  PRIMA_CUDA_TRY(cudaMemsetAsync(a.arrive_groups, 0,
                                 sizeof(unsigned long long) * dev::kArriveGroups * dev::kArriveStride, s));
  if (a.prof) PRIMA_CUDA_TRY(cudaMemsetAsync(a.prof, 0, sizeof(dev::Prof), s));

  dev::Params &P = a.P;
  P.eps_abs = p->eps_abs;
  P.eps_rel = p->eps_rel;
  P.rhs_norm = L.rhs_norm;
  P.obj_norm = L.obj_norm;
  P.max_iterations = p->max_iterations;
  P.eval_freq = p->evaluation_frequency;
  P.time_limit_ms = p->time_limit_ms;
  P.infeas_tol = p->infeasibility_tolerance;
  P.r_suff = p->restart_sufficient_reduction;
  P.r_nec = p->restart_necessary_reduction;
  P.r_art = p->restart_artificial_fraction;
  P.smoothing = p->primal_weight_smoothing;
  P.matrix_norm = L.orig_spectral_bound;
  P.offset = L.host ? L.host->objective_offset : 0.0;
  P.round_rho = anchored ? req.round_rho : 0.0;
  P.spin_limit = c->wait_limit > 0 ? (long long)c->wait_limit : dev::kDefaultSpinLimit;
  a.cancel = c->cancel_mapped_dev;
  a.progress = progress_record(true);
  PRIMA_CUDA_TRY(cudaStreamSynchronize(s));
  j.setup_ms = ms_since(j.t0);
  P.setup_ms = j.setup_ms;
  return PRIMA_OK;
}

// After the launch: the final Control record, the solution in caller units
// and the info fields.  kms: the launch's device time.
template <typename T>
int32_t finish_job(Ctx * /*c*/, Job<T> &j, float kms, int blocks) {
  const SolveRequest &req = j.req;
  const dev::Args<T> &a = j.a;
  const int32_t n = j.L->n, m = j.L->m;
  dev::Control ctl;
  dev::Sync sync;
  PRIMA_CUDA_TRY(cudaMemcpy(&ctl, a.ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  PRIMA_CUDA_TRY(cudaMemcpy(&sync, a.sync, sizeof(sync), cudaMemcpyDeviceToHost));
  if (sync.abort) ctl.error = PRIMA_ERR_TIMEOUT;
  if (req.x_out && n) PRIMA_CUDA_TRY(cudaMemcpy(req.x_out, a.xo, (size_t)n * 8, cudaMemcpyDeviceToHost));
  if (req.y_out && m) PRIMA_CUDA_TRY(cudaMemcpy(req.y_out, a.yo, (size_t)m * 8, cudaMemcpyDeviceToHost));
  if (req.rc_out && n) PRIMA_CUDA_TRY(cudaMemcpy(req.rc_out, a.rco, (size_t)n * 8, cudaMemcpyDeviceToHost));
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
  info->setup_ms = j.setup_ms;
  info->trials = ctl.total_trials;
  info->solve_ms = (int64_t)ms_since(j.t0);
  info->blocks = blocks;
  info->tile_rows = kTableRows[req.table];
  if (req.rounds) *req.rounds = ctl.rounds;
  if (a.prof) {
    dev::Prof prof;
    PRIMA_CUDA_TRY(cudaMemcpy(&prof, a.prof, sizeof(prof), cudaMemcpyDeviceToHost));
    static const char *names[8] = {"init", "A", "B", "F", "R", "W", "-", "R2"};
    std::fprintf(stderr, "[prima] blocks=%d tiles=%d/%d trials=%lld decide %.2f us/barrier:", blocks, a.ntiles_k,
                 a.ntiles_t, (long long)ctl.total_trials,
                 1e-3 * (double)prof.decide_ns / std::max<int64_t>(1, 2 * ctl.total_trials));
    if (prof.decide_b_count) {
      const double nb = (double)prof.decide_b_count;
      std::fprintf(stderr, " | decide B %.2f us (partials %.2f) |", 1e-3 * (double)prof.decide_b_ns / nb,
                   1e-3 * (double)prof.reduce_b_ns / nb);
    }
    std::fprintf(stderr, " | mean arrival:");
    for (int k = 0; k < 8; k++)
      if (prof.phase_count[k] && prof.arrive_ns[k])
        std::fprintf(stderr, " %s %.2f us", names[k], 1e-3 * (double)prof.arrive_ns[k] / ((double)prof.phase_count[k] * blocks));
    std::fprintf(stderr, " |");
    for (int k = 0; k < 8; k++)
      if (prof.phase_count[k])
        std::fprintf(stderr, " %s %.2f us x%lld", names[k], 1e-3 * (double)prof.phase_ns[k] / (double)prof.phase_count[k],
                     (long long)prof.phase_count[k]);
    std::fprintf(stderr, "\n");
    // per-block arrival spread: the slowest blocks, their SMs and tile counts
    const int nbp = std::min(blocks, dev::kProfBlocks);
    for (int ph = 0; ph < 2 && nbp > 1; ph++) {
      const int64_t cnt = prof.phase_count[ph == 0 ? dev::PH_A : dev::PH_B];
      if (!cnt) continue;
      std::vector<std::pair<double, int>> v;
      for (int b = 0; b < nbp; b++) v.push_back({1e-3 * (double)prof.block_arrive[ph][b] / (double)cnt, b});
      std::sort(v.begin(), v.end());
      const int32_t nt = ph == 0 ? a.ntiles_t : a.ntiles_k;
      auto tiles_of = [&](int b) { return b < nt ? (nt - b + blocks - 1) / blocks : 0; };
      std::fprintf(stderr, "[prima] phase %s arrival per block: min %.2f p10 %.2f median %.2f p90 %.2f max %.2f us; slowest:",
                   ph == 0 ? "A" : "B", v.front().first, v[nbp / 10].first, v[nbp / 2].first, v[(9 * nbp) / 10].first,
                   v.back().first);
      for (int k = 0; k < 8 && k < nbp; k++) {
        const int b = v[nbp - 1 - k].second;
        std::fprintf(stderr, " b%d(sm%d,%dt)=%.2f", b, prof.block_sm[b], tiles_of(b), v[nbp - 1 - k].first);
      }
      std::fprintf(stderr, " fastest:");
      for (int k = 0; k < 4 && k < nbp; k++) {
        const int b = v[k].second;
        std::fprintf(stderr, " b%d(sm%d,%dt)=%.2f", b, prof.block_sm[b], tiles_of(b), v[k].first);
      }
      {  // the phase's own work, the barrier wait and (after B) the decision, per block
        double wsum = 0, wmax = 0, tsum = 0, dsum = 0;
        for (int b = 0; b < nbp; b++) {
          const double w = 1e-3 * (double)prof.block_work[ph][b] / (double)cnt;
          wsum += w;
          wmax = std::max(wmax, w);
          tsum += 1e-3 * (double)prof.block_wait[ph][b] / (double)cnt;
          if (ph == 1) dsum += 1e-3 * (double)prof.block_decide[b] / (double)cnt;
        }
        std::fprintf(stderr, " | work mean %.2f max %.2f, barrier wait mean %.2f", wsum / nbp, wmax, tsum / nbp);
        if (ph == 1) std::fprintf(stderr, ", decision mean %.2f", dsum / nbp);
      }
      // mean arrival by SM group of 8 consecutive SM ids (a GPC-sized bucket)
      double by[32] = {0};
      int nby[32] = {0};
      for (int b = 0; b < nbp; b++) {
        const int g = std::min(31, std::max(0, prof.block_sm[b] / 8));
        by[g] += 1e-3 * (double)prof.block_arrive[ph][b] / (double)cnt;
        nby[g]++;
      }
      std::fprintf(stderr, " | by sm/8:");
      for (int g = 0; g < 32; g++)
        if (nby[g]) std::fprintf(stderr, " %.1f", by[g] / nby[g]);
      std::fprintf(stderr, "\n");
    }
  }
  if (a.prof && std::getenv("PRIMA_PHASE_TIMES_CSV")) {
    // the per-block record as a table, one row per block, times in us per trial
    dev::Prof prof;
    PRIMA_CUDA_TRY(cudaMemcpy(&prof, a.prof, sizeof(prof), cudaMemcpyDeviceToHost));
    if (FILE *f = std::fopen(std::getenv("PRIMA_PHASE_TIMES_CSV"), "w")) {
      const double ca = (double)std::max<int64_t>(1, prof.phase_count[dev::PH_A]);
      const double cb = (double)std::max<int64_t>(1, prof.phase_count[dev::PH_B]);
      std::fprintf(f, "block,sm,work_a,work_b,wait_a,wait_b,arrive_a,arrive_b,decide\n");
      for (int b = 0; b < std::min(blocks, dev::kProfBlocks); b++)
        std::fprintf(f, "%d,%d,%.4f,%.4f,%.4f,%.4f,%.4f,%.4f,%.4f\n", b, prof.block_sm[b],
                     1e-3 * (double)prof.block_work[0][b] / ca, 1e-3 * (double)prof.block_work[1][b] / cb,
                     1e-3 * (double)prof.block_wait[0][b] / ca, 1e-3 * (double)prof.block_wait[1][b] / cb,
                     1e-3 * (double)prof.block_arrive[0][b] / ca, 1e-3 * (double)prof.block_arrive[1][b] / cb,
                     1e-3 * (double)prof.block_decide[b] / cb);
      std::fclose(f);
    }
  }
  if (ctl.error) {
    std::string msg = "a bounded device-side wait gave up; the solve was abandoned";
    if (sync.diag[0]) {
      static const char *tags[4] = {"?", "phase A", "phase B", "SpMV"};
      char buf[256];
      std::snprintf(buf, sizeof(buf), " (first failure: a %s stage wait, stage %d, parity %d, tile %d of %d, block %d)",
                    tags[sync.diag[1] & 3], sync.diag[3], sync.diag[4], sync.diag[5], sync.diag[6], sync.diag[7]);
      msg += buf;
    }
    set_error(msg);
    return PRIMA_ERR_TIMEOUT;
  }
  return PRIMA_OK;
}

void print_progress() {
  volatile int32_t *p = progress_record(false);
  if (!p) return;
  std::fprintf(stderr, "[prima progress]");
  for (int b = 0; b < 4; b++) {
    std::fprintf(stderr, " | b%d:", b);
    for (int w = 0; w < 10; w++) std::fprintf(stderr, " %d", p[b * 16 + w]);
  }
  std::fprintf(stderr, "\n");
  std::fflush(stderr);
}

// Waits for the event ending a launch, forwarding the caller's cancel flag
// to the mapped flag the device polls at evaluation points.
int32_t wait_forwarding_cancel(Ctx *c, cudaEvent_t done, const volatile int32_t *cancel) {
  auto last = Clock::now();
  for (int spin = 0;; spin++) {
    const cudaError_t q = cudaEventQuery(done);
    if (q == cudaSuccess) return PRIMA_OK;
    if (q != cudaErrorNotReady) {
      set_error(std::string("solver kernel: ") + cudaGetErrorString(q));
      return PRIMA_ERR_CUDA;
    }
    if (cancel && *cancel) *(volatile int32_t *)c->cancel_mapped = 1;
    if (spin > 200) std::this_thread::sleep_for(std::chrono::microseconds(20));
    if (progress_record(false) && ms_since(last) > 2000.0) {
      print_progress();
      last = Clock::now();
    }
  }
}

// One cooperative launch of `kernel` with the given arguments, timed by CUDA
// events on the context stream.
template <typename T>
int32_t launch_timed(Ctx *c, const void *kernel, int blocks, void **kargs, const volatile int32_t *cancel,
                     float *kms) {
  NvtxRange range("prima: persistent PDHG launch");
  cudaStream_t s = c->stream;
  cudaEvent_t e0, e1;
  PRIMA_CUDA_TRY(cudaEventCreate(&e0));
  PRIMA_CUDA_TRY(cudaEventCreate(&e1));
  int32_t rc = PRIMA_OK;
  cudaEventRecord(e0, s);
  const cudaError_t le =
      cudaLaunchCooperativeKernel(kernel, dim3(blocks), dim3(dev::kThreads), kargs, dyn_smem<T>(), s);
  if (le != cudaSuccess) {
    set_error(std::string("cooperative launch: ") + cudaGetErrorString(le));
    rc = PRIMA_ERR_CUDA;
  } else {
    cudaEventRecord(e1, s);
    rc = wait_forwarding_cancel(c, e1, cancel);
    if (!rc) cudaEventElapsedTime(kms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Pdhg.Solve on a prepared problem: the host prologue, then the whole
// iteration in one cooperative launch.
template <typename T>
int32_t solve_with_layout(Ctx *c, PreparedLp &L, const SolveRequest &req, Clock::time_point t_start, int bps,
                          int table);

// The solver layout for a multi-block problem: blocks per SM (the most that
// fit, or one fewer: fewer blocks, more tiles each) and the tile table (full
// or half tiles).  Unless the context pins one, each candidate runs a short
// bounded solve of this problem (no outputs) and the fastest per step-size
// trial is kept for the problem and precision; another candidate must beat
// the first (the most blocks, full tiles) by 5 % to be chosen, so that timing
// noise between close candidates does not change the layout, and with it the
// grouping of the team's sums, from run to run.
template <typename T>
int32_t choose_layout(Ctx *c, PreparedLp &L, const SolveRequest &req, int per_sm, int *bps, int *table) {
  const int w = sizeof(T) == 8;
  if (c->pin_bps > 0) {
    *bps = std::min(c->pin_bps, per_sm);
    *table = c->pin_rows > 0 && c->pin_rows <= kTableRows[1] ? 1 : 0;
    return PRIMA_OK;
  }
  if (L.layout_bps[w] > 0) {
    *bps = L.layout_bps[w];
    *table = L.layout_rows[w];
    return PRIMA_OK;
  }
  struct Cand {
    int bps, table;
  } cands[3] = {{per_sm, 0}, {per_sm - 1, 0}, {per_sm, 1}};
  prima_params tp = *req.params;
  tp.max_iterations = 96;
  tp.time_limit_ms = -1.0;
  double best = 0.0;
  int pick = 0;
  for (int k = 0; k < 3; k++) {
    if (cands[k].bps < 1) continue;
    prima_solution_info info;
    SolveRequest tr{&tp, nullptr, nullptr, nullptr, nullptr, nullptr, &info};
    int32_t rc = solve_with_layout<T>(c, L, tr, Clock::now(), cands[k].bps, cands[k].table);
    if (rc) return rc;
    const double per_trial = info.device_ms / (double)std::max<int64_t>(1, info.trials);
    if (k == 0 || per_trial < best * 0.95) {
      best = per_trial;
      pick = k;
    }
  }
  L.layout_bps[w] = cands[pick].bps;
  L.layout_rows[w] = cands[pick].table;
  *bps = cands[pick].bps;
  *table = cands[pick].table;
  return PRIMA_OK;
}

template <typename T>
int32_t solve_on_device(Ctx *c, PreparedLp &L, const SolveRequest &req, Clock::time_point t_start) {
  int32_t rc;
  {
    Job<T> j;
    j.L = &L;
    j.req = req;
    if ((rc = prepare_job(c, j))) return rc;  // the tile tables the layouts need
  }
  int max_blocks = 0;
  if ((rc = max_coresident_blocks<T>(c, &max_blocks))) return rc;
  const int per_sm = max_blocks / c->num_sms;
  int bps = per_sm, table = 0;
  if (team_blocks(L.n, L.m, max_blocks) > 1 && (rc = choose_layout<T>(c, L, req, per_sm, &bps, &table))) return rc;
  return solve_with_layout<T>(c, L, req, t_start, bps, table);
}

template <typename T>
int32_t solve_with_layout(Ctx *c, PreparedLp &L, const SolveRequest &req_in, Clock::time_point t_start, int bps,
                          int table) {
  SolveRequest req = req_in;
  req.table = table;
  Job<T> j;
  j.L = &L;
  j.req = req;
  j.t0 = t_start;
  int32_t rc;
  if ((rc = prepare_job(c, j))) return rc;
  int max_blocks = 0;
  if ((rc = max_coresident_blocks<T>(c, &max_blocks))) return rc;
  max_blocks = std::min(max_blocks, bps * c->num_sms);
  const int blocks = team_blocks(L.n, L.m, max_blocks);
  const StateLayout<T> S(L.n, L.m, blocks, req.anchored);
  if ((rc = c->solver_arena.reserve(S.bytes))) return rc;
  *(volatile int32_t *)c->cancel_mapped = (req.cancel && *req.cancel) ? 1 : 0;
  if ((rc = setup_job(c, j, (char *)c->solver_arena.ptr, S, blocks))) return rc;
  void *kargs[] = {(void *)&j.a};
  float kms = 0.f;
  if ((rc = launch_timed<T>(c, (const void *)dev::pdhg_kernel<T>, blocks, kargs, req.cancel, &kms))) return rc;
  return finish_job(c, j, kms, blocks);
}

template <typename T>
int32_t max_coresident_batch_blocks(Ctx *c, int *out) {
  int per_sm = 0;
  PRIMA_CUDA_TRY(cudaFuncSetAttribute(dev::pdhg_batch_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)dyn_smem<T>()));
  PRIMA_CUDA_TRY(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::pdhg_batch_kernel<T>, dev::kThreads, dyn_smem<T>()));
  if (per_sm < 1) {
    set_error("batch solver kernel cannot be resident on an SM");
    return PRIMA_ERR_CUDA;
  }
  *out = per_sm * c->num_sms;
  return PRIMA_OK;
}

// Team size for a batch: the power of two that minimises a simple model of
// the makespan per iteration round.  An iteration of an instance with w tiles
// (K and K' together) on tb blocks costs about c0 + c1 w / tb: c0 for the two
// team barriers, c1 for a block to stream one tile.  With `teams` teams the
// round takes at least the slowest instance's iteration and at least the
// total spread over the teams.
// No team is larger than the largest instance would use alone (a problem of
// up to 4096 rows and columns runs as one block), so a batch of small LPs
// solves each exactly as its own solve would.
inline int batch_team_blocks(const std::vector<int64_t> &tiles, int max_blocks, int largest_solo) {
  constexpr double c0 = 20.0, c1 = 2.0;  // microseconds, measured on config-2-sized teams
  int best = 1;
  double best_cost = std::numeric_limits<double>::infinity();
  for (int tb = 1; tb <= std::min(max_blocks, largest_solo); tb *= 2) {
    const int teams = std::min<int64_t>((int64_t)tiles.size(), max_blocks / tb);
    double slowest = 0.0, sum = 0.0;
    for (int64_t w : tiles) {
      const double t = c0 + c1 * (double)((w + tb - 1) / tb);
      slowest = std::max(slowest, t);
      sum += t;
    }
    const double cost = std::max(slowest, sum / std::max(teams, 1));
    if (cost < best_cost) best_cost = cost, best = tb;
  }
  return best;
}

// Many solves in one cooperative launch of pdhg_batch_kernel (see there).
// Every job is prepared and set up as a single solve would be, with its own
// state in the batch arena; the Args records go to the device in order of
// decreasing size, the order in which the teams take them.
template <typename T>
int32_t solve_batch_on_device(Ctx *c, std::vector<Job<T>> &jobs, const volatile int32_t *cancel) {
  const int count = (int)jobs.size();
  if (count == 0) return PRIMA_OK;
  int32_t rc;
  for (auto &j : jobs)
    if ((rc = prepare_job(c, j))) return rc;
  int max_blocks = 0;
  if ((rc = max_coresident_batch_blocks<T>(c, &max_blocks))) return rc;
  std::vector<int64_t> tiles((size_t)count), size((size_t)count);
  const int w = sizeof(T) == 8;
  int largest_solo = 1;
  for (int i = 0; i < count; i++) {
    const PreparedLp &L = *jobs[i].L;
    tiles[i] = (int64_t)L.ntiles[w][0][0] + L.ntiles[w][0][1];
    size[i] = (int64_t)L.n + L.m + L.nnz;
    largest_solo = std::max(largest_solo, team_blocks(L.n, L.m, max_blocks));
  }
  const int tb = batch_team_blocks(tiles, max_blocks, largest_solo);
  const int teams = std::min(count, max_blocks / tb);
  std::vector<int> order((size_t)count);
  for (int i = 0; i < count; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return size[x] > size[y]; });

  std::vector<StateLayout<T>> layouts;
  std::vector<size_t> offs;
  layouts.reserve((size_t)count);
  size_t total = 0;
  for (int i = 0; i < count; i++) {
    layouts.emplace_back(jobs[i].L->n, jobs[i].L->m, tb, jobs[i].req.anchored);
    offs.push_back(total);
    total += (layouts.back().bytes + 255) & ~(size_t)255;
  }
  const size_t off_args = total;
  total += ((size_t)count * sizeof(dev::Args<T>) + 255) & ~(size_t)255;
  const size_t off_queue = total;
  total += ((size_t)(teams + 1) * 4 + 255) & ~(size_t)255;
  if ((rc = c->batch_arena.reserve(total))) return rc;
  char *base = (char *)c->batch_arena.ptr;
  *(volatile int32_t *)c->cancel_mapped = (cancel && *cancel) ? 1 : 0;
  for (int i = 0; i < count; i++)
    if ((rc = setup_job(c, jobs[i], base + offs[i], layouts[i], tb))) return rc;

  std::vector<dev::Args<T>> args((size_t)count);
  for (int i = 0; i < count; i++) args[i] = jobs[order[i]].a;
  std::vector<int32_t> queue((size_t)teams + 1, 0);
  queue[0] = teams;  // team k starts with instance k; the queue hands out the rest
  PRIMA_CUDA_TRY(cudaMemcpyAsync(base + off_args, args.data(), (size_t)count * sizeof(dev::Args<T>),
                                 cudaMemcpyHostToDevice, c->stream));
  PRIMA_CUDA_TRY(cudaMemcpyAsync(base + off_queue, queue.data(), queue.size() * 4, cudaMemcpyHostToDevice, c->stream));
  const dev::Args<T> *d_args = (const dev::Args<T> *)(base + off_args);
  int32_t *d_queue = (int32_t *)(base + off_queue);
  int32_t *d_team_next = d_queue + 1;
  int cnt = count, tbv = tb;
  void *kargs[] = {(void *)&d_args, (void *)&cnt, (void *)&tbv, (void *)&d_queue, (void *)&d_team_next};
  float kms = 0.f;
  if ((rc = launch_timed<T>(c, (const void *)dev::pdhg_batch_kernel<T>, teams * tb, kargs, cancel, &kms))) return rc;
  int32_t first_error = PRIMA_OK;
  for (int i = 0; i < count; i++) {
    dev::Control ctl;
    PRIMA_CUDA_TRY(cudaMemcpy(&ctl, jobs[i].a.ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
    rc = finish_job(c, jobs[i], kms, tb);
    // this instance's own device time, from the timer readings it took
    if (ctl.t_end > ctl.t0 && ctl.t0) jobs[i].req.info->device_ms = 1e-6 * (double)(ctl.t_end - ctl.t0);
    if (rc && !first_error) first_error = rc;
  }
  if (std::getenv("PRIMA_PHASE_TIMES"))
    std::fprintf(stderr, "[prima batch] %d instances, %d teams x %d blocks, %.2f ms\n", count, teams, tb, kms);
  return first_error;
}

// Equilibrate (again) if the prepared problem was scaled differently.
int32_t ensure_prepared(Ctx *c, PreparedLp &L, const prima_lp *lp, const prima_params *p) {
  if (L.host == lp && L.scaled_like(p)) return PRIMA_OK;
  const int32_t rc = L.prepare(lp, p, c->stream);
  L.host = lp;
  return rc;
}

int32_t solve_prepared(Ctx *c, PreparedLp &L, const prima_lp *lp, const SolveRequest &req, int bits,
                       Clock::time_point t0) {
  if (!req.info) return (set_error("requirement failed: info is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  int32_t rc;
  if ((rc = validate_params(req.params))) return rc;
  if ((rc = ensure_prepared(c, L, lp, req.params))) return rc;
  return bits == 64 ? solve_on_device<double>(c, L, req, t0) : solve_on_device<float>(c, L, req, t0);
}

// MixedPrecision.solve (MixedPrecision.scala:104-199), reference scheme: a
// reduced-precision pass on the device (FP32, loosened tolerances), an FP64
// re-check of any certificate at the caller's tolerance, and an FP64
// warm-started finish -- also on the device, on the same prepared problem.
//
// REFINEMENT scheme: the same reduced pass and certificate re-check, then the
// finish in FP32 too -- PDHG on the residual problem around an FP64 anchor
// placed at the reduced pass's answer (step size and primal weight carried),
// with the anchor re-centred at every restart and convergence judged in FP64
// on anchor + correction.  Each restart period only has to gain about a
// decade, far inside FP32's precision, so the FP32 iterations reach any
// tolerance FP64 could.  A Farkas ray is another matter: certifying
// infeasibility to a tight tolerance needs the diverging iterate itself to
// 1e-8 or better, beyond an FP32 correction's rounding, so when the reduced
// pass did not end Optimal the finish stays in FP64, as in the reference.
int32_t mixed_passes(Ctx *c, PreparedLp &L, const prima_lp *lp, const prima_params *p,
                     const prima_mixed_params *mp, const volatile int32_t *cancel, double *x_out, double *y_out,
                     double *rc_out, prima_solution_info *info, prima_mixed_info *minfo, Clock::time_point t0) {
  const int32_t n = lp->num_variables, m = lp->num_constraints;
  prima_params rp = *p;
  rp.eps_abs = std::max(p->eps_abs, mp->reduced_tolerance);
  rp.eps_rel = std::max(p->eps_rel, mp->reduced_tolerance);
  rp.max_iterations = std::min(p->max_iterations, mp->reduced_max_iterations);
  if (p->time_limit_ms >= 0) rp.time_limit_ms = std::max(1.0, std::floor(p->time_limit_ms * mp->reduced_time_share));
  rp.infeasibility_tolerance = std::max(p->infeasibility_tolerance, mp->reduced_tolerance);
  std::vector<double> rx((size_t)n), ry((size_t)m), rrc((size_t)n);
  prima_solution_info rinfo;
  int32_t rc = solve_prepared(c, L, lp, SolveRequest{&rp, nullptr, cancel, rx.data(), ry.data(), rrc.data(), &rinfo},
                              32, t0);
  if (rc) return rc;
  const int st = rinfo.status;
  const bool conclusive = st == PRIMA_STATUS_OPTIMAL || st == PRIMA_STATUS_PRIMAL_INFEASIBLE ||
                          st == PRIMA_STATUS_DUAL_INFEASIBLE;
  const bool cert_holds = conclusive && st != PRIMA_STATUS_OPTIMAL &&
                          classify_fp64(lp, rx.data(), ry.data(), p->infeasibility_tolerance) == st;
  std::memset(minfo, 0, sizeof(*minfo));
  minfo->reduced_iterations = rinfo.iterations;
  minfo->reduced_restarts = rinfo.restarts;
  minfo->reduced_ms = rinfo.solve_ms;
  if (!mp->always_refine && cert_holds) {
    *info = rinfo;
    if (x_out) std::memcpy(x_out, rx.data(), (size_t)n * 8);
    if (y_out) std::memcpy(y_out, ry.data(), (size_t)m * 8);
    if (rc_out) std::memcpy(rc_out, rrc.data(), (size_t)n * 8);
    return PRIMA_OK;
  }
  prima_params fp = *p;
  if (p->time_limit_ms >= 0) fp.time_limit_ms = std::max(1.0, p->time_limit_ms - (double)rinfo.solve_ms);
  bool usable = true;
  for (double v : rx) usable = usable && std::isfinite(v);
  for (double v : ry) usable = usable && std::isfinite(v);
  prima_warm_start ws;
  ws.primal = rx.data();
  ws.dual = ry.data();
  // WarmStart(solution) keeps the adaptive state only when finite and positive
  ws.step_size = (std::isfinite(rinfo.final_step_size) && rinfo.final_step_size > 0.0) ? rinfo.final_step_size : NAN;
  ws.primal_weight =
      (std::isfinite(rinfo.final_primal_weight) && rinfo.final_primal_weight > 0.0) ? rinfo.final_primal_weight : NAN;
  const auto t1 = Clock::now();
  SolveRequest finish{&fp, usable ? &ws : nullptr, cancel, x_out, y_out, rc_out, info};
  if (mp->scheme == PRIMA_MIXED_REFINEMENT && st == PRIMA_STATUS_OPTIMAL) {
    finish.anchored = true;
    finish.round_rho = mp->round_reduction > 0.0 ? 1.0 / mp->round_reduction : 0.0;
    finish.rounds = &minfo->refinement_rounds;
    rc = solve_prepared(c, L, lp, finish, 32, t1);
  } else {
    rc = solve_prepared(c, L, lp, finish, 64, t1);
  }
  if (rc) return rc;
  minfo->refinement_iterations = info->iterations;
  minfo->refinement_ms = info->solve_ms;
  minfo->refined = 1;
  info->device_ms += rinfo.device_ms;
  info->trials += rinfo.trials;
  info->solve_ms = (int64_t)ms_since(t0);
  return PRIMA_OK;
}

int32_t validate_mixed(const prima_mixed_params *mixed) {
  if (!mixed) return (set_error("requirement failed: NULL argument"), PRIMA_ERR_INVALID_ARGUMENT);
  if (!(mixed->reduced_tolerance > 0.0))
    return (set_error("requirement failed: reducedTolerance must be positive"), PRIMA_ERR_INVALID_ARGUMENT);
  if (mixed->reduced_max_iterations <= 0)
    return (set_error("requirement failed: reducedMaxIterations must be positive"), PRIMA_ERR_INVALID_ARGUMENT);
  if (!(mixed->reduced_time_share > 0.0 && mixed->reduced_time_share < 1.0))
    return (set_error("requirement failed: reducedTimeShare must lie in (0, 1)"), PRIMA_ERR_INVALID_ARGUMENT);
  if (mixed->scheme != PRIMA_MIXED_TWO_PASS && mixed->scheme != PRIMA_MIXED_REFINEMENT)
    return (set_error("requirement failed: unknown mixed-precision scheme"), PRIMA_ERR_INVALID_ARGUMENT);
  if (!(mixed->round_reduction == 0.0 || mixed->round_reduction > 1.0))
    return (set_error("requirement failed: roundReduction must be 0 (off) or greater than 1"), PRIMA_ERR_INVALID_ARGUMENT);
  return PRIMA_OK;
}

int32_t mixed_dispatch(Ctx *c, PreparedLp &L, const prima_lp *lp, const prima_params *params,
                       const prima_mixed_params *mixed, const volatile int32_t *cancel, double *x_out, double *y_out,
                       double *rc_out, prima_solution_info *info, prima_mixed_info *minfo, Clock::time_point t0) {
  int32_t rc;
  if (!info || !minfo) return (set_error("requirement failed: NULL argument"), PRIMA_ERR_INVALID_ARGUMENT);
  if ((rc = validate_mixed(mixed)) || (rc = validate_params(params))) return rc;
  if (c->bits == 64) {
    // a float64 device skips the reduced pass entirely (MixedPrecision.scala:111-113)
    rc = solve_prepared(c, L, lp, SolveRequest{params, nullptr, cancel, x_out, y_out, rc_out, info}, 64, t0);
    if (rc) return rc;
    std::memset(minfo, 0, sizeof(*minfo));
    minfo->refinement_iterations = info->iterations;
    minfo->refinement_ms = info->solve_ms;
    return PRIMA_OK;
  }
  return mixed_passes(c, L, lp, params, mixed, cancel, x_out, y_out, rc_out, info, minfo, t0);
}

// mixed_passes for many instances: each pass runs for every instance that
// needs it in one batch launch.  Per instance the decisions are exactly
// mixed_passes' (certificate re-check, refinement only after an Optimal
// reduced pass, otherwise the FP64 finish).
int32_t mixed_passes_batch(Ctx *c, std::vector<std::unique_ptr<PreparedLp>> &Ls, const prima_lp *lps,
                           const prima_params *p, const prima_mixed_params *mp, const volatile int32_t *cancel,
                           double *const *x_out, double *const *y_out, double *const *rc_out,
                           prima_solution_info *infos, prima_mixed_info *minfos, Clock::time_point t0) {
  const int32_t count = (int32_t)Ls.size();
  prima_params rp = *p;
  rp.eps_abs = std::max(p->eps_abs, mp->reduced_tolerance);
  rp.eps_rel = std::max(p->eps_rel, mp->reduced_tolerance);
  rp.max_iterations = std::min(p->max_iterations, mp->reduced_max_iterations);
  if (p->time_limit_ms >= 0) rp.time_limit_ms = std::max(1.0, std::floor(p->time_limit_ms * mp->reduced_time_share));
  rp.infeasibility_tolerance = std::max(p->infeasibility_tolerance, mp->reduced_tolerance);
  std::vector<std::vector<double>> rx((size_t)count), ry((size_t)count), rrc((size_t)count);
  std::vector<prima_solution_info> rinfo((size_t)count);
  int32_t rc;
  {
    std::vector<Job<float>> jobs((size_t)count);
    for (int32_t i = 0; i < count; i++) {
      rx[i].resize((size_t)Ls[i]->n);
      ry[i].resize((size_t)Ls[i]->m);
      rrc[i].resize((size_t)Ls[i]->n);
      jobs[i].L = Ls[i].get();
      jobs[i].req = SolveRequest{&rp, nullptr, cancel, rx[i].data(), ry[i].data(), rrc[i].data(), &rinfo[i]};
      jobs[i].t0 = t0;
    }
    if ((rc = solve_batch_on_device(c, jobs, cancel))) return rc;
  }
  prima_params fp = *p;
  const auto t1 = Clock::now();
  std::vector<prima_warm_start> ws((size_t)count);
  std::vector<Job<float>> anchored;
  std::vector<Job<double>> fp64;
  std::vector<int32_t> who32, who64;
  for (int32_t i = 0; i < count; i++) {
    const prima_lp *lp = &lps[i];
    const int st = rinfo[i].status;
    const bool conclusive = st == PRIMA_STATUS_OPTIMAL || st == PRIMA_STATUS_PRIMAL_INFEASIBLE ||
                            st == PRIMA_STATUS_DUAL_INFEASIBLE;
    const bool cert_holds = conclusive && st != PRIMA_STATUS_OPTIMAL &&
                            classify_fp64(lp, rx[i].data(), ry[i].data(), p->infeasibility_tolerance) == st;
    prima_mixed_info &mi = minfos[i];
    std::memset(&mi, 0, sizeof(mi));
    mi.reduced_iterations = rinfo[i].iterations;
    mi.reduced_restarts = rinfo[i].restarts;
    mi.reduced_ms = rinfo[i].solve_ms;
    double *xo = x_out ? x_out[i] : nullptr, *yo = y_out ? y_out[i] : nullptr, *rco = rc_out ? rc_out[i] : nullptr;
    if (!mp->always_refine && cert_holds) {
      infos[i] = rinfo[i];
      if (xo) std::memcpy(xo, rx[i].data(), (size_t)lp->num_variables * 8);
      if (yo) std::memcpy(yo, ry[i].data(), (size_t)lp->num_constraints * 8);
      if (rco) std::memcpy(rco, rrc[i].data(), (size_t)lp->num_variables * 8);
      continue;
    }
    bool usable = true;
    for (double v : rx[i]) usable = usable && std::isfinite(v);
    for (double v : ry[i]) usable = usable && std::isfinite(v);
    prima_warm_start &w = ws[i];
    w.primal = rx[i].data();
    w.dual = ry[i].data();
    w.step_size = (std::isfinite(rinfo[i].final_step_size) && rinfo[i].final_step_size > 0.0) ? rinfo[i].final_step_size
                                                                                             : NAN;
    w.primal_weight = (std::isfinite(rinfo[i].final_primal_weight) && rinfo[i].final_primal_weight > 0.0)
                          ? rinfo[i].final_primal_weight
                          : NAN;
    SolveRequest finish{&fp, usable ? &w : nullptr, cancel, xo, yo, rco, &infos[i]};
    if (mp->scheme == PRIMA_MIXED_REFINEMENT && st == PRIMA_STATUS_OPTIMAL) {
      finish.anchored = true;
      finish.round_rho = mp->round_reduction > 0.0 ? 1.0 / mp->round_reduction : 0.0;
      finish.rounds = &mi.refinement_rounds;
      Job<float> j;
      j.L = Ls[i].get();
      j.req = finish;
      j.t0 = t1;
      anchored.push_back(j);
      who32.push_back(i);
    } else {
      Job<double> j;
      j.L = Ls[i].get();
      j.req = finish;
      j.t0 = t1;
      fp64.push_back(j);
      who64.push_back(i);
    }
  }
  if ((rc = solve_batch_on_device(c, anchored, cancel))) return rc;
  if ((rc = solve_batch_on_device(c, fp64, cancel))) return rc;
  auto close = [&](int32_t i) {
    prima_mixed_info &mi = minfos[i];
    mi.refinement_iterations = infos[i].iterations;
    mi.refinement_ms = infos[i].solve_ms;
    mi.refined = 1;
    infos[i].device_ms += rinfo[i].device_ms;
    infos[i].trials += rinfo[i].trials;
    infos[i].solve_ms = (int64_t)ms_since(t0);
  };
  for (int32_t i : who32) close(i);
  for (int32_t i : who64) close(i);
  return PRIMA_OK;
}

// CUDA events on the context stream bracketing a whole coarse call.
struct Span {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit Span(cudaStream_t st) : s(st) {
    if (cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) cudaEventRecord(a, s);
  }
  double stop() {
    float ms = 0.f;
    if (a && b && cudaEventRecord(b, s) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess)
      cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~Span() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

LpHostCopy *copy_lp(const prima_lp *lp) {
  auto *h = new LpHostCopy();
  const int32_t n = lp->num_variables, m = lp->num_constraints;
  const int64_t nnz = lp->row_ptr[m];
  h->row_ptr.assign(lp->row_ptr, lp->row_ptr + m + 1);
  h->col_idx.assign(lp->col_idx, lp->col_idx + nnz);
  h->values.assign(lp->values, lp->values + nnz);
  h->objective.assign(lp->objective, lp->objective + n);
  h->lower.assign(lp->lower, lp->lower + n);
  h->upper.assign(lp->upper, lp->upper + n);
  h->rhs.assign(lp->rhs, lp->rhs + m);
  h->lp = *lp;
  h->lp.row_ptr = h->row_ptr.data();
  h->lp.col_idx = h->col_idx.data();
  h->lp.values = h->values.data();
  h->lp.objective = h->objective.data();
  h->lp.lower = h->lower.data();
  h->lp.upper = h->upper.data();
  h->lp.rhs = h->rhs.data();
  return h;
}

}  // namespace
}  // namespace prima

using namespace prima;

#define CTX_OR_RETURN(h)        \
  clear_error();                \
  int32_t rc_;                  \
  Ctx *c = lookup_ctx(h, &rc_); \
  if (!c) return rc_;           \
  cudaSetDevice(c->device)

extern "C" int32_t prima_pdhg_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                                    const prima_warm_start *warm, const volatile int32_t *cancel, double *x_out,
                                    double *y_out, double *rc_out, prima_solution_info *info) {
  CTX_OR_RETURN(ctx);
  const auto t0 = Clock::now();
  int32_t rc;
  if ((rc = validate_lp(lp))) return rc;
  c->scratch_lp.host = nullptr;  // a one-shot call always re-prepares
  Span span(c->stream);
  rc = solve_prepared(c, c->scratch_lp, lp, SolveRequest{params, warm, cancel, x_out, y_out, rc_out, info}, c->bits, t0);
  c->scratch_lp.host = nullptr;
  if (!rc) info->span_ms = span.stop();
  return rc;
}

extern "C" int32_t prima_mixed_solve(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                                     const prima_mixed_params *mixed, const volatile int32_t *cancel,
                                     double *x_out, double *y_out, double *rc_out, prima_solution_info *info,
                                     prima_mixed_info *minfo) {
  CTX_OR_RETURN(ctx);
  const auto t0 = Clock::now();
  int32_t rc;
  if ((rc = validate_lp(lp))) return rc;
  c->scratch_lp.host = nullptr;
  Span span(c->stream);
  rc = mixed_dispatch(c, c->scratch_lp, lp, params, mixed, cancel, x_out, y_out, rc_out, info, minfo, t0);
  c->scratch_lp.host = nullptr;
  if (!rc) info->span_ms = span.stop();
  return rc;
}

extern "C" int32_t prima_problem_create(prima_handle ctx, const prima_lp *lp, const prima_params *params,
                                        prima_handle *problem) {
  CTX_OR_RETURN(ctx);
  int32_t rc;
  if (!problem) return (set_error("requirement failed: output is NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  if ((rc = validate_lp(lp)) || (rc = validate_params(params))) return rc;
  auto L = std::make_unique<PreparedLp>();
  L->owned.reset(copy_lp(lp));
  if ((rc = ensure_prepared(c, *L, &L->owned->lp, params))) return rc;
  *problem = c->next_id++;
  c->problems[*problem] = std::move(L);
  return PRIMA_OK;
}

extern "C" int32_t prima_problem_free(prima_handle ctx, prima_handle problem) {
  CTX_OR_RETURN(ctx);
  auto it = c->problems.find(problem);
  if (it == c->problems.end()) return (set_error("unknown problem handle"), PRIMA_ERR_CLOSED);
  cudaStreamSynchronize(c->stream);
  c->problems.erase(it);
  return PRIMA_OK;
}

extern "C" int32_t prima_problem_set_bounds(prima_handle ctx, prima_handle problem, const double *lower,
                                            const double *upper) {
  CTX_OR_RETURN(ctx);
  auto it = c->problems.find(problem);
  if (it == c->problems.end()) return (set_error("unknown problem handle"), PRIMA_ERR_CLOSED);
  PreparedLp &L = *it->second;
  const int32_t n = L.n;
  if (n > 0 && (!lower || !upper)) return (set_error("requirement failed: bounds are NULL"), PRIMA_ERR_INVALID_ARGUMENT);
  for (int32_t i = 0; i < n; i++)
    if (!(lower[i] <= upper[i])) {
      set_error("variable " + std::to_string(i) + " has empty bound interval [" + std::to_string(lower[i]) + ", " +
                std::to_string(upper[i]) + "]");
      return PRIMA_ERR_INVALID_ARGUMENT;
    }
  LpHostCopy &h = *L.owned;
  h.lower.assign(lower, lower + n);
  h.upper.assign(upper, upper + n);
  h.lp.lower = h.lower.data();
  h.lp.upper = h.upper.data();
  return L.set_bounds(lower, upper, c->stream);
}

extern "C" int32_t prima_problem_scaled(prima_handle ctx, prima_handle problem, double *values, double *objective,
                                        double *rhs, double *lower, double *upper, double *row_scale,
                                        double *col_scale) {
  CTX_OR_RETURN(ctx);
  auto it = c->problems.find(problem);
  if (it == c->problems.end()) return (set_error("unknown problem handle"), PRIMA_ERR_CLOSED);
  const PreparedLp &L = *it->second;
  const struct {
    double *dst;
    const void *src;
    int64_t count;
  } outs[] = {{values, L.kv(), L.nnz}, {objective, L.sc(), L.n}, {rhs, L.sq(), L.m}, {lower, L.sl(), L.n},
              {upper, L.su(), L.n}, {row_scale, L.rs(), L.m}, {col_scale, L.cs(), L.n}};
  for (const auto &o : outs)
    if (o.dst && o.count > 0)
      PRIMA_CUDA_TRY(cudaMemcpyAsync(o.dst, o.src, (size_t)o.count * 8, cudaMemcpyDeviceToHost, c->stream));
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return PRIMA_OK;
}

extern "C" int32_t prima_problem_solve(prima_handle ctx, prima_handle problem, const prima_params *params,
                                       const prima_warm_start *warm, const volatile int32_t *cancel, double *x_out,
                                       double *y_out, double *rc_out, prima_solution_info *info) {
  CTX_OR_RETURN(ctx);
  auto it = c->problems.find(problem);
  if (it == c->problems.end()) return (set_error("unknown problem handle"), PRIMA_ERR_CLOSED);
  PreparedLp &L = *it->second;
  Span span(c->stream);
  const int32_t rc = solve_prepared(c, L, &L.owned->lp, SolveRequest{params, warm, cancel, x_out, y_out, rc_out, info},
                                    c->bits, Clock::now());
  if (!rc) info->span_ms = span.stop();
  return rc;
}

extern "C" int32_t prima_problem_mixed_solve(prima_handle ctx, prima_handle problem, const prima_params *params,
                                             const prima_mixed_params *mixed, const volatile int32_t *cancel,
                                             double *x_out, double *y_out, double *rc_out, prima_solution_info *info,
                                             prima_mixed_info *minfo) {
  CTX_OR_RETURN(ctx);
  auto it = c->problems.find(problem);
  if (it == c->problems.end()) return (set_error("unknown problem handle"), PRIMA_ERR_CLOSED);
  PreparedLp &L = *it->second;
  Span span(c->stream);
  const int32_t rc = mixed_dispatch(c, L, &L.owned->lp, params, mixed, cancel, x_out, y_out, rc_out, info, minfo,
                                    Clock::now());
  if (!rc) info->span_ms = span.stop();
  return rc;
}

extern "C" int32_t prima_pdhg_solve_batch(prima_handle ctx, int32_t count, const prima_lp *lps,
                                          const prima_params *params, const volatile int32_t *cancel,
                                          double *const *x_out, double *const *y_out, double *const *rc_out,
                                          prima_solution_info *infos) {
  CTX_OR_RETURN(ctx);
  const auto t0 = Clock::now();
  int32_t rc;
  if (count < 0 || (count > 0 && (!lps || !infos)))
    return (set_error("requirement failed: count must be non-negative and lps, infos non-NULL"),
            PRIMA_ERR_INVALID_ARGUMENT);
  if ((rc = validate_params(params))) return rc;
  for (int32_t i = 0; i < count; i++)
    if ((rc = validate_lp(&lps[i]))) return rc;
  Span span(c->stream);
  std::vector<std::unique_ptr<PreparedLp>> prepared((size_t)count);
  for (int32_t i = 0; i < count; i++) {
    prepared[i] = std::make_unique<PreparedLp>();
    if ((rc = ensure_prepared(c, *prepared[i], &lps[i], params))) return rc;
  }
  auto request = [&](int32_t i) {
    return SolveRequest{params, nullptr, cancel, x_out ? x_out[i] : nullptr, y_out ? y_out[i] : nullptr,
                        rc_out ? rc_out[i] : nullptr, &infos[i]};
  };
  if (c->bits == 64) {
    std::vector<Job<double>> jobs((size_t)count);
    for (int32_t i = 0; i < count; i++) jobs[i].L = prepared[i].get(), jobs[i].req = request(i), jobs[i].t0 = t0;
    rc = solve_batch_on_device(c, jobs, cancel);
  } else {
    std::vector<Job<float>> jobs((size_t)count);
    for (int32_t i = 0; i < count; i++) jobs[i].L = prepared[i].get(), jobs[i].req = request(i), jobs[i].t0 = t0;
    rc = solve_batch_on_device(c, jobs, cancel);
  }
  const double span_ms = span.stop();
  for (int32_t i = 0; i < count; i++) infos[i].span_ms = span_ms;
  return rc;
}

extern "C" int32_t prima_mixed_solve_batch(prima_handle ctx, int32_t count, const prima_lp *lps,
                                           const prima_params *params, const prima_mixed_params *mixed,
                                           const volatile int32_t *cancel, double *const *x_out,
                                           double *const *y_out, double *const *rc_out, prima_solution_info *infos,
                                           prima_mixed_info *minfos) {
  CTX_OR_RETURN(ctx);
  const auto t0 = Clock::now();
  int32_t rc;
  if (count < 0 || (count > 0 && (!lps || !infos || !minfos)))
    return (set_error("requirement failed: count must be non-negative and lps, infos, mixed_infos non-NULL"),
            PRIMA_ERR_INVALID_ARGUMENT);
  if ((rc = validate_mixed(mixed)) || (rc = validate_params(params))) return rc;
  for (int32_t i = 0; i < count; i++)
    if ((rc = validate_lp(&lps[i]))) return rc;
  if (c->bits == 64) {  // a float64 device skips the reduced pass (MixedPrecision.scala:111-113)
    rc = prima_pdhg_solve_batch(ctx, count, lps, params, cancel, x_out, y_out, rc_out, infos);
    for (int32_t i = 0; i < count && !rc; i++) {
      std::memset(&minfos[i], 0, sizeof(minfos[i]));
      minfos[i].refinement_iterations = infos[i].iterations;
      minfos[i].refinement_ms = infos[i].solve_ms;
    }
    return rc;
  }
  Span span(c->stream);
  std::vector<std::unique_ptr<PreparedLp>> prepared((size_t)count);
  for (int32_t i = 0; i < count; i++) {
    prepared[i] = std::make_unique<PreparedLp>();
    if ((rc = ensure_prepared(c, *prepared[i], &lps[i], params))) return rc;
  }
  rc = mixed_passes_batch(c, prepared, lps, params, mixed, cancel, x_out, y_out, rc_out, infos, minfos, t0);
  const double span_ms = span.stop();
  for (int32_t i = 0; i < count; i++) infos[i].span_ms = span_ms;
  return rc;
}
