// The kernel seam: a Kernels backend (core/kernels/Kernels.scala:42-125) on a
// B200.  Contexts own a CUDA stream and every vector / matrix they hand out;
// handles are integer ids that are never reused, so a stale handle is caught
// rather than dereferenced.
//
// Element semantics follow the reference backends exactly: in a 64-bit
// context each operation is the IEEE double expression ScalaKernels
// evaluates; in a 32-bit context it is the binary32 expression Float32Kernels
// evaluates (inputs narrowed, every product and sum rounded to binary32).
// The library is built with --fmad=false so no a*b+c is fused.  Reductions
// accumulate in double (a tree, not the reference's index order).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <sstream>

#include "prima_internal.h"

namespace prima {

// ---- device buffers -------------------------------------------------------
DeviceBuffer::~DeviceBuffer() { release(); }

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

// Every buffer carries 64 bytes of slack past its logical end: bulk copies
// into shared memory move whole 16-byte granules, so a copy of a range that
// ends mid-granule reads (and discards) up to 12 bytes beyond it.
int32_t DeviceBuffer::reserve(size_t b) {
  if (b <= bytes && ptr) return PRIMA_OK;
  release();
  if (b == 0) b = 256;
  cudaError_t e = cudaMalloc(&ptr, b + 64);
  if (e != cudaSuccess) {
    // The failure is reported here; take it off the thread's last-error slot,
    // where the next launch check would otherwise find it and blame that
    // launch.
    (void)cudaGetLastError();
    ptr = nullptr;
    set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PRIMA_ERR_OUT_OF_MEMORY : PRIMA_ERR_CUDA;
  }
  bytes = b;
  return PRIMA_OK;
}

// ---- registry -------------------------------------------------------------
static std::mutex g_mu;
static std::unordered_map<int64_t, std::unique_ptr<Ctx>> g_ctx;
static int64_t g_next_ctx = 1;

Ctx *lookup_ctx(prima_handle h, int32_t *code) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_ctx.find(h);
  if (it == g_ctx.end() || it->second->closed) {
    set_error("unknown or closed context handle");
    *code = PRIMA_ERR_CLOSED;
    return nullptr;
  }
  *code = PRIMA_OK;
  return it->second.get();
}

static Vec *lookup_vec(Ctx *c, prima_handle h) {
  auto it = c->vecs.find(h);
  if (it == c->vecs.end()) {
    set_error("unknown vector handle");
    return nullptr;
  }
  return it->second.get();
}

static Mat *lookup_mat(Ctx *c, prima_handle h) {
  auto it = c->mats.find(h);
  if (it == c->mats.end()) {
    set_error("unknown matrix handle");
    return nullptr;
  }
  return it->second.get();
}

static size_t esize(const Ctx *c) { return c->bits == 64 ? 8 : 4; }

// ---- kernels --------------------------------------------------------------
constexpr int kOpThreads = 256;

static unsigned grid_for(int64_t n, const Ctx *c) {
  int64_t b = (n + kOpThreads - 1) / kOpThreads;
  int64_t cap = (int64_t)c->num_sms * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// Float32Kernels.upload (:43-52): narrowing keeps infinities (the cast does).
template <typename T>
__global__ void k_from_double(const double *__restrict__ in, T *__restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)in[i];
}

template <typename T>
__global__ void k_to_double(const T *__restrict__ in, double *__restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// axpby: (alpha*x) + (beta*y) in T; out may alias x or y (each element is
// read before it is written by the same thread).
template <typename T>
__global__ void k_axpby(T a, const T *x, T b, const T *y, T *out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (a * x[i]) + (b * y[i]);
}

template <typename T>
__global__ void k_scale(T a, const T *x, T *out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a * x[i];
}

// ScalaKernels.primalStep (:78-98) / Float32Kernels.primalStep (:117-134)
template <typename T>
__global__ void k_primal_step(const T *x, const T *kty, const T *c, const T *l, const T *u, T tau, T *out,
                              int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T step = x[i] - (tau * (c[i] - kty[i]));
    const T lo = l[i], hi = u[i];
    out[i] = step < lo ? lo : (step > hi ? hi : step);
  }
}

// ScalaKernels.dualStep (:100-118) / Float32Kernels.dualStep (:136-153)
template <typename T>
__global__ void k_dual_step(const T *y, const T *kxbar, const T *q, T sigma, int64_t neq, T *out, int64_t m) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const T step = y[i] + (sigma * (q[i] - kxbar[i]));
    out[i] = i < neq ? step : (step > T(0) ? step : T(0));
  }
}

// Deterministic two-pass reduction: per-block partial sums (in double) in a
// fixed tree, then one block sums the partials in a fixed order.
template <typename T, bool kSquare>
__global__ void k_dot_partial(const T *x, const T *y, int64_t n, double *partial) {
  __shared__ double sh[kOpThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a = (double)x[i];
    const double b = kSquare ? a : (double)y[i];
    s += a * b;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kOpThreads / 32 ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
  }
}

__global__ void k_sum_partials(const double *partial, int nb, double *out) {
  __shared__ double sh[kOpThreads / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partial[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kOpThreads / 32 ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *out = t;
  }
}

// CSR SpMV, one thread per row: each row summed in index order starting
// from zero -- the reference's multiplyInto / Float32Kernels.spmv order.
template <typename T>
__global__ void k_spmv_row(int32_t rows, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                           const T *__restrict__ v, const T *__restrict__ x, T *__restrict__ out) {
  for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    T acc = T(0);
    const int32_t e = rp[r + 1];
    for (int32_t p = rp[r]; p < e; p++) acc = acc + (v[p] * x[ci[p]]);
    out[r] = acc;
  }
}

// CSR SpMV by row tiles (CSR-stream): a block takes kStreamRows consecutive
// rows at a time; its threads first form the tile's products v[k] * x[col[k]]
// (rounded to T) with coalesced index and value loads and every gather of
// the tile in flight at once, into shared memory; then each thread sums its
// rows' products in index order from zero -- the same sum, bit for bit, as
// one thread per row, with the memory traffic of a streaming kernel.  A tile
// whose nonzeros do not fit is summed straight from global memory, in the
// same order.
constexpr int kStreamRows = 512;   // rows per tile (two per thread)
constexpr int kStreamCap = 4096;   // products a tile stages

template <typename T>
__global__ void __launch_bounds__(kOpThreads) k_spmv_stream(int32_t rows, const int32_t *__restrict__ rp,
                                                            const int32_t *__restrict__ ci, const T *__restrict__ v,
                                                            const T *__restrict__ x, T *__restrict__ out) {
  __shared__ T prod[kStreamCap];
  static_assert(kStreamRows == 2 * kOpThreads, "two rows per thread");
  for (int64_t r0 = (int64_t)blockIdx.x * kStreamRows; r0 < rows; r0 += (int64_t)gridDim.x * kStreamRows) {
    const int32_t r1 = (int32_t)min((int64_t)rows, r0 + kStreamRows);
    const int32_t k0 = rp[r0], k1 = rp[r1];
    int32_t ra[2], rb[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int64_t r = r0 + threadIdx.x + q * kOpThreads;
      ra[q] = r < r1 ? rp[r] : 0;
      rb[q] = r < r1 ? rp[r + 1] : 0;
    }
    const bool staged = k1 - k0 <= kStreamCap;
    if (staged) {
#pragma unroll 4
      for (int32_t k = k0 + threadIdx.x; k < k1; k += kOpThreads) prod[k - k0] = v[k] * x[ci[k]];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int64_t r = r0 + threadIdx.x + q * kOpThreads;
      if (r < r1) {
        T acc = T(0);
        if (staged) {
          for (int32_t k = ra[q]; k < rb[q]; k++) acc = acc + prod[k - k0];
        } else {
          for (int32_t k = ra[q]; k < rb[q]; k++) acc = acc + (v[k] * x[ci[k]]);
        }
        out[r] = acc;
      }
    }
    __syncthreads();
  }
}

template <typename T>
static void launch_spmv(const Ctx *c, const Mat *a, const T *x, T *out) {
  const int32_t rows = a->rows;
  if (rows == 0) return;
  const int32_t *rp = (const int32_t *)a->row_ptr.ptr;
  const int32_t *ci = (const int32_t *)a->col_idx.ptr;
  const T *v = (const T *)a->vals.ptr;
  if (a->lanes == 0) {  // CSR-stream tiles
    const int64_t tiles = ((int64_t)rows + kStreamRows - 1) / kStreamRows;
    const unsigned g = (unsigned)std::min<int64_t>(tiles, (int64_t)c->num_sms * 8);
    k_spmv_stream<T><<<g, kOpThreads, 0, c->stream>>>(rows, rp, ci, v, x, out);
  } else {
    k_spmv_row<T><<<grid_for(rows, c), kOpThreads, 0, c->stream>>>(rows, rp, ci, v, x, out);
  }
}

int32_t seam_spmv(Ctx *c, const Mat *a, const void *x, void *out) {
  if (c->bits == 64) launch_spmv<double>(c, a, (const double *)x, (double *)out);
  else launch_spmv<float>(c, a, (const float *)x, (float *)out);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}

// Autotuner for the seam SpMV: both kernels sum every row in the
// reference's index order (bit-exact in either precision), so the choice is
// by speed alone -- each is timed on the uploaded matrix (a few launches
// between CUDA events) and the faster kept.
template <typename T>
static int32_t time_spmv(Ctx *c, Mat *a, const T *x, T *out, int variant, float *ms) {
  a->lanes = variant;
  launch_spmv<T>(c, a, x, out);  // warm-up
  cudaEvent_t e0, e1;
  PRIMA_CUDA_TRY(cudaEventCreate(&e0));
  PRIMA_CUDA_TRY(cudaEventCreate(&e1));
  cudaEventRecord(e0, c->stream);
  for (int rep = 0; rep < 5; rep++) launch_spmv<T>(c, a, x, out);
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  *ms = 0.f;
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}

static int32_t autotune_spmv(Ctx *c, Mat *a) {
  a->lanes = 0;
  if (a->rows == 0 || a->nnz < (int64_t)1 << 16) return PRIMA_OK;
  const size_t es = c->bits == 64 ? 8 : 4;
  DeviceBuffer xb, ob;
  int32_t rc;
  if ((rc = xb.reserve((size_t)a->cols * es + 16)) || (rc = ob.reserve((size_t)a->rows * es + 16))) return rc;
  PRIMA_CUDA_TRY(cudaMemsetAsync(xb.ptr, 0, (size_t)a->cols * es, c->stream));
  float t_stream = 0.f, t_row = 0.f;
  if (c->bits == 64) {
    if ((rc = time_spmv<double>(c, a, (const double *)xb.ptr, (double *)ob.ptr, 0, &t_stream)) ||
        (rc = time_spmv<double>(c, a, (const double *)xb.ptr, (double *)ob.ptr, 1, &t_row)))
      return rc;
  } else {
    if ((rc = time_spmv<float>(c, a, (const float *)xb.ptr, (float *)ob.ptr, 0, &t_stream)) ||
        (rc = time_spmv<float>(c, a, (const float *)xb.ptr, (float *)ob.ptr, 1, &t_row)))
      return rc;
  }
  a->lanes = t_row < t_stream ? 1 : 0;
  return PRIMA_OK;
}

}  // namespace prima

using namespace prima;

// ---- context --------------------------------------------------------------
extern "C" int32_t prima_open(int32_t device, int32_t precision_bits, prima_handle *out) {
  clear_error();
  if (!out) {
    set_error("requirement failed: output handle is NULL");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (precision_bits != 32 && precision_bits != 64) {
    set_error("requirement failed: precision_bits must be 32 or 64");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return PRIMA_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) {
    set_error("requirement failed: device ordinal out of range");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  PRIMA_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  PRIMA_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_error(std::string("device ") + prop.name + " is not sm_100 class");
    return PRIMA_ERR_NO_DEVICE;
  }
  auto c = std::make_unique<Ctx>();
  c->device = device;
  c->bits = precision_bits;
  c->num_sms = prop.multiProcessorCount;
  c->device_name = prop.name;
  PRIMA_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  PRIMA_CUDA_TRY(cudaMallocHost((void **)&c->host_scalar, 64 * sizeof(double)));
  PRIMA_CUDA_TRY(cudaHostAlloc((void **)&c->cancel_mapped, 64, cudaHostAllocMapped));
  *c->cancel_mapped = 0;
  PRIMA_CUDA_TRY(cudaHostGetDevicePointer((void **)&c->cancel_mapped_dev, c->cancel_mapped, 0));
  int32_t rc = c->scratch.reserve(4096 * sizeof(double));
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  const int64_t id = g_next_ctx++;
  g_ctx[id] = std::move(c);
  *out = id;
  return PRIMA_OK;
}

extern "C" int32_t prima_close(prima_handle h) {
  clear_error();
  std::unique_ptr<Ctx> c;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_ctx.find(h);
    if (it == g_ctx.end() || it->second->closed) return PRIMA_OK;  // idempotent
    it->second->closed = true;
    c = std::move(it->second);  // keep the id known as closed
    g_ctx[h] = std::make_unique<Ctx>();
    g_ctx[h]->closed = true;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->vecs.clear();
  c->mats.clear();
  c->scratch.release();
  c->solver_arena.release();
  if (c->host_scalar) cudaFreeHost(c->host_scalar);
  if (c->cancel_mapped) cudaFreeHost(c->cancel_mapped);
  cudaStreamDestroy(c->stream);
  return PRIMA_OK;
}

extern "C" int32_t prima_capabilities_get(prima_handle h, prima_capabilities *out) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(h, &rc);
  if (!c) return rc;
  if (!out) {
    set_error("requirement failed: output is NULL");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  std::memset(out, 0, sizeof(*out));
  std::snprintf(out->name, sizeof(out->name), "prima-cuda-fp%d", c->bits);
  std::snprintf(out->device, sizeof(out->device), "cuda:%d %s sm_100a", c->device, c->device_name.c_str());
  out->supports_float64 = c->bits == 64;
  out->precision_bits = c->bits;
  return PRIMA_OK;
}

extern "C" int32_t prima_set_device_wait_limit(prima_handle h, int64_t polls) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(h, &rc);
  if (!c) return rc;
  if (polls < 0) {
    set_error("requirement failed: the wait limit must be non-negative (0 restores the default)");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  c->wait_limit = polls;
  return PRIMA_OK;
}

extern "C" int32_t prima_set_solver_layout(prima_handle h, int32_t blocks_per_sm, int32_t tile_rows) {
  clear_error();
  int32_t rc;
  Ctx *c = lookup_ctx(h, &rc);
  if (!c) return rc;
  if (blocks_per_sm < 0 || (blocks_per_sm > 0 && tile_rows != 512 && tile_rows != 256) ||
      (blocks_per_sm == 0 && tile_rows != 0)) {
    set_error("requirement failed: a pinned layout is blocks_per_sm > 0 with tile_rows 512 or 256; (0, 0) "
              "restores the choice by timing");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  c->pin_bps = blocks_per_sm;
  c->pin_rows = tile_rows;
  return PRIMA_OK;
}

// ---- memory ---------------------------------------------------------------
#define CTX_OR_RETURN(h)        \
  clear_error();                \
  int32_t rc_;                  \
  Ctx *c = lookup_ctx(h, &rc_); \
  if (!c) return rc_;           \
  cudaSetDevice(c->device)

static int32_t new_vec(Ctx *c, int64_t n, Vec **out, prima_handle *h) {
  if (n < 0) {
    set_error("requirement failed: negative length");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  auto v = std::make_unique<Vec>();
  v->n = n;
  int32_t rc = v->buf.reserve((size_t)n * esize(c) + 16);
  if (rc) return rc;
  *out = v.get();
  *h = c->next_id++;
  c->vecs[*h] = std::move(v);
  return PRIMA_OK;
}

extern "C" int32_t prima_vec_alloc(prima_handle ctx, int64_t n, prima_handle *out) {
  CTX_OR_RETURN(ctx);
  if (!out) {
    set_error("requirement failed: output is NULL");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  Vec *v;
  int32_t rc = new_vec(c, n, &v, out);
  if (rc) return rc;
  PRIMA_CUDA_TRY(cudaMemsetAsync(v->buf.ptr, 0, (size_t)n * esize(c), c->stream));
  return PRIMA_OK;
}

// Stages doubles through the context scratch and narrows on the device.
static int32_t upload_into(Ctx *c, void *dst, const double *data, int64_t n) {
  if (n == 0) return PRIMA_OK;
  if (c->bits == 64) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(dst, data, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
    return PRIMA_OK;
  }
  DeviceBuffer stage;
  int32_t rc = stage.reserve((size_t)n * 8);
  if (rc) return rc;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(stage.ptr, data, (size_t)n * 8, cudaMemcpyHostToDevice, c->stream));
  k_from_double<float><<<grid_for(n, c), kOpThreads, 0, c->stream>>>((const double *)stage.ptr, (float *)dst, n);
  PRIMA_CUDA_TRY(cudaGetLastError());
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return PRIMA_OK;
}

extern "C" int32_t prima_vec_upload(prima_handle ctx, const double *data, int64_t n, prima_handle *out) {
  CTX_OR_RETURN(ctx);
  if (!out || (n > 0 && !data)) {
    set_error("requirement failed: NULL argument");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  Vec *v;
  int32_t rc = new_vec(c, n, &v, out);
  if (rc) return rc;
  rc = upload_into(c, v->buf.ptr, data, n);
  if (rc) return rc;
  // the caller may overwrite `data` as soon as this returns
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return PRIMA_OK;
}

extern "C" int32_t prima_vec_download(prima_handle ctx, prima_handle vh, double *into, int64_t n) {
  CTX_OR_RETURN(ctx);
  Vec *v = lookup_vec(c, vh);
  if (!v) return PRIMA_ERR_CLOSED;
  if (n != v->n || (n > 0 && !into)) {
    set_error("requirement failed: download length differs from the vector length");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (n == 0) return PRIMA_OK;
  if (c->bits == 64) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(into, v->buf.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
  } else {
    DeviceBuffer stage;
    int32_t rc = stage.reserve((size_t)n * 8);
    if (rc) return rc;
    k_to_double<float><<<grid_for(n, c), kOpThreads, 0, c->stream>>>((const float *)v->buf.ptr,
                                                                       (double *)stage.ptr, n);
    PRIMA_CUDA_TRY(cudaGetLastError());
    PRIMA_CUDA_TRY(cudaMemcpyAsync(into, stage.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return PRIMA_OK;
}

extern "C" int32_t prima_vec_length(prima_handle ctx, prima_handle vh, int64_t *n) {
  CTX_OR_RETURN(ctx);
  Vec *v = lookup_vec(c, vh);
  if (!v) return PRIMA_ERR_CLOSED;
  if (!n) {
    set_error("requirement failed: output is NULL");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  *n = v->n;
  return PRIMA_OK;
}

extern "C" int32_t prima_vec_free(prima_handle ctx, prima_handle vh) {
  CTX_OR_RETURN(ctx);
  auto it = c->vecs.find(vh);
  if (it == c->vecs.end()) {
    set_error("unknown vector handle");
    return PRIMA_ERR_CLOSED;
  }
  cudaStreamSynchronize(c->stream);
  c->vecs.erase(it);
  return PRIMA_OK;
}

extern "C" int32_t prima_mat_upload_csr(prima_handle ctx, int32_t rows, int32_t cols, const int32_t *row_ptr,
                                        const int32_t *col_idx, const double *values, prima_handle *out) {
  CTX_OR_RETURN(ctx);
  if (rows < 0 || cols < 0 || !row_ptr || !out) {
    set_error("requirement failed: bad matrix arguments");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (row_ptr[0] != 0) {
    set_error("requirement failed: row_ptr[0] must be 0");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  for (int32_t r = 0; r < rows; r++)
    if (row_ptr[r + 1] < row_ptr[r]) {
      set_error("requirement failed: row_ptr must be non-decreasing");
      return PRIMA_ERR_INVALID_ARGUMENT;
    }
  const int64_t nnz = row_ptr[rows];
  if (nnz > 0 && (!col_idx || !values)) {
    set_error("requirement failed: missing matrix entries");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  for (int64_t k = 0; k < nnz; k++)
    if (col_idx[k] < 0 || col_idx[k] >= cols) {
      set_error("requirement failed: column index out of range");
      return PRIMA_ERR_INVALID_ARGUMENT;
    }
  auto m = std::make_unique<Mat>();
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  int32_t rc;
  if ((rc = m->row_ptr.reserve(((size_t)rows + 1) * 4)) || (rc = m->col_idx.reserve((size_t)nnz * 4 + 16)) ||
      (rc = m->vals.reserve((size_t)nnz * esize(c) + 16)))
    return rc;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(m->row_ptr.ptr, row_ptr, ((size_t)rows + 1) * 4, cudaMemcpyHostToDevice, c->stream));
  if (nnz) {
    PRIMA_CUDA_TRY(cudaMemcpyAsync(m->col_idx.ptr, col_idx, (size_t)nnz * 4, cudaMemcpyHostToDevice, c->stream));
    if ((rc = upload_into(c, m->vals.ptr, values, nnz))) return rc;
  }
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if ((rc = autotune_spmv(c, m.get()))) return rc;
  *out = c->next_id++;
  c->mats[*out] = std::move(m);
  return PRIMA_OK;
}

// ---- the eight operations -------------------------------------------------
static int32_t same_len(int64_t a, int64_t b) {
  if (a != b) {
    set_error("requirement failed: vector lengths differ");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  return PRIMA_OK;
}

#define VEC_OR_RETURN(name, h)  \
  Vec *name = lookup_vec(c, h); \
  if (!name) return PRIMA_ERR_CLOSED

extern "C" int32_t prima_spmv(prima_handle ctx, prima_handle mh, prima_handle xh, prima_handle oh) {
  CTX_OR_RETURN(ctx);
  Mat *a = lookup_mat(c, mh);
  if (!a) return PRIMA_ERR_CLOSED;
  VEC_OR_RETURN(x, xh);
  VEC_OR_RETURN(o, oh);
  if (x->n != a->cols || o->n != a->rows) {
    set_error("requirement failed: spmv shape mismatch");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (x == o) {
    set_error("requirement failed: spmv output may not alias its input");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  return seam_spmv(c, a, x->buf.ptr, o->buf.ptr);
}

extern "C" int32_t prima_axpby(prima_handle ctx, double alpha, prima_handle xh, double beta, prima_handle yh,
                               prima_handle oh) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(x, xh);
  VEC_OR_RETURN(y, yh);
  VEC_OR_RETURN(o, oh);
  int32_t rc;
  if ((rc = same_len(x->n, y->n)) || (rc = same_len(x->n, o->n))) return rc;
  if (o->n == 0) return PRIMA_OK;
  if (c->bits == 64)
    k_axpby<double><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        alpha, (const double *)x->buf.ptr, beta, (const double *)y->buf.ptr, (double *)o->buf.ptr, o->n);
  else
    k_axpby<float><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        (float)alpha, (const float *)x->buf.ptr, (float)beta, (const float *)y->buf.ptr, (float *)o->buf.ptr, o->n);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}

extern "C" int32_t prima_scale(prima_handle ctx, double alpha, prima_handle xh, prima_handle oh) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(x, xh);
  VEC_OR_RETURN(o, oh);
  int32_t rc;
  if ((rc = same_len(x->n, o->n))) return rc;
  if (o->n == 0) return PRIMA_OK;
  if (c->bits == 64)
    k_scale<double><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(alpha, (const double *)x->buf.ptr,
                                                                       (double *)o->buf.ptr, o->n);
  else
    k_scale<float><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>((float)alpha, (const float *)x->buf.ptr,
                                                                      (float *)o->buf.ptr, o->n);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}

extern "C" int32_t prima_copy(prima_handle ctx, prima_handle sh, prima_handle dh) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(s, sh);
  VEC_OR_RETURN(d, dh);
  int32_t rc;
  if ((rc = same_len(s->n, d->n))) return rc;
  if (s->n == 0 || s == d) return PRIMA_OK;
  PRIMA_CUDA_TRY(cudaMemcpyAsync(d->buf.ptr, s->buf.ptr, (size_t)s->n * esize(c), cudaMemcpyDeviceToDevice, c->stream));
  return PRIMA_OK;
}

static int32_t reduce(Ctx *c, const Vec *x, const Vec *y, bool square, double *out) {
  if (!out) {
    set_error("requirement failed: output is NULL");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (x->n == 0) {
    *out = 0.0;
    return PRIMA_OK;
  }
  const unsigned g = grid_for(x->n, c);
  double *partial = (double *)c->scratch.ptr;
  double *result = partial + 2048;
  if (c->bits == 64) {
    if (square) k_dot_partial<double, true><<<g, kOpThreads, 0, c->stream>>>((const double *)x->buf.ptr, nullptr, x->n, partial);
    else k_dot_partial<double, false><<<g, kOpThreads, 0, c->stream>>>((const double *)x->buf.ptr, (const double *)y->buf.ptr, x->n, partial);
  } else {
    if (square) k_dot_partial<float, true><<<g, kOpThreads, 0, c->stream>>>((const float *)x->buf.ptr, nullptr, x->n, partial);
    else k_dot_partial<float, false><<<g, kOpThreads, 0, c->stream>>>((const float *)x->buf.ptr, (const float *)y->buf.ptr, x->n, partial);
  }
  k_sum_partials<<<1, kOpThreads, 0, c->stream>>>(partial, (int)g, result);
  PRIMA_CUDA_TRY(cudaGetLastError());
  PRIMA_CUDA_TRY(cudaMemcpyAsync(c->host_scalar, result, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PRIMA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out = *c->host_scalar;
  return PRIMA_OK;
}

extern "C" int32_t prima_dot(prima_handle ctx, prima_handle xh, prima_handle yh, double *out) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(x, xh);
  VEC_OR_RETURN(y, yh);
  int32_t rc;
  if ((rc = same_len(x->n, y->n))) return rc;
  return reduce(c, x, y, false, out);
}

extern "C" int32_t prima_squared_norm(prima_handle ctx, prima_handle xh, double *out) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(x, xh);
  return reduce(c, x, nullptr, true, out);
}

extern "C" int32_t prima_primal_step(prima_handle ctx, prima_handle xh, prima_handle kh, prima_handle ch,
                                     prima_handle lh, prima_handle uh, double tau, prima_handle oh) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(x, xh);
  VEC_OR_RETURN(k, kh);
  VEC_OR_RETURN(cc, ch);
  VEC_OR_RETURN(l, lh);
  VEC_OR_RETURN(u, uh);
  VEC_OR_RETURN(o, oh);
  int32_t rc;
  if ((rc = same_len(x->n, k->n)) || (rc = same_len(x->n, cc->n)) || (rc = same_len(x->n, l->n)) ||
      (rc = same_len(x->n, u->n)) || (rc = same_len(x->n, o->n)))
    return rc;
  if (o->n == 0) return PRIMA_OK;
  if (c->bits == 64)
    k_primal_step<double><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        (const double *)x->buf.ptr, (const double *)k->buf.ptr, (const double *)cc->buf.ptr,
        (const double *)l->buf.ptr, (const double *)u->buf.ptr, tau, (double *)o->buf.ptr, o->n);
  else
    k_primal_step<float><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        (const float *)x->buf.ptr, (const float *)k->buf.ptr, (const float *)cc->buf.ptr,
        (const float *)l->buf.ptr, (const float *)u->buf.ptr, (float)tau, (float *)o->buf.ptr, o->n);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}

extern "C" int32_t prima_dual_step(prima_handle ctx, prima_handle yh, prima_handle kh, prima_handle qh,
                                   double sigma, int32_t num_equalities, prima_handle oh) {
  CTX_OR_RETURN(ctx);
  VEC_OR_RETURN(y, yh);
  VEC_OR_RETURN(k, kh);
  VEC_OR_RETURN(q, qh);
  VEC_OR_RETURN(o, oh);
  int32_t rc;
  if ((rc = same_len(y->n, k->n)) || (rc = same_len(y->n, q->n)) || (rc = same_len(y->n, o->n))) return rc;
  if (num_equalities < 0) {
    set_error("requirement failed: numEqualities must be non-negative");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (o->n == 0) return PRIMA_OK;
  if (c->bits == 64)
    k_dual_step<double><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        (const double *)y->buf.ptr, (const double *)k->buf.ptr, (const double *)q->buf.ptr, sigma,
        num_equalities, (double *)o->buf.ptr, o->n);
  else
    k_dual_step<float><<<grid_for(o->n, c), kOpThreads, 0, c->stream>>>(
        (const float *)y->buf.ptr, (const float *)k->buf.ptr, (const float *)q->buf.ptr, (float)sigma,
        num_equalities, (float *)o->buf.ptr, o->n);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}
