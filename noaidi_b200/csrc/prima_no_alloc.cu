// prima_dot_no_alloc: the dot product of two caller-owned device arrays with
// no allocation of any kind.  It is the prima_dot reduction reworked for
// callers that cannot allocate device memory or hold a context handle: a
// host that manages device memory through its own pool or arena and must not
// have a library call cudaMalloc/cudaFree behind its back (cudaFree
// synchronises the whole device, and cudaMalloc can, stalling every stream
// the host has in flight), or that runs inside a fixed memory budget where
// every device byte is accounted for in advance.
//
// The per-block partial sums live in g_dot_partials, a file-scope device
// array of kDotPartials doubles (16 KiB), which every GPU that loads this
// library holds until the process exits.  Host code cannot use the array's
// name as a device address, so the first call on each device (with that
// device current) looks up the array's device address with
// cudaGetSymbolAddress and caches it, keyed by the current CUDA context's
// ID; that first call should come before any stream capture.  A reset of the
// device (cudaDeviceReset, or a reset of the primary context) loads the
// module again at a new address: the next call sees the new context ID and
// looks the address up again.  All calls on a device share the array: calls
// whose kernels overlap on the GPU (two streams, two threads) race on it.
// Nothing in it has to start at zero: a call writes every partial it reads.
//
// The arrays come from the caller, so each pointer is checked to be memory
// of the current device (cudaPointerGetAttributes, which allocates nothing)
// before any kernel is queued; a host pointer or another GPU's memory is
// refused, not read.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "prima_internal.h"

namespace prima {
namespace {

constexpr int kDotThreads = 256;
constexpr int kDotPerThread = 32;
constexpr int64_t kDotSpan = (int64_t)kDotThreads * kDotPerThread;  // elements per block
constexpr int kDotPartials = 2048;                                   // blocks per call, at most
constexpr int64_t kDotMaxElements = kDotSpan * kDotPartials;         // 16,777,216
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dot_partials[kDotPartials];

// Block b sums x[i]*y[i] (in double) over its span [b*kDotSpan, ...): each
// thread strides through the span, then a fixed shuffle tree combines the
// threads.  The block's total goes to partials[b].
template <typename T>
__global__ void __launch_bounds__(kDotThreads) k_dot_span(const T *__restrict__ x, const T *__restrict__ y,
                                                          int64_t n, double *__restrict__ partials) {
  __shared__ double sh[kDotThreads / 32];
  const int64_t lo = (int64_t)blockIdx.x * kDotSpan;
  const int64_t hi = lo + kDotSpan < n ? lo + kDotSpan : n;
  double s = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kDotThreads) s += (double)x[i] * (double)y[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kDotThreads / 32 ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
  }
}

// One block: the total of partials[0, nb) into *out.
__global__ void __launch_bounds__(kDotThreads) k_dot_total(const double *__restrict__ partials, int nb,
                                                           double *__restrict__ out) {
  __shared__ double sh[kDotThreads / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += kDotThreads) s += partials[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kDotThreads / 32 ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) *out = t;
  }
}

std::mutex g_setup_mu;
struct PartialsAddress {
  unsigned long long ctx_id = 0;  // the context the address belongs to
  double *ptr = nullptr;
};
PartialsAddress g_partials[kMaxDevices];

// The ID of the calling thread's current CUDA context, through the driver
// entry points the runtime hands out (the library does not link libcuda).
typedef int (*CtxGetCurrentFn)(void **ctx);
typedef int (*CtxGetIdFn)(void *ctx, unsigned long long *id);
int32_t current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void *f0 = nullptr, *f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    PRIMA_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0));
    PRIMA_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1));
    if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1) {
      set_error("prima_dot_no_alloc: the driver offers no cuCtxGetCurrent/cuCtxGetId");
      return PRIMA_ERR_CUDA;
    }
    get_current = (CtxGetCurrentFn)f0;
    get_id = (CtxGetIdFn)f1;
  }
  void *ctx = nullptr;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
    set_error("prima_dot_no_alloc: no current CUDA context on this thread");
    return PRIMA_ERR_CUDA;
  }
  return PRIMA_OK;
}

// The device address of g_dot_partials in the current context, looked up on
// the first call per device and again whenever the device's context changed.
int32_t partials_on_current_device(int dev, double **out) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("prima_dot_no_alloc: device ordinal " + std::to_string(dev) + " is beyond the supported " +
              std::to_string(kMaxDevices));
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  unsigned long long id = 0;
  int32_t rc = current_context_id(&id);
  if (rc) return rc;
  if (!g_partials[dev].ptr || g_partials[dev].ctx_id != id) {
    void *ptr = nullptr;
    PRIMA_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_dot_partials));
    g_partials[dev].ptr = (double *)ptr;
    g_partials[dev].ctx_id = id;
  }
  *out = g_partials[dev].ptr;
  return PRIMA_OK;
}

// True when p is memory the current device's kernels may read or write:
// device memory of that device, or managed memory.
bool on_device(const void *p, int dev) {
  cudaPointerAttributes attr;
  const cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // an unrecognised pointer: refused, not the caller's pending error
    return false;
  }
  if (attr.type == cudaMemoryTypeManaged) return true;
  return attr.type == cudaMemoryTypeDevice && attr.device == dev;
}

}  // namespace
}  // namespace prima

using namespace prima;

extern "C" int32_t prima_dot_no_alloc(const void *x, const void *y, int64_t n, int32_t element_bits, double *out,
                                      void *stream) {
  clear_error();
  if (element_bits != 32 && element_bits != 64) {
    set_error("prima_dot_no_alloc: element_bits must be 32 (float) or 64 (double), got " +
              std::to_string(element_bits));
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (n < 0 || n > kDotMaxElements) {
    set_error("prima_dot_no_alloc: n = " + std::to_string(n) + " is outside [0, " + std::to_string(kDotMaxElements) +
              "], the most elements its fixed scratch of " + std::to_string(kDotPartials) +
              " block partials can reduce");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  if (!out || (n > 0 && (!x || !y))) {
    set_error("prima_dot_no_alloc: x, y and out must be device pointers (x and y may be NULL only when n = 0)");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  const size_t esz = element_bits / 8;
  if (((uintptr_t)x % esz) || ((uintptr_t)y % esz) || ((uintptr_t)out % 8)) {
    set_error("prima_dot_no_alloc: x and y must be aligned to their element size and out to 8 bytes");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  int dev = -1;
  PRIMA_CUDA_TRY(cudaGetDevice(&dev));
  if (!on_device(out, dev) || (n > 0 && (!on_device(x, dev) || !on_device(y, dev)))) {
    set_error("prima_dot_no_alloc: x, y and out must be memory of the current device (device " + std::to_string(dev) +
              ") or managed memory; a host pointer or another GPU's memory is refused");
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  double *partials = nullptr;
  int32_t rc = partials_on_current_device(dev, &partials);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    PRIMA_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return PRIMA_OK;
  }
  // Each launch's own status is checked (not the thread's last-error slot,
  // which may hold an error the caller left there earlier).
  int nb = (int)((n + kDotSpan - 1) / kDotSpan);
  void *span_args[] = {(void *)&x, (void *)&y, (void *)&n, (void *)&partials};
  const void *span = element_bits == 64 ? (const void *)k_dot_span<double> : (const void *)k_dot_span<float>;
  PRIMA_CUDA_TRY(cudaLaunchKernel(span, dim3(nb), dim3(kDotThreads), span_args, 0, s));
  void *total_args[] = {(void *)&partials, (void *)&nb, (void *)&out};
  PRIMA_CUDA_TRY(cudaLaunchKernel((const void *)k_dot_total, dim3(1), dim3(kDotThreads), total_args, 0, s));
  return PRIMA_OK;
}
