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
// cudaGetSymbolAddress and caches it; that first call should come before any
// stream capture.  All calls on a device share the array: calls whose
// kernels overlap on the GPU (two streams, two threads) race on it.  Nothing
// in it has to start at zero: a call writes every partial it reads.
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
double *g_partials_ptr[kMaxDevices] = {};

// The device address of g_dot_partials on the current device, looked up on
// the first call per device.
int32_t partials_on_current_device(double **out) {
  int dev = -1;
  PRIMA_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("prima_dot_no_alloc: device ordinal " + std::to_string(dev) + " is beyond the supported " +
              std::to_string(kMaxDevices));
    return PRIMA_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_partials_ptr[dev]) {
    void *ptr = nullptr;
    PRIMA_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_dot_partials));
    g_partials_ptr[dev] = (double *)ptr;
  }
  *out = g_partials_ptr[dev];
  return PRIMA_OK;
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
  double *partials = nullptr;
  int32_t rc = partials_on_current_device(&partials);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {
    PRIMA_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(double), s));
    return PRIMA_OK;
  }
  const int nb = (int)((n + kDotSpan - 1) / kDotSpan);
  if (element_bits == 64)
    k_dot_span<double><<<nb, kDotThreads, 0, s>>>((const double *)x, (const double *)y, n, partials);
  else
    k_dot_span<float><<<nb, kDotThreads, 0, s>>>((const float *)x, (const float *)y, n, partials);
  k_dot_total<<<1, kDotThreads, 0, s>>>(partials, nb, out);
  PRIMA_CUDA_TRY(cudaGetLastError());
  return PRIMA_OK;
}
