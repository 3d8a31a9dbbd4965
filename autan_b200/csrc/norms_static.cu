// Exact-sum RMS norms of device-resident arrays with no device allocation: the word scratch of the
// exact sums is a file-scope device array, so the call makes no cudaMalloc / cudaFree (nor any
// call into a library that allocates).
//
// Callers that need this are the ones for whom an allocation is not an option at the point of the
// call: a caller whose device memory is held by its own pool allocator (every free byte already
// reserved, so a cudaMalloc would fail or fragment the pool), and a caller on a latency-critical
// path where a cudaFree is out because it waits for the whole device. The per-handle norms of
// autan_euler_device_* keep their scratch in the handle's own allocation and are not affected.
//
// The sums are the same as those of the stepper's residual norms (k_norm_sums / k_norm_finish in
// euler_device.cu): the exact sum of the squared terms, rounded once to nearest even, divided by
// the count and square-rooted, so the result matches autan_euler_device_evaluate bit for bit on
// the same residual.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "autan_euler_device.h"
#include "exact_sum.cuh"

namespace autan_b200 {
namespace {

constexpr int kStaticComponents = 8;          // components one call may hold
constexpr long long kStaticMaxTerms = 1LL << 30;  // terms per component
constexpr int kStaticDevices = 64;
constexpr int kSumBlock = 256;
constexpr int kSumBlocksMax = 148 * 8;

// 8 components x 71 words x 8 bytes = 4544 bytes of device memory, loaded with the module.
// Every word must be zero when a call's sums start: the entry point clears the words of the
// components it uses on the caller's stream before it adds.
static __device__ __align__(256) unsigned long long g_rms_words[kStaticComponents * kWords];

// Component k of term i at values[k * stride + i]; the warp-merged limb atomics of warp_exact_add
// per block into shared words, then one global atomic per non-zero word.
__global__ void __launch_bounds__(kSumBlock) k_static_sums(const double* values, long long n,
                                                           long long stride, int components,
                                                           unsigned long long* words) {
  __shared__ unsigned long long sh[kStaticComponents * kWords];
  const int used = components * kWords;
  for (int i = threadIdx.x; i < used; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < n; base += step) {
    const long long i = base + threadIdx.x;
    for (int k = 0; k < components; ++k) {
      const double v = i < n ? values[k * stride + i] : 0.0;
      warp_exact_add(sh + k * kWords, v * v);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < used; i += blockDim.x) {
    const unsigned long long v = sh[i];
    if (v != 0) atomicAdd(&words[i], v);
  }
}

// rms_k = sqrt(sum_k / n), one thread per component.
__global__ void k_static_finish(const unsigned long long* words, long long n, int components,
                                double* rms) {
  const int k = threadIdx.x;
  if (k < components) rms[k] = sqrt(exact_value(words + k * kWords) / static_cast<double>(n));
}

// The device address of g_rms_words per device, found once with that device current.
std::mutex g_lock;
unsigned long long* g_address[kStaticDevices] = {};

int report(char* err, size_t len, const char* msg, cudaError_t e = cudaSuccess) {
  if (err != nullptr && len > 0) {
    if (e != cudaSuccess) {
      snprintf(err, len, "%s: %s", msg, cudaGetErrorString(e));
    } else {
      snprintf(err, len, "%s", msg);
    }
  }
  return 1;
}

}  // namespace
}  // namespace autan_b200

using namespace autan_b200;

extern "C" int autan_exact_rms_static(const double* values, int64_t n, int64_t stride,
                                      int32_t components, double* rms, void* stream, char* err,
                                      size_t err_len) {
  if (values == nullptr || rms == nullptr) return report(err, err_len, "E1101: null argument");
  if (components < 1 || components > kStaticComponents)
    return report(err, err_len, "E1101: components must be 1 to 8");
  if (n < 1) return report(err, err_len, "E1101: n must be positive");
  if (n > kStaticMaxTerms) return report(err, err_len, "E1101: n above 2^30 terms per component");
  if (components > 1 && stride < n) return report(err, err_len, "E1101: stride below n");
  int device = -1;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return report(err, err_len, "E1300: cudaGetDevice", e);
  if (device < 0 || device >= kStaticDevices)
    return report(err, err_len, "E1101: device index above 63");
  unsigned long long* words = nullptr;
  {
    std::lock_guard<std::mutex> hold(g_lock);
    if (g_address[device] == nullptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_rms_words);
      if (e != cudaSuccess) return report(err, err_len, "E1300: cudaGetSymbolAddress", e);
      g_address[device] = static_cast<unsigned long long*>(p);
    }
    words = g_address[device];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(words, 0, sizeof(unsigned long long) * kWords * components, s);
  if (e != cudaSuccess) return report(err, err_len, "E1300: clearing the scratch words", e);
  long long blocks = (n + kSumBlock - 1) / kSumBlock;
  if (blocks > kSumBlocksMax) blocks = kSumBlocksMax;
  k_static_sums<<<static_cast<unsigned>(blocks), kSumBlock, 0, s>>>(values, n, stride, components,
                                                                    words);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(err, err_len, "E1300: launching the sums", e);
  k_static_finish<<<1, 32, 0, s>>>(words, n, components, rms);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(err, err_len, "E1300: launching the finish", e);
  return 0;
}
