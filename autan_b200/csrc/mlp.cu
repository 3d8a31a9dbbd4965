// The learned warm start: a small MLP (BF16 weights and activations, FP32 accumulation) trained
// and evaluated by this file's own tensor-core kernels, and the exact wall distance it takes as an
// input. C ABI: include/autan_mlp.h.
//
// Layout: activations are row-major [rows x padded width] BF16, every layer's width padded to a
// multiple of 16 (inputs) or 8 (outputs) with zeros; weights W [out x in] BF16 (and their
// transposes for the backward pass), FP32 master copies with Adam moments. The dense kernel is
// C[M x N] = A[M x K] B[N x K]^T with warp-level mma.sync m16n8k16 (BF16 in, FP32 accumulate),
// bias and GELU fused in its epilogue; the weight gradient C[N x K] = dZ^T A sums 128-row chunks
// into per-chunk partials that a second kernel adds in chunk order, so training is deterministic.
// Three engines: that warp-level mma.sync path, the same GEMMs a launch per layer on tcgen05, and
// (width 128, the default) the fused tcgen05 kernel of mlp_fused.cuh that takes each 128-row tile
// through the whole forward and backward pass in one launch.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "autan_mlp.h"

namespace autan_b200 {
namespace mlp {

using bf16 = __nv_bfloat16;

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};
[[noreturn]] void fail(const std::string& what) { throw Failure(what); }
// A failed CUDA call: the runtime's (non-sticky) last-error state is cleared before reporting, so
// that the next launch's check sees that launch's own result.
void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(std::string("E1300: ") + what + ": " + cudaGetErrorString(e));
  }
}

// Allows `kernel` launches with up to `bytes` of dynamic shared memory: its limit raised to the
// device's opt-in maximum less the kernel's static shared memory, the same value from every
// handle and thread (a limit set to each
// launch's own size would race with another handle's launch of the same kernel at a larger size).
template <class K>
void allow_smem(K kernel, size_t bytes) {
  int dev = 0, optin = 0;
  check(cudaGetDevice(&dev), "device");
  check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "device");
  cudaFuncAttributes fa{};
  check(cudaFuncGetAttributes(&fa, kernel), "smem");
  const long long limit = static_cast<long long>(optin) - static_cast<long long>(fa.sharedSizeBytes);
  if (static_cast<long long>(bytes) > limit) fail("E1300: shared memory above the device's limit");
  check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(limit)), "smem");
}

constexpr int kMaxWidth = 128;
constexpr int kRowsPerBlock = 64;  // dense kernel: 4 warps x 16 rows
constexpr int kChunk = 128;        // weight-gradient rows per partial

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return static_cast<uint32_t>(__bfloat16_as_ushort(lo)) |
         (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
}

// D = A B + C for one m16n8k16 tile (PTX mma.sync, row.col, BF16 operands, FP32 accumulators).
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = expf(-0.5f * z * z) * 0.39894228040143268f;
  return cdf + z * pdf;
}

// C[M x N] = A[M x K] B[N x K]^T + bias: A (lda), B (ldb) BF16 row-major, K a multiple of 16, N a
// multiple of 8 and at most 128. Epilogue: z = C + bias into Z (FP32, ldz, may be null); then
// GELU(z) (ACT) or z, into Y (BF16, ldy) or Yf (FP32, ldy). 128 threads: warp w the rows
// [16 w, 16 w + 16) of the block's 64.
template <bool ACT>
__global__ void __launch_bounds__(128) k_dense(const bf16* A, int lda, int M, int K, const bf16* B,
                                               int ldb, int N, const float* bias, float* Z, int ldz,
                                               bf16* Y, float* Yf, int ldy) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int sk = K + 8;  // padded row stride (bank spread)
  bf16* As = reinterpret_cast<bf16*>(smem);
  bf16* Bs = As + kRowsPerBlock * sk;
  const int row0 = blockIdx.x * kRowsPerBlock;
  // staged in 16-byte pieces (K, lda, ldb multiples of 8 elements; rows of sk elements stay
  // 16-byte aligned)
  const int kv = K / 8;
  for (int i = threadIdx.x; i < kRowsPerBlock * kv; i += blockDim.x) {
    const int r = i / kv, v = i % kv;
    const uint4 val = row0 + r < M
                          ? *reinterpret_cast<const uint4*>(A + static_cast<long long>(row0 + r) * lda + 8 * v)
                          : make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(As + r * sk + 8 * v) = val;
  }
  for (int i = threadIdx.x; i < N * kv; i += blockDim.x) {
    const int n = i / kv, v = i % kv;
    *reinterpret_cast<uint4*>(Bs + n * sk + 8 * v) =
        *reinterpret_cast<const uint4*>(B + static_cast<long long>(n) * ldb + 8 * v);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  float acc[16][4];
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.0f;
  const bf16* ar = As + (16 * warp) * sk;
  for (int k0 = 0; k0 < K; k0 += 16) {
    // fragments as 32-bit pairs of adjacent elements (even offsets: 4-byte aligned)
    auto pair = [](const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); };
    uint32_t a[4];
    a[0] = pair(ar + g * sk + k0 + 2 * t);
    a[1] = pair(ar + (g + 8) * sk + k0 + 2 * t);
    a[2] = pair(ar + g * sk + k0 + 2 * t + 8);
    a[3] = pair(ar + (g + 8) * sk + k0 + 2 * t + 8);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (8 * j < N) {
        const bf16* br = Bs + (8 * j + g) * sk + k0;
        uint32_t b[2];
        b[0] = pair(br + 2 * t);
        b[1] = pair(br + 2 * t + 8);
        mma16816(acc[j], a, b);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (8 * j >= N) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = row0 + 16 * warp + g + (q >= 2 ? 8 : 0);
      const int n = 8 * j + 2 * t + (q & 1);
      if (r >= M) continue;
      const float z = acc[j][q] + (bias != nullptr ? bias[n] : 0.0f);
      if (Z != nullptr) Z[static_cast<long long>(r) * ldz + n] = z;
      const float y = ACT ? gelu(z) : z;
      if (Y != nullptr) Y[static_cast<long long>(r) * ldy + n] = __float2bfloat16(y);
      if (Yf != nullptr) Yf[static_cast<long long>(r) * ldy + n] = y;
    }
  }
}

// Partial weight gradients: for the 128-row chunk blockIdx.x, P[chunk][N x K] = dZ_chunk^T A_chunk
// (dZ BF16 [M x N], A BF16 [M x K]; N, K multiples of 16, at most 128). 256 threads: warp w the
// gradient rows [16 w, 16 w + 16) (warps beyond N / 16 idle).
constexpr int kWgradSmem = 2 * kChunk * (kMaxWidth + 8) * 2;

__global__ void __launch_bounds__(256) k_wgrad(const bf16* dZ, int ldz, const bf16* A, int lda,
                                               int M, int N, int K, float* partial) {
  extern __shared__ __align__(16) unsigned char wsm[];
  auto Ds = reinterpret_cast<bf16 (*)[kMaxWidth + 8]>(wsm);
  auto As = reinterpret_cast<bf16 (*)[kMaxWidth + 8]>(wsm + kChunk * (kMaxWidth + 8) * 2);
  const int m0 = blockIdx.x * kChunk;
  // staged in 16-byte pieces (N, K, ldz, lda multiples of 8 elements)
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int i = threadIdx.x; i < kChunk * (N / 8); i += blockDim.x) {
    const int r = i / (N / 8), v = i % (N / 8);
    *reinterpret_cast<uint4*>(&Ds[r][8 * v]) =
        m0 + r < M ? *reinterpret_cast<const uint4*>(dZ + static_cast<long long>(m0 + r) * ldz + 8 * v) : zero;
  }
  for (int i = threadIdx.x; i < kChunk * (K / 8); i += blockDim.x) {
    const int r = i / (K / 8), v = i % (K / 8);
    *reinterpret_cast<uint4*>(&As[r][8 * v]) =
        m0 + r < M ? *reinterpret_cast<const uint4*>(A + static_cast<long long>(m0 + r) * lda + 8 * v) : zero;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  if (16 * warp >= N) return;
  float acc[16][4];
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[j][q] = 0.0f;
  const int n0 = 16 * warp;
  for (int r0 = 0; r0 < kChunk; r0 += 16) {
    // A operand (m16 x k16): element (i, r) = dZ[r0 + r][n0 + i]
    uint32_t a[4];
    a[0] = pack2(Ds[r0 + 2 * t][n0 + g], Ds[r0 + 2 * t + 1][n0 + g]);
    a[1] = pack2(Ds[r0 + 2 * t][n0 + g + 8], Ds[r0 + 2 * t + 1][n0 + g + 8]);
    a[2] = pack2(Ds[r0 + 2 * t + 8][n0 + g], Ds[r0 + 2 * t + 9][n0 + g]);
    a[3] = pack2(Ds[r0 + 2 * t + 8][n0 + g + 8], Ds[r0 + 2 * t + 9][n0 + g + 8]);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (8 * j < K) {
        // B operand (k16 x n8): element (r, c) = A[r0 + r][8 j + c]
        uint32_t b[2];
        b[0] = pack2(As[r0 + 2 * t][8 * j + g], As[r0 + 2 * t + 1][8 * j + g]);
        b[1] = pack2(As[r0 + 2 * t + 8][8 * j + g], As[r0 + 2 * t + 9][8 * j + g]);
        mma16816(acc[j], a, b);
      }
    }
  }
  float* out = partial + static_cast<long long>(blockIdx.x) * N * K;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (8 * j >= K) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int n = n0 + g + (q >= 2 ? 8 : 0);
      const int k = 8 * j + 2 * t + (q & 1);
      out[n * K + k] = acc[j][q];
    }
  }
}

// grad[i] = sum over chunks c (in order) of partial[c][i]; the bias gradient of the layer's
// columns likewise from the column sums of dZ (FP32) over the rows.
__global__ void k_sum_partials(const float* partial, int chunks, int size, float* grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= size) return;
  float s = 0.0f;
  for (int c = 0; c < chunks; ++c) s += partial[static_cast<long long>(c) * size + i];
  grad[i] = s;
}
// Column sums of dz [M x ld] over the rows of chunk blockIdx.y (kChunk rows), columns
// 32 blockIdx.x + threadIdx.x: each of the block's 8 row lanes sums every 8th row, the lanes are
// then added in lane order; partial[chunk][n] (summed over the chunks in order by k_sum_partials).
__global__ void __launch_bounds__(256) k_column_partials(const float* dz, int ld, int M, int N,
                                                         float* partial) {
  __shared__ float lane_sum[8][33];
  const int n = blockIdx.x * 32 + threadIdx.x;
  const long long r0 = static_cast<long long>(blockIdx.y) * kChunk;
  const long long r1 = min(r0 + kChunk, static_cast<long long>(M));
  float s = 0.0f;
  if (n < N)
    for (long long r = r0 + threadIdx.y; r < r1; r += 8) s += dz[r * ld + n];
  lane_sum[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && n < N) {
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += lane_sum[k][threadIdx.x];
    partial[static_cast<long long>(blockIdx.y) * N + n] = t;
  }
}

// Standardised inputs of rows idx (or 0..n-1) as BF16 [n x ldx] (zero padding).
__global__ void k_inputs(const float* x, int inputs, const int* idx, int n, const float* mean,
                         const float* sd, bf16* out, int ldx) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<long long>(n) * ldx) return;
  const long long r = i / ldx;
  const int c = static_cast<int>(i % ldx);
  float v = 0.0f;
  if (c < inputs) {
    const long long src = idx != nullptr ? idx[r] : r;
    v = (x[src * inputs + c] - mean[c]) / sd[c];
  }
  out[i] = __float2bfloat16(v);
}

// Output layer loss and gradient: pred (FP32 [n x ld]) against the standardised targets of rows
// idx; dpred = 2 (pred - t) / (n outputs) as FP32 and BF16; per-row squared errors into se.
__global__ void k_loss(const float* pred, int ld, const float* y, int outputs, const int* idx,
                       int n, const float* mean, const float* sd, float* dz, bf16* dzb, float* se) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const long long src = idx != nullptr ? idx[r] : r;
  float s = 0.0f;
  const float scale = 2.0f / (static_cast<float>(n) * outputs);
  for (int c = 0; c < ld; ++c) {
    float g = 0.0f;
    if (c < outputs) {
      const float t = (y[src * outputs + c] - mean[c]) / sd[c];
      const float d = pred[static_cast<long long>(r) * ld + c] - t;
      s += d * d;
      g = scale * d;
    }
    dz[static_cast<long long>(r) * ld + c] = g;
    dzb[static_cast<long long>(r) * ld + c] = __float2bfloat16(g);
  }
  se[r] = s;
}

// dZ of a hidden layer from the gradient of its activation dA (FP32): dZ = dA GELU'(Z).
__global__ void k_gelu_back(const float* dA, const float* Z, long long count, float* dz, bf16* dzb) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float g = dA[i] * gelu_grad(Z[i]);
  dz[i] = g;
  dzb[i] = __float2bfloat16(g);
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, long long count, float lr,
                       float c1, float c2) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  m[i] = 0.9f * m[i] + 0.1f * gi;
  v[i] = 0.999f * v[i] + 0.001f * gi * gi;
  const float mh = m[i] / c1, vh = v[i] / c2;
  p[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// BF16 weights W [np x kp] and W^T [kp x np] (zero padded) from the FP32 master W [out x in].
__global__ void k_round_weights(const float* w, int out, int in, bf16* wb, int kp, bf16* wt, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np * kp) return;
  const int n = i / kp, k = i % kp;
  const float x = n < out && k < in ? w[n * in + k] : 0.0f;
  wb[n * kp + k] = __float2bfloat16(x);
  wt[k * np + n] = __float2bfloat16(x);
}

__global__ void k_outputs(const float* pred, int ld, int outputs, int n, const float* mean,
                          const float* sd, float* y) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<long long>(n) * outputs) return;
  const long long r = i / outputs;
  const int c = static_cast<int>(i % outputs);
  y[i] = pred[r * ld + c] * sd[c] + mean[c];
}


// ---------------------------------------------------------------- tcgen05 engine
//
// The same GEMMs on the 5th-generation tensor cores: C[128 x N] = P[128 x K] Q[N x K]^T for one
// 128-row tile per CTA (4 warps). Both operands are written to shared memory in the K-major
// canonical layout without swizzle (8-row x 16-byte core matrices: rows 16 bytes apart, row groups
// 128 bytes apart, 8-element K groups R * 16 bytes apart for an R-row operand); one thread issues
// K / 16 tcgen05.mma (kind::f16, BF16 in, FP32 accumulator in tensor memory) and commits them to
// an mbarrier; after a bounded wait each warp reads its 32 accumulator lanes with tcgen05.ld.

constexpr int kTcRows = 128;
constexpr int kTcWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in a K-major operand of R rows.
__device__ __forceinline__ uint32_t kmajor(int r, int k, int R) {
  return static_cast<uint32_t>((k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: start >> 4 at bits [0, 14), leading byte offset (the K-group
// step) >> 4 at [16, 30), stride byte offset (the row-group step, 128) >> 4 at [32, 46), version 1
// at [46, 48), no swizzle (layout 0) at [61, 64).
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, int R) {
  uint64_t d = static_cast<uint64_t>((start >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(((R * 16) >> 4) & 0x3FFF) << 16;
  d |= static_cast<uint64_t>((128 >> 4) & 0x3FFF) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits [4, 6) = 1), BF16 A and B ([7, 10)
// and [10, 13) = 1), both K-major, N >> 3 at [17, 23), M >> 4 at [24, 29).
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u)
      : "memory");
}

__device__ __forceinline__ bool tc_try_wait(unsigned long long* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, "
      "p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// MODE 0: P rows from A (row-major, lda) at row0 + r, Q = B (row-major [N x K], ldb); epilogue as
// k_dense. MODE 1 (weight-gradient partial of chunk blockIdx.x): P[n][r] = A[m0 + r][n] (dZ, the
// tile's 128 rows the output neurons, N0 of them real), Q[k][r] = B[m0 + r][k] (the layer input);
// the partial [N0 x N] into Yf.
template <int MODE, bool ACT>
__global__ void __launch_bounds__(128) k_tc_gemm(const bf16* A, int lda, int M, int K, const bf16* B,
                                                 int ldb, int N, int N0, const float* bias, float* Z,
                                                 int ldz, bf16* Y, float* Yf, int ldy, int ncols,
                                                 unsigned int* fault) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t tmem_slot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int inner = MODE == 0 ? K : kTcRows;  // the contracted dimension
  unsigned char* ps = tsm;
  unsigned char* qs = tsm + kTcRows * inner * 2;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const long long r0 = static_cast<long long>(blockIdx.x) * kTcRows;
  if constexpr (MODE == 0) {
    const int groups = K >> 3;
    for (int i = threadIdx.x; i < kTcRows * groups; i += blockDim.x) {
      const int r = i / groups, g = i % groups;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (r0 + r < M) v = *reinterpret_cast<const uint4*>(A + (r0 + r) * lda + 8 * g);
      *reinterpret_cast<uint4*>(ps + kmajor(r, 8 * g, kTcRows)) = v;
    }
    for (int i = threadIdx.x; i < N * groups; i += blockDim.x) {
      const int n = i / groups, g = i % groups;
      *reinterpret_cast<uint4*>(qs + kmajor(n, 8 * g, N)) =
          *reinterpret_cast<const uint4*>(B + static_cast<long long>(n) * ldb + 8 * g);
    }
  } else {
    // Both operands transposed (the contraction runs over the chunk's rows): 8 x 8 blocks in two
    // halves, eight 8-byte loads of 8 rows' 4 columns, transposed in registers, four 16-byte
    // stores of one column's 8 rows (contiguous in the K-major layout). Columns n >= N0 of A are zero (N0 and
    // N multiples of 8; lda, ldb multiples of 8 elements).
    auto block8 = [&](const bf16* src, int ld, int cols, int bound, unsigned char* dst, int R) {
      const int nb = cols >> 3;
      for (int i = threadIdx.x; i < (kTcRows >> 3) * nb; i += blockDim.x) {
        const int rb = i / nb, cb = i % nb;
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // columns 4 h .. 4 h + 3 of the block
          uint32_t w[8][2];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const long long r = r0 + 8 * rb + q;
            uint2 v = make_uint2(0u, 0u);
            if (8 * cb < bound && r < M) v = *reinterpret_cast<const uint2*>(src + r * ld + 8 * cb + 4 * h);
            w[q][0] = v.x;
            w[q][1] = v.y;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const unsigned sel = (j & 1) ? 0x7632u : 0x5410u;  // high or low halves of two words
            uint4 o;
            o.x = __byte_perm(w[0][j >> 1], w[1][j >> 1], sel);
            o.y = __byte_perm(w[2][j >> 1], w[3][j >> 1], sel);
            o.z = __byte_perm(w[4][j >> 1], w[5][j >> 1], sel);
            o.w = __byte_perm(w[6][j >> 1], w[7][j >> 1], sel);
            *reinterpret_cast<uint4*>(dst + kmajor(8 * cb + 4 * h + j, 8 * rb, R)) = o;
          }
        }
      }
    };
    block8(A, lda, kTcRows, N0, ps, kTcRows);  // element (n, r) of dZ^T
    block8(B, ldb, N, N, qs, N);               // element (k, r) of A_prev^T
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  if (threadIdx.x == 0) {
    const uint32_t idesc = tc_idesc(N);
    for (int k0 = 0; k0 < inner; k0 += 16) {
      const uint64_t a = smem_desc(smem_addr(ps) + (k0 >> 3) * (kTcRows * 16), kTcRows);
      const uint64_t b = smem_desc(smem_addr(qs) + (k0 >> 3) * (N * 16), N);
      tc_mma(tmem, a, b, idesc, k0 > 0 ? 1u : 0u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(&bar))
                 : "memory");
  }
  bool done = false;
  for (int it = 0; it < kTcWaitLimit && !done; ++it) done = tc_try_wait(&bar, 0);
  // one decision per warp (the tensor-memory loads below are warp-collective): a phase seen
  // complete by any lane is complete
  done = __any_sync(0xffffffffu, done);
  if (!done) {
    // the accumulator never completed: record it, give the MMAs one more bounded wait, free the
    // tensor memory and leave without an epilogue
    if (threadIdx.x == 0) atomicExch(fault, 1u);
    for (int it = 0; it < kTcWaitLimit && !done; ++it) done = tc_try_wait(&bar, 0);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = 32 * warp + lane;
    for (int c0 = 0; c0 < N; c0 += 8) {
      uint32_t v[8];
      const uint32_t addr = tmem + (static_cast<uint32_t>(32 * warp) << 16) + static_cast<uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if constexpr (MODE == 0) {
        const long long r = r0 + row;
        if (r < M) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int n = c0 + j;
            const float z = __uint_as_float(v[j]) + (bias != nullptr ? bias[n] : 0.0f);
            if (Z != nullptr) Z[r * ldz + n] = z;
            const float y = ACT ? gelu(z) : z;
            if (Y != nullptr) Y[r * ldy + n] = __float2bfloat16(y);
            if (Yf != nullptr) Yf[r * ldy + n] = y;
          }
        }
      } else {
        if (row < N0) {
          float* out = Yf + static_cast<long long>(blockIdx.x) * N0 * N;
#pragma unroll
          for (int j = 0; j < 8; ++j) out[row * N + c0 + j] = __uint_as_float(v[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
}

#include "mlp_fused.cuh"

// ---------------------------------------------------------------- wall distance

struct V3 {
  double x, y, z;
};
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 axpy(V3 a, double s, V3 d) {
  return {a.x + s * d.x, a.y + s * d.y, a.z + s * d.z};
}

// Distance from p to triangle (a, b, c): the closest point by the Voronoi regions of the
// triangle's vertices, edges and face (Ericson, Real-Time Collision Detection, 2005, sec. 5.1.5).
__device__ double point_triangle(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  V3 q;
  if (d1 <= 0.0 && d2 <= 0.0) {
    q = a;
  } else {
    const V3 bp = sub3(p, b);
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    const V3 cp = sub3(p, c);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    const double vc = d1 * d4 - d3 * d2;
    const double vb = d5 * d2 - d1 * d6;
    const double va = d3 * d6 - d5 * d4;
    if (d3 >= 0.0 && d4 <= d3) {
      q = b;
    } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
      q = axpy(a, d1 / (d1 - d3), ab);
    } else if (d6 >= 0.0 && d5 <= d6) {
      q = c;
    } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
      q = axpy(a, d2 / (d2 - d6), ac);
    } else if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
      q = axpy(b, (d4 - d3) / ((d4 - d3) + (d5 - d6)), sub3(c, b));
    } else {
      const double den = 1.0 / (va + vb + vc);
      q = axpy(axpy(a, vb * den, ab), vc * den, ac);
    }
  }
  const V3 d = sub3(p, q);
  return sqrt(dot(d, d));
}

__global__ void k_wall_distance(const double* tri, const int64_t* tri_off, const double* pts,
                                const int* case_of, long long n, double* out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = case_of[i];
  const V3 p{pts[i], pts[n + i], pts[2 * n + i]};
  double best = __longlong_as_double(0x7ff0000000000000LL);
  for (int64_t t = tri_off[k]; t < tri_off[k + 1]; ++t) {
    const double* q = tri + 9 * t;
    const double d = point_triangle(p, {q[0], q[1], q[2]}, {q[3], q[4], q[5]}, {q[6], q[7], q[8]});
    if (d < best) best = d;
  }
  out[i] = best;
}

// ---------------------------------------------------------------- host

struct Buf {
  void* p = nullptr;
  size_t n = 0;
  Buf() = default;
  explicit Buf(size_t bytes) { alloc(bytes); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p != nullptr) cudaFree(p);
  }
  void alloc(size_t bytes) {
    if (p != nullptr) cudaFree(p);
    p = nullptr;
    n = bytes;
    if (bytes > 0) check(cudaMalloc(&p, bytes), "cudaMalloc");
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

int pad(int x, int m) { return (x + m - 1) / m * m; }
int blocks(long long n, int b) { return static_cast<int>(std::max<long long>(1, (n + b - 1) / b)); }

struct Layer {
  int in, out;   // logical sizes
  int kp, np;    // padded (K multiple of 16; N multiple of 16, 8 for the output)
  long long w0;  // offset of W in the parameter vector, then b at w0 + out * in
};

class Net {
 public:
  Net(int inputs, int width, int layers, int outputs, uint64_t seed, int device)
      : inputs_(inputs), width_(width), outputs_(outputs), device_(device) {
    if (width < 16 || width > kMaxWidth || width % 16 != 0) fail("E1101: width is 16 to 128, a multiple of 16");
    if (inputs < 1 || inputs > width || outputs < 1 || outputs > width || layers < 1)
      fail("E1101: inputs and outputs 1 to width, at least one hidden layer");
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    fault_.alloc(sizeof(unsigned int));
    check(cudaMemset(fault_.p, 0, sizeof(unsigned int)), "fault");
    long long off = 0;
    for (int l = 0; l <= layers; ++l) {
      Layer L;
      L.in = l == 0 ? inputs : width;
      L.out = l == layers ? outputs : width;
      L.kp = pad(L.in, 16);
      L.np = l == layers ? pad(L.out, 16) : width;
      L.w0 = off;
      off += static_cast<long long>(L.out) * L.in + L.out;
      layers_.push_back(L);
    }
    count_ = off;
    std::vector<float> p(count_, 0.0f);
    std::mt19937_64 rng(seed);
    for (const Layer& L : layers_) {
      const float a = std::sqrt(6.0f / static_cast<float>(L.in + L.out));
      std::uniform_real_distribution<float> u(-a, a);
      for (long long i = 0; i < static_cast<long long>(L.out) * L.in; ++i) p[L.w0 + i] = u(rng);
    }
    params_.alloc(count_ * 4);
    grad_.alloc(count_ * 4);
    {
      int dev = 0;
      check(cudaGetDevice(&dev), "device");
      check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev), "device");
    }
    fused_ok_ = width == kMaxWidth && static_cast<int>(layers_.size()) <= fused::kLayersMax;
    fused_ = fused_ok_;  // the fused tcgen05 engine is the default where it applies
    m_.alloc(count_ * 4);
    v_.alloc(count_ * 4);
    check(cudaMemsetAsync(m_.p, 0, count_ * 4, stream_), "memset");
    check(cudaMemsetAsync(v_.p, 0, count_ * 4, stream_), "memset");
    for (const Layer& L : layers_) {
      wb_.emplace_back(std::make_unique<Buf>(static_cast<size_t>(L.np) * L.kp * 2));
      wt_.emplace_back(std::make_unique<Buf>(static_cast<size_t>(L.np) * L.kp * 2));
      // the fused engine's operand images (zero padding stays zero: packing writes the weights)
      wk_img_.emplace_back(std::make_unique<Buf>(static_cast<size_t>(L.np) * L.kp * 2));
      wt_img_.emplace_back(std::make_unique<Buf>(static_cast<size_t>(L.np) * L.kp * 2));
      check(cudaMemsetAsync(wk_img_.back()->p, 0, wk_img_.back()->n, stream_), "memset");
      check(cudaMemsetAsync(wt_img_.back()->p, 0, wt_img_.back()->n, stream_), "memset");
    }
    std::vector<float> ones(std::max(inputs, outputs), 1.0f), zeros(std::max(inputs, outputs), 0.0f);
    in_mean_.alloc(inputs * 4);
    in_sd_.alloc(inputs * 4);
    out_mean_.alloc(outputs * 4);
    out_sd_.alloc(outputs * 4);
    build_layout();
    set_scaling(zeros.data(), ones.data(), zeros.data(), ones.data());
    set_parameters(p.data());
  }
  ~Net() {
    cudaStreamSynchronize(stream_);
    if (se_host_ != nullptr) cudaFreeHost(se_host_);
    cudaStreamDestroy(stream_);
  }

  long long count() const { return count_; }

  void set_scaling(const float* im, const float* is, const float* om, const float* os) {
    for (int i = 0; i < inputs_; ++i)
      if (!(is[i] > 0.0f)) fail("E1101: input standard deviations must be positive");
    for (int i = 0; i < outputs_; ++i)
      if (!(os[i] > 0.0f)) fail("E1101: output standard deviations must be positive");
    copy(in_mean_, im, inputs_ * 4);
    copy(in_sd_, is, inputs_ * 4);
    copy(out_mean_, om, outputs_ * 4);
    copy(out_sd_, os, outputs_ * 4);
    sync();
  }

  void set_parameters(const float* p) {
    copy(params_, p, count_ * 4);
    round_weights();
    sync();
  }
  void get_parameters(float* p) {
    check(cudaMemcpyAsync(p, params_.p, count_ * 4, cudaMemcpyDeviceToHost, stream_), "params");
    sync();
  }

  void set_data(const float* x, const float* y, long long n) {
    if (n < 1) fail("E1101: empty training set");
    n_data_ = n;
    x_.alloc(static_cast<size_t>(n) * inputs_ * 4);
    y_.alloc(static_cast<size_t>(n) * outputs_ * 4);
    copy(x_, x, static_cast<size_t>(n) * inputs_ * 4);
    copy(y_, y, static_cast<size_t>(n) * outputs_ * 4);
    sync();
  }

  // Forward and backward of `rows` rows (x: raw inputs, y: raw targets, idx: rows of them or null);
  // the gradient into grad_, the loss returned.
  // The minibatch loss (mean squared error of the standardised outputs). With se_host (pinned,
  // rows floats) the per-row squared errors are copied there asynchronously and 0 is returned:
  // the caller sums them (loss_of) after a synchronisation.
  float forward_backward(const float* x, const float* y, const int* idx, int rows,
                         float* se_host = nullptr) {
    if (rows > 65535LL * kChunk) fail("E1101: at most 65535 x 128 rows in one forward-backward pass");
    if (fused_) {
      fused_pass(x, y, idx, rows, false, 0.0f, 0.0f, 0.0f);
      return take_loss(fse_, rows, se_host);
    }
    ensure_work(rows);
    const int L = static_cast<int>(layers_.size());
    launch_inputs(x, idx, rows);
    forward(rows, true);
    const Layer& last = layers_[L - 1];
    k_loss<<<blocks(rows, 128), 128, 0, stream_>>>(zf(L - 1), last.np, y, outputs_, idx, rows,
                                                   out_mean_.as<float>(), out_sd_.as<float>(),
                                                   dz_.as<float>(), dzb_.as<bf16>(), se_.as<float>());
    check(cudaGetLastError(), "loss");
    for (int l = L - 1; l >= 0; --l) {
      const Layer& Ly = layers_[l];
      const bf16* a_prev = act(l - 1);
      const int lda = l == 0 ? layers_[0].kp : width_;
      // weight gradient, padded [np x kp], then the logical [out x in] part and the bias
      const int chunks = blocks(rows, kChunk);
      const int size = Ly.np * Ly.kp;
      ensure(partial_, static_cast<size_t>(chunks) * size * 4);
      ensure(wfull_, static_cast<size_t>(size) * 4);
      if (tc_) {
        const size_t smem = static_cast<size_t>(kTcRows + Ly.kp) * kTcRows * 2;
        allow_smem(k_tc_gemm<1, false>, smem);
        k_tc_gemm<1, false><<<chunks, 128, smem, stream_>>>(
            dzb_.as<bf16>(), Ly.np, rows, kTcRows, a_prev, lda, Ly.kp, Ly.np, nullptr, nullptr, 0,
            nullptr, partial_.as<float>(), 0, tmem_cols(Ly.kp), fault_.as<unsigned int>());
      } else {
        if (!wgrad_attr_) {
          allow_smem(k_wgrad, kWgradSmem);
          wgrad_attr_ = true;
        }
        k_wgrad<<<chunks, 256, kWgradSmem, stream_>>>(dzb_.as<bf16>(), Ly.np, a_prev, lda, rows, Ly.np,
                                                     Ly.kp, partial_.as<float>());
      }
      check(cudaGetLastError(), "wgrad");
      k_sum_partials<<<blocks(size, 256), 256, 0, stream_>>>(partial_.as<float>(), chunks, size,
                                                             wfull_.as<float>());
      check(cudaGetLastError(), "wgrad sum");
      check(cudaMemcpy2DAsync(grad_.as<float>() + Ly.w0, Ly.in * 4, wfull_.as<float>(), Ly.kp * 4,
                              Ly.in * 4, Ly.out, cudaMemcpyDeviceToDevice, stream_),
            "wgrad copy");
      // bias gradient: column sums of dZ per row chunk into the (now free) partials, then summed
      k_column_partials<<<dim3((Ly.out + 31) / 32, chunks), dim3(32, 8), 0, stream_>>>(
          dz_.as<float>(), Ly.np, rows, Ly.out, partial_.as<float>());
      check(cudaGetLastError(), "bias grad");
      k_sum_partials<<<blocks(Ly.out, 256), 256, 0, stream_>>>(
          partial_.as<float>(), chunks, Ly.out,
          grad_.as<float>() + Ly.w0 + static_cast<long long>(Ly.out) * Ly.in);
      check(cudaGetLastError(), "bias grad sum");
      if (l == 0) break;
      // dA_{l-1} = dZ_l W_l: the dense kernel on W^T [kp x np]
      const Layer& Lp = layers_[l - 1];
      launch_dense<false>(dzb_.as<bf16>(), Ly.np, rows, Ly.np, wt_[l]->as<bf16>(), Ly.np, Ly.kp,
                          nullptr, da_.as<float>(), Ly.kp, nullptr, nullptr, Ly.kp);
      k_gelu_back<<<blocks(static_cast<long long>(rows) * Lp.np, 256), 256, 0, stream_>>>(
          da_.as<float>(), zf(l - 1), static_cast<long long>(rows) * Lp.np, dz_.as<float>(),
          dzb_.as<bf16>());
      check(cudaGetLastError(), "gelu back");
    }
    return take_loss(se_, rows, se_host);
  }

  // The loss of a pass from its per-row squared errors (se, device): with se_host (pinned) they
  // are copied there asynchronously and 0 is returned.
  float take_loss(const Buf& se_dev, int rows, float* se_host) {
    if (se_host != nullptr) {
      check(cudaMemcpyAsync(se_host, se_dev.p, rows * 4, cudaMemcpyDeviceToHost, stream_), "loss");
      return 0.0f;
    }
    std::vector<float> se(rows);
    check(cudaMemcpyAsync(se.data(), se_dev.p, rows * 4, cudaMemcpyDeviceToHost, stream_), "loss");
    sync();
    return loss_of(se.data(), rows);
  }

  // The fused engine's pass over `rows` rows (fused::k_fused): the gradient into grad_ and the
  // per-row squared errors into fse_; with `update`, also the Adam step at rate lr (bias
  // corrections c1, c2) and the re-packed operand images, in the same second launch.
  void fused_pass(const float* x, const float* y, const int* idx, int rows, bool update, float lr,
                  float c1, float c2) {
    const int tiles = blocks(rows, 128);
    const int grid = std::min(tiles, sms_);
    const long long L = static_cast<long long>(layers_.size());
    ensure(zbuf_, static_cast<size_t>(grid) * (L - 1) * 128 * 128 * 4);
    ensure(atbuf_, static_cast<size_t>(grid) * lay_.at_bytes);
    ensure(fpartial_, static_cast<size_t>(grid) * count_ * 4);
    ensure(fse_, static_cast<size_t>(rows) * 4);
    fused_attrs();
    fused::k_fused<true><<<grid, fused::kThreads, fused::kSmem, stream_>>>(
        lay_, x, y, idx, rows, tiles, zbuf_.as<float>(), atbuf_.as<unsigned char>(),
        fpartial_.as<float>(), count_, fse_.as<float>(),
        2.0f / (static_cast<float>(rows) * outputs_), nullptr, fault_.as<unsigned int>());
    check(cudaGetLastError(), "fused pass");
    if (update) {
      fused::k_fused_update<true, true><<<blocks(count_, 256), 256, 0, stream_>>>(
          lay_, fpartial_.as<float>(), grid, count_, grad_.as<float>(), params_.as<float>(),
          m_.as<float>(), v_.as<float>(), lr, c1, c2, fault_.as<unsigned int>());
    } else {
      fused::k_fused_update<false, false><<<blocks(count_, 256), 256, 0, stream_>>>(
          lay_, fpartial_.as<float>(), grid, count_, grad_.as<float>(), params_.as<float>(),
          nullptr, nullptr, 0.0f, 1.0f, 1.0f, fault_.as<unsigned int>());
    }
    check(cudaGetLastError(), "fused update");
  }
  void fused_attrs() {
    if (fused_attr_) return;
    allow_smem(fused::k_fused<true>, fused::kSmem);
    allow_smem(fused::k_fused<false>, fused::kSmem);
    fused_attr_ = true;
  }

  float loss_of(const float* se, int rows) const {
    double s = 0.0;
    for (int i = 0; i < rows; ++i) s += se[i];
    return static_cast<float>(s / (static_cast<double>(rows) * outputs_));
  }

  void train(int epochs, int batch, float lr, uint64_t seed, float* loss) {
    if (n_data_ == 0) fail("E1101: no training data");
    if (batch < 128 || batch % 128 != 0) fail("E1101: batch must be a positive multiple of 128");
    std::mt19937_64 rng(seed);
    std::vector<int> perm(n_data_);
    const long long per_epoch = n_data_ / batch;
    const long long total = std::max<long long>(1, per_epoch * epochs);
    long long done = 0;
    for (long long i = 0; i < n_data_; ++i) perm[i] = static_cast<int>(i);
    ensure(idx_, static_cast<size_t>(n_data_) * 4);
    // an epoch's per-row squared errors, copied without a synchronisation per step
    const size_t staged = static_cast<size_t>(per_epoch) * batch;
    if (staged > se_host_n_) {
      if (se_host_ != nullptr) cudaFreeHost(se_host_);
      se_host_ = nullptr;
      se_host_n_ = 0;
      check(cudaMallocHost(reinterpret_cast<void**>(&se_host_), staged * sizeof(float)), "cudaMallocHost");
      se_host_n_ = staged;
    }
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(perm.begin(), perm.end(), rng);
      copy(idx_, perm.data(), static_cast<size_t>(n_data_) * 4);
      long long steps = 0;
      for (long long r0 = 0; r0 + batch <= n_data_; r0 += batch) {
        if (fused_) {
          // one fused pass and one update launch a step
          ++t_;
          const float rate = lr * 0.5f * (1.0f + std::cos(3.14159265358979f * static_cast<float>(done) / total));
          ++done;
          const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(t_));
          const float c2 = 1.0f - std::pow(0.999f, static_cast<float>(t_));
          fused_pass(x_.as<float>(), y_.as<float>(), idx_.as<int>() + r0, batch, true, rate, c1, c2);
          take_loss(fse_, batch, se_host_ + static_cast<size_t>(steps) * batch);
          ++steps;
          continue;
        }
        forward_backward(x_.as<float>(), y_.as<float>(), idx_.as<int>() + r0, batch,
                         se_host_ + static_cast<size_t>(steps) * batch);
        ++t_;
        // cosine decay of the learning rate over the call's steps
        const float rate = lr * 0.5f * (1.0f + std::cos(3.14159265358979f * static_cast<float>(done) / total));
        ++done;
        const float c1 = 1.0f - std::pow(0.9f, static_cast<float>(t_));
        const float c2 = 1.0f - std::pow(0.999f, static_cast<float>(t_));
        k_adam<<<blocks(count_, 256), 256, 0, stream_>>>(params_.as<float>(), grad_.as<float>(),
                                                         m_.as<float>(), v_.as<float>(), count_, rate, c1,
                                                         c2);
        check(cudaGetLastError(), "adam");
        round_weights();
        ++steps;
      }
      sync();
      double sum = 0.0;
      for (long long q = 0; q < steps; ++q) sum += loss_of(se_host_ + static_cast<size_t>(q) * batch, batch);
      if (loss != nullptr) loss[e] = static_cast<float>(steps > 0 ? sum / steps : 0.0);
    }
    sync();
  }

  void predict(const float* x, long long n, float* y, bool device_ptrs) {
    const long long chunk = 1 << 18;
    Buf xd, yd;
    if (!device_ptrs) {
      xd.alloc(static_cast<size_t>(n) * inputs_ * 4);
      yd.alloc(static_cast<size_t>(n) * outputs_ * 4);
      copy(xd, x, static_cast<size_t>(n) * inputs_ * 4);
    }
    const float* xs = device_ptrs ? x : xd.as<float>();
    float* ys = device_ptrs ? y : yd.as<float>();
    const int L = static_cast<int>(layers_.size());
    for (long long r0 = 0; r0 < n; r0 += chunk) {
      const int rows = static_cast<int>(std::min(chunk, n - r0));
      if (fused_) {
        const int tiles = blocks(rows, 128);
        fused_attrs();
        fused::k_fused<false><<<std::min(tiles, sms_), fused::kThreads, fused::kSmem, stream_>>>(
            lay_, xs + r0 * inputs_, nullptr, nullptr, rows, tiles, nullptr, nullptr, nullptr, 0,
            nullptr, 0.0f, ys + r0 * outputs_, fault_.as<unsigned int>());
        check(cudaGetLastError(), "fused predict");
        continue;
      }
      ensure_work(rows);
      launch_inputs(xs + r0 * inputs_, nullptr, rows);
      forward(rows, false);
      k_outputs<<<blocks(static_cast<long long>(rows) * outputs_, 256), 256, 0, stream_>>>(
          zf(L - 1), layers_[L - 1].np, outputs_, rows, out_mean_.as<float>(), out_sd_.as<float>(),
          ys + r0 * outputs_);
      check(cudaGetLastError(), "outputs");
    }
    if (!device_ptrs)
      check(cudaMemcpyAsync(y, yd.p, static_cast<size_t>(n) * outputs_ * 4, cudaMemcpyDeviceToHost, stream_),
            "predict");
    sync();
  }

  // One forward and backward pass on host rows, no update: the loss and the gradient.
  float gradient(const float* x, const float* y, int n, float* g) {
    Buf xd(static_cast<size_t>(n) * inputs_ * 4), yd(static_cast<size_t>(n) * outputs_ * 4);
    copy(xd, x, static_cast<size_t>(n) * inputs_ * 4);
    copy(yd, y, static_cast<size_t>(n) * outputs_ * 4);
    const float l = forward_backward(xd.as<float>(), yd.as<float>(), nullptr, n);
    grad_to(g);
    return l;
  }

  void grad_to(float* g) {
    check(cudaMemcpyAsync(g, grad_.p, count_ * 4, cudaMemcpyDeviceToHost, stream_), "grad");
    sync();
  }
  void copy_in(Buf& b, const void* host, size_t bytes) { copy(b, host, bytes); }
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }

 private:
  template <bool ACT>
  void launch_dense(const bf16* A, int lda, int M, int K, const bf16* B, int ldb, int N,
                    const float* bias, float* Z, int ldz, bf16* Y, float* Yf, int ldy) {
    if (tc_) {
      const size_t smem = static_cast<size_t>(kTcRows + N) * K * 2;
      allow_smem(k_tc_gemm<0, ACT>, smem);
      k_tc_gemm<0, ACT><<<blocks(M, kTcRows), 128, smem, stream_>>>(A, lda, M, K, B, ldb, N, N, bias,
                                                                   Z, ldz, Y, Yf, ldy, tmem_cols(N),
                                                                   fault_.as<unsigned int>());
      check(cudaGetLastError(), "tc dense");
      return;
    }
    const size_t smem = static_cast<size_t>(kRowsPerBlock + N) * (K + 8) * 2;
    if (smem > 48 * 1024)
      allow_smem(k_dense<ACT>, smem);
    k_dense<ACT><<<blocks(M, kRowsPerBlock), 128, smem, stream_>>>(A, lda, M, K, B, ldb, N, bias, Z,
                                                                  ldz, Y, Yf, ldy);
    check(cudaGetLastError(), "dense");
  }
  void forward(int rows, bool keep) {
    (void)keep;
    const int L = static_cast<int>(layers_.size());
    for (int l = 0; l < L; ++l) {
      const Layer& Ly = layers_[l];
      const bf16* a = act(l - 1);
      const int lda = l == 0 ? layers_[0].kp : width_;
      const float* bias = params_.as<float>() + Ly.w0 + static_cast<long long>(Ly.out) * Ly.in;
      // biases of padded output columns: the parameter vector holds `out` of them; padded
      // columns read beyond into the next layer's weights, so the output layer uses its own pad
      const float* b = Ly.np == Ly.out ? bias : padded_bias(l);
      if (l < L - 1) {
        launch_dense<true>(a, lda, rows, Ly.kp, wb_[l]->as<bf16>(), Ly.kp, Ly.np, b, zf(l), Ly.np,
                           act_b(l), nullptr, Ly.np);
      } else {
        launch_dense<false>(a, lda, rows, Ly.kp, wb_[l]->as<bf16>(), Ly.kp, Ly.np, b, zf(l), Ly.np,
                            nullptr, nullptr, Ly.np);
      }
    }
  }
  const float* padded_bias(int l) {
    const Layer& Ly = layers_[l];
    ensure(pbias_, static_cast<size_t>(kMaxWidth) * 4);
    check(cudaMemsetAsync(pbias_.p, 0, kMaxWidth * 4, stream_), "bias");
    check(cudaMemcpyAsync(pbias_.p, params_.as<float>() + Ly.w0 + static_cast<long long>(Ly.out) * Ly.in,
                          Ly.out * 4, cudaMemcpyDeviceToDevice, stream_), "bias");
    return pbias_.as<float>();
  }
  void launch_inputs(const float* x, const int* idx, int rows) {
    const int ldx = layers_[0].kp;
    k_inputs<<<blocks(static_cast<long long>(rows) * ldx, 256), 256, 0, stream_>>>(
        x, inputs_, idx, rows, in_mean_.as<float>(), in_sd_.as<float>(), x0_.as<bf16>(), ldx);
    check(cudaGetLastError(), "inputs");
  }
  void round_weights() {
    for (size_t l = 0; l < layers_.size(); ++l) {
      const Layer& Ly = layers_[l];
      k_round_weights<<<blocks(static_cast<long long>(Ly.np) * Ly.kp, 256), 256, 0, stream_>>>(
          params_.as<float>() + Ly.w0, Ly.out, Ly.in, wb_[l]->as<bf16>(), Ly.kp, wt_[l]->as<bf16>(),
          Ly.np);
      check(cudaGetLastError(), "round weights");
    }
    if (fused_ok_) {  // the fused engine's operand images
      fused::k_fused_update<false, true><<<blocks(count_, 256), 256, 0, stream_>>>(
          lay_, nullptr, 0, count_, nullptr, params_.as<float>(), nullptr, nullptr, 0.0f, 1.0f, 1.0f,
          nullptr);
      check(cudaGetLastError(), "pack weights");
    }
  }
  void build_layout() {
    if (!fused_ok_) return;
    fused::Layout& P = lay_;
    P = fused::Layout{};
    P.layers = static_cast<int>(layers_.size());
    P.inputs = inputs_;
    P.outputs = outputs_;
    long long at = 0;
    for (size_t l = 0; l < layers_.size(); ++l) {
      const Layer& Ly = layers_[l];
      P.in[l] = Ly.in;
      P.out[l] = Ly.out;
      P.kp[l] = Ly.kp;
      P.np[l] = Ly.np;
      P.w0[l] = Ly.w0;
      P.at0[l] = at;
      at += static_cast<long long>(Ly.kp) * 128 * 2;
      P.wk[l] = P.wkw[l] = wk_img_[l]->as<bf16>();
      P.wtk[l] = P.wtkw[l] = wt_img_[l]->as<bf16>();
    }
    P.at_bytes = at;
    P.params = params_.as<float>();
    P.in_mean = in_mean_.as<float>();
    P.in_sd = in_sd_.as<float>();
    P.out_mean = out_mean_.as<float>();
    P.out_sd = out_sd_.as<float>();
  }
  const bf16* act(int l) { return l < 0 ? x0_.as<bf16>() : act_b(l); }
  bf16* act_b(int l) { return acts_.as<bf16>() + static_cast<long long>(l) * work_rows_ * width_; }
  float* zf(int l) { return zs_.as<float>() + static_cast<long long>(l) * work_rows_ * kMaxWidth; }
  void ensure_work(int rows) {
    if (rows <= work_rows_) return;
    work_rows_ = rows;
    const long long L = static_cast<long long>(layers_.size());
    x0_.alloc(static_cast<size_t>(rows) * layers_[0].kp * 2);
    acts_.alloc(static_cast<size_t>(L) * rows * width_ * 2);
    zs_.alloc(static_cast<size_t>(L) * rows * kMaxWidth * 4);
    dz_.alloc(static_cast<size_t>(rows) * kMaxWidth * 4);
    dzb_.alloc(static_cast<size_t>(rows) * kMaxWidth * 2);
    da_.alloc(static_cast<size_t>(rows) * kMaxWidth * 4);
    se_.alloc(static_cast<size_t>(rows) * 4);
  }
  void ensure(Buf& b, size_t bytes) {
    if (b.n < bytes) b.alloc(bytes);
  }
  void copy(Buf& b, const void* host, size_t bytes) {
    check(cudaMemcpyAsync(b.p, host, bytes, cudaMemcpyHostToDevice, stream_), "copy");
  }
  void sync() {
    check(cudaStreamSynchronize(stream_), "sync");
    unsigned int f = 0;
    check(cudaMemcpy(&f, fault_.p, sizeof(f), cudaMemcpyDeviceToHost), "fault");
    if (f != 0) {
      // reported once: the word is cleared so that the handle's next call starts clean
      check(cudaMemset(fault_.p, 0, sizeof(unsigned int)), "fault");
      fail("E1201: a tensor-core wait timed out; results are invalid");
    }
  }
  static int tmem_cols(int n) {
    int c = 32;
    while (c < n) c *= 2;
    return c;
  }

 public:
  void set_engine(int engine) {
    if (engine < 0 || engine > 2)
      fail("E1101: engine 0 (mma.sync), 1 (tcgen05 per layer) or 2 (fused tcgen05)");
    if (engine == 2 && !fused_ok_)
      fail("E1101: the fused tcgen05 engine takes width 128 and at most 8 weight layers");
    tc_ = engine == 1;
    fused_ = engine == 2;
  }
  int engine() const { return fused_ ? 2 : (tc_ ? 1 : 0); }
  // Test hook (0 in normal use): the fused kernel's first wait polls a barrier nothing arrives on,
  // at most `polls` times, and runs out (the call then fails with E1201).
  void set_stall_test(int polls) {
    if (polls < 0) fail("E1101: polls must be >= 0");
    lay_.stall_polls = polls;
  }

 private:

  int inputs_, width_, outputs_, device_;
  cudaStream_t stream_ = nullptr;
  std::vector<Layer> layers_;
  long long count_ = 0;
  long long t_ = 0;
  long long n_data_ = 0;
  int work_rows_ = 0;
  bool wgrad_attr_ = false;
  bool tc_ = false;  // tcgen05 engine, layer per launch
  bool fused_ = false;     // fused tcgen05 engine (fused::k_fused)
  bool fused_ok_ = false;  // the network's shape suits it (width 128)
  bool fused_attr_ = false;
  int sms_ = 148;
  fused::Layout lay_{};
  Buf zbuf_, atbuf_, fpartial_, fse_;
  std::vector<std::unique_ptr<Buf>> wk_img_, wt_img_;
  Buf params_, grad_, m_, v_, in_mean_, in_sd_, out_mean_, out_sd_, x_, y_, idx_, fault_;
  float* se_host_ = nullptr;  // pinned: an epoch's per-row squared errors
  size_t se_host_n_ = 0;
  Buf x0_, acts_, zs_, dz_, dzb_, da_, se_, partial_, wfull_, pbias_;
  std::vector<std::unique_ptr<Buf>> wb_, wt_;
};

int fail_to(char* err, size_t len, const std::string& what) {
  if (err != nullptr && len > 0) snprintf(err, len, "%s", what.c_str());
  return 1;
}

template <class F>
int guarded(char* err, size_t len, F&& body) {
  try {
    body();
    return 0;
  } catch (const Failure& e) {
    return fail_to(err, len, e.what());
  } catch (const std::bad_alloc&) {
    return fail_to(err, len, "E1103: out of host memory");
  } catch (const std::exception& e) {
    return fail_to(err, len, std::string("E1100: ") + e.what());
  }
}

Net* as_net(void* h) {
  if (h == nullptr) fail("E1101: null handle");
  return static_cast<Net*>(h);
}

}  // namespace mlp
}  // namespace autan_b200

using namespace autan_b200::mlp;

extern "C" {

int autan_mlp_create(int32_t inputs, int32_t width, int32_t layers, int32_t outputs, uint64_t seed,
                     int32_t device, void** handle, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (handle == nullptr) fail("E1101: null handle");
    *handle = new Net(inputs, width, layers, outputs, seed, device < 0 ? 0 : device);
  });
}

void autan_mlp_destroy(void* handle) { delete static_cast<Net*>(handle); }

int autan_mlp_set_engine(void* handle, int32_t engine, char* err, size_t err_len) {
  return guarded(err, err_len, [&] { as_net(handle)->set_engine(engine); });
}

int autan_mlp_set_stall_test(void* handle, int32_t polls, char* err, size_t err_len) {
  return guarded(err, err_len, [&] { as_net(handle)->set_stall_test(polls); });
}

int autan_mlp_set_scaling(void* handle, const float* in_mean, const float* in_std,
                          const float* out_mean, const float* out_std, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!in_mean || !in_std || !out_mean || !out_std) fail("E1101: null scaling");
    as_net(handle)->set_scaling(in_mean, in_std, out_mean, out_std);
  });
}

int64_t autan_mlp_parameter_count(void* handle) {
  return handle == nullptr ? 0 : static_cast<Net*>(handle)->count();
}

int autan_mlp_get_parameters(void* handle, float* params, int64_t count, char* err,
                             size_t err_len) {
  return guarded(err, err_len, [&] {
    Net* n = as_net(handle);
    if (params == nullptr || count != n->count()) fail("E1101: parameter count mismatch");
    n->get_parameters(params);
  });
}

int autan_mlp_set_parameters(void* handle, const float* params, int64_t count, char* err,
                             size_t err_len) {
  return guarded(err, err_len, [&] {
    Net* n = as_net(handle);
    if (params == nullptr || count != n->count()) fail("E1101: parameter count mismatch");
    n->set_parameters(params);
  });
}

int autan_mlp_set_data(void* handle, const float* x, const float* y, int64_t n, char* err,
                       size_t err_len) {
  return guarded(err, err_len, [&] {
    if (x == nullptr || y == nullptr) fail("E1101: null data");
    as_net(handle)->set_data(x, y, n);
  });
}

int autan_mlp_train(void* handle, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                    float* loss, char* err, size_t err_len) {
  return guarded(err, err_len, [&] { as_net(handle)->train(epochs, batch, lr, seed, loss); });
}

int autan_mlp_gradient(void* handle, const float* x, const float* y, int64_t n, float* loss,
                       float* grad, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    Net* net = as_net(handle);
    if (x == nullptr || y == nullptr || grad == nullptr || n < 1 || n > (1 << 20))
      fail("E1101: 1 to 2^20 rows and non-null arrays");
    const float l = net->gradient(x, y, static_cast<int>(n), grad);
    if (loss != nullptr) *loss = l;
  });
}

int autan_mlp_predict(void* handle, const float* x, int64_t n, float* y, int32_t device_ptrs,
                      char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (x == nullptr || y == nullptr || n < 0) fail("E1101: null arrays");
    if (n == 0) return;
    as_net(handle)->predict(x, n, y, device_ptrs != 0);
  });
}

int autan_wall_distance(const double* triangles, const int64_t* tri_offsets, const double* points,
                        const int64_t* point_offsets, int32_t n_cases, int64_t n_points,
                        double* distance, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (!tri_offsets || !points || !point_offsets || !distance || n_cases < 1 || n_points < 0)
      fail("E1101: null or empty arguments");
    if (point_offsets[0] != 0 || point_offsets[n_cases] != n_points)
      fail("E1101: point offsets must span the points");
    const int64_t nt = tri_offsets[n_cases];
    std::vector<int> case_of(std::max<int64_t>(n_points, 1), 0);
    for (int k = 0; k < n_cases; ++k)
      for (int64_t i = point_offsets[k]; i < point_offsets[k + 1]; ++i) case_of[i] = k;
    Buf t(static_cast<size_t>(std::max<int64_t>(nt, 1)) * 9 * 8), to((n_cases + 1) * 8),
        p(static_cast<size_t>(std::max<int64_t>(n_points, 1)) * 3 * 8),
        c(case_of.size() * 4), d(static_cast<size_t>(std::max<int64_t>(n_points, 1)) * 8);
    if (nt > 0) check(cudaMemcpy(t.p, triangles, nt * 9 * 8, cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(to.p, tri_offsets, (n_cases + 1) * 8, cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(p.p, points, n_points * 3 * 8, cudaMemcpyHostToDevice), "copy");
    check(cudaMemcpy(c.p, case_of.data(), case_of.size() * 4, cudaMemcpyHostToDevice), "copy");
    k_wall_distance<<<blocks(n_points, 128), 128>>>(t.as<double>(), to.as<int64_t>(), p.as<double>(),
                                                    c.as<int>(), n_points, d.as<double>());
    check(cudaGetLastError(), "wall distance");
    check(cudaMemcpy(distance, d.p, n_points * 8, cudaMemcpyDeviceToHost), "copy");
  });
}

}  // extern "C"
