// The fused tcgen05 engine of the warm-start MLP (included by mlp.cu, inside its namespace; width
// 128). One CTA of 8 warps takes a 128-row tile through the whole network in one launch:
//
//   forward   for every layer l: A_l (shared memory, K-major BF16 image) x W_l (shared memory)
//             -> accumulator in tensor memory -> epilogue: + bias, GELU, BF16 into the image of
//             A_{l+1}; Z_l (FP32) kept in the CTA's scratch for GELU' (training);
//   loss      the output layer's epilogue: squared errors per row, dZ = 2 (pred - t) / (n outputs);
//   backward  for every layer from the last: dW_l = dZ_l^T A_l (or its transpose, so that the
//             MMA's M is always 128) and dA_l = dZ_l W_l, both into tensor memory by one batch of
//             MMAs; the epilogue adds dW_l and the FP32 column sums of dZ_l (the bias gradient)
//             to the CTA's partial, and forms dZ_{l-1} = dA_l GELU'(Z_{l-1}).
//
// Every layer's weights (the packed BF16 images W_l and W_l^T, L2-resident) are staged into shared
// memory by TMA bulk copies (cp.async.bulk, no tensor map, no multicast) on mbarriers, double
// buffered: the next layer's image lands while this layer computes. The transposed operands the
// weight gradient needs (A_l^T, dZ_l^T) are made by ldmatrix.trans + stmatrix; A_l^T goes to the
// CTA's scratch by a bulk store during the forward pass and comes back by a bulk copy in the
// backward pass. One thread issues the MMAs (kind::f16: BF16 operands, FP32 accumulators) and
// commits them to an mbarrier; every wait is bounded and a wait that runs out sets the fault word
// (E1201 on the host) and ends the CTA's work after bounded waits for what it has in flight.
//
// The CTA adds its tiles' gradients into its own partial (grid-stride over tiles, in tile order);
// k_fused_update then sums the CTAs' partials in CTA order (deterministic for a given grid), and
// for a training step applies Adam and re-packs the BF16 images.

namespace fused {

constexpr int kLayersMax = 8;
constexpr int kThreads = 512;             // warp w: TMEM lanes 32 (w % 4), column group w / 4
constexpr int kGroups = kThreads / 128;   // column groups of an accumulator's epilogue
constexpr int kImg = 128 * 128 * 2;       // bytes of a 128 x 128 BF16 operand image
constexpr int kTmemCols = 256;            // [0, 128) forward / dA accumulator, [128, 256) dW
constexpr int kWgradCol = 128;
// shared memory: A / dZ image, dZ^T (and the forward's A^T staging), W images x 2, A^T images x 2,
// column sums [4 lane quarters][128] and the squared-error parts [kGroups][128] (FP32)
constexpr int kOffA = 0;
constexpr int kOffDzt = kImg;
constexpr int kOffW = 2 * kImg;
constexpr int kOffAt = 4 * kImg;
constexpr int kOffCol = 6 * kImg;
constexpr int kOffSe = kOffCol + 4 * 128 * 4;
constexpr int kOffBias = kOffSe + kGroups * 128 * 4;  // the current layer's bias, 128 FP32
constexpr int kSmem = kOffBias + 128 * 4;

// The columns [c0, c1) of an N-column accumulator that column group h reads in the epilogues: N
// split into kGroups parts of at least 8 (groups past N read none).
__device__ __forceinline__ int group_cols(int N) { return N / kGroups > 8 ? N / kGroups : 8; }

struct Layout {
  int layers;  // weight layers: hidden layers + the output layer
  int inputs, outputs;
  int in[kLayersMax], out[kLayersMax], kp[kLayersMax], np[kLayersMax];
  long long w0[kLayersMax];    // W_l at w0 in the parameter vector ([out x in]), then its bias
  long long at0[kLayersMax];   // byte offset of the A_l^T image in a CTA's A^T scratch
  long long at_bytes;          // a CTA's A^T scratch
  const bf16* wk[kLayersMax];  // W_l as the forward B operand: [np x kp], K-major image
  bf16* wkw[kLayersMax];       // the same, writable (k_fused_update)
  const bf16* wtk[kLayersMax];  // W_l^T as the dA B operand: [kp x np], K-major image
  bf16* wtkw[kLayersMax];
  const float* params;  // FP32 master parameters (the biases are read from here)
  const float *in_mean, *in_sd, *out_mean, *out_sd;
  // Test hook of the failure detection (0 in normal use): with n > 0 every thread first waits, n
  // polls at most, on an mbarrier that nothing arrives on, so that the bounded wait runs out and
  // the kernel takes its fault path (fault word, no stores) before any copy or MMA is issued.
  int stall_polls;
};

__device__ __forceinline__ void bar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void bar_expect(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared completing on `bar` (TMA engine; no tensor map, no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// 1-D bulk copy shared -> global, in the issuing thread's bulk group.
__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_store_read_done() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_store_done() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void proxy_fence_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}
// Eight FP32 accumulator columns [col, col + 8) of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float* out) {
  uint32_t v[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 8; ++j) out[j] = __uint_as_float(v[j]);
}

// 32 FP32 accumulator columns [col, col + 32) of this warp's 32 TMEM lanes: one load, one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float* out) {
  uint32_t v[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
        "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
        "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) out[j] = __uint_as_float(v[j]);
}

// 16 FP32 accumulator columns [col, col + 16) of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* out) {
  uint32_t v[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) out[j] = __uint_as_float(v[j]);
}

// This warp's part of an accumulator: columns [c, c + 8 n) for n = cw / 8 (cw 32: one 32-column
// load; cw 8: one 8-column load; columns at or past `end`: none).
__device__ __forceinline__ void tmem_part(uint32_t addr, int cw, int c, int end, float* out) {
  if (c >= end) return;
  if (cw == 32) {
    tmem_ld32(addr + static_cast<uint32_t>(c), out);
  } else {
    tmem_ld8(addr + static_cast<uint32_t>(c), out);
  }
}

// A bounded wait on `bar`'s phase `parity` by every thread; true (uniformly) when it completed.
__device__ __forceinline__ bool wait_all(unsigned long long* bar, uint32_t parity) {
  bool done = false;
  for (int it = 0; it < kTcWaitLimit && !done; ++it) done = tc_try_wait(bar, parity);
  return __syncthreads_and(done ? 1 : 0) != 0;
}

// Eight BF16 values of a row into an image (16 bytes at kmajor(r, c0, 128)).
__device__ __forceinline__ void put8(unsigned char* img, int r, int c0, const float* v) {
  uint4 o;
  o.x = pack2(__float2bfloat16(v[0]), __float2bfloat16(v[1]));
  o.y = pack2(__float2bfloat16(v[2]), __float2bfloat16(v[3]));
  o.z = pack2(__float2bfloat16(v[4]), __float2bfloat16(v[5]));
  o.w = pack2(__float2bfloat16(v[6]), __float2bfloat16(v[7]));
  *reinterpret_cast<uint4*>(img + kmajor(r, c0, 128)) = o;
}

// dst [C x 128] (K-major, R = C) = src [128 x C]^T (K-major, R = 128), C a multiple of 8: every
// 8 x 8 core matrix transposed by ldmatrix.trans and written by stmatrix, four per warp at a time.
// Call from every thread; the caller synchronises around it.
__device__ __forceinline__ void transpose_img(const unsigned char* src, unsigned char* dst, int C) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mats = 16 * (C >> 3);  // core matrices m = 16 cb + rb
  for (int m0 = 4 * warp; m0 < mats; m0 += 4 * (kThreads / 32)) {
    const int m = m0 + (lane >> 3), i = lane & 7;
    const int rb = m & 15, cb = m >> 4;
    const bool live = m < mats;  // mats is a multiple of 4 (C >= 8): every group is whole
    const uint32_t a = smem_addr(src + (live ? kmajor(8 * rb + i, 8 * cb, 128) : 0));
    uint32_t r0, r1, r2, r3;
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
    const uint32_t b = smem_addr(dst + (live ? kmajor(8 * cb + i, 8 * rb, C) : 0));
    asm volatile("stmatrix.sync.aligned.m8n8.x4.shared.b16 [%0], {%1, %2, %3, %4};" ::"r"(b),
                 "r"(r0), "r"(r1), "r"(r2), "r"(r3)
                 : "memory");
  }
}

// Column sums over this warp's 32 lanes of eight values per lane (a fixed tree): the sum of
// column (lane >> 2) & 7 ... returned in lanes with (lane & 3) == 0, column index in *col.
__device__ __forceinline__ float warp_colsum8(const float* g, int* col) {
  const int lane = threadIdx.x & 31;
  const bool b4 = (lane >> 4) & 1, b3 = (lane >> 3) & 1, b2 = (lane >> 2) & 1;
  float a[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float send = b4 ? g[i] : g[i + 4];
    const float keep = b4 ? g[i + 4] : g[i];
    a[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float b[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float send = b3 ? a[i] : a[i + 2];
    const float keep = b3 ? a[i + 2] : a[i];
    b[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  const float send = b2 ? b[0] : b[1];
  float c = (b2 ? b[1] : b[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
  c += __shfl_xor_sync(0xffffffffu, c, 2);
  c += __shfl_xor_sync(0xffffffffu, c, 1);
  *col = (b4 ? 4 : 0) + (b3 ? 2 : 0) + (b2 ? 1 : 0);
  return c;
}

// Whether job j stages a weight image: the forward jobs (W_l) and the backward jobs of layers
// l > 0 (W_l^T); the backward jobs also stage A_l^T.
__device__ __forceinline__ int job_layer(const Layout& P, int j) {
  return j < P.layers ? j : 2 * P.layers - 1 - j;
}

template <bool TRAIN>
__global__ void __launch_bounds__(kThreads, 1)
    k_fused(Layout P, const float* x, const float* y, const int* idx, int rows, int tiles,
            float* zbuf, unsigned char* atbuf, float* partial, long long count, float* se,
            float scale, float* yout, unsigned int* fault) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) unsigned long long mma_bar, ld_bar[2], dead_bar;
  __shared__ uint32_t tmem_slot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, h = warp >> 2;  // TMEM lane quarter, column group
  const int row = 32 * q + lane;          // this thread's row of the tile
  unsigned char* const aimg = sm + kOffA;  // A_l (forward), dZ_l (backward)
  unsigned char* const dzt = sm + kOffDzt;
  auto wimg = [&](int b) { return sm + kOffW + b * kImg; };    // W_l / W_l^T, double-buffered
  auto atimg = [&](int b) { return sm + kOffAt + b * kImg; };  // A_l^T, double-buffered
  float* const colsum = reinterpret_cast<float*>(sm + kOffCol);  // [4][128]
  float* const separt = reinterpret_cast<float*>(sm + kOffSe);   // [kGroups][128]
  float* const sbias = reinterpret_cast<float*>(sm + kOffBias);  // [128]
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    bar_init(&mma_bar);
    bar_init(&ld_bar[0]);
    bar_init(&ld_bar[1]);
    bar_init(&dead_bar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = static_cast<uint32_t>(32 * q) << 16;
  const int L = P.layers;
  const int jobs = TRAIN ? 2 * L : L;
  float* const zc = TRAIN ? zbuf + static_cast<long long>(blockIdx.x) * (L - 1) * 128 * 128 : nullptr;
  unsigned char* const atc = TRAIN ? atbuf + static_cast<long long>(blockIdx.x) * P.at_bytes : nullptr;
  float* const part = TRAIN ? partial + static_cast<long long>(blockIdx.x) * count : nullptr;
  // phases: bit b of ld_par is the parity of buffer b's next load; ld_busy bit b: a load issued
  // into buffer b and not yet waited for (thread 0's record, for the fault path)
  uint32_t mma_par = 0, ld_par = 0, ld_busy = 0;
  bool mma_pending = false;
  bool ok = true;
  if (P.stall_polls > 0) {  // the test hook: a wait that cannot complete, bounded
    bool done = false;
    for (int it = 0; it < P.stall_polls && !done; ++it) done = tc_try_wait(&dead_bar, 0);
    ok = __syncthreads_and(done ? 1 : 0) != 0;
  }

  // job j's staging (thread 0): W_l or W_l^T, and A_l^T for the backward jobs, into buffer j % 2
  auto issue = [&](int j) {
    const int l = job_layer(P, j), b = j & 1;
    if (j < L) {
      const uint32_t wb = static_cast<uint32_t>(P.np[l] * P.kp[l] * 2);
      bar_expect(&ld_bar[b], wb);
      bulk_load(wimg(b), P.wk[l], wb, &ld_bar[b]);
    } else {
      const uint32_t wb = l > 0 ? static_cast<uint32_t>(P.np[l] * P.kp[l] * 2) : 0u;
      const uint32_t ab = static_cast<uint32_t>(P.kp[l] * 128 * 2);
      bulk_store_done();  // the forward pass's A^T stores complete before they are read back
      bar_expect(&ld_bar[b], wb + ab);
      if (wb > 0) bulk_load(wimg(b), P.wtk[l], wb, &ld_bar[b]);
      bulk_load(atimg(b), atc + P.at0[l], ab, &ld_bar[b]);
    }
    ld_busy |= 1u << b;
  };
  // A^T of the image in aimg ([128 x C]) to the scratch slot of layer l, through dzt
  auto save_at = [&](int l, int C) {
    if (threadIdx.x == 0) bulk_store_read_done();  // dzt free of the previous store
    __syncthreads();
    transpose_img(aimg, dzt, C);
    proxy_fence_shared();
    __syncthreads();
    if (threadIdx.x == 0) bulk_store(atc + P.at0[l], dzt, static_cast<uint32_t>(C * 128 * 2));
  };
  // the bias gradient of layer l from colsum (every warp has written its columns): summed over the
  // four lane quarters in order, added to the partial
  auto bias_grad = [&](int l, bool first) {
    __syncthreads();
    const int t = threadIdx.x;
    if (t < P.out[l]) {
      const float s = ((colsum[t] + colsum[128 + t]) + colsum[256 + t]) + colsum[384 + t];
      float* dst = part + P.w0[l] + static_cast<long long>(P.out[l]) * P.in[l] + t;
      *dst = first ? s : *dst + s;
    }
  };
  auto colsum_chunk = [&](int c0, const float* g) {
    int col;
    const float s = warp_colsum8(g, &col);
    if ((lane & 3) == 0) colsum[q * 128 + c0 + col] = s;
  };

  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const long long r0 = static_cast<long long>(tile) * 128;
    const bool first = tile == static_cast<int>(blockIdx.x);
    const bool valid = r0 + row < rows;
    long long src = 0;
    if (valid) src = idx != nullptr ? idx[r0 + row] : r0 + row;
    if (threadIdx.x == 0) issue(0);
    // the standardised inputs: A_0 [128 x kp_0] (zero padding, zero rows past the end)
    {
      const int groups = P.kp[0] >> 3;
      for (int i = threadIdx.x; i < 128 * groups; i += kThreads) {
        const int r = i / groups, g = i % groups;
        float v[8];
        const bool in = r0 + r < rows;
        const long long s = !in ? 0 : (idx != nullptr ? idx[r0 + r] : r0 + r);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int c = 8 * g + e;
          v[e] = in && c < P.inputs ? (x[s * P.inputs + c] - P.in_mean[c]) / P.in_sd[c] : 0.0f;
        }
        put8(aimg, r, 8 * g, v);
      }
    }
    if (TRAIN) save_at(0, P.kp[0]);

    for (int j = 0; j < jobs && ok; ++j) {
      const int l = job_layer(P, j), b = j & 1;
      const bool forward = j < L;
      // the next job's staging into the other buffer (its last reader, job j - 1, is complete)
      if (threadIdx.x == 0 && j + 1 < jobs) issue(j + 1);
      ok = wait_all(&ld_bar[b], (ld_par >> b) & 1u);
      if (!ok) break;
      ld_par ^= 1u << b;
      ld_busy &= ~(1u << b);
      // operands written by this CTA's threads (images, transposes) -> the tensor cores
      proxy_fence_shared();
      tc_before();
      __syncthreads();
      tc_after();
      if (threadIdx.x == 0) {
        if (forward) {
          const uint32_t idesc = tc_idesc(P.np[l]);
          for (int k0 = 0; k0 < P.kp[l]; k0 += 16)
            tc_mma(tmem, smem_desc(smem_addr(aimg) + (k0 >> 3) * (128 * 16), 128),
                   smem_desc(smem_addr(wimg(b)) + (k0 >> 3) * (P.np[l] * 16), P.np[l]), idesc,
                   k0 > 0 ? 1u : 0u);
        } else {
          // dW_l (M = np = 128: dZ^T x A^T rows) or dW_l^T (M = kp = 128: A^T x dZ^T rows)
          const bool direct = P.np[l] == 128;
          const int nw = direct ? P.kp[l] : P.np[l];
          const unsigned char* ma = direct ? dzt : atimg(b);
          const unsigned char* mb = direct ? atimg(b) : dzt;
          const uint32_t idw = tc_idesc(nw);
          for (int k0 = 0; k0 < 128; k0 += 16)
            tc_mma(tmem + kWgradCol, smem_desc(smem_addr(ma) + (k0 >> 3) * (128 * 16), 128),
                   smem_desc(smem_addr(mb) + (k0 >> 3) * (nw * 16), nw), idw, k0 > 0 ? 1u : 0u);
          if (l > 0) {  // dA_l = dZ_l W_l: [128 x np] x (W^T image [kp x np])
            const uint32_t ida = tc_idesc(P.kp[l]);
            for (int k0 = 0; k0 < P.np[l]; k0 += 16)
              tc_mma(tmem, smem_desc(smem_addr(aimg) + (k0 >> 3) * (128 * 16), 128),
                     smem_desc(smem_addr(wimg(b)) + (k0 >> 3) * (P.kp[l] * 16), P.kp[l]), ida,
                     k0 > 0 ? 1u : 0u);
          }
        }
        tc_commit(&mma_bar);
      }
      mma_pending = true;
      // loaded while the MMAs run: the forward epilogue's bias into shared memory (visible after
      // the wait's barrier); the backward epilogue's GELU'(Z_{l-1}) of this thread's 32 columns
      // (the input of a layer l > 0 is 128 wide) into registers
      float pre[32];
      if (forward) {
        if (threadIdx.x < 128) {
          const float* bias = P.params + P.w0[l] + static_cast<long long>(P.out[l]) * P.in[l];
          sbias[threadIdx.x] = static_cast<int>(threadIdx.x) < P.out[l] ? __ldg(bias + threadIdx.x) : 0.0f;
        }
      } else if constexpr (TRAIN) {
        if (l > 0) {
#pragma unroll
          for (int e = 0; e < 32; ++e)
            pre[e] = zc[(static_cast<long long>(l - 1) * 128 + h * 32 + e) * 128 + row];
        }
      }
      ok = wait_all(&mma_bar, mma_par);
      if (!ok) break;
      mma_par ^= 1u;
      mma_pending = false;
      tc_after();

      if (forward) {
        const int N = P.np[l];
        const bool last = l == L - 1;
        float s_err = 0.0f;
        const int cw = group_cols(N);
        float acc[32];
        tmem_part(tmem + lane_base, cw, h * cw, N, acc);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int c0 = h * cw + 8 * j;
          if (8 * j >= cw || c0 >= N) break;
          float z[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) z[e] = acc[8 * j + e] + sbias[c0 + e];
          if (!last) {
            if constexpr (TRAIN) {
              // GELU'(Z) for the backward pass (the same erf as the activation's)
#pragma unroll
              for (int e = 0; e < 8; ++e)
                zc[(static_cast<long long>(l) * 128 + c0 + e) * 128 + row] = gelu_grad(z[e]);
            }
            float a[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) a[e] = gelu(z[e]);
            put8(aimg, row, c0, a);
          } else if constexpr (!TRAIN) {
            if (valid)
#pragma unroll
              for (int e = 0; e < 8; ++e) {
                const int c = c0 + e;
                if (c < P.outputs) yout[(r0 + row) * P.outputs + c] = z[e] * P.out_sd[c] + P.out_mean[c];
              }
          } else {
            // the loss (mean squared error of the standardised outputs) and dZ of the output
            float g[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int c = c0 + e;
              float d = 0.0f;
              if (valid && c < P.outputs) {
                const float t = (y[src * P.outputs + c] - P.out_mean[c]) / P.out_sd[c];
                d = z[e] - t;
                s_err += d * d;
              }
              g[e] = scale * d;
            }
            colsum_chunk(c0, g);
            put8(aimg, row, c0, g);
          }
        }
        if (!last) {
          if (TRAIN) save_at(l + 1, N);
        } else if constexpr (TRAIN) {
          separt[h * 128 + row] = s_err;
          bias_grad(l, first);  // synchronises first
          if (h == 0 && valid) {
            float t = separt[row];
            for (int g = 1; g < kGroups; ++g) t += separt[g * 128 + row];
            se[r0 + row] = t;
          }
          if (threadIdx.x == 0) bulk_store_read_done();  // dzt free of the last A^T store
          __syncthreads();
          transpose_img(aimg, dzt, N);
        }
      } else {
        // dW_l into the partial
        const bool direct = P.np[l] == 128;
        const int nw = direct ? P.kp[l] : P.np[l];
        float* const pw = part + P.w0[l];
        const int cw = group_cols(nw);
        // in two loads of up to 16 columns (the GELU' values held for the next part bound the
        // registers)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const int cb = h * cw + 16 * half;
          if (16 * half >= cw || cb >= nw) break;
          float wv[16];
          if (cw == 32) {
            tmem_ld16(tmem + lane_base + static_cast<uint32_t>(kWgradCol + cb), wv);
          } else {
            tmem_ld8(tmem + lane_base + static_cast<uint32_t>(kWgradCol + cb), wv);
          }
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int c0 = cb + 8 * j;
            if (16 * half + 8 * j >= cw || c0 >= nw) break;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int o = direct ? row : c0 + e, i = direct ? c0 + e : row;
              if (o < P.out[l] && i < P.in[l]) {
                float* dst = pw + static_cast<long long>(o) * P.in[l] + i;
                *dst = first ? wv[8 * j + e] : *dst + wv[8 * j + e];
              }
            }
          }
        }
        if (l > 0) {
          // dZ_{l-1} = dA_l GELU'(Z_{l-1}), its column sums (bias gradient of layer l - 1)
          constexpr int N = 128;  // = kp[l] = np[l - 1] at width 128
          float da[32];
          tmem_ld32(tmem + lane_base + static_cast<uint32_t>(h * 32), da);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int c0 = h * 32 + 8 * j;
            float g[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) g[e] = da[8 * j + e] * pre[8 * j + e];
            colsum_chunk(c0, g);
            put8(aimg, row, c0, g);
          }
          bias_grad(l - 1, first);  // synchronises first
          transpose_img(aimg, dzt, N);
        }
      }
      tc_before();
      __syncthreads();
      tc_after();
    }
  }
  if (!ok) {
    // a wait ran out: record it, let what is in flight land (bounded), then free the accumulators
    if (threadIdx.x == 0) atomicExch(fault, 1u);
    // (ld_busy is thread 0's record; the other threads' copy only lacks its issues)
    for (int b = 0; b < 2; ++b)
      if ((ld_busy >> b) & 1u) {
        bool done = false;
        for (int it = 0; it < kTcWaitLimit && !done; ++it) done = tc_try_wait(&ld_bar[b], (ld_par >> b) & 1u);
      }
    if (mma_pending) {
      bool done = false;
      for (int it = 0; it < kTcWaitLimit && !done; ++it) done = tc_try_wait(&mma_bar, mma_par);
    }
  }
  if (threadIdx.x == 0) bulk_store_done();
  tc_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
}

// grad[p] = the CTAs' partials summed in CTA order; with ADAM, the Adam step of parameter p
// (as k_adam); with PACK, its BF16 copies into the layer's two operand images (weights only).
// Nothing is written after a fault of the pass (fault word set; null: no pass).
template <bool ADAM, bool PACK>
__global__ void k_fused_update(Layout P, const float* partial, int ctas, long long count,
                               float* grad, float* params, float* m, float* v, float lr, float c1,
                               float c2, const unsigned int* fault) {
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= count) return;
  if (fault != nullptr && *reinterpret_cast<const volatile unsigned int*>(fault) != 0u) return;
  if (partial != nullptr) {
    float s = 0.0f;
    for (int c = 0; c < ctas; ++c) s += partial[static_cast<long long>(c) * count + p];
    grad[p] = s;
    if constexpr (ADAM) {
      m[p] = 0.9f * m[p] + 0.1f * s;
      v[p] = 0.999f * v[p] + 0.001f * s * s;
      const float mh = m[p] / c1, vh = v[p] / c2;
      params[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
    }
  }
  if constexpr (PACK) {
    int l = 0;
    while (l + 1 < P.layers && p >= P.w0[l + 1]) ++l;
    const long long local = p - P.w0[l];
    if (local < static_cast<long long>(P.out[l]) * P.in[l]) {
      const int o = static_cast<int>(local / P.in[l]), i = static_cast<int>(local % P.in[l]);
      const bf16 w = __float2bfloat16(params[p]);
      *reinterpret_cast<bf16*>(reinterpret_cast<unsigned char*>(P.wkw[l]) + kmajor(o, i, P.np[l])) = w;
      *reinterpret_cast<bf16*>(reinterpret_cast<unsigned char*>(P.wtkw[l]) + kmajor(i, o, P.kp[l])) = w;
    }
  }
}

}  // namespace fused
