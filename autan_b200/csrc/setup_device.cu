// The gradient set-up on the GPU (include/autan_b200_setup.h, autan_setup_device_*): the face2
// stencil of every cell and the least-squares weights of the owned cells, with the per-cell rules
// of setup_rules.cuh that the host set-up (setup.cpp) also runs, so the two give the same bits.
//
//   k_face2_count   one thread per cell: its stencil's length (candidates gathered into a
//                   per-thread buffer in local memory, sorted, repeats dropped);
//   k_scan_*        exclusive prefix sum of the lengths into the CSR offsets (per-block sums in
//                   shared memory, one block over the block totals, then the block offsets added);
//   k_face2_fill    one thread per cell: its entries written at its offset;
//   k_lsq_weights   one thread per owned cell: the FP64 normal matrix over the stencil, the
//                   inverse, the weights (a second attempt with every boundary face where the
//                   first fit is singular).
// Set-up work is per cell with no reuse between cells, so plain per-thread loads are used.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "autan_b200_setup.h"
#include "setup_rules.cuh"

namespace autan_b200 {
namespace {

namespace S = setup;

constexpr int kCellBlock = 128;
constexpr int kScanBlock = 1024;

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

// Status words of a set-up: [0] cells whose candidates overflowed the buffer, [1] cells whose
// weights needed every boundary face, [2] cells with no accepted fit.
__global__ void __launch_bounds__(kCellBlock) k_face2_count(S::MeshView m, int64_t* len,
                                                            unsigned long long* status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.n_cells) return;
  int32_t buf[S::kMaxCandidates];
  const int n = S::face2_entries(m, c, buf, S::kMaxCandidates, nullptr);
  if (n < 0) atomicAdd(&status[0], 1ULL);
  len[c] = n < 0 ? 0 : n;
}

__global__ void __launch_bounds__(kCellBlock) k_face2_fill(S::MeshView m, const int64_t* offsets,
                                                           int32_t* entries) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.n_cells) return;
  int32_t buf[S::kMaxCandidates];
  S::face2_entries(m, c, buf, S::kMaxCandidates, entries + offsets[c]);
}

__global__ void __launch_bounds__(kCellBlock) k_lsq_weights(S::MeshView m, const int64_t* offsets,
                                                            const int32_t* entries,
                                                            const uint8_t* bc_kind, double* w,
                                                            int64_t n_stencil,
                                                            unsigned long long* status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.n_owned) return;
  const int r = S::lsq_cell_weights(m, c, offsets, entries, bc_kind, w, n_stencil);
  if (r == 1) atomicAdd(&status[1], 1ULL);
  if (r == 2) atomicAdd(&status[2], 1ULL);
}

// Exclusive scan of v[0..n) into out[0..n] (out[n] the total), three phases.
__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(const int64_t* v, int64_t n, int64_t* out,
                                                            int64_t* block_sum) {
  __shared__ int64_t s[kScanBlock];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanBlock + threadIdx.x;
  s[threadIdx.x] = i < n ? v[i] : 0;
  __syncthreads();
  // Hillis-Steele inclusive scan in shared memory
  for (int off = 1; off < kScanBlock; off <<= 1) {
    const int64_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += add;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v[i];  // exclusive within the block
  if (threadIdx.x == kScanBlock - 1) block_sum[blockIdx.x] = s[threadIdx.x];
}

// One block: the block totals scanned in order, chunk by chunk (exclusive), the grand total last.
__global__ void __launch_bounds__(kScanBlock) k_scan_totals(int64_t* block_sum, int64_t n_blocks,
                                                            int64_t* total) {
  __shared__ int64_t s[kScanBlock];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < n_blocks; base += kScanBlock) {
    const int64_t i = base + threadIdx.x;
    const int64_t x = i < n_blocks ? block_sum[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
      const int64_t add = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
      __syncthreads();
      s[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < n_blocks) block_sum[i] = carry + s[threadIdx.x] - x;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry += s[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int64_t* out, int64_t n, const int64_t* block_sum, const int64_t* total) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_sum[i / kScanBlock];
  if (i == n) out[n] = *total;
}

// Device memory owned by a set-up handle.
struct DeviceBuffer {
  void* p = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() {
    if (p != nullptr) cudaFree(p);
  }
  void alloc(size_t n) {
    if (p != nullptr) cudaFree(p);
    p = nullptr;
    bytes = n;
    check(cudaMalloc(&p, n < 1 ? 1 : n), "cudaMalloc");
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
void upload(DeviceBuffer& b, const T* src, size_t count, cudaStream_t s) {
  b.alloc(count * sizeof(T));
  if (count > 0)
    check(cudaMemcpyAsync(b.p, src, count * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
}

struct Setup {
  int device = 0;
  cudaStream_t stream = nullptr;
  S::MeshView view{};
  DeviceBuffer cfo, cf, owner, neighbour, cc, fc;
  DeviceBuffer len, offsets, entries, block_sum, total, status, kind, weights;
  int64_t n_stencil = 0;
  float ms[3] = {0.f, 0.f, 0.f};  // upload, stencil, weights
  cudaEvent_t ev[4] = {};

  ~Setup() {
    for (auto& e : ev)
      if (e != nullptr) cudaEventDestroy(e);
    if (stream != nullptr) cudaStreamDestroy(stream);
  }

  static unsigned blocks(int64_t n, int b) { return static_cast<unsigned>((n + b - 1) / b); }

  void create(const autan_setup_mesh& m) {
    if (m.n_cells < 1 || m.n_owned_cells < 1 || m.n_owned_cells > m.n_cells ||
        m.n_interior_faces < 0 || m.n_faces < m.n_interior_faces)
      fail("E1101: inconsistent mesh counts");
    if (m.cell_face_offsets == nullptr || m.cell_faces == nullptr || m.owner == nullptr ||
        m.cell_centroid == nullptr || m.face_centroid == nullptr ||
        (m.n_interior_faces > 0 && m.neighbour == nullptr))
      fail("E1101: a required mesh array is NULL");
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto& e : ev) check(cudaEventCreate(&e), "cudaEventCreate");
    const int64_t nc = m.n_cells, nf = m.n_faces;
    const int64_t ninc = m.cell_face_offsets[nc];
    check(cudaEventRecord(ev[0], stream), "event");
    upload(cfo, m.cell_face_offsets, static_cast<size_t>(nc + 1), stream);
    upload(cf, m.cell_faces, static_cast<size_t>(ninc), stream);
    upload(owner, m.owner, static_cast<size_t>(nf), stream);
    upload(neighbour, m.neighbour, static_cast<size_t>(m.n_interior_faces), stream);
    upload(cc, m.cell_centroid, static_cast<size_t>(3 * nc), stream);
    upload(fc, m.face_centroid, static_cast<size_t>(3 * nf), stream);
    view = {m.n_cells, m.n_owned_cells, m.n_faces, m.n_interior_faces, cfo.as<int64_t>(),
            cf.as<int32_t>(), owner.as<int32_t>(), neighbour.as<int32_t>(), cc.as<double>(),
            fc.as<double>()};
    check(cudaEventRecord(ev[1], stream), "event");
    // the stencil: lengths, offsets, entries
    status.alloc(3 * sizeof(unsigned long long));
    check(cudaMemsetAsync(status.p, 0, status.bytes, stream), "memset");
    len.alloc(static_cast<size_t>(nc) * sizeof(int64_t));
    offsets.alloc(static_cast<size_t>(nc + 1) * sizeof(int64_t));
    const int64_t nblocks = (nc + kScanBlock - 1) / kScanBlock;
    block_sum.alloc(static_cast<size_t>(nblocks) * sizeof(int64_t));
    total.alloc(sizeof(int64_t));
    k_face2_count<<<blocks(nc, kCellBlock), kCellBlock, 0, stream>>>(view, len.as<int64_t>(),
                                                                    status.as<unsigned long long>());
    check(cudaGetLastError(), "k_face2_count");
    k_scan_blocks<<<static_cast<unsigned>(nblocks), kScanBlock, 0, stream>>>(
        len.as<int64_t>(), nc, offsets.as<int64_t>(), block_sum.as<int64_t>());
    check(cudaGetLastError(), "k_scan_blocks");
    k_scan_totals<<<1, kScanBlock, 0, stream>>>(block_sum.as<int64_t>(), nblocks, total.as<int64_t>());
    check(cudaGetLastError(), "k_scan_totals");
    k_scan_add<<<blocks(nc + 1, 256), 256, 0, stream>>>(offsets.as<int64_t>(), nc,
                                                        block_sum.as<int64_t>(), total.as<int64_t>());
    check(cudaGetLastError(), "k_scan_add");
    unsigned long long st[3] = {0, 0, 0};
    check(cudaMemcpyAsync(&n_stencil, total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, stream),
          "total");
    check(cudaMemcpyAsync(st, status.p, sizeof(st), cudaMemcpyDeviceToHost, stream), "status");
    check(cudaStreamSynchronize(stream), "stencil lengths");
    if (st[0] != 0) fail("E1102: a cell's face2 stencil has more than 512 candidates");
    entries.alloc(static_cast<size_t>(n_stencil) * sizeof(int32_t));
    k_face2_fill<<<blocks(nc, kCellBlock), kCellBlock, 0, stream>>>(view, offsets.as<int64_t>(),
                                                                   entries.as<int32_t>());
    check(cudaGetLastError(), "k_face2_fill");
    check(cudaEventRecord(ev[2], stream), "event");
    check(cudaStreamSynchronize(stream), "stencil");
    check(cudaEventElapsedTime(&ms[0], ev[0], ev[1]), "event time");
    check(cudaEventElapsedTime(&ms[1], ev[1], ev[2]), "event time");
  }

  int64_t compute_weights(const uint8_t* bc_kind) {
    check(cudaSetDevice(device), "cudaSetDevice");
    const int64_t nb = view.n_faces - view.n_interior;
    upload(kind, bc_kind, static_cast<size_t>(nb), stream);
    weights.alloc(static_cast<size_t>(3 * n_stencil) * sizeof(double));
    check(cudaMemsetAsync(weights.p, 0, weights.bytes, stream), "memset");
    check(cudaMemsetAsync(status.p, 0, status.bytes, stream), "memset");
    check(cudaEventRecord(ev[2], stream), "event");
    k_lsq_weights<<<blocks(view.n_owned, kCellBlock), kCellBlock, 0, stream>>>(
        view, offsets.as<int64_t>(), entries.as<int32_t>(), kind.as<uint8_t>(),
        weights.as<double>(), n_stencil, status.as<unsigned long long>());
    check(cudaGetLastError(), "k_lsq_weights");
    check(cudaEventRecord(ev[3], stream), "event");
    unsigned long long st[3] = {0, 0, 0};
    check(cudaMemcpyAsync(st, status.p, sizeof(st), cudaMemcpyDeviceToHost, stream), "status");
    check(cudaStreamSynchronize(stream), "weights");
    check(cudaEventElapsedTime(&ms[2], ev[2], ev[3]), "event time");
    return static_cast<int64_t>(st[1]);
  }

  void download(int64_t* off, int32_t* ent, double* w) {
    check(cudaSetDevice(device), "cudaSetDevice");
    const int64_t nc = view.n_cells;
    if (off != nullptr)
      check(cudaMemcpyAsync(off, offsets.p, static_cast<size_t>(nc + 1) * sizeof(int64_t),
                            cudaMemcpyDeviceToHost, stream), "download");
    if (ent != nullptr && n_stencil > 0)
      check(cudaMemcpyAsync(ent, entries.p, static_cast<size_t>(n_stencil) * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, stream), "download");
    if (w != nullptr) {
      if (weights.p == nullptr) fail("E1101: no weights computed");
      check(cudaMemcpyAsync(w, weights.p, static_cast<size_t>(3 * n_stencil) * sizeof(double),
                            cudaMemcpyDeviceToHost, stream), "download");
    }
    check(cudaStreamSynchronize(stream), "download");
  }
};

int fail_to(char* err, size_t len, const std::string& what) {
  if (err != nullptr && len > 0) {
    std::strncpy(err, what.c_str(), len - 1);
    err[len - 1] = '\0';
  }
  return 1;
}

template <class F>
int guarded(char* err, size_t len, F&& body) {
  try {
    body();
    return 0;
  } catch (const std::exception& e) {
    return fail_to(err, len, e.what());
  } catch (...) {
    return fail_to(err, len, "E1300: unknown failure");
  }
}

}  // namespace
}  // namespace autan_b200

using autan_b200::Setup;

extern "C" {

int autan_setup_device_create(const struct autan_setup_mesh* mesh, int32_t device, void** handle,
                              int64_t* n_stencil, char* err, size_t err_len) {
  return autan_b200::guarded(err, err_len, [&]() {
    if (mesh == nullptr || handle == nullptr) throw autan_b200::Failure("E1101: null argument");
    auto s = std::make_unique<Setup>();
    s->device = device;
    s->create(*mesh);
    if (n_stencil != nullptr) *n_stencil = s->n_stencil;
    *handle = s.release();
  });
}

int autan_setup_device_weights(void* handle, const uint8_t* bc_kind, int64_t* retried, char* err,
                               size_t err_len) {
  return autan_b200::guarded(err, err_len, [&]() {
    if (handle == nullptr || bc_kind == nullptr) throw autan_b200::Failure("E1101: null argument");
    const int64_t r = static_cast<Setup*>(handle)->compute_weights(bc_kind);
    if (retried != nullptr) *retried = r;
  });
}

int autan_setup_device_download(void* handle, int64_t* stencil_offsets, int32_t* stencil,
                                double* weights, char* err, size_t err_len) {
  return autan_b200::guarded(err, err_len, [&]() {
    if (handle == nullptr) throw autan_b200::Failure("E1101: null handle");
    static_cast<Setup*>(handle)->download(stencil_offsets, stencil, weights);
  });
}

void autan_setup_device_times(void* handle, double* ms) {
  const auto* s = static_cast<const Setup*>(handle);
  for (int k = 0; k < 3; ++k) ms[k] = s->ms[k];
}

void autan_setup_device_free(void* handle) { delete static_cast<Setup*>(handle); }

}  // extern "C"
