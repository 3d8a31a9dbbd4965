// The explicit Euler residual-and-update path on B200 (sm_100a), behind the C ABI of
// include/autan_euler_device.h.
//
// Data layout in HBM (owned cells only: a periodic image reads its owned cell's values, so the
// reference's three ghost fills per residual disappear):
//   cell records     one 32-element record per cell (128 B in fp32+acc64): primitives W at words
//                    0-4, limiter phi at 8-12, gradient grad W at 13-27 (row-major 5 x 3): a
//                    neighbour's whole reconstruction data is one cache line, read with 16-byte
//                    vector loads; three record buffers rotate through the RK stages;
//   FP64 SoA         u (conserved), RK stage, RK4 accumulator, residual, volume (streamed);
//   stencil          face2 entries, each {w_x, w_y, w_z, cell or n + b} in 16 B (fp32), in a
//                    sliced ELLPACK layout (32 cells per slice, entry j of cell c at
//                    start[c / 32] + 32 j + c % 32): a warp reads entry j of its cells as 512
//                    contiguous bytes;
//   incidences       each cell's faces in increasing face index (the reference's scatter order),
//                    sliced the same way, coded 2 f + side (interior) or -(b + 1) (boundary);
//   face records     per interior face {n, A, rel(x_f, x_l), l, rel(x_f, x_r), r} (48 B), per
//                    boundary face {n, A, rel(x_f, x_o), kind, data, owner} (64 B): the `rel`
//                    offsets already in the compute type, as the bodies' rel() computes them;
//                    moments (warped faces only) apart.
//
// Kernels per RK stage:
//   k_boundary_states  prim_b of every boundary face;
//   k_gradients        per cell: LSQ gradient over the stencil (FP64 sums), bounds, then the
//                      Venkatakrishnan limiter over the cell's faces (wmin/wmax never stored); at
//                      stage 0 also the spectral radius, the CFL step and its block minimum;
//   k_faces            per cell: every face flux of the cell recomputed (gather-recompute: no float
//                      atomics, no face scratch), summed in face order from the source term, then
//                      the RK stage update in FP64 and the next stage's primitives.
// Per step: the exact-sum residual norms of stage 0. A step is captured in one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "autan_euler_device.h"
#include "euler_bodies.cuh"
#include "convergence.hpp"
#include "exact_sum.cuh"

namespace autan_b200 {

struct Fp64 {
  using C = double;  // compute, and storage of states, gradients and geometry values
  using V = double2; // 16-byte vector of C
  static constexpr int kVec = 2;
};
struct Fp32Acc64 {
  using C = float;
  using V = float4;
  static constexpr int kVec = 4;
};

constexpr int kSlice = 32;
constexpr int kHistory = 4096;
constexpr int kBlock = 256;
constexpr int kPrimW = 8;   // primitive record width: rho, u, v, w, p, then padding
constexpr int kGroup = 8;   // words per cell in each group of the reconstruction array
constexpr int kRecon = 24;  // reconstruction words per cell: phi 0-4, grad 5-19, padding 20-23
constexpr int kFace = 12;   // interior face record width
constexpr int kBface = 16;  // boundary face record width
constexpr int kPrimB = 8;   // boundary state record width
static_assert(kPrimB == kPrimW, "boundary states share the primitive buffers' record index (n + b)");

// Step control in device memory: written by the kernels, read by the host after a batch.
struct Control {
  unsigned long long dt_bits;    // atomicMin of the local steps' bits (positive doubles)
  unsigned long long bad_state;  // least cell with an invalid state (~0: none)
  unsigned long long bad_res;    // least cell with a non-finite residual
  long long step;                // steps taken since the last reset
  double dt;                     // the global step of the current step
  unsigned long long fault;      // a bounded device wait timed out
  // Nonzero once a primitive record written since the last state upload holds a value that is not
  // finite or whose magnitude reaches 2^60 (sticky until the next upload): the gradient kernels'
  // scaled integer-pipe widening is exact only below that bound and falls back to cvt above it.
  unsigned long long special;
  double rms[5];
  unsigned long long words[5][kWords];
  double hist_rms[kHistory][5];
  double hist_dt[kHistory];
};
// The part of Control a step's result needs (read back after every step call).
constexpr size_t kControlHead = offsetof(Control, words);

template <class P>
struct Dev {
  using C = typename P::C;
  int n;     // owned cells
  int nb;    // boundary faces
  int n_if;  // owned interior faces
  Params<C> p;
  double ref[5];
  const C* prim;      // kPrimW x n: the primitives this stage reads, then its boundary states
  C* prim_next;       // the primitives this stage writes
  C* recon;           // phi and grad of this stage: kRecon / kGroup groups of kGroup x n words
  long long rstride;  // words from one group to the next (kGroup x n)
  C* prim_b;       // kPrimB x nb: this stage's boundary states (prim's buffer after n records)
  double* u;
  double* stage;
  double* racc;
  double* res;
  const double* volume;
  double* dt_local;
  const C* source;  // 5 x n, or null
  const int* st_start;
  const int* st_len;
  const C* st;      // 4 per entry, sliced
  const int* inc_start;
  const int* inc_len;
  const int* inc_code;
  const C* inc_rec;  // 4 per incidence, sliced: rel(x_f, x_c) of the cell's side, the other side
                     // (its cell's value index, or n + b for boundary face b: the primitive
                     // buffers hold the boundary states after the cells)
  const C* inc_dt;   // 4 per incidence, sliced: the face's unit normal and area
  int n_slices;
  const C* face;    // kFace per owned interior face
  const C* bface;   // kBface per boundary face
  const C* f_m;     // 9 x n_if, warped meshes only
  const C* b_m;     // 9 x nb
  Control* ctl;
  // Batched cases (null without): the case of each owned cell and whether each case still steps.
  const int* case_of;
  const unsigned char* active;
  // Per 32 consecutive owned interior (boundary) faces: the case of all their owners, or -1 when
  // they span two cases; a warp of a stopped case leaves before reading its face records.
  const int* face_warp_case;
  const int* bface_warp_case;
  // Per case, the AUSM+-up cut-off Mach number (each case's own freestream Mach), or null for the
  // scheme's one value.
  const typename P::C* case_minf;
  // 1 when every LSQ weight is finite and below 2^40 in magnitude (checked at create): with
  // Control::special clear, the gradient sums may then be widened on the integer pipe.
  int wide_ok;
  // Re-packed launches of batched cases (null: the launch covers every item): the warp tiles
  // (32 consecutive cells, owned interior faces or owned boundary faces) that hold an item of a
  // case still stepping; a launch's warp w takes tile w.
  const int* cell_tiles;
  const int* face_tiles;
  const int* bface_tiles;
  int n_cell_tiles, n_face_tiles, n_bface_tiles;
  // Test hook of the failure detection (0 in normal use): with n > 0 every warp of the mode-5
  // gradient kernel also waits, n polls at most, on an mbarrier that nothing arrives on, so that
  // the bounded wait runs out and takes the timeout path (fault word, no stores).
  int stall_polls;
};

// Whether owned cell c takes part (its case has not stopped).
template <class P>
__device__ __forceinline__ bool cell_active(const Dev<P>& d, int c) {
  return d.active == nullptr || d.active[d.case_of[c]] != 0;
}

// Whether this block's cells (blockDim.x consecutive owned cells) all belong to one stopped case:
// the block then leaves before prefetching or staging its stencil rows. Uniform over the block.
template <class P>
__device__ __forceinline__ bool block_idle(const Dev<P>& d) {
  if (d.active == nullptr) return false;
  const long long c0 = static_cast<long long>(blockIdx.x) * blockDim.x;
  if (c0 >= d.n) return true;
  const long long c1 = min(c0 + static_cast<long long>(blockDim.x), static_cast<long long>(d.n)) - 1;
  const int k0 = d.case_of[c0];
  return k0 == d.case_of[c1] && d.active[k0] == 0;
}

// The item (cell or face) of this thread: blockIdx.x * blockDim.x + threadIdx.x, or, with a tile
// list, item lane of the list's tile for this thread's warp; -1 past the list's end.
__device__ __forceinline__ int tile_item(const int* tiles, int n_tiles) {
  if (tiles == nullptr) return blockIdx.x * blockDim.x + threadIdx.x;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  return w < n_tiles ? (__ldg(tiles + w) << 5) + static_cast<int>(threadIdx.x & 31) : -1;
}

__device__ __forceinline__ int index_of(float x) { return __float_as_int(x); }
__device__ __forceinline__ int index_of(double x) {
  return static_cast<int>(__double_as_longlong(x));
}

// Interior face records start on 32-byte boundaries in FP64 (96 bytes) but not in fp32 (48).
template <class P>
constexpr bool kFaceA32 = (kFace * sizeof(typename P::C)) % 32 == 0;

// 32-byte vector loads and stores (the 256-bit ld / st of sm_100): one L1 wavefront per lane
// where two 16-byte vectors take two. The address must be 32-byte aligned.
__device__ __forceinline__ void ld32(const float* p, float* o) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]), "=f"(o[6]),
        "=f"(o[7])
      : "l"(p));
}
__device__ __forceinline__ void ld32(const double* p, double* o) {
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3])
      : "l"(p));
}
// L2 eviction priority (createpolicy): data a launch reads once marked first out, so that it does
// not push the records many threads read out of L2.
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// 16 bytes read once: not allocated in L1, under L2 policy `pol`.
__device__ __forceinline__ float4 ld16_once(const float* p, unsigned long long pol) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ void st32(float* p, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]),
               "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}
__device__ __forceinline__ void st32(double* p, const double* v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]),
               "d"(v[3])
               : "memory");
}

// Vector loads of a record's words [w, w + count), count a multiple of the 16-byte vector width:
// with A32 (base + w 32-byte aligned) 32-byte vectors first, then 16-byte ones.
template <class P, bool A32 = false>
__device__ __forceinline__ void load_words(const typename P::C* base, int w, int count,
                                           typename P::C* out) {
  using V = typename P::V;
  constexpr int kW32 = 32 / static_cast<int>(sizeof(typename P::C));
  if constexpr (A32) {
#pragma unroll
    for (int q = 0; q < count / kW32; ++q) ld32(base + w + kW32 * q, out + kW32 * q);
    const int done = (count / kW32) * kW32;
    base += done;
    out += done;
    count -= done;
  }
  const V* v = reinterpret_cast<const V*>(base + w);
#pragma unroll
  for (int q = 0; q < count / P::kVec; ++q) {
    const V x = __ldg(v + q);
    if constexpr (P::kVec == 4) {
      out[4 * q] = x.x;
      out[4 * q + 1] = x.y;
      out[4 * q + 2] = x.z;
      out[4 * q + 3] = x.w;
    } else {
      out[2 * q] = x.x;
      out[2 * q + 1] = x.y;
    }
  }
}

template <class P, bool A32 = false>
__device__ __forceinline__ void store_words(typename P::C* base, int w, int count,
                                            const typename P::C* in) {
  using V = typename P::V;
  constexpr int kW32 = 32 / static_cast<int>(sizeof(typename P::C));
  if constexpr (A32) {
#pragma unroll
    for (int q = 0; q < count / kW32; ++q) st32(base + w + kW32 * q, in + kW32 * q);
    const int done = (count / kW32) * kW32;
    base += done;
    in += done;
    count -= done;
  }
  V* v = reinterpret_cast<V*>(base + w);
#pragma unroll
  for (int q = 0; q < count / P::kVec; ++q) {
    V x;
    if constexpr (P::kVec == 4) {
      x.x = in[4 * q];
      x.y = in[4 * q + 1];
      x.z = in[4 * q + 2];
      x.w = in[4 * q + 3];
    } else {
      x.x = in[2 * q];
      x.y = in[2 * q + 1];
    }
    v[q] = x;
  }
}

// The primitives of cell c (words 0-4 of its primitive record).
template <class P>
__device__ __forceinline__ void load_prim(const typename P::C* prim, int c, typename P::C* w) {
  typename P::C t[8];
  load_words<P, true>(prim + static_cast<long long>(c) * kPrimW, 0, 8, t);
#pragma unroll
  for (int k = 0; k < 5; ++k) w[k] = t[k];
}

// Primitives, limiter and gradient of cell c: its primitive record and its word group of each of
// the reconstruction array's groups (cell-contiguous within a group, so that the records of
// consecutive cells share cache lines).
template <class P>
__device__ __forceinline__ void load_recon(const Dev<P>& d, int c, typename P::C* w,
                                           typename P::C* phi, typename P::C* g) {
  typename P::C t[kRecon], q[8];
  load_words<P, true>(d.prim + static_cast<long long>(c) * kPrimW, 0, 8, q);
#pragma unroll
  for (int k = 0; k < kRecon / kGroup; ++k)
    load_words<P, true>(d.recon + k * d.rstride + static_cast<long long>(c) * kGroup, 0, kGroup,
                        t + kGroup * k);
#pragma unroll
  for (int k = 0; k < 5; ++k) w[k] = q[k];
#pragma unroll
  for (int k = 0; k < 5; ++k) phi[k] = t[k];
#pragma unroll
  for (int k = 0; k < 15; ++k) g[k] = t[5 + k];
}

// Writes phi (out[0-4]) and grad (out[5-19]) of cell c; out[20-23] are the padding.
template <class P>
__device__ __forceinline__ void store_recon(const Dev<P>& d, int c, const typename P::C* out) {
#pragma unroll
  for (int k = 0; k < kRecon / kGroup; ++k)
    store_words<P, true>(d.recon + k * d.rstride + static_cast<long long>(c) * kGroup, 0, kGroup,
                         out + kGroup * k);
}

// Whether a primitive value is one the scaled widening of the gradient sums cannot take exactly
// (not finite, or of magnitude 2^60 or more); recorded in Control::special by every writer of
// primitive records.
__device__ __forceinline__ bool special_value(float x) { return !(fabsf(x) < 0x1p60f); }
__device__ __forceinline__ bool special_value(double x) { return !(fabs(x) < 0x1p60); }

template <class C>
__device__ __forceinline__ void note_special(const C* w, Control* ctl) {
  bool s = false;
#pragma unroll
  for (int k = 0; k < 5; ++k) s = s || special_value(w[k]);
  if (s && ctl != nullptr) atomicOr(&ctl->special, 1ULL);
}

// Writes the primitives of cell c (words 0-7, the padding 5-7 zero).
template <class P>
__device__ __forceinline__ void store_prim(typename P::C* prim, int c, const typename P::C* w,
                                           Control* ctl) {
  using C = typename P::C;
  const C t[8] = {w[0], w[1], w[2], w[3], w[4], C(0), C(0), C(0)};
  store_words<P, true>(prim + static_cast<long long>(c) * kPrimW, 0, 8, t);
  note_special(w, ctl);
}

// Euler<P>::state then to_primitive: W of the stored state S(u - U_ref) (euler.cpp:925-932,
// kernels/euler.py:94-104, 433).
template <class P>
__device__ __forceinline__ void prim_of_state(const Dev<P>& d, const double* u, typename P::C* w,
                                              typename P::C* dq) {
  using C = typename P::C;
#pragma unroll
  for (int k = 0; k < 5; ++k) dq[k] = static_cast<C>(u[k] - d.ref[k]);
  to_primitive(dq, d.p, w);
}

// CudaStepper::invalid (device_stepper.cuh:107-164): cell c's state as the kernels read it (dq
// the gauge difference State(u - U_ref) in the compute type: density and pressure finite and
// positive), then its residual (finite); the least such cells go to Control::bad_state and
// bad_res.
template <class P>
__device__ __forceinline__ void mark_invalid(const Dev<P>& d, int c, const typename P::C* dq,
                                             const double* res) {
  using C = typename P::C;
  const C g = d.p.g;
  const C r0 = static_cast<C>(d.ref[0]);
  const C rho = r0 + dq[0];
  C dm_m = C(0), mr_mr = C(0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const C mr = static_cast<C>(d.ref[k + 1]);
    dm_m = dm_m + dq[k + 1] * (C(2) * mr + dq[k + 1]);
    mr_mr = mr_mr + mr * mr;
  }
  const C dk = (dm_m * r0 - mr_mr * dq[0]) / (rho * r0);
  const C pr = (g - C(1)) * (dq[4] - C(0.5) * dk) + d.p.pref;
  const bool bad = !isfinite(static_cast<double>(rho)) || !isfinite(static_cast<double>(pr)) ||
                   !(rho > C(0)) || !(pr > C(0));
  if (bad) atomicMin(&d.ctl->bad_state, static_cast<unsigned long long>(c));
  bool badr = false;
#pragma unroll
  for (int k = 0; k < 5; ++k) badr = badr || !isfinite(res[k]);
  if (badr) atomicMin(&d.ctl->bad_res, static_cast<unsigned long long>(c));
}

// ---------------------------------------------------------------- kernels

// The divergence marks of the device state u and the residual res (FP64 SoA) for evaluate().
template <class P>
__global__ void __launch_bounds__(kBlock) k_invalid(Dev<P> d, const double* u, const double* res) {
  using C = typename P::C;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  C dq[5];
  double r[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const long long i = static_cast<long long>(k) * d.n + c;
    dq[k] = static_cast<C>(u[i] - d.ref[k]);
    r[k] = res[i];
  }
  mark_invalid(d, c, dq, r);
}

// The primitives of a host state (upload, residual): records of u.
template <class P>
__global__ void __launch_bounds__(kBlock) k_store(Dev<P> d, const double* u, typename P::C* rec) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.n) return;
  double uc[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) uc[k] = u[static_cast<long long>(k) * d.n + c];
  typename P::C w[5], dq[5];
  prim_of_state(d, uc, w, dq);
  store_prim<P>(rec, c, w, d.ctl);
}

// boundary_states (kernels/euler.py:455-466): prim_b of boundary face b.
template <class P>
__device__ __forceinline__ void boundary_state(const Dev<P>& d, int b) {
  using C = typename P::C;
  C r[kBface], w[5], out[8];
  load_words<P, true>(d.bface + static_cast<long long>(b) * kBface, 0, kBface, r);
  load_prim<P>(d.prim, index_of(r[13]), w);
  boundary_value(w, r[7], r + 8, r, d.p, out);
  out[5] = out[6] = out[7] = C(0);
  store_words<P, true>(d.prim_b + static_cast<long long>(b) * kPrimB, 0, 8, out);
  note_special(out, d.ctl);
}

// ... of every boundary face.
template <class P>
__global__ void __launch_bounds__(kBlock) k_boundary_states(Dev<P> d) {
  const int b = tile_item(d.bface_tiles, d.n_bface_tiles);
  if (b < 0 || b >= d.nb) return;
  boundary_state(d, b);
}

// The minimum over a block of positive doubles' bits, then one atomicMin. Every thread of the
// block calls it.
__device__ __forceinline__ void block_min_dt(double dt, bool valid, unsigned long long* target) {
  __shared__ unsigned long long warp_min[kBlock / 32];
  unsigned long long b = valid && dt > 0.0 ? static_cast<unsigned long long>(__double_as_longlong(dt))
                                           : ~0ULL;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, b, off);
    b = o < b ? o : b;
  }
  if ((threadIdx.x & 31) == 0) warp_min[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = warp_min[0];
    for (int i = 1; i < static_cast<int>(blockDim.x >> 5); ++i) m = warp_min[i] < m ? warp_min[i] : m;
    if (m != ~0ULL) atomicMin(target, m);
  }
}

// spectral_radius (kernels/euler.py:1103-1112) and the cell's CFL step (device_stepper.cuh:84-89):
// lambda_c = sum over its faces of max(|v . n| + c) A (FP64 sum, stored as State), dt_c = (cfl V)
// / lambda_c.
template <class P>
__device__ __forceinline__ double cell_time_step(const Dev<P>& d, int c, const typename P::C* wc,
                                                 double cfl) {
  using C = typename P::C;
  double acc = 0.0;
  const int ib = __ldg(d.inc_start + (c >> 5)) + (c & 31);
  const int il = __ldg(d.inc_len + c);
  for (int j = 0; j < il; ++j) {
    const int code = __ldg(d.inc_code + ib + static_cast<long long>(j) * kSlice);
    C wn[5], rec[kFace];
    if (code >= 0) {
      const int f = code >> 1;
      load_words<P, kFaceA32<P>>(d.face + static_cast<long long>(f) * kFace, 0, kFace, rec);
      const int o = (code & 1) ? index_of(rec[7]) : index_of(rec[11]);
      load_prim<P>(d.prim, o, wn);
    } else {
      const int b = -code - 1;
      load_words<P>(d.bface + static_cast<long long>(b) * kBface, 0, 4, rec);
      C t[8];
      load_words<P, true>(d.prim_b + static_cast<long long>(b) * kPrimB, 0, 8, t);
#pragma unroll
      for (int k = 0; k < 5; ++k) wn[k] = t[k];
    }
    acc += static_cast<double>(wave_speed(wc, wn, rec, rec[3], d.p.g, d.p.pref));
  }
  const double lam = static_cast<double>(static_cast<C>(acc));
  return cfl * d.volume[c] / lam;
}

// The primitives of a cell (words 0-4), of a boundary face's state or of a face's flux, five
// values only; src is 32-byte aligned (record, prim_b and flux strides are multiples of 32 bytes).
template <class P>
__device__ __forceinline__ void load5(const typename P::C* src, typename P::C* w) {
  if constexpr (P::kVec == 4) {
    float t[8];
    ld32(src, t);
#pragma unroll
    for (int k = 0; k < 5; ++k) w[k] = t[k];
  } else {
    double t[4];
    ld32(src, t);
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = t[k];
    w[4] = __ldg(src + 4);
  }
}

// The stencil bounds (min and max over the stencil values, kernels/euler.py:510-521) with the
// hardware min/max. They can differ from the keep-the-first rule only in the sign of a zero bound
// (a NaN value is passed over by both), and the limiter uses a bound only as dp = bound - w_c:
// when the sign differs dp is zero, and venkat adds dp only as dp * dp (+0) or as a zero product
// to a sum of eps2 > 0 and d^2 terms, so phi has the same bits either way.
__device__ __forceinline__ float bound_min(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float bound_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double bound_min(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double bound_max(double a, double b) { return fmax(a, b); }

// Fire-and-forget TMA prefetch of a contiguous range into L2 (cp.async.bulk.prefetch.L2, no shared
// memory, no completion to wait for): ptr 16-byte aligned, bytes a multiple of 16, issued in
// pieces of at most 32 KB.
__device__ __forceinline__ void prefetch_l2(const void* ptr, long long bytes) {
  const char* p = static_cast<const char*>(ptr);
  for (long long off = 0; off < bytes; off += 32768) {
    const long long left = bytes - off;
    const unsigned n = static_cast<unsigned>(left < 32768 ? left : 32768);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p + off), "r"(n) : "memory");
  }
}

// The block's stencil rows and incidence records (contiguous in the sliced layout) to L2; with a
// tile list, each warp's own slice (call from one lane of each warp, c its cell or -1).
template <class P, bool LIMIT, bool DT>
__device__ __forceinline__ void prefetch_tile_rows(const Dev<P>& d, int c) {
  using C = typename P::C;
  if (c < 0) return;
  const int s0 = c >> 5;
  if (s0 >= d.n_slices) return;
  const long long e0 = __ldg(d.st_start + s0), e1 = __ldg(d.st_start + s0 + 1);
  const long long i0 = __ldg(d.inc_start + s0), i1 = __ldg(d.inc_start + s0 + 1);
  prefetch_l2(d.st + 4 * e0, (e1 - e0) * 4 * static_cast<long long>(sizeof(C)));
  if (LIMIT || DT) prefetch_l2(d.inc_rec + 4 * i0, (i1 - i0) * 4 * static_cast<long long>(sizeof(C)));
  if (DT) prefetch_l2(d.inc_dt + 4 * i0, (i1 - i0) * 4 * static_cast<long long>(sizeof(C)));
}


template <class P, bool LIMIT, bool DT>
__device__ __forceinline__ void prefetch_block_rows(const Dev<P>& d) {
  using C = typename P::C;
  const int s0 = static_cast<int>((static_cast<long long>(blockIdx.x) * blockDim.x) >> 5);
  const int s1 = min(s0 + static_cast<int>(blockDim.x >> 5), d.n_slices);
  if (s0 < s1) {
    const long long e0 = __ldg(d.st_start + s0), e1 = __ldg(d.st_start + s1);
    const long long i0 = __ldg(d.inc_start + s0), i1 = __ldg(d.inc_start + s1);
    prefetch_l2(d.st + 4 * e0, (e1 - e0) * 4 * static_cast<long long>(sizeof(C)));
    if (LIMIT || DT) prefetch_l2(d.inc_rec + 4 * i0, (i1 - i0) * 4 * static_cast<long long>(sizeof(C)));
    if (DT) prefetch_l2(d.inc_dt + 4 * i0, (i1 - i0) * 4 * static_cast<long long>(sizeof(C)));
  }
}

// Prefetch of a gradient block's rows: the block's slices, or (TILES) each warp's tile's.
template <class P, bool LIMIT, bool DT, bool TILES = false>
__device__ __forceinline__ void prefetch_rows(const Dev<P>& d, int c) {
  if constexpr (!TILES) {
    if (threadIdx.x == 0) prefetch_block_rows<P, LIMIT, DT>(d);
  } else {
    if ((threadIdx.x & 31) == 0) prefetch_tile_rows<P, LIMIT, DT>(d, c);
  }
}

// The owned cell of this thread in a gradient launch: the launch index, or (TILES, re-packed
// batched launches) the warp's tile's cell. The gradient kernels other than k_gradients_tiles
// never run over tiles; their cell index then stays a function of the launch index, which the
// compiler recomputes instead of holding it in a register through the stencil loop.
template <bool TILES, class P>
__device__ __forceinline__ int gradient_cell(const Dev<P>& d) {
  if constexpr (TILES) {
    return tile_item(d.cell_tiles, d.n_cell_tiles);
  } else {
    return static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
  }
}

// The end of a cell's gradient loop (kernels/euler.py:517-521, :563-608, :1103-1112): the FP64
// sums rounded to the gradient, the bounds with the cell's own value, then one pass over the
// cell's incidences for the limiter and, with DT, the spectral radius and the cell's CFL step
// (returned; 0 without DT); the reconstruction record stored.
template <class P, bool LIMIT, bool DT, bool S = false>
__device__ __forceinline__ double gradient_tail(const Dev<P>& d, int c, const typename P::C* wc,
                                                const double* acc, typename P::C* lo,
                                                typename P::C* hi, double cfl, int local) {
  using C = typename P::C;
  static_assert(!S || sizeof(C) == 4, "streamed loads of the fp32+acc64 records only");
  unsigned long long pol_first = 0;
  if constexpr (S) pol_first = l2_evict_first();
  // include_own_value (:517-521); out: phi, then grad, then padding.
  C out[kRecon];
#pragma unroll
  for (int k = 0; k < 15; ++k) out[5 + k] = static_cast<C>(acc[k]);
  const C* g = out + 5;
  // phi, and the limiter's per-cell arguments (the same in every face's venkat call): the
  // bounds' distances from the cell value and eps^2.
  C phi[5], dmax[5], dmin[5], eps2[5];
  if constexpr (LIMIT) {
    const C vol = static_cast<C>(__ldg(d.volume + c));
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      dmax[i] = maxv(hi[i], wc[i]) - wc[i];
      dmin[i] = minv(lo[i], wc[i]) - wc[i];
      eps2[i] = d.p.scale[i] * vol;
      phi[i] = C(INFINITY);
    }
  }
  // One pass over the cell's incidences for both the limiter (its record: rel(x_f, x_c) of this
  // side) and, with DT, spectral_radius (:1103-1112: the other side's state, the face's normal
  // and area), each in incidence order.
  double lam = 0.0;
  if constexpr (LIMIT || DT) {
    const long long ib = __ldg(d.inc_start + (c >> 5)) + (c & 31);
    const int il = __ldg(d.inc_len + c);
    for (int j = 0; j < il; ++j) {
      const long long at = 4 * (ib + static_cast<long long>(j) * kSlice);
      C r[4];
      if constexpr (S) {
        const float4 v = ld16_once(d.inc_rec + at, pol_first);
        r[0] = v.x, r[1] = v.y, r[2] = v.z, r[3] = v.w;
      } else {
        load_words<P, sizeof(C) == 8>(d.inc_rec + at, 0, 4, r);
      }
      C nd[4], wn[5];
      if constexpr (DT) {
        if constexpr (S) {
          const float4 v = ld16_once(d.inc_dt + at, pol_first);
          nd[0] = v.x, nd[1] = v.y, nd[2] = v.z, nd[3] = v.w;
        } else {
          load_words<P, sizeof(C) == 8>(d.inc_dt + at, 0, 4, nd);
        }
        const int o = index_of(r[3]);
        load5<P>(d.prim + static_cast<long long>(o) * kPrimW, wn);
      }
      if constexpr (LIMIT) {
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          const C dd = g[3 * i] * r[0] + g[3 * i + 1] * r[1] + g[3 * i + 2] * r[2];
          // venkat's value is >= 0 and never -0 (its numerator adds 2 d dp, >= 0, to
          // dp^2 + eps2 >= +0), or NaN: the hardware min is then the keep-the-first min
          phi[i] = bound_min(phi[i], venkat(dd, dmax[i], dmin[i], eps2[i]));
        }
      }
      if constexpr (DT) lam += static_cast<double>(wave_speed(wc, wn, nd, nd[3], d.p.g, d.p.pref));
    }
  }
  if constexpr (LIMIT) {
    // at_most_one (:591-593)
#pragma unroll
    for (int i = 0; i < 5; ++i) out[i] = minv(phi[i], C(1.0));
  } else {
    // Second order without limiter: phi = 1 (physics/src/euler.cpp:195).
#pragma unroll
    for (int i = 0; i < 5; ++i) out[i] = C(1.0);
  }
#pragma unroll
  for (int k = 20; k < kRecon; ++k) out[k] = C(0);
  store_recon<P>(d, c, out);
  if constexpr (DT) {
    // The cell's CFL step (device_stepper.cuh:84-89).
    const double dt = cfl * d.volume[c] / static_cast<double>(static_cast<C>(lam));
    if (local) d.dt_local[c] = dt;
    return dt;
  }
  return 0.0;
}

// gradients (kernels/euler.py:540-549) then limiter (:596-608), one thread per owned cell: the LSQ
// gradient over the face2 stencil with FP64 sums, the bounds over the stencil and the cell, then
// phi_k = min(1, min over the cell's faces of venkat(grad W . rel(x_f, x_c), ...)); the entries
// are read CHUNK at a time (their loads, then the neighbours' loads, all in flight together) and
// added in stencil order. With DT, also the cell's CFL step and the block's minimum.
// S (fp32+acc64): the stencil rows and incidence records, each read once, streamed: not allocated
// in L1 and first out of L2 (createpolicy evict_first), so that they do not push the neighbours'
// records, each read by about 20 cells, out of the caches. The 8 M-cell channel's gradient
// launches: 4.07 -> 3.93 ms per step; marking the neighbours' records evict_last as well measured
// slower (4.05 ms).
template <class P, bool LIMIT, bool DT, int CHUNK, bool S = false>
__device__ __forceinline__ double gradient_cell_body(const Dev<P>& d, int c, double cfl, int local);

template <class P, bool LIMIT, bool DT, int CHUNK, bool TILES = false, bool S = false>
__device__ __forceinline__ void gradients_cells(const Dev<P>& d, double cfl, int local) {
  if (!TILES && block_idle(d)) return;
  const int c = gradient_cell<TILES>(d);
  const bool live = c >= 0 && c < d.n && cell_active(d, c);
  double dt = 0.0;
  prefetch_rows<P, LIMIT, DT, TILES>(d, c);
  if (live) dt = gradient_cell_body<P, LIMIT, DT, CHUNK, S>(d, c, cfl, local);
  if constexpr (DT) block_min_dt(dt, live, &d.ctl->dt_bits);
}

// One owned cell's gradient, bounds and limiter (and, with DT, its CFL step, returned).
template <class P, bool LIMIT, bool DT, int CHUNK, bool S>
__device__ __forceinline__ double gradient_cell_body(const Dev<P>& d, int c, double cfl, int local) {
  using C = typename P::C;
  static_assert(!S || sizeof(C) == 4, "streamed loads of the fp32+acc64 records only");
  unsigned long long pol_first = 0;
  if constexpr (S) pol_first = l2_evict_first();
  {
    C wc[5];
    load5<P>(d.prim + static_cast<long long>(c) * kPrimW, wc);
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    C lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      lo[k] = C(INFINITY);
      hi[k] = -C(INFINITY);
    }
    const int base = __ldg(d.st_start + (c >> 5)) + (c & 31);
    const int len = __ldg(d.st_len + c);
    // One stencil entry {w, index} and its value wn, added in stencil order.
    auto add_entry = [&](const C* e, const C* wn) {
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const C dw = wn[i] - wc[i];
        acc[3 * i] += static_cast<double>(dw * e[0]);
        acc[3 * i + 1] += static_cast<double>(dw * e[1]);
        acc[3 * i + 2] += static_cast<double>(dw * e[2]);
      }
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        lo[i] = bound_min(lo[i], wn[i]);
        hi[i] = bound_max(hi[i], wn[i]);
      }
    };
    auto row = [&](int j, C* e) {
      if constexpr (S) {
        const float4 v = ld16_once(d.st + 4 * (base + static_cast<long long>(j) * kSlice), pol_first);
        e[0] = v.x, e[1] = v.y, e[2] = v.z, e[3] = v.w;
      } else {
        load_words<P, sizeof(C) == 8>(d.st + 4 * (base + static_cast<long long>(j) * kSlice), 0, 4, e);
      }
    };
    auto gather = [&](const C* e, C* w) {
      const int x = index_of(e[3]);
      load5<P>(d.prim + static_cast<long long>(x) * kPrimW, w);
    };
    if constexpr (CHUNK == 0) {
      // Software pipeline: while entry j is added, the gather of entry j + 1 and the row of entry
      // j + 2 are in flight.
      C eC[4], eN[4], wC[5], wN[5];
      if (len > 0) {
        row(0, eC);
        gather(eC, wC);
      }
      if (len > 1) row(1, eN);
#pragma unroll 2
      for (int j = 0; j < len; ++j) {
        C eF[4];
        if (j + 1 < len) gather(eN, wN);
        if (j + 2 < len) row(j + 2, eF);
        add_entry(eC, wC);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          eC[k] = eN[k];
          eN[k] = eF[k];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) wC[k] = wN[k];
      }
    } else {
      for (int j0 = 0; j0 < len; j0 += CHUNK) {
        C e4[CHUNK][4], wn[CHUNK][5];
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q < len) row(j0 + q, e4[q]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q < len) gather(e4[q], wn[q]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q < len) add_entry(e4[q], wn[q]);
      }
    }
    return gradient_tail<P, LIMIT, DT, S>(d, c, wc, acc, lo, hi, cfl, local);
  }
}

template <class P, bool LIMIT, bool DT, int CHUNK>
__global__ void __launch_bounds__(256) k_gradients(Dev<P> d, double cfl, int local) {
  gradients_cells<P, LIMIT, DT, CHUNK>(d, cfl, local);
}

// Two entries in flight in fp32+acc64, registers sized for 7 blocks of 128 per SM (at most 128
// threads a block): 72 registers instead of 80. Only this form gets the bound; given to the
// others it makes them spill.
template <class P, bool LIMIT, bool DT>
__global__ void __launch_bounds__(128, 7) k_gradients_occ7(Dev<P> d, double cfl, int local) {
  gradients_cells<P, LIMIT, DT, 2, false, sizeof(typename P::C) == 4>(d, cfl, local);
}

// The gradient launch of re-packed batched steps (whatever the tuning): each warp takes the cells
// of its tile, two entries in flight, 128 threads per block (the fp32+acc64 form bounded for 7
// blocks per SM as k_gradients_occ7).
template <class P>
constexpr int kTilesMinBlocks = sizeof(typename P::C) == 4 ? 7 : 1;
template <class P, bool LIMIT, bool DT>
__global__ void __launch_bounds__(128, kTilesMinBlocks<P>) k_gradients_tiles(Dev<P> d, double cfl,
                                                                             int local) {
  gradients_cells<P, LIMIT, DT, 2, true>(d, cfl, local);
}

// ---------------------------------------------------------------- integer-pipe widening

// 2^-896 p as a double, exactly, for every finite float p (normal, subnormal or zero, of either
// sign): the float's sign, exponent and fraction bits placed in a double whose 11-bit exponent
// field holds the float's 8-bit one (bias 127 read against bias 1023, hence the factor). A signed
// 32 x 32 -> 64 multiply by 2^29 shifts the bits (its sign extension fills the top three bits of
// the exponent field with the sign), one AND clears those three bits: two integer instructions in
// place of one cvt.f64.f32 on the conversion (XU) pipe, which the 15 products of every stencil
// entry otherwise keep half busy. An infinity or NaN p maps to a finite double: callers take
// this path only where no product can be one.
//
// FP64 sums of these values are 2^-896 times the sums of the same products widened by cvt, bit
// for bit: while a partial sum is at least 2^-1022 both are rounded to 53 bits at the same
// relative position; below it the unscaled partial sum is a multiple of 2^-149 under 2^-126
// (23 significant bits, exact) and the scaled one a multiple of 2^-1045 under 2^-1022, which a
// subnormal double holds exactly. Multiplying a scaled sum by 2^896 restores it exactly.
__device__ __forceinline__ double widen_scaled(float p) {
  double out;
  asm("{\n\t.reg .b64 t;\n\t.reg .b32 l, h;\n\t"
      "mul.wide.s32 t, %1, 536870912;\n\t"
      "mov.b64 {l, h}, t;\n\t"
      "and.b32 h, h, 0x8FFFFFFF;\n\t"
      "mov.b64 %0, {l, h};\n\t}"
      : "=d"(out)
      : "r"(__float_as_int(p)));
  return out;
}
constexpr double kUnscale = 0x1p896;

// A product widened for the FP64 sums: scaled on the integer pipe (SCALED) or by cvt.
template <bool SCALED>
__device__ __forceinline__ double widen(float p) {
  if constexpr (SCALED) {
    return widen_scaled(p);
  } else {
    return static_cast<double>(p);
  }
}

// The products of a stencil entry in the gradient sums are finite and below 2^101 when every
// primitive read is below 2^60 in magnitude (Control::special clear) and every LSQ weight below
// 2^40 (Dev::wide_ok, checked at create); their sums then stay below 2^120, so the scaled
// widening is exact.

// Five words of a record as one 16-byte and one 4-byte load: 5 registers held while the gather is
// in flight where the 32-byte load holds 8. The two loads read one 32-byte sector.
__device__ __forceinline__ void load5_narrow(const float* src, float* w) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(src));
  w[0] = a.x;
  w[1] = a.y;
  w[2] = a.z;
  w[3] = a.w;
  w[4] = __ldg(src + 4);
}

template <bool G5>
__device__ __forceinline__ void gather5(const float* src, float* w) {
  if constexpr (G5) {
    load5_narrow(src, w);
  } else {
    load5<Fp32Acc64>(src, w);
  }
}

// gradient_tail with the pass over the incidences software-pipelined: the record (and the
// normal and area) of incidence j + 1 is loaded, and with DT the other side's primitives of
// incidence j gathered, before incidence j's limiter terms are computed. Same operations in the
// same order as gradient_tail.
template <bool LIMIT, bool DT, bool G5>
__device__ __forceinline__ double gradient_tail_pipelined(const Dev<Fp32Acc64>& d, int c,
                                                          const float* wc, const double* acc,
                                                          const float* lo, const float* hi,
                                                          double cfl, int local) {
  using P = Fp32Acc64;
  using C = float;
  C out[kRecon];
#pragma unroll
  for (int k = 0; k < 15; ++k) out[5 + k] = static_cast<C>(acc[k]);
  const C* g = out + 5;
  C phi[5], dmax[5], dmin[5], eps2[5];
  if constexpr (LIMIT) {
    const C vol = static_cast<C>(__ldg(d.volume + c));
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      dmax[i] = maxv(hi[i], wc[i]) - wc[i];
      dmin[i] = minv(lo[i], wc[i]) - wc[i];
      eps2[i] = d.p.scale[i] * vol;
      // min(1, min over the faces of venkat) as a min from 1: the same value, and a face whose
      // venkat cannot go below the running min skips its quotient (venkat_min)
      phi[i] = C(1.0);
    }
  }
  double lam = 0.0;
  C cc = C(0);
  if constexpr (DT) cc = sound_speed(wc, d.p.g, d.p.pref);
  if constexpr (LIMIT || DT) {
    const long long ib = __ldg(d.inc_start + (c >> 5)) + (c & 31);
    const int il = __ldg(d.inc_len + c);
    C r[4];
    if (il > 0) load_words<P>(d.inc_rec + 4 * ib, 0, 4, r);
    for (int j = 0; j < il; ++j) {
      C rn[4], nd[4], wn[5];
      if constexpr (DT) {
        gather5<G5>(d.prim + static_cast<long long>(index_of(r[3])) * kPrimW, wn);
        load_words<P>(d.inc_dt + 4 * (ib + static_cast<long long>(j) * kSlice), 0, 4, nd);
      }
      if (j + 1 < il)
        load_words<P>(d.inc_rec + 4 * (ib + static_cast<long long>(j + 1) * kSlice), 0, 4, rn);
      if constexpr (LIMIT) {
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          const C dd = g[3 * i] * r[0] + g[3 * i + 1] * r[1] + g[3 * i + 2] * r[2];
          phi[i] = venkat_min(phi[i], dd, dmax[i], dmin[i], eps2[i]);
        }
      }
      if constexpr (DT)
        lam += static_cast<double>(wave_speed_cc(wc, cc, wn, nd, nd[3], d.p.g, d.p.pref));
#pragma unroll
      for (int k = 0; k < 4; ++k) r[k] = rn[k];
    }
  }
  if constexpr (LIMIT) {
#pragma unroll
    for (int i = 0; i < 5; ++i) out[i] = minv(phi[i], C(1.0));
  } else {
#pragma unroll
    for (int i = 0; i < 5; ++i) out[i] = C(1.0);
  }
#pragma unroll
  for (int k = 20; k < kRecon; ++k) out[k] = C(0);
  store_recon<P>(d, c, out);
  if constexpr (DT) {
    const double dt = cfl * d.volume[c] / static_cast<double>(static_cast<C>(lam));
    if (local) d.dt_local[c] = dt;
    return dt;
  }
  return 0.0;
}

// gradients + limiter (as k_gradients) in fp32+acc64 with the product widening on the integer
// pipe: WIDE = 1 widens the x and y products of each entry (10 of 15) with widen_scaled, WIDE = 2
// all 15, the rest through cvt; G5 gathers neighbours with load5_narrow; CHUNK entries are
// loaded together. Where Control::special is set or a weight is out of range the cells take the
// cvt loop instead (the same sums, bit for bit).
template <bool LIMIT, bool DT, int WIDE, bool G5, int CHUNK>
__device__ __forceinline__ void gradients_w_cells(const Dev<Fp32Acc64>& d, double cfl, int local) {
  using P = Fp32Acc64;
  using C = float;
  if (block_idle(d)) return;
  const int c = gradient_cell<false>(d);
  const bool live = c < d.n && cell_active(d, c);
  const bool fast = WIDE > 0 && d.wide_ok != 0 && __ldg(&d.ctl->special) == 0ULL;
  double dt = 0.0;
  prefetch_rows<P, LIMIT, DT>(d, c);
  if (live) {
    C wc[5];
    load5<P>(d.prim + static_cast<long long>(c) * kPrimW, wc);
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    C lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      lo[k] = C(INFINITY);
      hi[k] = -C(INFINITY);
    }
    const int base = __ldg(d.st_start + (c >> 5)) + (c & 31);
    const int len = __ldg(d.st_len + c);
    auto walk = [&](auto scaled) {
      constexpr int W = decltype(scaled)::value;
      for (int j0 = 0; j0 < len; j0 += CHUNK) {
        C e4[CHUNK][4], wn[CHUNK][5];
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q < len)
            load_words<P>(d.st + 4 * (base + static_cast<long long>(j0 + q) * kSlice), 0, 4, e4[q]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q < len)
            gather5<G5>(d.prim + static_cast<long long>(index_of(e4[q][3])) * kPrimW, wn[q]);
#pragma unroll
        for (int q = 0; q < CHUNK; ++q) {
          if (j0 + q < len) {
#pragma unroll
            for (int i = 0; i < 5; ++i) {
              const C dw = wn[q][i] - wc[i];
              acc[3 * i] += widen<(W >= 1)>(dw * e4[q][0]);
              acc[3 * i + 1] += widen<(W >= 1)>(dw * e4[q][1]);
              acc[3 * i + 2] += widen<(W >= 2)>(dw * e4[q][2]);
            }
#pragma unroll
            for (int i = 0; i < 5; ++i) {
              lo[i] = bound_min(lo[i], wn[q][i]);
              hi[i] = bound_max(hi[i], wn[q][i]);
            }
          }
        }
      }
    };
    if (fast) {
      walk(std::integral_constant<int, WIDE>{});
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        acc[3 * i] *= kUnscale;
        acc[3 * i + 1] *= kUnscale;
        if (WIDE >= 2) acc[3 * i + 2] *= kUnscale;
      }
    } else {
      walk(std::integral_constant<int, 0>{});
    }
    dt = gradient_tail_pipelined<LIMIT, DT, G5>(d, c, wc, acc, lo, hi, cfl, local);
  }
  if constexpr (DT) block_min_dt(dt, live, &d.ctl->dt_bits);
}

template <bool LIMIT, bool DT, int WIDE, bool G5, int CHUNK, int MINB>
__global__ void __launch_bounds__(128, MINB) k_gradients_w(Dev<Fp32Acc64> d, double cfl, int local) {
  gradients_w_cells<LIMIT, DT, WIDE, G5, CHUNK>(d, cfl, local);
}

// ---------------------------------------------------------------- TMA bulk staging

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// One 1-D bulk copy global -> shared (TMA, no tensor map, no multicast), completing on `bar`.
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, unsigned bytes,
                                               unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, "
      "p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

constexpr int kWaitLimit = 1 << 20;  // polls of an mbarrier before a kernel gives up

// Waits for phase 0 of `bar` with an iteration limit. On a timeout it marks the control's fault
// word and waits once more, again bounded, so that no copy into this block's shared memory is
// left in flight when the block exits.
__device__ __forceinline__ bool bounded_wait(unsigned long long* bar, Control* ctl) {
  for (int it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, 0)) return true;
  if (threadIdx.x == 0 && ctl != nullptr) atomicExch(&ctl->fault, 1ULL);
  for (int it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, 0)) break;
  return false;
}

// gradients + limiter (as k_gradients) for the cells of blockDim.x / 32 consecutive slices, their
// stencil rows and per-incidence limiter records staged into shared memory by one TMA bulk copy
// each (the slices' rows are contiguous in the sliced layout): the block's whole streaming input
// is in flight at once, and the threads then only gather their neighbours' primitives (L2).
template <class P, bool LIMIT, bool DT, int CHUNK>
__device__ __forceinline__ void gradients_staged_cells(const Dev<P>& d, double cfl, int local) {
  using C = typename P::C;
  if (block_idle(d)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bar;
  const int per_block = blockDim.x / 32;
  const int s0 = blockIdx.x * per_block;
  const int s1 = min(s0 + per_block, d.n_slices);
  const long long e0 = __ldg(d.st_start + s0), e1 = __ldg(d.st_start + s1);
  const long long i0 = __ldg(d.inc_start + s0), i1 = __ldg(d.inc_start + s1);
  C* ent = reinterpret_cast<C*>(smem_raw);
  C* inc = ent + 4 * (e1 - e0);
  C* ndt = inc + 4 * (i1 - i0);
  const unsigned eb = static_cast<unsigned>((e1 - e0) * 4 * sizeof(C));
  const unsigned ib = (LIMIT || DT) ? static_cast<unsigned>((i1 - i0) * 4 * sizeof(C)) : 0u;
  const unsigned db = DT ? static_cast<unsigned>((i1 - i0) * 4 * sizeof(C)) : 0u;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, eb + ib + db);
    if (eb > 0) bulk_to_shared(ent, d.st + 4 * e0, eb, &bar);
    if (ib > 0) bulk_to_shared(inc, d.inc_rec + 4 * i0, ib, &bar);
    if (db > 0) bulk_to_shared(ndt, d.inc_dt + 4 * i0, db, &bar);
  }
  if (!bounded_wait(&bar, d.ctl)) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = c < d.n && cell_active(d, c);
  double dt = 0.0;
  if (live) {
    C wc[5];
    load5<P>(d.prim + static_cast<long long>(c) * kPrimW, wc);
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    C lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      lo[k] = C(INFINITY);
      hi[k] = -C(INFINITY);
    }
    const C* row = ent + 4 * (__ldg(d.st_start + (c >> 5)) - e0 + (c & 31));
    const int len = __ldg(d.st_len + c);
    constexpr int kChunk = CHUNK;
    for (int j0 = 0; j0 < len; j0 += kChunk) {
      C wn[kChunk][5];
#pragma unroll
      for (int q = 0; q < kChunk; ++q) {
        if (j0 + q < len) {
          const int e = index_of(row[4 * kSlice * (j0 + q) + 3]);
          load5<P>(d.prim + static_cast<long long>(e) * kPrimW, wn[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < kChunk; ++q) {
        if (j0 + q < len) {
          const C* w = row + 4 * kSlice * (j0 + q);
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            const C dw = wn[q][i] - wc[i];
            acc[3 * i] += static_cast<double>(dw * w[0]);
            acc[3 * i + 1] += static_cast<double>(dw * w[1]);
            acc[3 * i + 2] += static_cast<double>(dw * w[2]);
          }
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            lo[i] = bound_min(lo[i], wn[q][i]);
            hi[i] = bound_max(hi[i], wn[q][i]);
          }
        }
      }
    }
    // include_own_value (:517-521); out: phi, then grad, then padding.
    C out[kRecon];
#pragma unroll
    for (int k = 0; k < 15; ++k) out[5 + k] = static_cast<C>(acc[k]);
    const C* g = out + 5;
    const C* irow = inc + 4 * (__ldg(d.inc_start + (c >> 5)) - i0 + (c & 31));
    const C* drow = ndt + (irow - inc);
    const int il = __ldg(d.inc_len + c);
    C phi[5], dmax[5], dmin[5], eps2[5];
    if constexpr (LIMIT) {
      const C vol = static_cast<C>(__ldg(d.volume + c));
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        dmax[i] = maxv(hi[i], wc[i]) - wc[i];
        dmin[i] = minv(lo[i], wc[i]) - wc[i];
        eps2[i] = d.p.scale[i] * vol;
        phi[i] = C(INFINITY);
      }
    }
    // One pass over the staged incidence records for the limiter and, with DT, spectral_radius
    // (:1103-1112: the other side's state from the limiter record, the normal and area staged).
    double lam = 0.0;
    if constexpr (LIMIT || DT) {
      for (int j = 0; j < il; ++j) {
        const C* r = irow + 4 * kSlice * j;
        C wn[5];
        if constexpr (DT) {
          const int o = index_of(r[3]);
          load5<P>(d.prim + static_cast<long long>(o) * kPrimW, wn);
        }
        if constexpr (LIMIT) {
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            const C dd = g[3 * i] * r[0] + g[3 * i + 1] * r[1] + g[3 * i + 2] * r[2];
            // venkat's value is >= 0 and never -0 (its numerator adds 2 d dp, >= 0, to
            // dp^2 + eps2 >= +0), or NaN: the hardware min is then the keep-the-first min
            phi[i] = bound_min(phi[i], venkat(dd, dmax[i], dmin[i], eps2[i]));
          }
        }
        if constexpr (DT) {
          const C* nd = drow + 4 * kSlice * j;
          lam += static_cast<double>(wave_speed(wc, wn, nd, nd[3], d.p.g, d.p.pref));
        }
      }
    }
    if constexpr (LIMIT) {
      // at_most_one (:591-593)
#pragma unroll
      for (int i = 0; i < 5; ++i) out[i] = minv(phi[i], C(1.0));
    } else {
      // Second order without limiter: phi = 1 (physics/src/euler.cpp:195).
#pragma unroll
      for (int i = 0; i < 5; ++i) out[i] = C(1.0);
    }
#pragma unroll
    for (int k = 20; k < kRecon; ++k) out[k] = C(0);
    store_recon<P>(d, c, out);
    if constexpr (DT) {
      // The cell's CFL step (device_stepper.cuh:84-89).
      dt = cfl * d.volume[c] / static_cast<double>(static_cast<C>(lam));
      if (local) d.dt_local[c] = dt;
    }
  }
  if constexpr (DT) block_min_dt(dt, live, &d.ctl->dt_bits);
}

template <class P, bool LIMIT, bool DT, int CHUNK>
__global__ void __launch_bounds__(128) k_gradients_tma(Dev<P> d, double cfl, int local) {
  gradients_staged_cells<P, LIMIT, DT, CHUNK>(d, cfl, local);
}

// ---------------------------------------------------------------- per-warp TMA row ring

// A warp's 32 cells are one slice: the rows of its entry j are 512 contiguous bytes. Each warp
// keeps its next R entries' rows in a ring of shared-memory slots, each filled by one 1-D TMA bulk
// copy (cp.async.bulk, no tensor map, no multicast) that completes on the slot's mbarrier; lane 0
// refills a slot once the warp has read it. The stencil stream from HBM then runs R entries ahead
// of the warp without holding registers, and an entry's neighbour index is in shared memory when
// the warp reaches it, so the gathers start at once: the row load no longer sits in front of every
// gather. Shared memory per block of 4 warps: 4 R (512 + 8) bytes.
constexpr int kRingWarps = 4;
constexpr size_t warp_ring_bytes(int R) {
  return static_cast<size_t>(kRingWarps) * R * (kSlice * 16 + 8);
}

// Waits for phase `parity` of a slot's mbarrier, polling at most `polls` times; false on a
// timeout.
__device__ __forceinline__ bool slot_wait(unsigned long long* bar, unsigned parity,
                                          int polls = kWaitLimit) {
  for (int it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// gradients + limiter (as k_gradients) in fp32+acc64 with the stencil rows streamed through the
// warp's slot ring; CHUNK entries' gathers in flight at once (their weights read from the slots
// after the gathers return); G5: 5-word gathers. A slot wait that times out marks Control::fault;
// the warp then waits, again bounded, for the copies it has issued and stores nothing.
template <bool LIMIT, bool DT, int R, int CHUNK, bool G5>
__global__ void __launch_bounds__(128, 7) k_gradients_wring(Dev<Fp32Acc64> d, double cfl, int local) {
  using P = Fp32Acc64;
  using C = float;
  static_assert(R >= CHUNK, "the ring holds at least one chunk");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  if (block_idle(d)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* ring = reinterpret_cast<float4*>(smem_raw) + warp * R * kSlice;
  unsigned long long* bar =
      reinterpret_cast<unsigned long long*>(smem_raw + kRingWarps * R * kSlice * 16) + warp * R;
  const int c = gradient_cell<false>(d);
  const bool live = c < d.n && cell_active(d, c);
  bool ok = true;
  double dt = 0.0;
  if (__any_sync(0xffffffffu, live)) {  // uniform over the warp
    const int s = c >> 5;
    const long long e0 = __ldg(d.st_start + s);
    const int L = static_cast<int>((__ldg(d.st_start + s + 1) - e0) / kSlice);
    const float4* src = reinterpret_cast<const float4*>(d.st) + e0;
    auto issue = [&](int j) {  // lane 0: entry j's rows into slot j % R
      const int k = j % R;
      mbar_expect_tx(&bar[k], kSlice * 16);
      bulk_to_shared(ring + k * kSlice, src + static_cast<long long>(j) * kSlice, kSlice * 16, &bar[k]);
    };
    if (lane == 0) {
      for (int k = 0; k < R; ++k) mbar_init(&bar[k], 1);
      for (int j = 0; j < R && j < L; ++j) issue(j);
    }
    __syncwarp();
    if (d.stall_polls > 0) {
      // test hook: a wait on a barrier nothing arrives on runs out after stall_polls polls
      __shared__ __align__(8) unsigned long long dead[kRingWarps];
      if (lane == 0) mbar_init(&dead[warp], 1);
      __syncwarp();
      ok = __all_sync(0xffffffffu, slot_wait(&dead[warp], 0, d.stall_polls));
    }
    const int len = live ? __ldg(d.st_len + c) : 0;
    C wc[5] = {C(0), C(0), C(0), C(0), C(0)};
    if (live) load5<P>(d.prim + static_cast<long long>(c) * kPrimW, wc);
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    C lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      lo[k] = C(INFINITY);
      hi[k] = -C(INFINITY);
    }
    int waited = 0;  // entries whose slot has been waited for
    for (int j0 = 0; ok && j0 < L; j0 += CHUNK) {
      bool got = true;
#pragma unroll
      for (int q = 0; q < CHUNK; ++q)
        if (j0 + q < L) got = got && slot_wait(&bar[(j0 + q) % R], ((j0 + q) / R) & 1);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      waited = j0 + CHUNK < L ? j0 + CHUNK : L;
      C wn[CHUNK][5];
#pragma unroll
      for (int q = 0; q < CHUNK; ++q)
        if (j0 + q < len) {
          const int x = __float_as_int(ring[((j0 + q) % R) * kSlice + lane].w);
          gather5<G5>(d.prim + static_cast<long long>(x) * kPrimW, wn[q]);
        }
#pragma unroll
      for (int q = 0; q < CHUNK; ++q) {
        if (j0 + q < len) {
          const float4 e = ring[((j0 + q) % R) * kSlice + lane];
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            const C dw = wn[q][i] - wc[i];
            acc[3 * i] += static_cast<double>(dw * e.x);
            acc[3 * i + 1] += static_cast<double>(dw * e.y);
            acc[3 * i + 2] += static_cast<double>(dw * e.z);
          }
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            lo[i] = bound_min(lo[i], wn[q][i]);
            hi[i] = bound_max(hi[i], wn[q][i]);
          }
        }
      }
      __syncwarp();  // every lane has read the chunk's slots
      if (lane == 0)
#pragma unroll
        for (int q = 0; q < CHUNK; ++q)
          if (j0 + q + R < L) issue(j0 + q + R);
    }
    if (!ok) {
      // a slot wait gave up: mark the fault and wait, bounded, for the copies still in flight
      if (lane == 0) atomicExch(&d.ctl->fault, 1ULL);
      for (int j = waited; j < L && j < waited + R; ++j) slot_wait(&bar[j % R], (j / R) & 1);
    } else if (live) {
      dt = gradient_tail_pipelined<LIMIT, DT, G5>(d, c, wc, acc, lo, hi, cfl, local);
    }
  }
  if constexpr (DT) block_min_dt(dt, live && ok, &d.ctl->dt_bits);
}

// fp32+acc64 with up to 4 entries in flight, registers sized for 6 blocks of 128 per SM: the
// stage-0 form (with the time step) drops from 94 to 80 registers. The 8-entry form and the FP64
// policy spill under that bound and keep k_gradients_tma.
template <class P, bool LIMIT, bool DT, int CHUNK>
__global__ void __launch_bounds__(128, 6) k_gradients_tma_occ6(Dev<P> d, double cfl, int local) {
  gradients_staged_cells<P, LIMIT, DT, CHUNK>(d, cfl, local);
}

// ---------------------------------------------------------------- asynchronous-copy ring

// Per-thread asynchronous copies into shared memory (cp.async): .cg (16 bytes, L2 only) for the
// streamed stencil rows, .ca (4, 8 or 16 bytes, through L1) for the gathered neighbour records,
// whose neighbours are shared by nearby cells. Completion is tracked per thread by commit groups.
__device__ __forceinline__ void cp_async_cg16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
template <int B>
__device__ __forceinline__ void cp_async_ca(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(B)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Bytes of shared memory per thread of k_gradients_ring at depth `depth` (C of `word` bytes):
// depth + 1 neighbour records of 5 words and 2 depth + 1 stencil rows of 4 words.
constexpr int ring_bytes(int depth, int word) {
  return (depth + 1) * 5 * word + (2 * depth + 1) * 4 * word;
}

// gradients + limiter (as k_gradients), the stencil walked with asynchronous copies: each thread
// keeps a ring in shared memory of its next D neighbour records and next 2D stencil rows, so D
// gathers are in flight without holding registers. Entry j's group (its neighbour record, and
// the row of entry j + D) is the D-th newest when entry j is added: cp.async.wait_group D - 1. A
// slot is refilled one entry after it was read (D + 1 record slots, 2D + 1 row slots). Entries
// are added in stencil order, so the sums are those of k_gradients bit for bit.
template <class P, bool LIMIT, bool DT, int D>
__global__ void __launch_bounds__(128, 6) k_gradients_ring(Dev<P> d, double cfl, int local) {
  using C = typename P::C;
  if (block_idle(d)) return;
  constexpr int kW = 16 / static_cast<int>(sizeof(C));   // words per 16-byte piece
  constexpr int kG16 = 5 / kW;                            // whole pieces of a record's 5 words
  constexpr int kGRem = (5 % kW) * static_cast<int>(sizeof(C));  // bytes after them
  constexpr int kR16 = 4 / kW;                            // pieces of a stencil row
  constexpr int kGS = D + 1, kRS = 2 * D + 1;             // record and row slots
  static_assert(kGRem == 4 || kGRem == 8, "a record's tail is one word");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nt = blockDim.x, t = threadIdx.x;
  // Regions, each piece interleaved over the block's threads (conflict-free 128-bit accesses):
  // records' whole pieces, records' tails, rows.
  unsigned char* const g16 = smem_raw;
  unsigned char* const grem = g16 + kGS * kG16 * nt * 16;
  unsigned char* const r16 = grem + kGS * nt * kGRem;
  const int c = gradient_cell<false>(d);
  const bool live = c < d.n && cell_active(d, c);
  double dt = 0.0;
  prefetch_rows<P, LIMIT, DT>(d, c);
  if (live) {
    C wc[5];
    load5<P>(d.prim + static_cast<long long>(c) * kPrimW, wc);
    double acc[15];
#pragma unroll
    for (int k = 0; k < 15; ++k) acc[k] = 0.0;
    C lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      lo[k] = C(INFINITY);
      hi[k] = -C(INFINITY);
    }
    const long long base = __ldg(d.st_start + (c >> 5)) + (c & 31);
    const int len = __ldg(d.st_len + c);
    const C* rows = d.st + 4 * base;
    auto rpiece = [&](int slot, int q) { return r16 + ((slot * kR16 + q) * nt + t) * 16; };
    auto issue_row = [&](int j, int slot) {
      const C* src = rows + 4LL * kSlice * j;
#pragma unroll
      for (int q = 0; q < kR16; ++q) cp_async_cg16(rpiece(slot, q), src + q * kW);
    };
    auto row_index = [&](int slot) {
      return index_of(reinterpret_cast<const C*>(rpiece(slot, kR16 - 1))[kW - 1]);
    };
    auto issue_gather = [&](int x, int slot) {
      const C* src = d.prim + static_cast<long long>(x) * kPrimW;
#pragma unroll
      for (int q = 0; q < kG16; ++q) cp_async_ca<16>(g16 + ((slot * kG16 + q) * nt + t) * 16, src + q * kW);
      cp_async_ca<kGRem>(grem + (slot * nt + t) * kGRem, src + kG16 * kW);
    };
    // Prologue: rows 0 .. D-1 (waited for), then per entry g < D its record and the row of g + D.
    for (int j = 0; j < D && j < len; ++j) issue_row(j, j);
    cp_async_commit();
    cp_async_wait<0>();
#pragma unroll
    for (int g = 0; g < D; ++g) {
      if (g < len) issue_gather(row_index(g), g);
      if (g + D < len) issue_row(g + D, g + D);
      cp_async_commit();
    }
    int gs = 0, rs = 0;           // slots of entry j's record and row
    int gw = D, rw = 2 * D;       // slots the next record and row go to
    int rn = D;                   // slot of the row of entry j + D
    for (int j = 0; j < len; ++j) {
      cp_async_wait<D - 1>();
      C wn[5], e[4];
#pragma unroll
      for (int q = 0; q < kG16; ++q) {
        const C* v = reinterpret_cast<const C*>(g16 + ((gs * kG16 + q) * nt + t) * 16);
#pragma unroll
        for (int w = 0; w < kW; ++w) wn[q * kW + w] = v[w];
      }
      wn[4] = *reinterpret_cast<const C*>(grem + (gs * nt + t) * kGRem);
#pragma unroll
      for (int q = 0; q < kR16; ++q) {
        const C* v = reinterpret_cast<const C*>(rpiece(rs, q));
#pragma unroll
        for (int w = 0; w < kW; ++w) e[q * kW + w] = v[w];
      }
      const int x = j + D < len ? row_index(rn) : 0;
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const C dw = wn[i] - wc[i];
        acc[3 * i] += static_cast<double>(dw * e[0]);
        acc[3 * i + 1] += static_cast<double>(dw * e[1]);
        acc[3 * i + 2] += static_cast<double>(dw * e[2]);
      }
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        lo[i] = bound_min(lo[i], wn[i]);
        hi[i] = bound_max(hi[i], wn[i]);
      }
      if (j + D < len) issue_gather(x, gw);
      if (j + 2 * D < len) issue_row(j + 2 * D, rw);
      cp_async_commit();
      gs = gs + 1 == kGS ? 0 : gs + 1;
      gw = gw + 1 == kGS ? 0 : gw + 1;
      rs = rs + 1 == kRS ? 0 : rs + 1;
      rw = rw + 1 == kRS ? 0 : rw + 1;
      rn = rn + 1 == kRS ? 0 : rn + 1;
    }
    cp_async_wait<0>();
    dt = gradient_tail<P, LIMIT, DT>(d, c, wc, acc, lo, hi, cfl, local);
  }
  if constexpr (DT) block_min_dt(dt, live, &d.ctl->dt_bits);
}

// The CFL step alone (first-order schemes), with the block minimum; `dt_out` for the host.
template <class P>
__global__ void __launch_bounds__(256) k_spectral(Dev<P> d, double cfl, int local,
                                                  double* dt_out) {
  using C = typename P::C;
  const int c = tile_item(d.cell_tiles, d.n_cell_tiles);
  const bool live = c >= 0 && c < d.n && cell_active(d, c);
  double dt = 0.0;
  if (live) {
    C wc[5];
    load_prim<P>(d.prim, c, wc);
    dt = cell_time_step(d, c, wc, cfl);
    if (local && d.dt_local != nullptr) d.dt_local[c] = dt;
    if (dt_out != nullptr) dt_out[c] = dt;
  }
  if (d.ctl != nullptr) block_min_dt(dt, live, &d.ctl->dt_bits);
}

// kFaceParts: the residual's face part alone (no sources, from zero), Euler<P>::face_parts.
enum Mode : int { kResidual = 0, kRk3 = 1, kRk4 = 2, kFaceParts = 3 };

// The reconstruction data of a cell: primitives, limiter and gradient (zero gradient and limiter
// for the first-order scheme).
template <class P, bool SECOND>
__device__ __forceinline__ void cell_recon(const Dev<P>& d, int c, typename P::C* w,
                                           typename P::C* phi, typename P::C* g) {
  using C = typename P::C;
  if constexpr (SECOND) {
    load_recon<P>(d, c, w, phi, g);
  } else {
    load5<P>(d.prim + static_cast<long long>(c) * kPrimW, w);
#pragma unroll
    for (int k = 0; k < 15; ++k) g[k] = C(0.0);
#pragma unroll
    for (int k = 0; k < 5; ++k) phi[k] = C(0.0);
  }
}

// The scheme's values for a face of owner cell `owner`: with per-case cut-offs, the AUSM+-up
// cut-off Mach number of the owner's case (M_co of ausm_up, kernels/euler.py:268-303).
template <int FLUX, class P>
__device__ __forceinline__ Params<typename P::C> face_params(const Dev<P>& d, int owner) {
  Params<typename P::C> p = d.p;
  if constexpr (FLUX == 2) {
    if (d.case_minf != nullptr) p.minf = d.case_minf[d.case_of[owner]];
  }
  return p;
}

// The flux of interior face f in its orientation (roe_face / hllc_face / ausm_face,
// kernels/euler.py:687-753, planar forms :783-844): both sides reconstructed, the numerical flux
// times the area, plus the warped-face term.
template <class P, int FLUX, bool PLANAR>
__device__ __forceinline__ void interior_flux(const Dev<P>& d, int f, const typename P::C* fr,
                                              const typename P::C* wl, const typename P::C* gl,
                                              const typename P::C* pl, const typename P::C* wr,
                                              const typename P::C* gr, const typename P::C* pr,
                                              typename P::C* out) {
  using C = typename P::C;
  const C* n = fr;
  const C area = fr[3];
  C fl[5], frr[5], fx[5];
  reconstruct(wl, gl, pl, fr + 4, d.p.pref, fl);
  reconstruct(wr, gr, pr, fr + 8, d.p.pref, frr);
  numerical_flux<FLUX>(fl, frr, n, face_params<FLUX>(d, index_of(fr[7])), fx);
  if constexpr (PLANAR) {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = area * fx[k];
  } else {
    C m[9], avg[5], wt[5];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = __ldg(d.f_m + static_cast<long long>(q) * d.n_if + f);
#pragma unroll
    for (int k = 0; k < 5; ++k) avg[k] = C(0.5) * (fl[k] + frr[k]);
    warp_term(avg, gl, pl, gr, pr, m, d.p.g, d.p.pref, wt);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = area * fx[k] + wt[k];
  }
}

// The flux of boundary face b (roe_boundary ..., kernels/euler.py:868-941, planar :967-1037):
// slip walls (and no-slip walls in the full loops) carry the pressure only.
template <class P, int FLUX, bool PLANAR>
__device__ __forceinline__ void boundary_flux(const Dev<P>& d, int b, const typename P::C* br,
                                              const typename P::C* wc, const typename P::C* gc,
                                              const typename P::C* pc, typename P::C* out) {
  using C = typename P::C;
  const C* n = br;
  const C area = br[3];
  const C kind = br[7];
  C wf[5];
  reconstruct(wc, gc, pc, br + 4, d.p.pref, wf);
  const bool slip = (kind > C(1.5)) & (kind < C(2.5));
  const bool wall = PLANAR ? slip : (slip | (kind > C(4.5)));
  if (wall) {
    const C wfl[5] = {C(0.0), wf[4] * n[0], wf[4] * n[1], wf[4] * n[2], C(0.0)};
    if constexpr (PLANAR) {
#pragma unroll
      for (int k = 0; k < 5; ++k) out[k] = area * wfl[k];
    } else {
      C m[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) m[q] = __ldg(d.b_m + static_cast<long long>(q) * d.nb + b);
      // wall_warp (:678-681): p_l M^T grad p.
      C ww[5] = {C(0.0), C(0.0), C(0.0), C(0.0), C(0.0)};
#pragma unroll
      for (int i = 0; i < 3; ++i)
        ww[1 + i] = pc[4] * (m[i] * gc[12] + m[3 + i] * gc[13] + m[6 + i] * gc[14]);
#pragma unroll
      for (int k = 0; k < 5; ++k) out[k] = area * wfl[k] + ww[k];
    }
  } else {
    C wbv[5], fx[5];
    boundary_value(wf, kind, br + 8, n, d.p, wbv);
    numerical_flux<FLUX>(wf, wbv, n, face_params<FLUX>(d, index_of(br[13])), fx);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = area * fx[k];
  }
}

// After a cell's residual: the residual output, the RK stage update of the FP64 state, the next
// stage's primitives and, after the last stage, the validity checks.
// The FP64 words of a cell that its update reads: u, the stage state (SSP-RK3) or the RK4
// accumulator (stages > 0), and the step h. The kernels load them before their flux sums, so that
// these loads are in flight together with the flux loads.
struct CellIn {
  double u[5], x[5], h;
};

template <class P>
__device__ __forceinline__ void load_cell_in(const Dev<P>& d, int c, int mode, int stage, int local,
                                             CellIn& in) {
  if (mode == kResidual || mode == kFaceParts) return;
#pragma unroll
  for (int k = 0; k < 5; ++k) in.u[k] = d.u[static_cast<long long>(k) * d.n + c];
  if (stage > 0) {
    const double* src = mode == kRk3 ? d.stage : d.racc;
#pragma unroll
    for (int k = 0; k < 5; ++k) in.x[k] = src[static_cast<long long>(k) * d.n + c];
  } else {
#pragma unroll
    for (int k = 0; k < 5; ++k) in.x[k] = 0.0;
  }
  // the global step from its minimum's bits (final once the stage-0 cell kernel has run)
  in.h = local ? d.dt_local[c] : __longlong_as_double(static_cast<long long>(d.ctl->dt_bits));
}

template <class P>
__device__ __forceinline__ void finish_cell(const Dev<P>& d, int c, const double* res,
                                            double vol, int mode, int stage, double wa, double wb,
                                            int last, const CellIn& in, bool store_res = true) {
  using C = typename P::C;
  const bool residual_only = mode == kResidual || mode == kFaceParts;
  if (residual_only || (stage == 0 && store_res)) {
#pragma unroll
    for (int k = 0; k < 5; ++k) d.res[static_cast<long long>(k) * d.n + c] = res[k];
  }
  if (residual_only) return;
  const double h = in.h;
  double nu[5];
  if (mode == kRk3) {
    // rk_stage (device_stepper.cuh:93-104): next = stage - (h / V) R; stage = a u + b next.
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const long long i = static_cast<long long>(k) * d.n + c;
      const double uk = in.u[k];
      const double sk = stage == 0 ? uk : in.x[k];
      const double next = sk - h / vol * res[k];
      nu[k] = wa * uk + wb * next;
      if (last) {
        d.u[i] = nu[k];
      } else {
        d.stage[i] = nu[k];
      }
    }
  } else {
    // Classical RK4: stage_s = u - ((c_s h) / V) R_s; u = u - ((h / 6) / V) (R_0 + 2 R_1 +
    // 2 R_2 + R_3).
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const long long i = static_cast<long long>(k) * d.n + c;
      const double uk = in.u[k];
      double a;
      if (stage == 0) {
        a = res[k];
      } else if (stage < 3) {
        a = in.x[k] + 2.0 * res[k];
      } else {
        a = in.x[k] + res[k];
      }
      if (stage < 3) {
        d.racc[i] = a;
        nu[k] = uk - wa * h / vol * res[k];
      } else {
        nu[k] = uk - h / 6.0 / vol * a;
        d.u[i] = nu[k];
      }
    }
  }
  C w[5], dq[5];
  prim_of_state(d, nu, w, dq);
  store_prim<P>(d.prim_next, c, w, d.ctl);
  if (last) mark_invalid(d, c, dq, res);
}

// Gather-recompute: the faces of one owned cell (roe/hllc/ausm _faces and _boundaries), every
// face flux of the cell recomputed here and added in increasing face index from the source term
// -V s, the order in which the reference's scatter adds them (emit_cpu.py emit_loop); then
// finish_cell.
template <class P, int FLUX, bool PLANAR, bool SECOND>
__global__ void __launch_bounds__(256) k_faces_cell(Dev<P> d, int mode, int stage, double wa,
                                                    double wb, int local, int last) {
  using C = typename P::C;
  const int c = tile_item(d.cell_tiles, d.n_cell_tiles);
  if (c < 0 || c >= d.n || !cell_active(d, c)) return;
  C wc[5], gc[15], pc[5];
  cell_recon<P, SECOND>(d, c, wc, pc, gc);
  const double vol = __ldg(d.volume + c);
  double res[5];
  {
    const C nv = -static_cast<C>(vol);  // sources (:611-616): res = -V s
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const C s = d.source != nullptr ? __ldg(d.source + static_cast<long long>(k) * d.n + c) : C(0.0);
      res[k] = static_cast<double>(nv * s);
    }
  }
  const int ib = __ldg(d.inc_start + (c >> 5)) + (c & 31);
  const int il = __ldg(d.inc_len + c);
  for (int j = 0; j < il; ++j) {
    const int code = __ldg(d.inc_code + ib + static_cast<long long>(j) * kSlice);
    C out[5];
    if (code >= 0) {
      const int f = code >> 1;
      const bool left = (code & 1) == 0;
      C fr[kFace], wo[5], go[15], po[5];
      load_words<P, kFaceA32<P>>(d.face + static_cast<long long>(f) * kFace, 0, kFace, fr);
      cell_recon<P, SECOND>(d, left ? index_of(fr[11]) : index_of(fr[7]), wo, po, go);
      if (left) {
        interior_flux<P, FLUX, PLANAR>(d, f, fr, wc, gc, pc, wo, go, po, out);
#pragma unroll
        for (int k = 0; k < 5; ++k) res[k] += static_cast<double>(out[k]);
      } else {
        interior_flux<P, FLUX, PLANAR>(d, f, fr, wo, go, po, wc, gc, pc, out);
#pragma unroll
        for (int k = 0; k < 5; ++k) res[k] -= static_cast<double>(out[k]);
      }
    } else {
      const int b = -code - 1;
      C br[kBface];
      load_words<P, true>(d.bface + static_cast<long long>(b) * kBface, 0, kBface, br);
      boundary_flux<P, FLUX, PLANAR>(d, b, br, wc, gc, pc, out);
#pragma unroll
      for (int k = 0; k < 5; ++k) res[k] += static_cast<double>(out[k]);
    }
  }
  CellIn in;
  load_cell_in(d, c, mode, stage, local, in);
  finish_cell(d, c, res, vol, mode, stage, wa, wb, last, in);
}

constexpr int kFlux = 8;  // flux record width (5 used): one 32-byte sector in fp32+acc64

// The flux of owned interior face f, in its orientation, into the face scratch (none for a face
// of a stopped case).
template <class P, int FLUX, bool PLANAR, bool SECOND>
__device__ __forceinline__ void face_flux_body(const Dev<P>& d, int f, typename P::C* flux) {
  using C = typename P::C;
  C fr[kFace], wl[5], gl[15], pl[5], wr[5], gr[15], pr[5], out[8];
  load_words<P, kFaceA32<P>>(d.face + static_cast<long long>(f) * kFace, 0, kFace, fr);
  if (!cell_active(d, index_of(fr[7]))) return;
  cell_recon<P, SECOND>(d, index_of(fr[7]), wl, pl, gl);
  cell_recon<P, SECOND>(d, index_of(fr[11]), wr, pr, gr);
  interior_flux<P, FLUX, PLANAR>(d, f, fr, wl, gl, pl, wr, gr, pr, out);
  out[5] = out[6] = out[7] = C(0);
  store_words<P, true>(flux + static_cast<long long>(f) * kFlux, 0, kFlux, out);
}

// The flux of boundary face b of an owned cell into the boundary-face scratch.
template <class P, int FLUX, bool PLANAR, bool SECOND>
__device__ __forceinline__ void bface_flux_body(const Dev<P>& d, int b, typename P::C* flux) {
  using C = typename P::C;
  C br[kBface], wc[5], gc[15], pc[5], out[8];
  load_words<P, true>(d.bface + static_cast<long long>(b) * kBface, 0, kBface, br);
  if (!cell_active(d, index_of(br[13]))) return;
  cell_recon<P, SECOND>(d, index_of(br[13]), wc, pc, gc);
  boundary_flux<P, FLUX, PLANAR>(d, b, br, wc, gc, pc, out);
  out[5] = out[6] = out[7] = C(0);
  store_words<P, true>(flux + static_cast<long long>(b) * kFlux, 0, kFlux, out);
}

// Store-gather, first half (the reference's store strategy, emit_gpu.py): the flux of every owned
// interior face, once, in its orientation, into the face scratch. The fp32+acc64 forms that fit 48
// registers without spilling (planar faces, or first order) are bounded for it: 42 warps per SM at
// 64 threads a block instead of 36 at 50 registers. The non-planar second-order and fp64 forms
// spill under that bound and keep their own allocation.
template <class P, bool PLANAR, bool SECOND>
constexpr int kFaceMinBlocks = (sizeof(typename P::C) == 4 && (PLANAR || !SECOND)) ? 5 : 1;
template <class P, int FLUX, bool PLANAR, bool SECOND>
__global__ void __launch_bounds__(256, (kFaceMinBlocks<P, PLANAR, SECOND>))
    k_face_flux(Dev<P> d, typename P::C* flux) {
  const int f = tile_item(d.face_tiles, d.n_face_tiles);
  if (f < 0 || f >= d.n_if) return;
  if (d.face_warp_case != nullptr) {
    const int kc = __ldg(d.face_warp_case + (f >> 5));
    if (kc >= 0 && d.active[kc] == 0) return;
  }
  face_flux_body<P, FLUX, PLANAR, SECOND>(d, f, flux);
}

// ... and of every boundary face of an owned cell (the first n_owned_faces - n_interior_faces).
template <class P, int FLUX, bool PLANAR, bool SECOND>
__global__ void __launch_bounds__(256) k_bface_flux(Dev<P> d, typename P::C* flux, int nbo) {
  const int b = tile_item(d.bface_tiles, d.n_bface_tiles);
  if (b < 0 || b >= nbo) return;
  if (d.bface_warp_case != nullptr) {
    const int kc = __ldg(d.bface_warp_case + (b >> 5));
    if (kc >= 0 && d.active[kc] == 0) return;
  }
  bface_flux_body<P, FLUX, PLANAR, SECOND>(d, b, flux);
}

// Store-gather, second half: each owned cell adds its faces' fluxes in increasing face index
// from the source term (loads of four faces in flight at a time), then finish_cell.
// Replicated exact-sum words of the stage-0 norms (NORMS gathers): block b adds its words to
// replica b % kNormReplicas, so that the blocks' atomics spread over this many copies of each
// word; k_norm_collect sums the replicas.
constexpr int kNormReplicas = 64;

template <class P, bool NORMS>
__device__ __forceinline__ void gather_cell(const Dev<P>& d, int c, const typename P::C* flux,
                                            const typename P::C* bflux, int mode, int stage,
                                            double wa, double wb, int local, int last,
                                            double* res_out);

// Store-gather sum: each cell's face fluxes added in increasing face index from the source term,
// then the RK stage (finish_cell). NORMS (face mode 2, a step's stage 0 without batched cases):
// the squares of the stage-0 residual also go into the exact sums of the RMS norms here, per warp
// in shared memory and per block into a replica of norm_words, instead of a separate pass over a
// stored residual (which is then not stored).
template <class P, bool NORMS>
__global__ void __launch_bounds__(256) k_gather(Dev<P> d, const typename P::C* flux,
                                                const typename P::C* bflux, int mode, int stage,
                                                double wa, double wb, int local, int last,
                                                unsigned long long* norm_words) {
  if constexpr (!NORMS) {
    const int c = tile_item(d.cell_tiles, d.n_cell_tiles);
    if (c >= 0 && c < d.n && cell_active(d, c))
      gather_cell<P, false>(d, c, flux, bflux, mode, stage, wa, wb, local, last, nullptr);
  } else {
    // grid-stride over the cells (never re-packed: fused only without batched cases), so that
    // each block clears and flushes its shared words once for many cells
    extern __shared__ unsigned long long warp_words[];  // (blockDim.x / 32) x 5 x kWords
    const int nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < nw * 5 * kWords; i += blockDim.x) warp_words[i] = 0ULL;
    __syncthreads();
    unsigned long long* mine = warp_words + (threadIdx.x >> 5) * 5 * kWords;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < d.n;
         base += stride) {  // block-uniform trip count: every lane reaches the warp adds
      const long long c = base + threadIdx.x;
      double res[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      if (c < d.n && cell_active(d, static_cast<int>(c)))
        gather_cell<P, true>(d, static_cast<int>(c), flux, bflux, mode, stage, wa, wb, local,
                             last, res);
#pragma unroll
      for (int k = 0; k < 5; ++k) warp_exact_add_nonneg<true>(mine + k * kWords, res[k] * res[k]);
    }
    __syncthreads();
    unsigned long long* replica = norm_words + (blockIdx.x % kNormReplicas) * 5 * kWords;
    for (int i = threadIdx.x; i < 5 * kWords; i += blockDim.x) {
      unsigned long long v = 0;
      for (int w = 0; w < nw; ++w) v += warp_words[w * 5 * kWords + i];
      if (v != 0) atomicAdd(&replica[i], v);
    }
  }
}

template <class P, bool NORMS>
__device__ __forceinline__ void gather_cell(const Dev<P>& d, int c, const typename P::C* flux,
                                            const typename P::C* bflux, int mode, int stage,
                                            double wa, double wb, int local, int last,
                                            double* res_out) {
  using C = typename P::C;
  const double vol = __ldg(d.volume + c);
  double res[5];
  {
    const C nv = -static_cast<C>(vol);  // sources (:611-616): res = -V s
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const C s = d.source != nullptr ? __ldg(d.source + static_cast<long long>(k) * d.n + c) : C(0.0);
      res[k] = mode == kFaceParts ? 0.0 : static_cast<double>(nv * s);  // face_parts: from zero
    }
  }
  const int ib = __ldg(d.inc_start + (c >> 5)) + (c & 31);
  const int il = __ldg(d.inc_len + c);
  constexpr int kChunk = 4;
  // the codes of the next chunk load with this chunk's flux records (two dependent loads a chunk
  // otherwise: its codes, then its records)
  int code[kChunk];
#pragma unroll
  for (int q = 0; q < kChunk; ++q)
    code[q] = q < il ? __ldg(d.inc_code + ib + static_cast<long long>(q) * kSlice) : 0;
  for (int j0 = 0; j0 < il; j0 += kChunk) {
    C fv[kChunk][5];
#pragma unroll
    for (int q = 0; q < kChunk; ++q)
      if (j0 + q < il)
        load5<P>(code[q] >= 0 ? flux + static_cast<long long>(code[q] >> 1) * kFlux
                              : bflux + static_cast<long long>(-code[q] - 1) * kFlux,
                 fv[q]);
    int next[kChunk];
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
      const int j = j0 + kChunk + q;
      next[q] = j < il ? __ldg(d.inc_code + ib + static_cast<long long>(j) * kSlice) : 0;
    }
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
      if (j0 + q < il) {
        if (code[q] >= 0 && (code[q] & 1)) {
#pragma unroll
          for (int k = 0; k < 5; ++k) res[k] -= static_cast<double>(fv[q][k]);
        } else {
#pragma unroll
          for (int k = 0; k < 5; ++k) res[k] += static_cast<double>(fv[q][k]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kChunk; ++q) code[q] = next[q];
  }
  // the cell's RK inputs after the faces (not held in registers through the face loop)
  CellIn in;
  load_cell_in(d, c, mode, stage, local, in);
  finish_cell(d, c, res, vol, mode, stage, wa, wb, last, in, !NORMS);
  if constexpr (NORMS) {
#pragma unroll
    for (int k = 0; k < 5; ++k) res_out[k] = res[k];
  }
}

// The replicas of the fused stage-0 norms summed into the control's words (one block).
__global__ void k_norm_collect(const unsigned long long* replicas, Control* ctl) {
  for (int i = threadIdx.x; i < 5 * kWords; i += blockDim.x) {
    unsigned long long v = 0;
    for (int r = 0; r < kNormReplicas; ++r) v += replicas[r * 5 * kWords + i];
    (&ctl->words[0][0])[i] = v;
  }
}

// The exact sums of R_k^2 over the owned cells (SquareTerm, device_stepper.cuh:168-176): each
// warp adds into words of its own in shared memory, the block then sums its warps' words and adds
// the non-zero ones to the global words.
// With batched cases (case_of, active not null) the cells of stopped cases are left out.
__global__ void __launch_bounds__(kBlock) k_norm_sums(const double* res, int n, Control* ctl,
                                                      const int* case_of,
                                                      const unsigned char* active) {
  constexpr int kWarps = kBlock / 32;
  __shared__ unsigned long long sh[kWarps][5 * kWords];
  for (int i = threadIdx.x; i < kWarps * 5 * kWords; i += blockDim.x) (&sh[0][0])[i] = 0;
  __syncthreads();
  unsigned long long* mine = sh[threadIdx.x >> 5];
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < n; base += stride) {
    const long long c = base + threadIdx.x;
    double r[5];
    const bool in = c < n && (active == nullptr || active[case_of[c]] != 0);
#pragma unroll
    for (int k = 0; k < 5; ++k) r[k] = in ? res[k * static_cast<long long>(n) + c] : 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) warp_exact_add_nonneg<true>(mine + k * kWords, r[k] * r[k]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 5 * kWords; i += blockDim.x) {
    unsigned long long v = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) v += sh[w][i];
    if (v != 0) atomicAdd(&ctl->words[i / kWords][i % kWords], v);
  }
}

// record_norms (euler_physics.cpp:1040-1054): rms_k = sqrt(sum / N), N the owned cells (of all
// ranks on a partitioned mesh); the step's history entry.
// With record (a step's stage 0): the step's dt from its minimum's bits (for the host and the
// history; the gathers read the bits themselves) and the history entry; with advance, the step
// count too (in place of k_end_step, where nothing later in the step reads it).
__global__ void k_norm_finish(Control* ctl, double n, int record, int advance) {
  const int k = threadIdx.x;
  __shared__ double rms[5];
  if (k < 5) rms[k] = sqrt(exact_value(ctl->words[k]) / n);
  __syncthreads();
  if (k == 0) {
    const long long slot = ctl->step % kHistory;
    for (int q = 0; q < 5; ++q) {
      ctl->rms[q] = rms[q];
      if (record) ctl->hist_rms[slot][q] = rms[q];
    }
    if (record) {
      ctl->dt = __longlong_as_double(static_cast<long long>(ctl->dt_bits));
      ctl->hist_dt[slot] = ctl->dt;
    }
    if (advance) ctl->step += 1;
  }
}

// Batched cases: for each 32 consecutive face records (`width` words, the owner's index at word
// `owner`), the case of all their owners, or -1 when they span two cases.
template <class C>
__global__ void k_warp_case(const C* rec, int width, int owner, int count, const int* case_of,
                            int* out) {
  const long long f = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int kc = f < count ? case_of[index_of(rec[f * width + owner])] : -2;
  const int first = __shfl_sync(0xffffffffu, kc, 0);
  const bool same = __all_sync(0xffffffffu, kc == first || kc == -2);
  if ((threadIdx.x & 31) == 0 && f < count) out[f >> 5] = same ? first : -1;
}

// Batched cases: the exact sums of R_k^2 per case. Each block walks kCaseSpan consecutive chunks
// of blockDim.x cells: a chunk inside one case adds into words private to each warp (shared
// memory), flushed to that case's global words when the case changes and at the end; a chunk over
// a case boundary adds each warp's terms, grouped by case, to the global words of their cases.
constexpr int kCaseSpan = 8;

__global__ void __launch_bounds__(kBlock) k_case_norm_sums(const double* res, int n,
                                                           const int* case_of,
                                                           const unsigned char* active,
                                                           unsigned long long* words) {
  constexpr int kWarps = kBlock / 32;
  __shared__ unsigned long long sh[kWarps][5 * kWords];
  unsigned long long* mine = sh[threadIdx.x >> 5];
  auto clear = [&]() {
    for (int i = threadIdx.x; i < kWarps * 5 * kWords; i += blockDim.x) (&sh[0][0])[i] = 0;
  };
  auto flush = [&](int kc) {
    unsigned long long* dst = words + static_cast<long long>(kc) * 5 * kWords;
    for (int i = threadIdx.x; i < 5 * kWords; i += blockDim.x) {
      unsigned long long v = 0;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) v += sh[w][i];
      if (v != 0) atomicAdd(&dst[i], v);
    }
  };
  clear();
  __syncthreads();
  int cur = -1;
  for (int s = 0; s < kCaseSpan; ++s) {
    const long long c0 = (static_cast<long long>(blockIdx.x) * kCaseSpan + s) * blockDim.x;
    if (c0 >= n) break;
    const long long c1 = min(c0 + static_cast<long long>(blockDim.x), static_cast<long long>(n)) - 1;
    const long long c = c0 + threadIdx.x;
    const int first = case_of[c0], last = case_of[c1];
    if (first == last) {
      if (active[first] == 0) continue;  // a stopped case: nothing to add
      if (first != cur) {
        if (cur >= 0) {
          __syncthreads();
          flush(cur);
          __syncthreads();
          clear();
          __syncthreads();
        }
        cur = first;
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const double r = c < n ? res[k * static_cast<long long>(n) + c] : 0.0;
        warp_exact_add_nonneg<true>(mine + k * kWords, r * r);
      }
    } else {
      const unsigned full = 0xffffffffu;
      const int kase = c < n && active[case_of[c]] != 0 ? case_of[c] : -1;
      unsigned todo = __ballot_sync(full, kase >= 0);
      while (todo != 0) {
        const int kc = __shfl_sync(full, kase, __ffs(todo) - 1);
        const bool in = kase == kc;
        const unsigned group = __ballot_sync(full, in);
        unsigned long long* dst = words + static_cast<long long>(kc) * 5 * kWords;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const double r = in ? res[k * static_cast<long long>(n) + c] : 0.0;
          warp_exact_add_nonneg(dst + k * kWords, r * r);
        }
        todo &= ~group;
      }
    }
  }
  __syncthreads();
  if (cur >= 0) flush(cur);
}

// The global exact words of a batched step from its cases' words (a sum of integers: the same
// total as a pass over the active cells), before k_case_norm_finish clears them.
__global__ void k_case_words_total(const unsigned long long* case_words, int n_cases,
                                   Control* ctl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 5 * kWords; i += gridDim.x * blockDim.x) {
    unsigned long long v = 0;
    for (int kc = 0; kc < n_cases; ++kc) v += case_words[static_cast<long long>(kc) * 5 * kWords + i];
    (&ctl->words[0][0])[i] = v;
  }
}

// Per case and equation (q = 5 case + k): rms = sqrt(sum / cells of the case) into this step's
// row of the case history; the words are cleared for the next step.
__global__ void k_case_norm_finish(unsigned long long* words, const double* cells, int n_cases,
                                   const Control* ctl, double* hist) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 5 * n_cases) return;
  unsigned long long* w = words + static_cast<long long>(q) * kWords;
  const double rms = sqrt(exact_value(w) / cells[q / 5]);
  hist[(ctl->step % kHistory) * 5LL * n_cases + q] = rms;
  for (int i = 0; i < kWords; ++i) w[i] = 0;
}

// The start of a step: clears the sums and the validity marks, sets the global step (fixed) or
// prepares its minimum (CFL).
__global__ void k_begin(Control* ctl, double dt_fixed, unsigned long long* norm_replicas) {
  const int t = threadIdx.x;
  for (int i = t; i < 5 * kWords; i += blockDim.x) (&ctl->words[0][0])[i] = 0;
  if (norm_replicas != nullptr)
    for (int i = t; i < kNormReplicas * 5 * kWords; i += blockDim.x) norm_replicas[i] = 0;
  if (t == 0) {
    ctl->dt_bits = dt_fixed > 0.0 ? static_cast<unsigned long long>(__double_as_longlong(dt_fixed))
                                  : 0x7ff0000000000000ULL;
    ctl->bad_state = ~0ULL;
    ctl->bad_res = ~0ULL;
  }
}

__global__ void k_end_step(Control* ctl) {
  if (threadIdx.x == 0) ctl->step += 1;
}

// Ghost exchange of a partitioned mesh (the forward halo exchange's pack and unpack,
// partition/include/autan/partition/halo_exchange.hpp:18-31): records of `groups` groups of
// kGroup words, group g of cell c at base + g gstride + kGroup c. PACK: the records of cells[i]
// into buf record after record; else the records buf[i] into the cells first + i. One thread per
// 16-byte piece (group strides, records and buf are 16-byte aligned).
template <class C, bool PACK>
__global__ void k_halo_records(C* base, long long gstride, int groups, const int* cells,
                               long long count, int first, C* buf) {
  constexpr int kPieces = kGroup * static_cast<int>(sizeof(C)) / 16;
  const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long per = static_cast<long long>(groups) * kPieces;
  if (t >= count * per) return;
  const long long i = t / per;
  const int r = static_cast<int>(t - i * per);
  const int g = r / kPieces, q = r % kPieces;
  const long long c = PACK ? static_cast<long long>(cells[i]) : first + i;
  uint4* rec = reinterpret_cast<uint4*>(base + g * gstride + c * kGroup) + q;
  uint4* packed = reinterpret_cast<uint4*>(buf + (i * groups + g) * kGroup) + q;
  if constexpr (PACK) {
    *packed = *rec;
  } else {
    *rec = *packed;
  }
}

// Gradients and limiter of the reconstruction array, as FP64 SoA (15 x n, 5 x n).
template <class P>
__global__ void k_unpack(const typename P::C* recon, int n, long long rstride, double* grad,
                         double* phi) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  auto word = [&](int w) {
    return static_cast<double>(recon[(w / kGroup) * rstride +
                                     static_cast<long long>(c) * kGroup + w % kGroup]);
  };
  for (int k = 0; k < 15; ++k) grad[static_cast<long long>(k) * n + c] = word(5 + k);
  for (int k = 0; k < 5; ++k) phi[static_cast<long long>(k) * n + c] = word(k);
}

// The face scratch as FP64 face fluxes, 5 x nf (owned interior faces, then owned boundary faces
// at ni + b): the write-only loops' face_flux (kernels/euler.py:1059-1085).
template <class P>
__global__ void k_unpack_flux(const typename P::C* flux, const typename P::C* bflux, int nif,
                              int nbo, int ni, int nf, double* out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nif) {
    for (int k = 0; k < 5; ++k)
      out[static_cast<long long>(k) * nf + i] = static_cast<double>(flux[i * kFlux + k]);
  } else if (i < static_cast<long long>(nif) + nbo) {
    const long long b = i - nif;
    for (int k = 0; k < 5; ++k)
      out[static_cast<long long>(k) * nf + ni + b] = static_cast<double>(bflux[b * kFlux + k]);
  }
}

// Euler<P>::boundary_pressure (physics/src/euler.cpp:1182-1223) for every boundary face, in FP64
// from the stored primitives, gradient and limiter of its owner: the face pressure
// p_f = p_c + phi_p (grad p . (x_f - x_c)), p_c when rho_f or p_f is not positive, and the force
// p_f S + phi_p M^T grad p. r64: the FP64 offsets x_f - x_c, 3 x nb; pref: p_ref in FP64.
template <class P>
__global__ void __launch_bounds__(kBlock) k_boundary_pressure(Dev<P> d, const double* r64,
                                                              int second, double pref, double* p,
                                                              double* force) {
  using C = typename P::C;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  const long long nb = d.nb;
  const C* br = d.bface + static_cast<long long>(b) * kBface;
  const int o = index_of(br[13]);
  C w[5], phi[5], g[15];
  if (second) {
    load_recon<P>(d, o, w, phi, g);
  } else {
    // set_second_order(false) zeroes grad and phi (physics/src/euler.cpp:903-912).
    load_prim<P>(d.prim, o, w);
#pragma unroll
    for (int k = 0; k < 5; ++k) phi[k] = C(0);
#pragma unroll
    for (int k = 0; k < 15; ++k) g[k] = C(0);
  }
  double drho = 0.0, dp = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double r = r64[j * nb + b];
    drho += static_cast<double>(g[j]) * r;
    dp += static_cast<double>(g[12 + j]) * r;
  }
  const double rho_c = static_cast<double>(w[0]);
  const double p_c = pref + static_cast<double>(w[4]);
  const double rho_f = rho_c + static_cast<double>(phi[0]) * drho;
  double p_f = p_c + static_cast<double>(phi[4]) * dp;
  if (!(rho_f > 0.0 && p_f > 0.0)) p_f = p_c;
  p[b] = p_f;
  if (force == nullptr) return;
  const double phi_p = static_cast<double>(phi[4]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double warp = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const C m = d.b_m != nullptr ? d.b_m[(3 * j + k) * nb + b] : C(0);
      warp += static_cast<double>(m) * static_cast<double>(g[12 + j]);
    }
    const double area_k = static_cast<double>(br[k]) * static_cast<double>(br[3]);
    force[k * nb + b] = p_f * area_k + phi_p * warp;
  }
}

// The sums of EulerPhysics::check_conservation (physics/src/euler_physics.cpp:1747-1779) on one
// rank, each exact: words of E_k (R^F and minus the boundary fluxes), D_k (|flux| per incidence of
// an owned cell: `mult` incidences of each owned interior face, one of each owned boundary face),
// boundary_k and faces_k, 20 x kWords in that order. res: the face parts of the owned cells.
template <class P>
__global__ void __launch_bounds__(kBlock) k_conservation(Dev<P> d, const typename P::C* flux,
                                                         const typename P::C* bflux,
                                                         const unsigned char* mult, int nbo,
                                                         unsigned long long* words) {
  __shared__ unsigned long long sh[20 * kWords];
  for (int i = threadIdx.x; i < 20 * kWords; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const long long total = max(max(static_cast<long long>(d.n), static_cast<long long>(d.n_if)),
                              static_cast<long long>(nbo));
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x; base < total;
       base += stride) {
    const long long i = base + threadIdx.x;
    const int mu = i < d.n_if ? mult[i] : 0;
    for (int k = 0; k < 5; ++k) {
      const double r = i < d.n ? d.res[k * static_cast<long long>(d.n) + i] : 0.0;
      const double fb = i < nbo ? static_cast<double>(bflux[i * kFlux + k]) : 0.0;
      const double fi = i < d.n_if ? static_cast<double>(flux[i * kFlux + k]) : 0.0;
      warp_exact_add(sh + k * kWords, r);
      warp_exact_add(sh + k * kWords, -fb);
      warp_exact_add(sh + (5 + k) * kWords, fabs(fb));
      warp_exact_add(sh + (5 + k) * kWords, mu >= 1 ? fabs(fi) : 0.0);
      warp_exact_add(sh + (5 + k) * kWords, mu >= 2 ? fabs(fi) : 0.0);
      warp_exact_add(sh + (10 + k) * kWords, fb);
      warp_exact_add(sh + (15 + k) * kWords, r);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 20 * kWords; i += blockDim.x) {
    const unsigned long long v = sh[i];
    if (v != 0) atomicAdd(&words[i], v);
  }
}

__global__ void k_conservation_finish(const unsigned long long* words, double* out) {
  const int q = threadIdx.x;
  if (q < 20) out[q] = exact_value(words + q * kWords);
}

// ---------------------------------------------------------------- host side

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const std::string& what) { throw Failure(what); }

// A failed CUDA call: the runtime's (non-sticky) last-error state is cleared before reporting, so
// that the next launch's check sees that launch's own result.
void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(std::string("E1200: ") + what + ": " + cudaGetErrorString(e));
  }
}

class Buffer {
 public:
  Buffer() = default;
  explicit Buffer(size_t bytes) { alloc(bytes); }
  Buffer(const Buffer&) = delete;
  Buffer& operator=(const Buffer&) = delete;
  Buffer(Buffer&& o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  Buffer& operator=(Buffer&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  ~Buffer() {
    if (p_ != nullptr) cudaFree(p_);
  }
  void alloc(size_t bytes) {
    if (p_ != nullptr) cudaFree(p_);
    p_ = nullptr;
    n_ = bytes;
    if (bytes > 0) check(cudaMalloc(&p_, bytes), "cudaMalloc");
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p_);
  }
  void* ptr() const { return p_; }
  size_t bytes() const { return n_; }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
};

template <class T>
Buffer upload(const std::vector<T>& v, cudaStream_t s) {
  Buffer b(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!v.empty())
    check(cudaMemcpyAsync(b.ptr(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s),
          "upload");
  return b;
}

// Sliced (ELLPACK by slices of 32) positions of CSR rows.
struct Sliced {
  std::vector<int> start;  // per slice
  std::vector<int> len;    // per row
  long long total = 0;
  long long at(int row, int j) const {
    return static_cast<long long>(start[row / kSlice]) + static_cast<long long>(j) * kSlice +
           row % kSlice;
  }
};

Sliced slice_rows(const std::vector<long long>& off) {
  Sliced s;
  const int n = static_cast<int>(off.size()) - 1;
  s.len.assign(std::max(n, 1), 0);
  s.start.assign((n + kSlice - 1) / kSlice + 1, 0);
  long long run = 0;
  for (int sl = 0; sl * kSlice < n; ++sl) {
    long long longest = 0;
    for (int l = 0; l < kSlice && sl * kSlice + l < n; ++l) {
      const int r = sl * kSlice + l;
      s.len[r] = static_cast<int>(off[r + 1] - off[r]);
      longest = std::max(longest, off[r + 1] - off[r]);
    }
    s.start[sl] = static_cast<int>(run);
    run += longest * kSlice;
    // Slice starts are int32 entries (word offsets, 4 per entry, are formed in 64 bits).
    if (run >= std::numeric_limits<int>::max() - 2 * kSlice)
      fail("E1101: stencil too large for int32 offsets");
  }
  s.start.back() = static_cast<int>(run);
  s.total = run;
  return s;
}

template <class C>
C index_bits(int i) {
  C x;
  if constexpr (sizeof(C) == 4) {
    std::memcpy(&x, &i, 4);
  } else {
    const long long l = i;
    std::memcpy(&x, &l, 8);
  }
  return x;
}

struct Counters {
  long long launches = 0, steps = 0, residuals = 0;
};

// Launch choices of the hot kernels; every choice computes the same bits (the summation order of
// each cell is fixed), so the autotuner picks by time alone.
struct Tuning {
  int grad_chunk = 4;    // stencil entries loaded together by the gradient kernel: 1, 2, 4 (8 staged)
  int grad_block = 128;  // its threads per block
  int face_mode = 1;     // 0: gather-recompute (each cell computes its faces' fluxes); 1: store-gather;
                         // 2: store-gather with a step's stage-0 norms summed in its gather
  int face_block = 128;  // threads per block of the face-flux (or gather-recompute) kernel
  int gather_block = 256;  // threads per block of the store-gather sum
  int grad_mode = 1;     // 0: stencil rows loaded by each thread; 1: staged by TMA bulk copies;
                         // 2: loaded by each thread, software-pipelined (chunk unused);
                         // 3: a per-thread ring of asynchronous copies, chunk entries deep;
                         // 4 (fp32+acc64): loaded by each thread with the products widened on the
                         // integer pipe (grad_widen), 5-word gathers (grad_narrow), registers
                         // bounded for grad_minb blocks of 128 per SM (chunk 2: 7 or 6; chunk 4: 5);
                         // 5 (fp32+acc64): each warp's stencil rows streamed by TMA bulk copies
                         // into a ring of grad_depth shared-memory slots, grad_chunk gathers in
                         // flight (5-word with grad_narrow)
  int grad_widen = 0;    // mode 4: products widened by widen_scaled: 0 none, 1 x and y, 2 all
  int grad_narrow = 0;   // mode 4: 1 gathers neighbours as 16 + 4 bytes instead of 32
  int grad_minb = 7;     // mode 4: blocks of 128 threads per SM the registers are bounded for
  int grad_depth = 4;    // mode 5: entries each warp's row ring holds (4 or 8)
  static constexpr int kCount = 10;
  static constexpr int kMinCount = 6;  // callers that predate mode 4 pass the first six
  void to(int32_t* p) const {
    p[0] = grad_chunk;
    p[1] = grad_block;
    p[2] = face_mode;
    p[3] = face_block;
    p[4] = gather_block;
    p[5] = grad_mode;
    p[6] = grad_widen;
    p[7] = grad_narrow;
    p[8] = grad_minb;
    p[9] = grad_depth;
  }
  static Tuning from(const int32_t* p, int count = kCount) {
    Tuning t;
    t.grad_chunk = p[0];
    t.grad_block = p[1];
    t.face_mode = p[2];
    t.face_block = p[3];
    t.gather_block = p[4];
    t.grad_mode = p[5];
    if (count >= kCount) {
      t.grad_widen = p[6];
      t.grad_narrow = p[7];
      t.grad_minb = p[8];
      t.grad_depth = p[9];
    }
    t.validate();
    return t;
  }
  void validate() const;
};

void Tuning::validate() const {
  auto block_ok = [](int b) { return b >= 32 && b <= 256 && b % 32 == 0; };
  if (grad_mode == 0 && grad_chunk != 1 && grad_chunk != 2 && grad_chunk != 4)
    fail("E1101: grad_chunk is 1, 2 or 4");
  if (grad_mode == 0 && grad_chunk == 2 && grad_block > 128)
    fail("E1101: the gradient kernel with 2 entries in flight takes <= 128 threads");
  if (grad_mode == 1 && grad_chunk != 2 && grad_chunk != 4 && grad_chunk != 8)
    fail("E1101: grad_chunk of the staged kernel is 2, 4 or 8");
  if (face_mode < 0 || face_mode > 2) fail("E1101: face_mode is 0, 1 or 2");
  if (grad_mode == 3 && grad_chunk != 2 && grad_chunk != 4 && grad_chunk != 8)
    fail("E1101: grad_chunk of the ring kernel is 2, 4 or 8");
  if (grad_mode < 0 || grad_mode > 5) fail("E1101: grad_mode is 0 to 5");
  if (grad_mode == 5) {
    if (grad_block != 128) fail("E1101: the mode-5 gradient kernel takes 128 threads");
    if (grad_chunk != 2 && grad_chunk != 3) fail("E1101: grad_chunk of mode 5 is 2 or 3");
    if (grad_depth != 4 && grad_depth != 8) fail("E1101: grad_depth is 4 or 8");
    if (grad_narrow != 0 && grad_narrow != 1) fail("E1101: grad_narrow is 0 or 1");
  }
  if (grad_mode == 4) {
    if (grad_block != 128) fail("E1101: the mode-4 gradient kernel takes 128 threads");
    if (grad_widen < 0 || grad_widen > 2) fail("E1101: grad_widen is 0, 1 or 2");
    if (grad_narrow != 0 && grad_narrow != 1) fail("E1101: grad_narrow is 0 or 1");
    if (!((grad_chunk == 2 && (grad_minb == 7 || grad_minb == 6)) || (grad_chunk == 4 && grad_minb == 5)))
      fail("E1101: mode 4 takes grad_chunk 2 with grad_minb 7 or 6, or grad_chunk 4 with grad_minb 5");
  }
  if (grad_mode == 3 && grad_block > 128) fail("E1101: the ring gradient kernel takes <= 128 threads");
  if (grad_mode == 1 && grad_block > 128) fail("E1101: the staged gradient kernel takes <= 128 threads");
  if (!block_ok(grad_block) || !block_ok(face_block) || !block_ok(gather_block))
    fail("E1101: block sizes are multiples of 32 in [32, 256]");
}

class Stepper {
 public:
  virtual ~Stepper() = default;
  virtual void set_boundary(const uint8_t* kind, const double* data) = 0;
  virtual void set_boundary_data(const double* data) = 0;
  virtual void set_source(const double* source) = 0;
  virtual void set_second_order(bool on) = 0;
  virtual void upload_state(const double* u) = 0;
  virtual void download_state(double* u) = 0;
  virtual void residual(const double* u, double* res) = 0;
  virtual void step(double cfl, double dt, bool local, int rk, long long n, bool graph,
                    autan_euler_step_result* out) = 0;
  virtual void evaluate(autan_euler_step_result* out) = 0;
  virtual void history(long long count, double* rms, double* dt) = 0;
  virtual void gradients(double* grad, double* phi) = 0;
  virtual void time_steps(double cfl, double* dt) = 0;
  virtual long long device_bytes() const = 0;
  virtual void kernel_times(double cfl, double dt, bool local, int rk, long long n, double* ms,
                            long long* launches) = 0;
  virtual void set_tuning(const Tuning& t) = 0;
  virtual Tuning tuning() const = 0;
  virtual double autotune(double cfl, double dt, bool local, int rk, int trial_steps) = 0;
  virtual void face_parts(const double* u, double* res_faces, double* face_flux) = 0;
  virtual void boundary_pressure(const double* u, double* p, double* force) = 0;
  virtual int conservation(double* sums) = 0;
  virtual void set_cases(int n_cases, const int64_t* cell_offsets) = 0;
  virtual void set_active(const uint8_t* active) = 0;
  virtual void set_case_mach_ref(const double* mach_ref) = 0;
  virtual void case_history(long long count, double* rms) = 0;
  virtual int n_cases() const = 0;
  virtual void set_stall_test(int polls) = 0;
  virtual void set_ranks(const autan_euler_ranks* ranks) = 0;
  // Whether any rank has `mine` set (this rank's alone without ranks): a stop every rank of a
  // partitioned march takes together.
  virtual bool any_rank(bool mine) = 0;
  virtual long long external_ghosts() const = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  Counters counters;
};

template <class P>
class Impl final : public Stepper {
  using C = typename P::C;

 public:
  Impl(const autan_euler_mesh& m, const autan_euler_scheme& sc, cudaStream_t st)
      : scheme_(sc), planar_(sc.planar != 0), second_(sc.second_order != 0),
        limiter_(sc.limiter != 0) {
    stream = st;
    nc_ = m.n_cells;
    n_ = m.n_owned_cells;
    nf_ = m.n_faces;
    ni_ = m.n_interior_faces;
    nif_ = m.n_owned_interior_faces;
    nb_ = m.n_faces - m.n_interior_faces;
    validate(m);
    // Value index of every mesh cell: owned cells themselves, images their owned cell, external
    // ghosts (ghost_owner -1: another rank's cell) records of their own after the owned cells'.
    std::vector<int> val(nc_);
    for (int c = 0; c < n_; ++c) val[c] = c;
    for (int g = n_; g < nc_; ++g)
      if (m.ghost_owner[g - n_] == -1) val[g] = n_ + n_ext_++;
    nv_ = n_ + n_ext_;
    for (int g = n_; g < nc_; ++g) {
      const int o = m.ghost_owner[g - n_];
      if (o == -1) continue;
      if (o < 0 || o >= n_) fail("E1101: a ghost cell's owner is not an owned cell");
      val[g] = o;
    }
    // Parameters (physics/src/euler.cpp:229-245).
    const double* r = sc.reference;
    if (!(r[0] > 0.0)) fail("E1101: reference density must be positive");
    if (!(sc.mach_ref > 0.0)) fail("E1101: AUSM+-up needs a positive cut-off Mach number");
    const double p_ref =
        (sc.gamma - 1.0) * (r[4] - 0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / r[0]);
    const double k3 = std::pow(sc.venkat_k / sc.length, 3);
    Params<C>& p = d_.p;
    p.g = static_cast<C>(sc.gamma);
    p.rgas = static_cast<C>(sc.gas_constant);
    p.pref = static_cast<C>(p_ref);
    pref64_ = p_ref;
    p.minf = static_cast<C>(sc.mach_ref);
    for (int k = 0; k < 5; ++k) {
      p.ur[k] = static_cast<C>(r[k]);
      p.scale[k] = static_cast<C>(k3 * sc.scale[k] * sc.scale[k]);
      d_.ref[k] = r[k];
    }
    if (planar_ && m.face_moment != nullptr) {
      for (long long i = 0; i < 9LL * nf_; ++i)
        if (m.face_moment[i] != 0.0)
          fail("E1101: planar loops on a mesh with a face not proven planar");
    }
    const long long NF = nf_, NC = nc_;
    // Interior face records.
    std::vector<C> face(static_cast<size_t>(kFace) * std::max(nif_, 1), C(0));
    std::vector<C> fm(planar_ ? 0 : 9LL * nif_);
    for (int f = 0; f < nif_; ++f) {
      const int l = m.owner[f], rr = m.neighbour[f];
      C* q = face.data() + static_cast<long long>(f) * kFace;
      for (int a = 0; a < 3; ++a) {
        q[a] = static_cast<C>(m.face_normal[a * NF + f]);
        const double xf = m.face_centroid[a * NF + f];
        q[4 + a] = static_cast<C>(xf - m.cell_centroid[a * NC + l]);
        q[8 + a] = static_cast<C>(xf - m.cell_centroid[a * NC + rr]);
      }
      q[3] = static_cast<C>(m.face_area_magnitude[f]);
      q[7] = index_bits<C>(val[l]);
      q[11] = index_bits<C>(val[rr]);
      if (!planar_)
        for (int j = 0; j < 9; ++j)
          fm[j * static_cast<long long>(nif_) + f] =
              m.face_moment != nullptr ? static_cast<C>(m.face_moment[j * NF + f]) : C(0);
    }
    // Boundary face records (all of them: the stencils of owned cells reach those of images).
    bface_host_.assign(static_cast<size_t>(kBface) * std::max(nb_, 1), C(0));
    std::vector<C> bm(planar_ ? 0 : 9LL * nb_);
    for (int b = 0; b < nb_; ++b) {
      const int f = ni_ + b;
      const int o = m.owner[f];
      C* q = bface_host_.data() + static_cast<long long>(b) * kBface;
      for (int a = 0; a < 3; ++a) {
        q[a] = static_cast<C>(m.face_normal[a * NF + f]);
        q[4 + a] = static_cast<C>(m.face_centroid[a * NF + f] - m.cell_centroid[a * NC + o]);
      }
      q[3] = static_cast<C>(m.face_area_magnitude[f]);
      q[7] = C(2);  // slip until set_boundary
      q[13] = index_bits<C>(val[o]);
      if (!planar_)
        for (int j = 0; j < 9; ++j)
          bm[j * static_cast<long long>(nb_) + b] =
              m.face_moment != nullptr ? static_cast<C>(m.face_moment[j * NF + f]) : C(0);
    }
    // Incidences of owned cells, in increasing face index, sliced.
    std::vector<long long> ioff(n_ + 1);
    for (int c = 0; c <= n_; ++c) ioff[c] = m.cell_face_offsets[c];
    inc_ = slice_rows(ioff);
    std::vector<int> code(std::max<long long>(inc_.total, 1), 0);
    std::vector<C> irec(4 * std::max<long long>(inc_.total, 1), C(0));
    std::vector<C> idt(4 * std::max<long long>(inc_.total, 1), C(0));
    for (int c = 0; c < n_; ++c) {
      int prev = -1;
      for (long long k = ioff[c]; k < ioff[c + 1]; ++k) {
        const int f = m.cell_faces[k];
        if (f <= prev) fail("E1101: cell_faces must list each cell's faces in increasing order");
        prev = f;
        int v = 0;
        if (f < ni_) {
          if (f >= nif_) fail("E1101: an owned cell's interior face lies beyond the owned faces");
          if (m.owner[f] == c) {
            v = 2 * f;
          } else if (m.neighbour[f] == c) {
            v = 2 * f + 1;
          } else {
            fail("E1101: cell_faces lists a face of another cell");
          }
        } else {
          if (f >= m.n_owned_faces) fail("E1101: an owned cell's boundary face lies beyond the owned faces");
          if (m.owner[f] != c) fail("E1101: cell_faces lists a boundary face of another cell");
          v = -(f - ni_ + 1);
        }
        const long long at = inc_.at(c, static_cast<int>(k - ioff[c]));
        code[at] = v;
        // The limiter's offset rel(x_f, x_c), as the face record holds it for this side.
        const C* rel = v >= 0 ? face.data() + static_cast<long long>(f) * kFace + ((v & 1) ? 8 : 4)
                              : bface_host_.data() + static_cast<long long>(f - ni_) * kBface + 4;
        for (int a = 0; a < 3; ++a) irec[4 * at + a] = rel[a];
        // The other side: the owner for the neighbour's incidence and the reverse, or the face.
        const C* q = v >= 0 ? face.data() + static_cast<long long>(f) * kFace
                            : bface_host_.data() + static_cast<long long>(f - ni_) * kBface;
        irec[4 * at + 3] = v >= 0 ? ((v & 1) ? q[7] : q[11]) : index_bits<C>(nv_ + (f - ni_));
        for (int a = 0; a < 4; ++a) idt[4 * at + a] = q[a];
      }
    }
    // Stencil of owned cells, sliced, each entry {w_x, w_y, w_z, record}: the record of a cell
    // value (its value index) or of boundary face b's state (n + external ghosts + b).
    const bool has_stencil =
        m.stencil != nullptr && m.stencil_offsets != nullptr && m.stencil_lsq_weight != nullptr;
    std::vector<long long> soff(n_ + 1, 0);
    if (has_stencil)
      for (int c = 0; c <= n_; ++c) soff[c] = m.stencil_offsets[c] - m.stencil_offsets[0];
    st_ = slice_rows(soff);
    const long long nst = has_stencil ? m.stencil_offsets[nc_] : 0;
    std::vector<C> ste(4 * std::max<long long>(st_.total, 1), C(0));
    bool weights_in_range = true;  // finite and below 2^40: the gradient's scaled widening holds
    for (int c = 0; c < (has_stencil ? n_ : 0); ++c) {
      for (long long k = m.stencil_offsets[c]; k < m.stencil_offsets[c + 1]; ++k) {
        const int e = m.stencil[k];
        int v;
        if (e >= 0) {
          if (e >= nc_) fail("E1101: a stencil entry is out of range");
          v = val[e];
        } else {
          const int f = -e - 1;
          if (f < ni_ || f >= nf_) fail("E1101: a stencil entry is not a boundary face");
          v = nv_ + (f - ni_);  // the boundary state's record, after the cells' records
        }
        C* q = ste.data() + 4 * st_.at(c, static_cast<int>(k - m.stencil_offsets[c]));
        for (int a = 0; a < 3; ++a) {
          q[a] = static_cast<C>(m.stencil_lsq_weight[a * nst + k]);
          if (!(std::fabs(static_cast<double>(q[a])) < 0x1p40)) weights_in_range = false;
        }
        q[3] = index_bits<C>(v);
      }
    }
    std::vector<double> vol(m.cell_volume, m.cell_volume + n_);
    nbo_ = m.n_owned_faces - m.n_interior_faces;
    // Boundary pressure and conservation data: the FP64 offsets x_f - x_o of every boundary face
    // (3 x nb), the owned cells of each owned interior face (1 or 2: an image counts as not
    // owned) and the most faces of an owned cell.
    std::vector<double> r64(3ULL * std::max(nb_, 1), 0.0);
    for (int b = 0; b < nb_; ++b) {
      const int f = ni_ + b, o = m.owner[f];
      for (int a = 0; a < 3; ++a)
        r64[a * static_cast<long long>(nb_) + b] = m.face_centroid[a * NF + f] - m.cell_centroid[a * NC + o];
    }
    std::vector<unsigned char> mult(std::max(nif_, 1), 0);
    for (int f = 0; f < nif_; ++f)
      mult[f] = static_cast<unsigned char>((m.owner[f] < n_ ? 1 : 0) + (m.neighbour[f] < n_ ? 1 : 0));
    for (int c = 0; c < n_; ++c)
      max_faces_ = std::max<int>(max_faces_, static_cast<int>(m.cell_face_offsets[c + 1] - m.cell_face_offsets[c]));
    // Device arrays.
    const size_t n5 = 5ULL * n_;
    // each primitive buffer holds the owned cells' records, the external ghosts', then the
    // boundary faces' states; the reconstruction array the cells' and the external ghosts'
    for (auto& b : prim_) b.alloc(static_cast<size_t>(kPrimW) * (nv_ + std::max(nb_, 1)) * sizeof(C));
    recon_.alloc(static_cast<size_t>(kRecon) * nv_ * sizeof(C));
    u_.alloc(n5 * sizeof(double));
    stage_.alloc(n5 * sizeof(double));
    racc_.alloc(n5 * sizeof(double));
    res_.alloc(n5 * sizeof(double));
    dt_local_.alloc(std::max(n_, 1) * sizeof(double));
    ctl_.alloc(sizeof(Control));
    volume_ = upload(vol, stream);
    st_start_ = upload(st_.start, stream);
    st_len_ = upload(st_.len, stream);
    st_e_ = upload(ste, stream);
    inc_start_ = upload(inc_.start, stream);
    inc_len_ = upload(inc_.len, stream);
    inc_code_ = upload(code, stream);
    inc_rec_ = upload(irec, stream);
    bface_r64_ = upload(r64, stream);
    face_mult_ = upload(mult, stream);
    cons_words_.alloc(20ULL * kWords * sizeof(unsigned long long));
    norm_words_.alloc(static_cast<size_t>(kNormReplicas) * 5 * kWords * sizeof(unsigned long long));
    check(cudaMemsetAsync(norm_words_.ptr(), 0, norm_words_.bytes(), stream), "memset");
    inc_dt_ = upload(idt, stream);
    face_ = upload(face, stream);
    f_m_ = upload(fm, stream);
    bface_ = upload(bface_host_, stream);
    b_m_ = upload(bm, stream);
    for (Buffer* b : {&u_, &stage_, &racc_, &res_, &dt_local_, &ctl_})
      check(cudaMemsetAsync(b->ptr(), 0, b->bytes(), stream), "memset");
    for (auto& b : prim_) check(cudaMemsetAsync(b.ptr(), 0, b.bytes(), stream), "memset");
    check(cudaMemsetAsync(recon_.ptr(), 0, recon_.bytes(), stream), "memset");
    d_.n = n_;
    d_.nb = nb_;
    d_.n_if = nif_;
    d_.prim_b = prim_[0].as<C>() + static_cast<long long>(kPrimW) * nv_;
    d_.recon = recon_.as<C>();
    d_.rstride = static_cast<long long>(kGroup) * nv_;
    d_.u = u_.as<double>();
    d_.stage = stage_.as<double>();
    d_.racc = racc_.as<double>();
    d_.res = res_.as<double>();
    d_.volume = volume_.as<double>();
    d_.dt_local = dt_local_.as<double>();
    d_.source = nullptr;
    d_.st_start = st_start_.as<int>();
    d_.st_len = st_len_.as<int>();
    d_.st = st_e_.as<C>();
    d_.inc_start = inc_start_.as<int>();
    d_.inc_len = inc_len_.as<int>();
    d_.inc_code = inc_code_.as<int>();
    d_.inc_rec = inc_rec_.as<C>();
    d_.inc_dt = inc_dt_.as<C>();
    d_.n_slices = slices();
    d_.face = face_.as<C>();
    d_.bface = bface_.as<C>();
    // No moments on a planar mesh: the pointers stay null (their buffers hold one placeholder
    // element), so that a kernel guarded by a null test never reads past them.
    d_.f_m = planar_ ? nullptr : f_m_.as<C>();
    d_.b_m = planar_ ? nullptr : b_m_.as<C>();
    d_.ctl = ctl_.as<Control>();
    d_.case_of = nullptr;
    d_.active = nullptr;
    d_.face_warp_case = nullptr;
    d_.bface_warp_case = nullptr;
    d_.case_minf = nullptr;
    d_.cell_tiles = d_.face_tiles = d_.bface_tiles = nullptr;
    d_.n_cell_tiles = d_.n_face_tiles = d_.n_bface_tiles = 0;
    d_.wide_ok = (sizeof(C) == 4 && weights_in_range) ? 1 : 0;
    wide_ok_mesh_ = d_.wide_ok;
    d_.stall_polls = 0;
    check(cudaMallocHost(reinterpret_cast<void**>(&head_), kControlHead), "cudaMallocHost");
    if (tuning_.face_mode != 0) ensure_flux_scratch();
    check(cudaStreamSynchronize(stream), "create");
  }

  ~Impl() override {
    drop_graph();
    if (head_ != nullptr) cudaFreeHost(head_);
  }

  long long device_bytes() const override {
    long long t = 0;
    for (const Buffer* b : {&u_, &stage_, &racc_, &res_, &dt_local_, &ctl_, &volume_,
                            &st_start_, &st_len_, &st_e_, &inc_start_, &inc_len_, &inc_code_,
                            &face_, &f_m_, &bface_, &b_m_, &source_, &flux_, &bflux_,
                            &inc_rec_, &inc_dt_, &bface_r64_, &face_mult_, &cons_words_})
      t += static_cast<long long>(b->bytes());
    for (const auto& b : prim_) t += static_cast<long long>(b.bytes());
    t += static_cast<long long>(recon_.bytes());
    return t;
  }

  void set_boundary(const uint8_t* kind, const double* data) override {
    for (int b = 0; b < nb_; ++b) {
      if (kind[b] > 5) fail("E1101: boundary code out of range");
      bface_host_[static_cast<long long>(b) * kBface + 7] = static_cast<C>(kind[b]);
    }
    set_boundary_data(data);
    drop_graph();
  }

  void set_boundary_data(const double* data) override {
    for (int b = 0; b < nb_; ++b)
      for (int k = 0; k < 5; ++k)
        bface_host_[static_cast<long long>(b) * kBface + 8 + k] =
            static_cast<C>(data[k * static_cast<long long>(nb_) + b]);
    check(cudaMemcpyAsync(bface_.ptr(), bface_host_.data(), bface_host_.size() * sizeof(C),
                          cudaMemcpyHostToDevice, stream), "boundary data");
    check(cudaStreamSynchronize(stream), "boundary data");
  }

  void set_source(const double* source) override {
    std::vector<C> v(5ULL * n_);
    bool any = false;
    for (int k = 0; k < 5; ++k)
      for (int c = 0; c < n_; ++c) {
        v[k * static_cast<long long>(n_) + c] = static_cast<C>(source[k * static_cast<long long>(nc_) + c]);
        any = any || v[k * static_cast<long long>(n_) + c] != C(0);
      }
    if (!any) {
      source_ = Buffer();
      d_.source = nullptr;
    } else {
      source_ = upload(v, stream);
      d_.source = source_.as<C>();
      check(cudaStreamSynchronize(stream), "source");
    }
    drop_graph();
  }

  void set_second_order(bool on) override {
    // As the host (physics/src/euler.cpp:903-912): without reconstruction the faces read no
    // gradients or limiter; unlimited, phi is 1 (written by the gradient kernel).
    second_ = on;
    drop_graph();
  }

  // Host state (5 x n_cells, caller-owned; pinned memory makes the copies asynchronous DMA):
  // one copy per component, of the owned cells.
  void copy_in(const double* host, double* dev) {
    const size_t per = static_cast<size_t>(n_) * sizeof(double);
    for (int k = 0; k < 5; ++k)
      check(cudaMemcpyAsync(dev + k * static_cast<long long>(n_), host + k * static_cast<long long>(nc_),
                            per, cudaMemcpyHostToDevice, stream), "upload");
  }
  void copy_out(const double* dev, double* host) {
    const size_t per = static_cast<size_t>(n_) * sizeof(double);
    for (int k = 0; k < 5; ++k)
      check(cudaMemcpyAsync(host + k * static_cast<long long>(nc_), dev + k * static_cast<long long>(n_),
                            per, cudaMemcpyDeviceToHost, stream), "download");
    check(cudaStreamSynchronize(stream), "download");
    for (int k = 0; k < 5; ++k)
      for (int g = n_; g < nc_; ++g)
        if (ghost_owner_[g - n_] >= 0)  // an external ghost's entry is left as it is
          host[k * static_cast<long long>(nc_) + g] = host[k * static_cast<long long>(nc_) + ghost_owner_[g - n_]];
  }

  // The primitives of the device state u_ into record buffer 0, where every step starts: a new
  // state, so Control::special is cleared first and set again by k_store if this state needs it.
  void store_state() {
    check(cudaMemsetAsync(&d_.ctl->special, 0, sizeof(unsigned long long), stream), "special");
    launch(k_store<P>, blocks(n_), kBlock, d_, static_cast<const double*>(u_.as<double>()),
           prim_[0].as<C>());
  }

  void upload_state(const double* u) override {
    copy_in(u, u_.as<double>());
    store_state();
    check(cudaStreamSynchronize(stream), "upload");
  }

  void download_state(double* u) override { copy_out(u_.as<double>(), u); }

  void residual(const double* u, double* res) override {
    single_rank_only("residual");
    copy_in(u, stage_.as<double>());
    launch(k_store<P>, blocks(n_), kBlock, d_, static_cast<const double*>(stage_.as<double>()),
           prim_[1].as<C>());
    enqueue_residual(1);
    copy_out(res_.as<double>(), res);
    for (int k = 0; k < 5; ++k)
      for (int g = n_; g < nc_; ++g) res[k * static_cast<long long>(nc_) + g] = 0.0;
  }

  void evaluate(autan_euler_step_result* out) override {
    need_ranks();
    launch(k_begin, 1, 256, d_.ctl, 1.0, static_cast<unsigned long long*>(nullptr));
    if (ranked()) {
      halo(0, prim_[0].as<C>());
      enqueue_cells(0, false, 0.0, false);
      if (second_) halo(1, recon_.as<C>());
      launch_faces(with_rec(0, 0), kResidual, 0, 0.0, 0.0, 0, 0);
      last_rec_ = 0;
      ++counters.residuals;
    } else {
      enqueue_residual(0);
    }
    launch(k_norm_sums, norm_blocks(), kBlock, static_cast<const double*>(res_.as<double>()), n_, d_.ctl,
           static_cast<const int*>(nullptr), static_cast<const unsigned char*>(nullptr));
    if (ranked()) reduce_words(&d_.ctl->words[0][0], 5 * kWords, 0);
    launch(k_norm_finish, 1, 32, d_.ctl, rms_cells(), 0, 0);
    // invalid(): the state, then the residual, marked on the device
    launch(k_invalid<P>, blocks(n_), kBlock, d_, static_cast<const double*>(u_.as<double>()),
           static_cast<const double*>(res_.as<double>()));
    check(cudaMemcpyAsync(head_, d_.ctl, kControlHead, cudaMemcpyDeviceToHost, stream), "control");
    check(cudaStreamSynchronize(stream), "evaluate");
    for (int k = 0; k < 5; ++k) out->residuals[k] = head_->rms[k];
    out->time_step = 0.0;
    out->steps = 0;
    out->invalid_cell = head_->bad_state != ~0ULL ? static_cast<int64_t>(head_->bad_state)
                        : head_->bad_res != ~0ULL ? static_cast<int64_t>(head_->bad_res)
                                                  : -1;
  }

  void step(double cfl, double dt, bool local, int rk, long long n, bool graph,
            autan_euler_step_result* out) override {
    if (rk != 3 && rk != 4) fail("E1101: rk must be 3 or 4");
    if (n < 1) fail("E1101: n_steps must be positive");
    if (!(dt > 0.0) && !(cfl > 0.0)) fail("E1101: a positive dt or CFL is needed");
    need_ranks();
    if (ranked()) graph = false;  // the exchange callbacks run on the host between launches
    // Reset the step count so that the history holds this call's steps, and the fault word.
    check(cudaMemsetAsync(&d_.ctl->step, 0, sizeof(long long), stream), "reset");
    check(cudaMemsetAsync(&d_.ctl->fault, 0, sizeof(unsigned long long), stream), "reset");
    const StepKey key{cfl, dt, local, rk};
    if (graph) {
      if (graph_exec_ == nullptr || !(key == graph_key_)) capture(key);
      for (long long i = 0; i < n; ++i) {
        check(cudaGraphLaunch(graph_exec_, stream), "cudaGraphLaunch");
        counters.launches += graph_nodes_;
      }
    } else {
      for (long long i = 0; i < n; ++i) enqueue_step(key);
    }
    counters.steps += n;
    last_rec_ = rk == 3 ? 2 : 1;
    // The result: the control's head (the last step's sums, step and marks) only.
    check(cudaMemcpyAsync(head_, d_.ctl, kControlHead, cudaMemcpyDeviceToHost, stream), "control");
    check(cudaStreamSynchronize(stream), "control");
    if (head_->fault != 0) fail("E1201: a bounded device wait timed out; results of this call are invalid");
    for (int k = 0; k < 5; ++k) out->residuals[k] = head_->rms[k];
    out->time_step = head_->dt;
    out->steps = head_->step;
    out->invalid_cell = head_->bad_state != ~0ULL ? static_cast<int64_t>(head_->bad_state)
                        : head_->bad_res != ~0ULL ? static_cast<int64_t>(head_->bad_res)
                                                  : -1;
  }

  void history(long long count, double* rms, double* dt) override {
    std::vector<Control> h(1);
    check(cudaMemcpyAsync(h.data(), d_.ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream), "control");
    check(cudaStreamSynchronize(stream), "control");
    const long long n = std::min<long long>({count, h[0].step, kHistory});
    for (long long i = 0; i < n; ++i) {
      if (rms != nullptr)
        for (int k = 0; k < 5; ++k) rms[5 * i + k] = h[0].hist_rms[i][k];
      if (dt != nullptr) dt[i] = h[0].hist_dt[i];
    }
  }

  void gradients(double* grad, double* phi) override {
    Buffer g(15ULL * n_ * sizeof(double)), f(5ULL * n_ * sizeof(double));
    launch(k_unpack<P>, blocks(n_), kBlock, static_cast<const C*>(recon_.as<C>()), n_, d_.rstride,
           g.as<double>(), f.as<double>());
    if (grad != nullptr)
      check(cudaMemcpyAsync(grad, g.ptr(), 15ULL * n_ * 8, cudaMemcpyDeviceToHost, stream), "grad");
    if (phi != nullptr)
      check(cudaMemcpyAsync(phi, f.ptr(), 5ULL * n_ * 8, cudaMemcpyDeviceToHost, stream), "phi");
    check(cudaStreamSynchronize(stream), "gradients");
  }

  void time_steps(double cfl, double* dt) override {
    single_rank_only("time_steps");
    Buffer tmp(std::max(n_, 1) * sizeof(double));
    Dev<P> d = with_rec(0, 0);
    if (nb_ > 0) launch(k_boundary_states<P>, blocks(nb_), kBlock, d);
    d.ctl = nullptr;
    launch(k_spectral<P>, blocks(n_), kBlock, d, cfl, 0, tmp.as<double>());
    check(cudaMemcpyAsync(dt, tmp.ptr(), n_ * sizeof(double), cudaMemcpyDeviceToHost, stream), "dt");
    check(cudaStreamSynchronize(stream), "time steps");
  }

  // Runs n steps with CUDA events around every launch on the handle's stream; per kind the total
  // milliseconds and the launches.
  void kernel_times(double cfl, double dt, bool local, int rk, long long n, double* ms,
                    long long* launches) override {
    need_ranks();
    for (int k = 0; k < 6; ++k) {
      ms[k] = 0.0;
      launches[k] = 0;
    }
    timing_ = true;
    const StepKey key{cfl, dt, local, rk};
    try {
      for (long long i = 0; i < n; ++i) enqueue_step(key);
    } catch (...) {
      timing_ = false;
      throw;
    }
    timing_ = false;
    check(cudaStreamSynchronize(stream), "kernel times");
    for (const auto& t : timed_) {
      float m = 0.0f;
      check(cudaEventElapsedTime(&m, t.before, t.after), "elapsed");
      ms[t.kind] += m;
      launches[t.kind] += 1;
      cudaEventDestroy(t.before);
      cudaEventDestroy(t.after);
    }
    timed_.clear();
    counters.steps += n;
  }

  void set_tuning(const Tuning& t) override {
    t.validate();
    tuning_ = t;
    if (t.face_mode != 0) ensure_flux_scratch();  // never inside a graph capture
    drop_graph();
  }

  Tuning tuning() const override { return tuning_; }

  // The autotuner: each candidate launch configuration steps the device state `trial_steps` times
  // (after one untimed step) with event timing; the gradient choices are picked by the gradient
  // kernel's time, then the face choices by the time of the face kernels and the norms (which
  // face mode 2 sums inside its gather). The state is restored after
  // every trial, so tuning leaves the solution unchanged. Returns the tuned ms per step.
  double autotune(double cfl, double dt, bool local, int rk, int trial_steps) override {
    need_ranks();  // with ranks, every rank tunes together: the trials make the same exchanges
    if (trial_steps < 1) fail("E1101: trial_steps must be positive");
    Buffer saved(5ULL * n_ * sizeof(double));
    check(cudaMemcpyAsync(saved.ptr(), u_.ptr(), saved.bytes(), cudaMemcpyDeviceToDevice, stream),
          "save state");
    auto restore = [&]() {
      check(cudaMemcpyAsync(u_.ptr(), saved.ptr(), saved.bytes(), cudaMemcpyDeviceToDevice, stream),
            "restore state");
      store_state();
      check(cudaStreamSynchronize(stream), "restore state");
    };
    ensure_flux_scratch();
    auto measure = [&](const Tuning& t, int kind) {
      tuning_ = t;
      double ms[6];
      long long l[6];
      kernel_times(cfl, dt, local, rk, 1, ms, l);
      kernel_times(cfl, dt, local, rk, trial_steps, ms, l);
      restore();
      double total = 0.0;
      for (int k = 0; k < 6; ++k) total += ms[k];
      const double picked = kind == kFaces ? ms[kFaces] + ms[kNorms] : ms[kind];
      return (kind < 0 ? total : picked) / trial_steps;
    };
    Tuning best = tuning_;
    if (second_) {
      double best_ms = 1e300;
      Tuning keep = best;
      for (int mode : {0, 1, 2, 3})
      for (int chunk : {1, 2, 4, 8})
        for (int block : {64, 128, 256}) {
          if (mode == 0 && chunk == 8) continue;
          if (mode == 0 && chunk == 2 && block > 128) continue;
          if (mode == 2 && chunk != 1) continue;
          if ((mode == 1 || mode == 3) && (chunk == 1 || block > 128)) continue;
          Tuning t = keep;
          t.grad_mode = mode;
          t.grad_chunk = chunk;
          t.grad_block = block;
          const double ms = measure(t, kGradients);
          if (ms < best_ms) {
            best_ms = ms;
            best = t;
          }
        }
      if (sizeof(C) == 4 && limiter_)
        for (int depth : {4, 8})
          for (int chunk : {2, 3})
            for (int narrow : {0, 1}) {
              Tuning t = keep;
              t.grad_mode = 5;
              t.grad_block = 128;
              t.grad_depth = depth;
              t.grad_chunk = chunk;
              t.grad_narrow = narrow;
              const double ms = measure(t, kGradients);
              if (ms < best_ms) {
                best_ms = ms;
                best = t;
              }
            }
      if (sizeof(C) == 4 && limiter_)
        for (int shape = 0; shape < 3; ++shape)  // (entries in flight, register bound)
        for (int widen : {0, 1, 2})
          for (int narrow : {0, 1})
            {
              Tuning t = keep;
              t.grad_mode = 4;
              t.grad_block = 128;
              t.grad_widen = widen;
              t.grad_narrow = narrow;
              t.grad_chunk = shape == 2 ? 4 : 2;
              t.grad_minb = shape == 0 ? 7 : (shape == 1 ? 6 : 5);
              const double ms = measure(t, kGradients);
              if (ms < best_ms) {
                best_ms = ms;
                best = t;
              }
            }
    }
    {
      double best_ms = 1e300;
      Tuning keep = best;
      for (int mode : {0, 1, 2})
        for (int block : {64, 128, 256})
          for (int gather : {128, 256}) {
            if (mode == 0 && gather != 256) continue;
            if (mode == 2 && n_cases_ > 0) continue;  // the same launches as mode 1
            Tuning t = keep;
            t.face_mode = mode;
            t.face_block = block;
            t.gather_block = gather;
            const double ms = measure(t, kFaces);
            if (ms < best_ms) {
              best_ms = ms;
              best = t;
            }
          }
    }
    const double total = measure(best, -1);
    tuning_ = best;
    drop_graph();
    return total;
  }

  std::vector<int> ghost_owner_;

 private:
  struct StepKey {
    double cfl, dt;
    bool local;
    int rk;
    bool operator==(const StepKey& o) const {
      return cfl == o.cfl && dt == o.dt && local == o.local && rk == o.rk;
    }
  };

  // Kernel kinds of autan_euler_device_kernel_times.
  enum Kind : int { kBoundary = 0, kGradients = 1, kSpectral = 2, kFaces = 3, kNorms = 4, kControl = 5 };

  void validate(const autan_euler_mesh& m) {
    if (m.n_owned_cells < 1 || m.n_cells < m.n_owned_cells || m.n_faces < m.n_interior_faces ||
        m.n_owned_interior_faces > m.n_interior_faces || m.n_owned_faces > m.n_faces ||
        m.n_owned_faces < m.n_interior_faces)
      fail("E1101: inconsistent mesh counts");
    if (m.owner == nullptr || m.cell_face_offsets == nullptr || m.cell_faces == nullptr ||
        m.face_normal == nullptr || m.face_area_magnitude == nullptr ||
        m.face_centroid == nullptr || m.cell_centroid == nullptr || m.cell_volume == nullptr ||
        (m.n_interior_faces > 0 && m.neighbour == nullptr))
      fail("E1101: a required mesh array is NULL");
    if (m.n_cells > m.n_owned_cells && m.ghost_owner == nullptr)
      fail("E1101: ghost cells need ghost_owner");
    if (second_ && (m.stencil == nullptr || m.stencil_offsets == nullptr ||
                    m.stencil_lsq_weight == nullptr))
      fail("E1101: a second-order scheme needs the stencil and its weights");
    if (scheme_.flux < 0 || scheme_.flux > 2) fail("E1101: unknown flux");
    for (int c = 0; c < m.n_owned_cells; ++c)
      if (!(m.cell_volume[c] > 0.0)) fail("E0121: an owned cell has a non-positive volume");
    if (m.n_cells > m.n_owned_cells)
      ghost_owner_.assign(m.ghost_owner, m.ghost_owner + (m.n_cells - m.n_owned_cells));
    if (static_cast<long long>(m.n_owned_cells) >= (1LL << 30)) fail("E1101: mesh too large");
  }

  int slices() const { return std::max(1, (n_ + kSlice - 1) / kSlice); }

  // Shared memory of the staged gradient kernel at `block` threads: the largest of its blocks'
  // stencil rows and incidence records (twice the incidences when it also stages their normals
  // and areas for the time step).
  size_t staged_smem(int block, bool dt) {
    const int per = block / kSlice;
    auto& cached = staged_smem_[dt ? 1 : 0][per];
    if (cached == 0) {
      long long most = 0;
      const int ns = slices();
      const int rows = dt ? 2 : 1;
      for (int s0 = 0; s0 < ns; s0 += per) {
        const int s1 = std::min(s0 + per, ns);
        most = std::max<long long>(most, static_cast<long long>(st_.start[s1] - st_.start[s0]) +
                                             rows * (inc_.start[s1] - inc_.start[s0]));
      }
      cached = static_cast<size_t>(most) * 4 * sizeof(C) + 16;
      if (cached > 220 * 1024) fail("E1101: stencil rows too long for the staged gradient kernel");
    }
    return cached;
  }

  static int blocks(long long n, int block = kBlock) {
    return static_cast<int>(std::max<long long>(1, (n + block - 1) / block));
  }
  int norm_blocks() const { return std::min(blocks(n_), 148 * 8); }

  // The grid-stride fused-norm gather: as many blocks as stay resident on the device at once.
  int norm_gather_grid(int gb, size_t smem) {
    int& cached = norm_gather_grid_[gb / 32];
    if (cached == 0) {
      int per_sm = 0, sms = 0, dev = 0;
      check(cudaGetDevice(&dev), "device");
      check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device");
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather<P, true>, gb, smem),
            "occupancy");
      cached = std::max(1, per_sm) * std::max(1, sms);
    }
    return std::min(cached, blocks(n_, gb));
  }

  template <class K, class... A>
  void launch(K kernel, int grid, int block, A... args) {
    launch_as(kControl, kernel, grid, block, args...);
  }

  template <class K, class... A>
  void launch_as(int kind, K kernel, int grid, int block, A... args) {
    launch_smem(kind, kernel, grid, block, 0, args...);
  }

  template <class K, class... A>
  void launch_smem(int kind, K kernel, int grid, int block, size_t smem, A... args) {
    cudaEvent_t before = nullptr, after = nullptr;
    if (smem > 48 * 1024) {
      // The kernel's dynamic shared-memory limit raised to the device's opt-in maximum less its
      // static shared memory, the same value from every handle and thread: a limit set to each
      // launch's own size would race with another handle's launch of the same kernel at a larger
      // size.
      if (smem_optin_ == 0) {
        int dev = 0;
        check(cudaGetDevice(&dev), "device");
        check(cudaDeviceGetAttribute(&smem_optin_, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
              "device");
      }
      cudaFuncAttributes fa{};
      check(cudaFuncGetAttributes(&fa, kernel), "shared memory");
      const long long limit =
          static_cast<long long>(smem_optin_) - static_cast<long long>(fa.sharedSizeBytes);
      if (static_cast<long long>(smem) > limit) fail("E1200: shared memory above the device's limit");
      check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(limit)), "shared memory");
    }
    if (timing_) {
      check(cudaEventCreate(&before), "event");
      check(cudaEventCreate(&after), "event");
      check(cudaEventRecord(before, stream), "event");
    }
    kernel<<<grid, block, smem, stream>>>(args...);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      char what[160];
      std::snprintf(what, sizeof(what), "kernel launch (kind %d, grid %d, block %d, %zu bytes shared)",
                    kind, grid, block, smem);
      check(e, what);
    }
    ++counters.launches;
    if (timing_) {
      check(cudaEventRecord(after, stream), "event");
      timed_.push_back({kind, before, after});
    }
  }

  Dev<P> with_rec(int in, int out) const {
    Dev<P> d = d_;
    if (repacked()) {
      d.cell_tiles = cell_tiles_.as<int>();
      d.face_tiles = face_tiles_.as<int>();
      d.bface_tiles = bface_tiles_.as<int>();
      d.n_cell_tiles = n_cell_tiles_;
      d.n_face_tiles = n_face_tiles_;
      d.n_bface_tiles = n_bface_tiles_;
    }
    d.prim = prim_[in].as<C>();
    d.prim_b = prim_[in].as<C>() + static_cast<long long>(kPrimW) * nv_;  // this stage's boundary states
    d.prim_next = prim_[out].as<C>();
    return d;
  }

  void launch_faces(const Dev<P>& d, int mode, int stage, double wa, double wb, int local,
                    int last, bool norms = false) {
    if (tuning_.face_mode == 0) {
      dispatch_faces([&](auto flux, auto planar, auto second) {
        constexpr int F = decltype(flux)::value;
        constexpr bool PL = decltype(planar)::value, SE = decltype(second)::value;
        const int bs = tuning_.face_block;
        launch_as(kFaces, k_faces_cell<P, F, PL, SE>, cell_grid(bs), bs, d, mode, stage, wa, wb,
                  local, last);
      });
      return;
    }
    launch_flux(d);
    C* fl = flux_.as<C>();
    C* bfl = bflux_.as<C>();
    const int gb = tuning_.gather_block;
    if (norms) {
      const size_t sm = static_cast<size_t>(gb / 32) * 5 * kWords * sizeof(unsigned long long);
      launch_smem(kFaces, k_gather<P, true>, norm_gather_grid(gb, sm), gb, sm, d,
                  static_cast<const C*>(fl),
                  static_cast<const C*>(bfl), mode, stage, wa, wb, local, last,
                  norm_words_.as<unsigned long long>());
    } else {
      launch_as(kFaces, k_gather<P, false>, cell_grid(gb), gb, d, static_cast<const C*>(fl),
                static_cast<const C*>(bfl), mode, stage, wa, wb, local, last,
                static_cast<unsigned long long*>(nullptr));
    }
  }

  // Every owned face's flux, once, into the face scratch (the store-gather strategy's first half).
  void launch_flux(const Dev<P>& d) {
    if (flux_.bytes() == 0) fail("E1200: face scratch missing");
    C* fl = flux_.as<C>();
    C* bfl = bflux_.as<C>();
    dispatch_faces([&](auto flux, auto planar, auto second) {
      constexpr int F = decltype(flux)::value;
      constexpr bool PL = decltype(planar)::value, SE = decltype(second)::value;
      const int bs = tuning_.face_block;
      launch_as(kFaces, k_face_flux<P, F, PL, SE>, face_grid(bs), bs, d, fl);
      if (nbo_ > 0) launch_as(kFaces, k_bface_flux<P, F, PL, SE>, bface_grid(bs, nbo_), bs, d, bfl, nbo_);
    });
  }

  // The primitives (in prim_[1]), boundary states, gradients and limiter of the host state u
  // (5 x n_cells) or, with u == nullptr, of the device state.
  void prepare(const double* u) {
    const double* src = u_.as<double>();
    if (u != nullptr) {
      copy_in(u, stage_.as<double>());
      src = stage_.as<double>();
    }
    launch(k_store<P>, blocks(n_), kBlock, d_, src, prim_[1].as<C>());
    enqueue_cells(1, false, 0.0, false);
  }

  // After prepare: each owned face's flux into the face scratch and the face parts R^F of the
  // owned cells into res_ (Euler<P>::face_parts, physics/src/euler.cpp:944-965).
  void enqueue_face_parts() {
    ensure_flux_scratch();
    const Dev<P> d = with_rec(1, 1);
    launch_flux(d);
    launch(k_gather<P, false>, blocks(n_), kBlock, d, static_cast<const C*>(flux_.as<C>()),
           static_cast<const C*>(bflux_.as<C>()), static_cast<int>(kFaceParts), 0, 0.0, 0.0, 0, 0,
           static_cast<unsigned long long*>(nullptr));
  }

  void face_parts(const double* u, double* res_faces, double* face_flux) override {
    single_rank_only("face_parts");
    prepare(u);
    enqueue_face_parts();
    if (res_faces != nullptr) {
      copy_out(res_.as<double>(), res_faces);
      for (int k = 0; k < 5; ++k)
        for (int g = n_; g < nc_; ++g) res_faces[k * static_cast<long long>(nc_) + g] = 0.0;
    }
    if (face_flux != nullptr) {
      Buffer out(5ULL * nf_ * sizeof(double));
      check(cudaMemsetAsync(out.ptr(), 0, out.bytes(), stream), "face_flux");
      launch(k_unpack_flux<P>, blocks(static_cast<long long>(nif_) + nbo_), kBlock,
             static_cast<const C*>(flux_.as<C>()), static_cast<const C*>(bflux_.as<C>()), nif_, nbo_,
             ni_, nf_, out.as<double>());
      check(cudaMemcpyAsync(face_flux, out.ptr(), out.bytes(), cudaMemcpyDeviceToHost, stream),
            "face_flux");
    }
    check(cudaStreamSynchronize(stream), "face_parts");
  }

  void boundary_pressure(const double* u, double* p, double* force) override {
    single_rank_only("boundary_pressure");
    prepare(u);
    Buffer pb(std::max<size_t>(1, static_cast<size_t>(nb_)) * sizeof(double));
    Buffer fb(force != nullptr ? 3ULL * std::max(nb_, 1) * sizeof(double) : 0);
    launch(k_boundary_pressure<P>, blocks(nb_), kBlock, with_rec(1, 1),
           static_cast<const double*>(bface_r64_.as<double>()), second_ ? 1 : 0, pref64_,
           pb.as<double>(), force != nullptr ? fb.as<double>() : static_cast<double*>(nullptr));
    if (p != nullptr && nb_ > 0)
      check(cudaMemcpyAsync(p, pb.ptr(), nb_ * sizeof(double), cudaMemcpyDeviceToHost, stream), "p");
    if (force != nullptr && nb_ > 0)
      check(cudaMemcpyAsync(force, fb.ptr(), 3ULL * nb_ * sizeof(double), cudaMemcpyDeviceToHost,
                            stream), "force");
    check(cudaStreamSynchronize(stream), "boundary_pressure");
  }

  int conservation(double* sums) override {
    single_rank_only("conservation");
    prepare(nullptr);
    enqueue_face_parts();
    check(cudaMemsetAsync(cons_words_.ptr(), 0, cons_words_.bytes(), stream), "conservation");
    const long long total = std::max<long long>({n_, nif_, nbo_});
    launch(k_conservation<P>, std::min(blocks(total), 148 * 4), kBlock, with_rec(1, 1),
           static_cast<const C*>(flux_.as<C>()), static_cast<const C*>(bflux_.as<C>()),
           static_cast<const unsigned char*>(face_mult_.as<unsigned char>()), nbo_,
           cons_words_.as<unsigned long long>());
    Buffer out(20 * sizeof(double));
    launch(k_conservation_finish, 1, 32, static_cast<const unsigned long long*>(
                                             cons_words_.as<unsigned long long>()),
           out.as<double>());
    check(cudaMemcpyAsync(sums, out.ptr(), 20 * sizeof(double), cudaMemcpyDeviceToHost, stream),
          "conservation");
    check(cudaStreamSynchronize(stream), "conservation");
    return max_faces_;
  }

  // Batched cases: owned cells [cell_offsets[k], cell_offsets[k + 1]) form case k.
  void set_cases(int n_cases, const int64_t* off) override {
    single_rank_only("set_cases");
    if (ranked()) fail("E1101: ranks and batched cases do not go together");
    if (n_cases < 1 || off == nullptr) fail("E1101: at least one case and its cell offsets");
    if (off[0] != 0 || off[n_cases] != n_) fail("E1101: case offsets must span the owned cells");
    std::vector<int> case_of(std::max(n_, 1), 0);
    std::vector<double> cells(n_cases);
    for (int k = 0; k < n_cases; ++k) {
      if (off[k + 1] <= off[k]) fail("E1101: every case needs at least one cell");
      cells[k] = static_cast<double>(off[k + 1] - off[k]);
      for (int64_t c = off[k]; c < off[k + 1]; ++c) case_of[c] = k;
    }
    drop_graph();
    n_cases_ = n_cases;
    case_of_ = upload(case_of, stream);
    case_cells_ = upload(cells, stream);
    case_words_.alloc(5ULL * kWords * n_cases * sizeof(unsigned long long));
    case_hist_.alloc(static_cast<size_t>(kHistory) * 5 * n_cases * sizeof(double));
    active_.alloc(static_cast<size_t>(n_cases));
    check(cudaMemsetAsync(case_words_.ptr(), 0, case_words_.bytes(), stream), "cases");
    check(cudaMemsetAsync(case_hist_.ptr(), 0, case_hist_.bytes(), stream), "cases");
    check(cudaMemsetAsync(active_.ptr(), 1, active_.bytes(), stream), "cases");
    d_.case_of = case_of_.as<int>();
    d_.active = active_.as<unsigned char>();
    face_warp_case_.alloc(static_cast<size_t>(std::max((nif_ + 31) / 32, 1)) * sizeof(int));
    bface_warp_case_.alloc(static_cast<size_t>(std::max((nbo_ + 31) / 32, 1)) * sizeof(int));
    if (nif_ > 0)
      launch(k_warp_case<C>, blocks(nif_), kBlock, static_cast<const C*>(face_.as<C>()), kFace, 7,
             nif_, static_cast<const int*>(case_of_.as<int>()), face_warp_case_.as<int>());
    if (nbo_ > 0)
      launch(k_warp_case<C>, blocks(nbo_), kBlock, static_cast<const C*>(bface_.as<C>()), kBface, 13,
             nbo_, static_cast<const int*>(case_of_.as<int>()), bface_warp_case_.as<int>());
    d_.face_warp_case = face_warp_case_.as<int>();
    d_.bface_warp_case = bface_warp_case_.as<int>();
    d_.case_minf = nullptr;
    case_offsets_.assign(off, off + n_cases + 1);
    face_warp_case_h_.assign(static_cast<size_t>((nif_ + 31) / 32), 0);
    bface_warp_case_h_.assign(static_cast<size_t>((nbo_ + 31) / 32), 0);
    if (!face_warp_case_h_.empty())
      check(cudaMemcpyAsync(face_warp_case_h_.data(), face_warp_case_.ptr(),
                            face_warp_case_h_.size() * sizeof(int), cudaMemcpyDeviceToHost, stream),
            "cases");
    if (!bface_warp_case_h_.empty())
      check(cudaMemcpyAsync(bface_warp_case_h_.data(), bface_warp_case_.ptr(),
                            bface_warp_case_h_.size() * sizeof(int), cudaMemcpyDeviceToHost, stream),
            "cases");
    n_cell_tiles_ = n_face_tiles_ = n_bface_tiles_ = -1;
    check(cudaStreamSynchronize(stream), "cases");
  }

  // The warp tiles of the cases still stepping (re-packed launches), or none when every case
  // steps: 32-cell slices overlapping an active case's cells, and the 32-face warps of interior and
  // boundary faces whose owners include an active case.
  void repack(const uint8_t* active) {
    bool all = true;
    for (int k = 0; k < n_cases_; ++k) all = all && active[k] != 0;
    drop_graph();
    if (all) {
      n_cell_tiles_ = n_face_tiles_ = n_bface_tiles_ = -1;
      return;
    }
    std::vector<int> cells, faces, bfaces;
    std::vector<uint8_t> mark(static_cast<size_t>((n_ + 31) / 32), 0);
    for (int k = 0; k < n_cases_; ++k)
      if (active[k])
        for (int64_t sl = case_offsets_[k] / 32; sl <= (case_offsets_[k + 1] - 1) / 32; ++sl) mark[sl] = 1;
    for (size_t sl = 0; sl < mark.size(); ++sl)
      if (mark[sl]) cells.push_back(static_cast<int>(sl));
    auto warps = [&](const std::vector<int>& wc, std::vector<int>& out) {
      for (size_t w = 0; w < wc.size(); ++w)
        if (wc[w] < 0 || active[wc[w]]) out.push_back(static_cast<int>(w));
    };
    warps(face_warp_case_h_, faces);
    warps(bface_warp_case_h_, bfaces);
    auto put = [&](Buffer& b, const std::vector<int>& v, int& n) {
      n = static_cast<int>(v.size());
      b = upload(v, stream);
    };
    put(cell_tiles_, cells, n_cell_tiles_);
    put(face_tiles_, faces, n_face_tiles_);
    put(bface_tiles_, bfaces, n_bface_tiles_);
  }

  // Grids of the step's launches: over the tiles while cases are re-packed, else every item.
  bool repacked() const { return step_tiles_ && n_cell_tiles_ >= 0; }
  int cell_grid(int bs) const {
    return repacked() ? blocks(32LL * std::max(n_cell_tiles_, 1), bs) : blocks(n_, bs);
  }
  int face_grid(int bs) const {
    return repacked() ? blocks(32LL * std::max(n_face_tiles_, 1), bs) : blocks(nif_, bs);
  }
  int bface_grid(int bs, int count) const {
    return repacked() ? blocks(32LL * std::max(n_bface_tiles_, 1), bs) : blocks(count, bs);
  }

  void set_case_mach_ref(const double* mach_ref) override {
    if (n_cases_ == 0) fail("E1101: no cases set");
    std::vector<C> v(n_cases_);
    for (int k = 0; k < n_cases_; ++k) {
      if (!(mach_ref[k] > 0.0)) fail("E1101: AUSM+-up needs a positive cut-off Mach number");
      v[k] = static_cast<C>(mach_ref[k]);
    }
    drop_graph();
    case_minf_ = upload(v, stream);
    d_.case_minf = case_minf_.as<C>();
    check(cudaStreamSynchronize(stream), "cases");
  }

  void set_active(const uint8_t* active) override {
    if (n_cases_ == 0) fail("E1101: no cases set");
    check(cudaMemcpyAsync(active_.ptr(), active, static_cast<size_t>(n_cases_), cudaMemcpyHostToDevice,
                          stream), "active");
    repack(active);
    check(cudaStreamSynchronize(stream), "active");
  }

  // The last `count` steps' per-case RMS (count x n_cases x 5), oldest first.
  void case_history(long long count, double* rms) override {
    if (n_cases_ == 0) fail("E1101: no cases set");
    long long step = 0;
    check(cudaMemcpyAsync(&step, &d_.ctl->step, sizeof(step), cudaMemcpyDeviceToHost, stream), "history");
    check(cudaStreamSynchronize(stream), "history");
    const long long n = std::min<long long>({count, step, kHistory});
    const size_t row = 5ULL * n_cases_ * sizeof(double);
    for (long long i = 0; i < n; ++i) {
      const long long slot = (step - n + i) % kHistory;
      check(cudaMemcpyAsync(rms + i * 5LL * n_cases_, case_hist_.as<double>() + slot * 5LL * n_cases_,
                            row, cudaMemcpyDeviceToHost, stream), "history");
    }
    check(cudaStreamSynchronize(stream), "history");
  }

  int n_cases() const override { return n_cases_; }

  void set_stall_test(int polls) override {
    if (polls < 0) fail("E1101: polls must be >= 0");
    d_.stall_polls = polls;
    drop_graph();
  }

  // ---- ranks of a partitioned mesh

  long long external_ghosts() const override { return n_ext_; }

  void set_ranks(const autan_euler_ranks* r) override {
    drop_graph();
    if (r == nullptr) {
      ranks_ = autan_euler_ranks{};
      send_cells_ = Buffer();
      d_.wide_ok = wide_ok_mesh_;
      return;
    }
    if (n_cases_ > 0) fail("E1101: ranks and batched cases do not go together");
    if (r->exchange == nullptr || r->reduce == nullptr) fail("E1101: ranks need both callbacks");
    if (r->n_send < 0 || (r->n_send > 0 && (r->send_cells == nullptr || r->send == nullptr)))
      fail("E1101: a send list needs its cells and its buffer");
    if (n_ext_ > 0 && r->recv == nullptr) fail("E1101: external ghosts need a receive buffer");
    if (r->words == nullptr) fail("E1101: ranks need the reduction words");
    auto misaligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) != 0; };
    if (misaligned(r->send) || misaligned(r->recv) || misaligned(r->words))
      fail("E1101: the exchange buffers must be 16-byte aligned");
    if (!(r->global_cells >= static_cast<double>(n_))) fail("E1101: global_cells below the owned cells");
    std::vector<int> cells(static_cast<size_t>(std::max<long long>(r->n_send, 1)), 0);
    for (long long i = 0; i < r->n_send; ++i) {
      if (r->send_cells[i] < 0 || r->send_cells[i] >= n_) fail("E1101: a send cell is not an owned cell");
      cells[i] = r->send_cells[i];
    }
    send_cells_ = upload(cells, stream);
    check(cudaStreamSynchronize(stream), "ranks");
    ranks_ = *r;
    d_.wide_ok = 0;
  }

  bool ranked() const { return ranks_.exchange != nullptr; }

  // The CUDA runtime's last-error state after a ranks' callback: an error the callee's own CUDA
  // calls left there (a communication library may leave one it has handled) is the callee's to
  // report through its return code, and must not be read as the failure of the library's next
  // launch. Sticky errors (a faulted context) stay visible to every later call.
  static void drop_callee_error() { (void)cudaGetLastError(); }

  bool any_rank(bool mine) override {
    if (!ranked()) return mine;
    long long word = mine ? 0 : 1;  // the minimum over the ranks is 0 where any rank has it set
    check(cudaMemcpyAsync(ranks_.words, &word, sizeof(word), cudaMemcpyHostToDevice, stream), "ranks");
    const int32_t rc = ranks_.reduce(ranks_.user, 1, 1, static_cast<void*>(stream));
    drop_callee_error();
    if (rc != 0) fail("E1301: the ranks' reduction failed");
    check(cudaMemcpyAsync(&word, ranks_.words, sizeof(word), cudaMemcpyDeviceToHost, stream), "ranks");
    check(cudaStreamSynchronize(stream), "ranks");
    return word == 0;
  }
  double rms_cells() const { return ranked() ? ranks_.global_cells : static_cast<double>(n_); }

  // An entry point that evaluates from a host state or tunes itself: owned cells only.
  void single_rank_only(const char* what) const {
    if (n_ext_ > 0) {
      std::string m = "E1101: ";
      m += what;
      m += " is not available on a mesh with external ghosts";
      fail(m.c_str());
    }
  }
  // A step or evaluation of a mesh with external ghosts needs the ranks' exchange.
  void need_ranks() const {
    if (n_ext_ > 0 && !ranked())
      fail("E1101: a mesh with external ghosts steps only with its ranks set");
  }

  // The forward ghost exchange of the primitive records in `prim` (what 0) or of the
  // reconstruction array (what 1): pack the send cells' records, the exchange callback, unpack
  // the external ghosts' records.
  void halo(int what, C* base) {
    const int groups = what == 0 ? 1 : kRecon / kGroup;
    const long long gstride = what == 0 ? 0 : d_.rstride;
    const long long per = static_cast<long long>(groups) * kGroup * static_cast<long long>(sizeof(C)) / 16;
    if (ranks_.n_send > 0)
      launch(k_halo_records<C, true>, blocks(ranks_.n_send * per), kBlock, base, gstride, groups,
             static_cast<const int*>(send_cells_.as<int>()), static_cast<long long>(ranks_.n_send), 0,
             static_cast<C*>(ranks_.send));
    const long long bytes = static_cast<long long>(groups) * kGroup * static_cast<long long>(sizeof(C));
    const int32_t rc = ranks_.exchange(ranks_.user, what, bytes, static_cast<void*>(stream));
    drop_callee_error();
    if (rc != 0) fail("E1301: the ranks' ghost exchange failed");
    if (n_ext_ > 0)
      launch(k_halo_records<C, false>, blocks(static_cast<long long>(n_ext_) * per), kBlock, base,
             gstride, groups, static_cast<const int*>(nullptr), static_cast<long long>(n_ext_), n_,
             static_cast<C*>(ranks_.recv));
  }

  // `count` words of the control block combined over the ranks in place (op 0 sum, 1 min).
  void reduce_words(unsigned long long* dev, int count, int op) {
    const size_t bytes = static_cast<size_t>(count) * sizeof(unsigned long long);
    check(cudaMemcpyAsync(ranks_.words, dev, bytes, cudaMemcpyDeviceToDevice, stream), "ranks");
    const int32_t rc = ranks_.reduce(ranks_.user, op, count, static_cast<void*>(stream));
    drop_callee_error();
    if (rc != 0) fail("E1301: the ranks' reduction failed");
    check(cudaMemcpyAsync(dev, ranks_.words, bytes, cudaMemcpyDeviceToDevice, stream), "ranks");
  }

  // Calls body(flux, planar, second) with the scheme's compile-time choices.
  template <class B>
  void dispatch_faces(B&& body) {
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using T = std::true_type;
    using Fa = std::false_type;
    auto by_flux = [&](auto pl, auto se) {
      if (scheme_.flux == 0) body(I0{}, pl, se);
      else if (scheme_.flux == 1) body(I1{}, pl, se);
      else body(I2{}, pl, se);
    };
    if (planar_) {
      if (second_) by_flux(T{}, T{});
      else by_flux(T{}, Fa{});
    } else {
      if (second_) by_flux(Fa{}, T{});
      else by_flux(Fa{}, Fa{});
    }
  }

  void ensure_flux_scratch() {
    if (flux_.bytes() == 0) {
      flux_.alloc(static_cast<size_t>(kFlux) * std::max(nif_, 1) * sizeof(C));
      bflux_.alloc(static_cast<size_t>(kFlux) * std::max(nbo_, 1) * sizeof(C));
    }
  }

  // The loops before the faces on record buffer `in`: boundary states, gradients and limiter;
  // with `dt`, the spectral radius and the CFL step of the step too.
  void enqueue_cells(int in, bool dt, double cfl, bool local) {
    const Dev<P> d = with_rec(in, in);
    if (nb_ > 0) launch_as(kBoundary, k_boundary_states<P>, bface_grid(kBlock, nb_), kBlock, d);
    const int g = cell_grid(kBlock);
    const int loc = local ? 1 : 0;
    if (second_) {
      const int bs = tuning_.grad_block;
      const int gs = cell_grid(bs);
      auto go = [&](auto lim, auto with_dt) {
        constexpr bool L = decltype(lim)::value, D = decltype(with_dt)::value;
        if (repacked()) {
          launch_as(kGradients, k_gradients_tiles<P, L, D>, cell_grid(128), 128, d, cfl, loc);
          return;
        }
        if (tuning_.grad_mode == 4 || tuning_.grad_mode == 5) {
          if constexpr (std::is_same_v<P, Fp32Acc64> && L) {
            if (tuning_.grad_mode == 5) launch_gradients_ring<D>(d, cfl, loc);
            else launch_gradients_w<D>(d, cfl, loc);
            return;
          }
          // fp64 or no limiter: the mode-0 form with two entries in flight
          if constexpr (sizeof(C) == 4)
            launch_as(kGradients, k_gradients_occ7<P, L, D>, cell_grid(128), 128, d, cfl, loc);
          else
            launch_as(kGradients, k_gradients<P, L, D, 2>, cell_grid(128), 128, d, cfl, loc);
          return;
        }
        if (tuning_.grad_mode == 1) {
          const int sm = static_cast<int>(staged_smem(bs, D));
          const int gb = blocks(n_, bs);
          if (tuning_.grad_chunk == 8) {
            launch_smem(kGradients, k_gradients_tma<P, L, D, 8>, gb, bs, sm, d, cfl, loc);
          } else if constexpr (sizeof(C) == 4) {  // fp32+acc64: the 6-blocks-per-SM bound
            if (tuning_.grad_chunk == 2)
              launch_smem(kGradients, k_gradients_tma_occ6<P, L, D, 2>, gb, bs, sm, d, cfl, loc);
            else
              launch_smem(kGradients, k_gradients_tma_occ6<P, L, D, 4>, gb, bs, sm, d, cfl, loc);
          } else {
            if (tuning_.grad_chunk == 2)
              launch_smem(kGradients, k_gradients_tma<P, L, D, 2>, gb, bs, sm, d, cfl, loc);
            else
              launch_smem(kGradients, k_gradients_tma<P, L, D, 4>, gb, bs, sm, d, cfl, loc);
          }
          return;
        }
        if (tuning_.grad_mode == 3) {
          const int w = static_cast<int>(sizeof(C));
          if (tuning_.grad_chunk == 2)
            launch_smem(kGradients, k_gradients_ring<P, L, D, 2>, gs, bs, bs * ring_bytes(2, w), d, cfl, loc);
          else if (tuning_.grad_chunk == 8)
            launch_smem(kGradients, k_gradients_ring<P, L, D, 8>, gs, bs, bs * ring_bytes(8, w), d, cfl, loc);
          else
            launch_smem(kGradients, k_gradients_ring<P, L, D, 4>, gs, bs, bs * ring_bytes(4, w), d, cfl, loc);
          return;
        }
        if (tuning_.grad_mode == 2) {
          launch_as(kGradients, k_gradients<P, L, D, 0>, gs, bs, d, cfl, loc);
        } else if (tuning_.grad_chunk == 1) {
          launch_as(kGradients, k_gradients<P, L, D, 1>, gs, bs, d, cfl, loc);
        } else if (tuning_.grad_chunk == 2) {
          if constexpr (sizeof(C) == 4)  // fp32+acc64: the 7-blocks-per-SM bound
            launch_as(kGradients, k_gradients_occ7<P, L, D>, gs, bs, d, cfl, loc);
          else
            launch_as(kGradients, k_gradients<P, L, D, 2>, gs, bs, d, cfl, loc);
        } else {
          launch_as(kGradients, k_gradients<P, L, D, 4>, gs, bs, d, cfl, loc);
        }
      };
      if (limiter_) {
        if (dt) go(std::true_type{}, std::true_type{});
        else go(std::true_type{}, std::false_type{});
      } else {
        if (dt) go(std::false_type{}, std::true_type{});
        else go(std::false_type{}, std::false_type{});
      }
    } else if (dt) {
      launch_as(kSpectral, k_spectral<P>, g, kBlock, d, cfl, loc, static_cast<double*>(nullptr));
    }
  }

  // The mode-4 gradient kernel of the tuning's widening, gathers and register bound (fp32+acc64,
  // limited second order).
  template <bool D>
  void launch_gradients_w(const Dev<P>& d, double cfl, int loc) {
    if constexpr (std::is_same_v<P, Fp32Acc64>) {
      const int gs = cell_grid(128);
      auto shape = [&](auto wide, auto narrow) {
        constexpr int W = decltype(wide)::value;
        constexpr bool G = decltype(narrow)::value;
        if (tuning_.grad_chunk == 4)
          launch_as(kGradients, k_gradients_w<true, D, W, G, 4, 5>, gs, 128, d, cfl, loc);
        else if (tuning_.grad_minb == 6)
          launch_as(kGradients, k_gradients_w<true, D, W, G, 2, 6>, gs, 128, d, cfl, loc);
        else
          launch_as(kGradients, k_gradients_w<true, D, W, G, 2, 7>, gs, 128, d, cfl, loc);
      };
      auto narrow = [&](auto wide) {
        if (tuning_.grad_narrow) shape(wide, std::true_type{});
        else shape(wide, std::false_type{});
      };
      if (tuning_.grad_widen == 2) narrow(std::integral_constant<int, 2>{});
      else if (tuning_.grad_widen == 1) narrow(std::integral_constant<int, 1>{});
      else narrow(std::integral_constant<int, 0>{});
    }
  }

  // The mode-5 gradient kernel (per-warp TMA row ring) of the tuning's depth, chunk and gathers.
  template <bool D>
  void launch_gradients_ring(const Dev<P>& d, double cfl, int loc) {
    if constexpr (std::is_same_v<P, Fp32Acc64>) {
      const int gs = cell_grid(128);
      auto go = [&](auto depth, auto chunk, auto narrow) {
        constexpr int R = decltype(depth)::value, CH = decltype(chunk)::value;
        constexpr bool G = decltype(narrow)::value;
        launch_smem(kGradients, k_gradients_wring<true, D, R, CH, G>, gs, 128, warp_ring_bytes(R),
                    d, cfl, loc);
      };
      using I2 = std::integral_constant<int, 2>;
      using I3 = std::integral_constant<int, 3>;
      using I4 = std::integral_constant<int, 4>;
      using I8 = std::integral_constant<int, 8>;
      auto by_chunk = [&](auto depth, auto narrow) {
        if (tuning_.grad_chunk == 3) go(depth, I3{}, narrow);
        else go(depth, I2{}, narrow);
      };
      auto by_narrow = [&](auto depth) {
        if (tuning_.grad_narrow) by_chunk(depth, std::true_type{});
        else by_chunk(depth, std::false_type{});
      };
      if (tuning_.grad_depth == 8) by_narrow(I8{});
      else by_narrow(I4{});
    }
  }

  void enqueue_residual(int in) {
    enqueue_cells(in, false, 0.0, false);
    launch_faces(with_rec(in, in), kResidual, 0, 0.0, 0.0, 0, 0);
    last_rec_ = in;
    ++counters.residuals;
  }

  // One step. Records rotate through three buffers so that a step starts and ends in buffer 0:
  // RK3 0 -> 1 -> 2 -> 0; RK4 0 -> 1 -> 2 -> 1 -> 0.
  void enqueue_step(const StepKey& k) {
    struct Tiles {  // the step's launches take the re-packed tiles, nothing else does
      bool& on;
      explicit Tiles(bool& f) : on(f) { on = true; }
      ~Tiles() { on = false; }
    } tiles(step_tiles_);
    const bool cfl_dt = !(k.dt > 0.0);
    const bool local = cfl_dt && k.local;
    // the stage-0 norms fused into the store-gather sum (not with batched cases, whose per-case
    // norms read the stored residual)
    const bool fused = tuning_.face_mode == 2 && n_cases_ == 0;
    launch(k_begin, 1, 256, d_.ctl, cfl_dt ? 0.0 : k.dt,
           fused ? norm_words_.as<unsigned long long>() : static_cast<unsigned long long*>(nullptr));
    const int stages = k.rk == 3 ? 3 : 4;
    static const int in3[3] = {0, 1, 2}, out3[3] = {1, 2, 0};
    static const int in4[4] = {0, 1, 2, 1}, out4[4] = {1, 2, 1, 0};
    static const double w3[3][2] = {{0.0, 1.0}, {0.75, 0.25}, {1.0 / 3.0, 2.0 / 3.0}};
    static const double c4[4] = {0.5, 0.5, 1.0, 0.0};
    for (int st = 0; st < stages; ++st) {
      const int in = k.rk == 3 ? in3[st] : in4[st];
      const int out = k.rk == 3 ? out3[st] : out4[st];
      if (ranked()) halo(0, prim_[in].as<C>());
      enqueue_cells(in, st == 0 && cfl_dt, k.cfl, local);
      if (ranked()) {
        if (st == 0 && cfl_dt) reduce_words(&d_.ctl->dt_bits, 1, 1);
        if (second_) halo(1, recon_.as<C>());
      }
      const double wa = k.rk == 3 ? w3[st][0] : c4[st];
      const double wb = k.rk == 3 ? w3[st][1] : 0.0;
      launch_faces(with_rec(in, out), k.rk == 3 ? kRk3 : kRk4, st, wa, wb, local ? 1 : 0,
                   st == stages - 1 ? 1 : 0, fused && st == 0);
      if (st == 0) {
        if (fused) {
          launch_as(kNorms, k_norm_collect, 1, 512,
                    static_cast<const unsigned long long*>(norm_words_.as<unsigned long long>()),
                    d_.ctl);
        } else if (n_cases_ > 0) {
          // per case, then the global words as the cases' total (one pass over the residual)
          launch_as(kNorms, k_case_norm_sums, blocks(n_, kBlock * kCaseSpan), kBlock,
                    static_cast<const double*>(res_.as<double>()), n_,
                    static_cast<const int*>(case_of_.as<int>()),
                    static_cast<const unsigned char*>(active_.as<unsigned char>()),
                    case_words_.as<unsigned long long>());
          launch_as(kNorms, k_case_words_total, 2, 256,
                    static_cast<const unsigned long long*>(case_words_.as<unsigned long long>()),
                    n_cases_, d_.ctl);
        } else {
          launch_as(kNorms, k_norm_sums, norm_blocks(), kBlock,
                    static_cast<const double*>(res_.as<double>()), n_, d_.ctl,
                    static_cast<const int*>(nullptr), static_cast<const unsigned char*>(nullptr));
        }
        if (ranked()) reduce_words(&d_.ctl->words[0][0], 5 * kWords, 0);
        launch_as(kNorms, k_norm_finish, 1, 32, d_.ctl, rms_cells(), 1, n_cases_ == 0 ? 1 : 0);
        if (n_cases_ > 0)
          launch_as(kNorms, k_case_norm_finish, blocks(5LL * n_cases_, 128), 128,
                    case_words_.as<unsigned long long>(), static_cast<const double*>(case_cells_.as<double>()),
                    n_cases_, static_cast<const Control*>(d_.ctl), case_hist_.as<double>());
      }
    }
    if (n_cases_ > 0) launch(k_end_step, 1, 32, d_.ctl);  // after the per-case history
  }

  void capture(const StepKey& k) {
    drop_graph();
    const long long before = counters.launches;
    check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      enqueue_step(k);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g != nullptr) cudaGraphDestroy(g);
      throw;
    }
    check(cudaStreamEndCapture(stream, &graph_), "end capture");
    check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "instantiate");
    graph_nodes_ = counters.launches - before;
    counters.launches = before;
    graph_key_ = k;
  }

  void drop_graph() {
    if (graph_exec_ != nullptr) cudaGraphExecDestroy(graph_exec_);
    if (graph_ != nullptr) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
  }

  autan_euler_scheme scheme_;
  bool planar_, second_, limiter_;
  int nc_ = 0, n_ = 0, nf_ = 0, ni_ = 0, nif_ = 0, nb_ = 0;
  int n_ext_ = 0, nv_ = 0;  // external ghosts; owned cells + external ghosts (value records)
  int smem_optin_ = 0;      // the device's opt-in shared memory per block (queried on first use)
  // The ranks of a partitioned mesh (null exchange: one rank), the send list on the device and
  // the widening choice of the mesh's own weights (off while ranks are set: the special-value word
  // would not see the other ranks' records).
  autan_euler_ranks ranks_{};
  Buffer send_cells_;
  int wide_ok_mesh_ = 0;
  Sliced st_, inc_;
  Dev<P> d_{};
  Buffer prim_[3];  // primitive records, rotated through the stages
  Buffer recon_;    // phi and grad of the current stage
  Buffer u_, stage_, racc_, res_, dt_local_, ctl_, volume_;
  Buffer st_start_, st_len_, st_e_, inc_start_, inc_len_, inc_code_, inc_rec_, inc_dt_;
  Buffer bface_r64_, face_mult_, cons_words_;  // boundary pressure and conservation
  Buffer case_of_, case_cells_, case_words_, case_hist_, active_;  // batched cases
  Buffer face_warp_case_, bface_warp_case_, case_minf_;
  int n_cases_ = 0;
  double pref64_ = 0.0;
  int max_faces_ = 0;
  Buffer face_, f_m_, bface_, b_m_, source_;
  std::vector<C> bface_host_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  long long graph_nodes_ = 0;
  StepKey graph_key_{0.0, 0.0, false, 0};
  int last_rec_ = 0;
  int nbo_ = 0;  // boundary faces of owned cells
  Tuning tuning_;
  size_t staged_smem_[2][5] = {};  // [time step staged][slices per block]
  Buffer flux_, bflux_;  // face scratch of the store-gather strategy
  Buffer norm_words_;    // kNormReplicas x 5 x kWords: the fused stage-0 norms' exact sums
  int norm_gather_grid_[9] = {};  // by gather_block / 32
  // Re-packed launches of batched cases (repack): tile lists, their lengths (-1: none), the
  // cases' cell offsets and the host copies of the 32-face warps' cases.
  Buffer cell_tiles_, face_tiles_, bface_tiles_;
  int n_cell_tiles_ = -1, n_face_tiles_ = -1, n_bface_tiles_ = -1;
  std::vector<int64_t> case_offsets_;
  std::vector<int> face_warp_case_h_, bface_warp_case_h_;
  bool step_tiles_ = false;  // set while enqueue_step records: its launches use the tiles
  Control* head_ = nullptr;  // pinned copy of the control's head
  struct Timed {
    int kind;
    cudaEvent_t before, after;
  };
  bool timing_ = false;
  std::vector<Timed> timed_;
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
  } catch (const Failure& e) {
    return fail_to(err, len, e.what());
  } catch (const std::bad_alloc&) {
    return fail_to(err, len, "E1103: out of host memory");
  } catch (const std::exception& e) {
    return fail_to(err, len, std::string("E1100: ") + e.what());
  }
}

struct DeviceGuard {
  int previous = -1;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    if (device >= 0 && device != previous) check(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int now = -1;
    if (cudaGetDevice(&now) == cudaSuccess && previous >= 0 && now != previous)
      cudaSetDevice(previous);
  }
};

Stepper* as_stepper(void* h) {
  if (h == nullptr) fail("E1101: null handle");
  return static_cast<Stepper*>(h);
}

}  // namespace autan_b200

namespace autan_b200 {

// A steady march to the convergence rule (runtime/src/run.cpp:2351-2389), `batch` steps per
// captured-graph call, the rule fed each step's residual RMS from the history.
void march(Stepper* h, double cfl, double dt, bool local, int rk, long long max_steps, int batch,
           double orders, const double* floors, autan_march_result* out) {
  if (out == nullptr) fail("E1101: null result");
  if (max_steps < 1 || batch < 1) fail("E1101: max_steps and batch must be positive");
  if (!(orders > 0.0)) fail("E1101: orders must be positive");
  Convergence conv(orders, floors);
  autan_march_result res{};
  res.invalid_cell = -1;
  std::vector<double> rms(5ULL * batch);
  std::vector<double> dts(static_cast<size_t>(batch));
  cudaEvent_t t0 = nullptr;
  cudaEvent_t t1 = nullptr;
  check(cudaEventCreate(&t0), "event");
  check(cudaEventCreate(&t1), "event");
  check(cudaEventRecord(t0, h->stream), "event");
  long long taken = 0;
  bool invalid = false;  // on any rank of a partitioned mesh
  while (taken < max_steps && !res.converged && !invalid) {
    const long long n = std::min<long long>(batch, max_steps - taken);
    autan_euler_step_result r{};
    h->step(cfl, dt, local, rk, n, true, &r);
    h->history(n, rms.data(), dts.data());
    for (long long i = 0; i < n; ++i) {
      for (int k = 0; k < 5; ++k) res.last[k] = rms[5 * i + k];
      res.time_step = dts[i];
      if (conv.add(rms.data() + 5 * i)) {
        res.converged = 1;
        res.iterations = taken + i + 1;
        res.plateau_mask = conv.plateau_mask();
        break;
      }
    }
    taken += n;
    res.invalid_cell = r.invalid_cell;
    invalid = h->any_rank(r.invalid_cell >= 0);
  }
  check(cudaEventRecord(t1, h->stream), "event");
  check(cudaEventSynchronize(t1), "event");
  float ms = 0.0f;
  check(cudaEventElapsedTime(&ms, t0, t1), "event");
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (!res.converged) res.iterations = taken;
  res.steps = taken;
  res.gpu_ms = ms;
  for (int k = 0; k < 5; ++k) res.first[k] = conv.first()[k];
  *out = res;
}

// The batched march: one convergence rule per case, fed that case's row of each step's per-case
// RMS; a case that meets its rule stops stepping (its cells are skipped from the next batch on).
void march_cases(Stepper* h, double cfl, double dt, bool local, int rk, long long max_steps,
                 int batch, double orders, const double* floors, const double* reference,
                 int64_t* iterations, int32_t* converged, double* first, int64_t* steps_taken,
                 double* gpu_ms, double* stop_ms) {
  const int nk = h->n_cases();
  if (nk == 0) fail("E1101: no cases set");
  if (max_steps < 1 || batch < 1) fail("E1101: max_steps and batch must be positive");
  if (!(orders > 0.0)) fail("E1101: orders must be positive");
  if (iterations == nullptr || converged == nullptr) fail("E1101: null outputs");
  std::vector<Convergence> conv;
  conv.reserve(nk);
  for (int k = 0; k < nk; ++k)
    conv.emplace_back(orders, floors != nullptr ? floors + 5 * k : nullptr,
                      reference != nullptr ? reference + 5 * k : nullptr);
  std::vector<uint8_t> active(nk, 1);
  for (int k = 0; k < nk; ++k) {
    iterations[k] = 0;
    converged[k] = 0;
    if (stop_ms != nullptr) stop_ms[k] = -1.0;
  }
  h->set_active(active.data());
  std::vector<double> rms(5ULL * nk * batch);
  cudaEvent_t t0 = nullptr;
  cudaEvent_t t1 = nullptr;
  cudaEvent_t tb = nullptr;
  check(cudaEventCreate(&t0), "event");
  check(cudaEventCreate(&t1), "event");
  check(cudaEventCreate(&tb), "event");
  check(cudaEventRecord(t0, h->stream), "event");
  long long taken = 0;
  int left = nk;
  const int workers = std::max(1, std::min<int>(static_cast<int>(std::thread::hardware_concurrency()),
                                                 nk / 32));
  while (taken < max_steps && left > 0) {
    const long long n = std::min<long long>(batch, max_steps - taken);
    autan_euler_step_result r{};
    h->step(cfl, dt, local, rk, n, true, &r);
    h->case_history(n, rms.data());
    // Each case's rule over this batch; the cases are independent, so interleaved subsets of
    // them go to host threads.
    std::vector<int> done(workers, 0);
    auto run = [&](int w) {
      for (int k = w; k < nk; k += workers) {
        if (!active[k]) continue;
        for (long long i = 0; i < n; ++i) {
          if (conv[k].add(rms.data() + (i * nk + k) * 5)) {
            iterations[k] = taken + i + 1;
            converged[k] = 1;
            active[k] = 0;
            ++done[w];
            break;
          }
        }
      }
    };
    if (workers == 1) {
      run(0);
    } else {
      std::vector<std::thread> pool;
      for (int w = 1; w < workers; ++w) pool.emplace_back(run, w);
      run(0);
      for (auto& t : pool) t.join();
    }
    int newly = 0;
    for (int v : done) newly += v;
    const bool changed = newly > 0;
    if (changed && stop_ms != nullptr) {
      // the device time so far (the batch's steps have completed: step() synchronised)
      check(cudaEventRecord(tb, h->stream), "event");
      check(cudaEventSynchronize(tb), "event");
      float now = 0.0f;
      check(cudaEventElapsedTime(&now, t0, tb), "event");
      for (int k = 0; k < nk; ++k)
        if (converged[k] && stop_ms[k] < 0.0) stop_ms[k] = now;
    }
    left -= newly;
    taken += n;
    if (changed) h->set_active(active.data());
    if (r.invalid_cell >= 0) break;
  }
  check(cudaEventRecord(t1, h->stream), "event");
  check(cudaEventSynchronize(t1), "event");
  float ms = 0.0f;
  check(cudaEventElapsedTime(&ms, t0, t1), "event");
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(tb);
  if (stop_ms != nullptr)
    for (int k = 0; k < nk; ++k)
      if (stop_ms[k] < 0.0) stop_ms[k] = ms;
  for (int k = 0; k < nk; ++k)
    if (!converged[k]) iterations[k] = taken;
  if (first != nullptr)
    for (int k = 0; k < nk; ++k)
      for (int e = 0; e < 5; ++e) first[5 * k + e] = conv[k].first()[e];
  // every case steps again (evaluations after the march see every case)
  std::fill(active.begin(), active.end(), static_cast<uint8_t>(1));
  h->set_active(active.data());
  if (steps_taken != nullptr) *steps_taken = taken;
  if (gpu_ms != nullptr) *gpu_ms = ms;
}

}  // namespace autan_b200

using namespace autan_b200;

extern "C" {

int autan_euler_device_create(const autan_euler_mesh* mesh, const autan_euler_scheme* scheme,
                              int32_t device, void* stream, void** handle, char* err,
                              size_t err_len) {
  return guarded(err, err_len, [&] {
    if (mesh == nullptr || scheme == nullptr || handle == nullptr) fail("E1101: null argument");
    int count = 0;
    check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (device >= count) fail("E1101: no such device");
    int dev = device;
    if (dev < 0) check(cudaGetDevice(&dev), "cudaGetDevice");
    DeviceGuard guard(dev);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    bool own = false;
    if (s == nullptr) {
      check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
      own = true;
    }
    std::unique_ptr<Stepper> h;
    try {
      if (scheme->precision == AUTAN_FP64) {
        h = std::make_unique<Impl<Fp64>>(*mesh, *scheme, s);
      } else if (scheme->precision == AUTAN_FP32_ACC64) {
        h = std::make_unique<Impl<Fp32Acc64>>(*mesh, *scheme, s);
      } else {
        fail("E1102: unknown precision policy");
      }
    } catch (...) {
      if (own) cudaStreamDestroy(s);
      throw;
    }
    h->own_stream = own;
    h->device = dev;
    *handle = h.release();
  });
}

void autan_euler_device_destroy(void* handle) {
  if (handle == nullptr) return;
  auto* h = static_cast<Stepper*>(handle);
  DeviceGuard guard(h->device);
  cudaStream_t s = h->stream;
  const bool own = h->own_stream;
  cudaStreamSynchronize(s);
  delete h;
  if (own) cudaStreamDestroy(s);
}

#define AUTAN_CALL(body)             \
  return guarded(err, err_len, [&] { \
    auto* h = as_stepper(handle);    \
    DeviceGuard guard(h->device);    \
    body;                            \
  })

int autan_euler_device_set_boundary(void* handle, const uint8_t* kind, const double* data,
                                    int64_t n_boundary, char* err, size_t err_len) {
  AUTAN_CALL({
    if (kind == nullptr || data == nullptr) fail("E1101: null boundary arrays");
    (void)n_boundary;
    h->set_boundary(kind, data);
  });
}

int autan_euler_device_set_boundary_data(void* handle, const double* data, int64_t n_boundary,
                                         char* err, size_t err_len) {
  AUTAN_CALL({
    if (data == nullptr) fail("E1101: null boundary data");
    (void)n_boundary;
    h->set_boundary_data(data);
  });
}

int autan_euler_device_set_source(void* handle, const double* source, char* err, size_t err_len) {
  AUTAN_CALL({
    if (source == nullptr) fail("E1101: null source");
    h->set_source(source);
  });
}

int autan_euler_device_set_second_order(void* handle, int32_t on, char* err, size_t err_len) {
  AUTAN_CALL(h->set_second_order(on != 0));
}

int autan_euler_device_upload(void* handle, const double* u, char* err, size_t err_len) {
  AUTAN_CALL({
    if (u == nullptr) fail("E1101: null state");
    h->upload_state(u);
  });
}

int autan_euler_device_download(void* handle, double* u, char* err, size_t err_len) {
  AUTAN_CALL({
    if (u == nullptr) fail("E1101: null state");
    h->download_state(u);
  });
}

int autan_euler_device_residual(void* handle, const double* u, double* res, char* err,
                                size_t err_len) {
  AUTAN_CALL({
    if (u == nullptr || res == nullptr) fail("E1101: null arrays");
    h->residual(u, res);
  });
}

int autan_euler_device_step(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                            int64_t n_steps, int32_t use_graph, autan_euler_step_result* out,
                            char* err, size_t err_len) {
  AUTAN_CALL({
    autan_euler_step_result r{};
    h->step(cfl, dt, local != 0, rk, n_steps, use_graph != 0, &r);
    if (out != nullptr) *out = r;
  });
}

int autan_euler_device_evaluate(void* handle, autan_euler_step_result* out, char* err,
                                size_t err_len) {
  AUTAN_CALL({
    autan_euler_step_result r{};
    h->evaluate(&r);
    if (out != nullptr) *out = r;
  });
}

int autan_euler_device_history(void* handle, int64_t count, double* rms, double* dt, char* err,
                               size_t err_len) {
  AUTAN_CALL(h->history(count, rms, dt));
}

int autan_euler_device_gradients(void* handle, double* grad, double* phi, char* err,
                                 size_t err_len) {
  AUTAN_CALL(h->gradients(grad, phi));
}

int autan_euler_device_time_steps(void* handle, double cfl, double* dt, char* err,
                                  size_t err_len) {
  AUTAN_CALL({
    if (dt == nullptr) fail("E1101: null output");
    h->time_steps(cfl, dt);
  });
}

int autan_euler_device_kernel_times(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                    int64_t n_steps, double* ms, int64_t* launches, char* err,
                                    size_t err_len) {
  AUTAN_CALL({
    if (ms == nullptr || launches == nullptr) fail("E1101: null output");
    if (rk != 3 && rk != 4) fail("E1101: rk must be 3 or 4");
    long long l[6];
    h->kernel_times(cfl, dt, local != 0, rk, n_steps, ms, l);
    for (int k = 0; k < 6; ++k) launches[k] = l[k];
  });
}

int autan_euler_device_set_tuning(void* handle, const int32_t* params, int32_t count, char* err,
                                  size_t err_len) {
  AUTAN_CALL({
    if (params == nullptr || (count != Tuning::kMinCount && count < Tuning::kCount))
      fail("E1101: 6 or 10 tuning parameters expected");
    int32_t all[Tuning::kCount];
    h->tuning().to(all);
    for (int i = 0; i < std::min<int>(count, Tuning::kCount); ++i) all[i] = params[i];
    h->set_tuning(Tuning::from(all));
  });
}

int autan_euler_device_get_tuning(void* handle, int32_t* params, int32_t count, char* err,
                                  size_t err_len) {
  AUTAN_CALL({
    if (params == nullptr || count < Tuning::kCount) fail("E1101: room for 10 parameters expected");
    h->tuning().to(params);
  });
}

int autan_euler_device_autotune(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                int32_t trial_steps, int32_t* params, double* ms_per_step,
                                char* err, size_t err_len) {
  AUTAN_CALL({
    if (rk != 3 && rk != 4) fail("E1101: rk must be 3 or 4");
    const double ms = h->autotune(cfl, dt, local != 0, rk, trial_steps);
    if (params != nullptr) h->tuning().to(params);
    if (ms_per_step != nullptr) *ms_per_step = ms;
  });
}

int autan_euler_device_face_parts(void* handle, const double* u, double* res_faces,
                                  double* face_flux, char* err, size_t err_len) {
  AUTAN_CALL(h->face_parts(u, res_faces, face_flux));
}

int autan_euler_device_boundary_pressure(void* handle, const double* u, double* p, double* force,
                                         char* err, size_t err_len) {
  AUTAN_CALL({
    if (p == nullptr) fail("E1101: null pressure output");
    h->boundary_pressure(u, p, force);
  });
}

int autan_euler_device_conservation(void* handle, double* sums, int32_t* max_faces, char* err,
                                    size_t err_len) {
  AUTAN_CALL({
    if (sums == nullptr) fail("E1101: null output");
    const int d = h->conservation(sums);
    if (max_faces != nullptr) *max_faces = d;
  });
}

int autan_euler_device_march(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                             int64_t max_steps, int32_t batch, double orders, const double* floors,
                             autan_march_result* out, char* err, size_t err_len) {
  AUTAN_CALL(march(h, cfl, dt, local != 0, rk, max_steps, batch, orders, floors, out));
}

int autan_euler_device_set_cases(void* handle, int32_t n_cases, const int64_t* cell_offsets,
                                 char* err, size_t err_len) {
  AUTAN_CALL(h->set_cases(n_cases, cell_offsets));
}

int autan_euler_device_set_case_mach_ref(void* handle, const double* mach_ref, char* err,
                                         size_t err_len) {
  AUTAN_CALL({
    if (mach_ref == nullptr) fail("E1101: null cut-off Mach numbers");
    h->set_case_mach_ref(mach_ref);
  });
}

int autan_euler_device_set_active(void* handle, const uint8_t* active, char* err, size_t err_len) {
  AUTAN_CALL({
    if (active == nullptr) fail("E1101: null active flags");
    h->set_active(active);
  });
}

int autan_euler_device_case_history(void* handle, int64_t count, double* rms, char* err,
                                    size_t err_len) {
  AUTAN_CALL({
    if (rms == nullptr) fail("E1101: null output");
    h->case_history(count, rms);
  });
}

int autan_euler_device_march_cases(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                   int64_t max_steps, int32_t batch, double orders,
                                   const double* floors, const double* reference,
                                   int64_t* iterations, int32_t* converged, double* first,
                                   int64_t* steps, double* gpu_ms, double* stop_ms, char* err,
                                   size_t err_len) {
  AUTAN_CALL(march_cases(h, cfl, dt, local != 0, rk, max_steps, batch, orders, floors, reference,
                         iterations, converged, first, steps, gpu_ms, stop_ms));
}

int autan_euler_device_set_stall_test(void* handle, int32_t polls, char* err, size_t err_len) {
  AUTAN_CALL({ h->set_stall_test(polls); });
}

int autan_euler_device_set_ranks(void* handle, const autan_euler_ranks* ranks, char* err,
                                 size_t err_len) {
  AUTAN_CALL({ h->set_ranks(ranks); });
}

int autan_euler_device_external_ghosts(void* handle, int64_t* count, char* err, size_t err_len) {
  AUTAN_CALL({
    if (count == nullptr) fail("E1101: null count");
    *count = h->external_ghosts();
  });
}

int autan_euler_device_sync(void* handle, char* err, size_t err_len) {
  AUTAN_CALL(check(cudaStreamSynchronize(h->stream), "sync"));
}

void* autan_euler_device_stream(void* handle) {
  return handle == nullptr ? nullptr : static_cast<void*>(static_cast<Stepper*>(handle)->stream);
}

int autan_euler_device_counters(void* handle, int64_t* counters, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    auto* h = as_stepper(handle);
    counters[0] = h->counters.launches;
    counters[1] = h->counters.steps;
    counters[2] = h->counters.residuals;
    counters[3] = h->device_bytes();
  });
}

}  // extern "C"
