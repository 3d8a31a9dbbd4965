// The per-cell rules of the gradient set-up, shared by the host set-up (setup.cpp) and the GPU
// set-up (setup_device.cu): one source, compiled by g++ with -ffp-contract=off and by nvcc with
// --fmad=false, so both give the same bits.
//
//   face2_entries    the face2 stencil of a cell (codegen/cpp/geometry.cpp:432, StencilKind::face2,
//                    no global keys): the cells across its faces and the cells across their faces,
//                    the cell itself left out, ascending; then the boundary faces of the cell and of
//                    those face neighbours, ascending, each written as -(f + 1).
//   lsq_cell_weights the least-squares gradient weights of one cell over its stencil
//                    (physics/src/euler.cpp:340-416, Euler::Impl::compute_gradient_weights).
//
// Both are written for one thread per cell with a fixed candidate buffer: the stencil gathers its
// candidates into the buffer and sorts them there (no marks over all cells, which a GPU thread
// cannot hold); the weights walk the stencil twice, the first pass forming the 3 x 3 normal matrix
// and the second recomputing each offset to write its weights (nothing stored per entry).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define AUTAN_HD __host__ __device__ __forceinline__
#else
#define AUTAN_HD inline
#endif

namespace autan_b200 {
namespace setup {

// Topology and geometry the rules read (device or host pointers, the mesh contract's layouts).
struct MeshView {
  int32_t n_cells, n_owned, n_faces, n_interior;
  const int64_t* cell_face_offsets;  // n_cells + 1
  const int32_t* cell_faces;
  const int32_t* owner;      // n_faces
  const int32_t* neighbour;  // n_interior
  const double* cell_centroid;  // 3 x n_cells
  const double* face_centroid;  // 3 x n_faces
};

// Largest number of candidates (with repeats) a cell's stencil may gather.
constexpr int kMaxCandidates = 512;

// Sorts v[0..n) ascending and drops repeats; returns the number kept.
AUTAN_HD int sort_unique(int32_t* v, int n) {
  for (int i = 1; i < n; ++i) {
    const int32_t x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
  int kept = 0;
  for (int i = 0; i < n; ++i)
    if (kept == 0 || v[kept - 1] != v[i]) v[kept++] = v[i];
  return kept;
}

// The face2 stencil of cell c into out (when not null) as the contract writes it; returns its
// length, or -1 when the candidates exceed `cap` (buf holds cap ints of scratch). Candidates:
// interior neighbours encoded as themselves, boundary faces as n_cells + f, so one sort orders
// cells before boundary faces, each ascending.
AUTAN_HD int face2_entries(const MeshView& m, int32_t c, int32_t* buf, int cap, int32_t* out) {
  int n = 0;
  const int32_t nc = m.n_cells, ni = m.n_interior;
  for (int64_t k = m.cell_face_offsets[c]; k < m.cell_face_offsets[c + 1]; ++k) {
    const int32_t f = m.cell_faces[k];
    if (f >= ni) {
      if (n >= cap) return -1;
      buf[n++] = nc + f;
      continue;
    }
    const int32_t nb = m.owner[f] == c ? m.neighbour[f] : m.owner[f];
    if (n >= cap) return -1;
    buf[n++] = nb;
    for (int64_t k2 = m.cell_face_offsets[nb]; k2 < m.cell_face_offsets[nb + 1]; ++k2) {
      const int32_t f2 = m.cell_faces[k2];
      int32_t x;
      if (f2 >= ni) {
        x = nc + f2;
      } else {
        x = m.owner[f2] == nb ? m.neighbour[f2] : m.owner[f2];
        if (x == c) continue;
      }
      if (n >= cap) return -1;
      buf[n++] = x;
    }
  }
  const int kept = sort_unique(buf, n);
  if (out != nullptr)
    for (int i = 0; i < kept; ++i) out[i] = buf[i] < nc ? buf[i] : -(buf[i] - nc) - 1;
  return kept;
}

// The offset of stencil entry e of cell c, FP64, component by component: the entry's point (a
// cell centroid, or for -(f + 1) boundary face f's centroid) minus the cell's centroid, a
// component within 64 ulps of the larger coordinate counted as zero (round-off across a
// one-cell-thick layer, not geometry). `fit`: whether the entry enters the fit (boundary faces
// only where their condition fixes the state, kind 0, or where `all_boundaries`).
AUTAN_HD void entry_offset(const MeshView& m, int32_t c, int32_t e, const uint8_t* bc_kind,
                           bool all_boundaries, double* d, bool* fit) {
  const double* px;
  int64_t stride, at;
  *fit = true;
  if (e >= 0) {
    px = m.cell_centroid;
    stride = m.n_cells;
    at = e;
  } else {
    const int32_t f = -e - 1;
    px = m.face_centroid;
    stride = m.n_faces;
    at = f;
    *fit = all_boundaries || bc_kind[f - m.n_interior] == 0;
  }
  const double eps = 2.220446049250313e-16;  // 2^-52, the FP64 coordinates' epsilon
  for (int j = 0; j < 3; ++j) {
    const double x = px[j * stride + at];
    const double xc = m.cell_centroid[j * static_cast<int64_t>(m.n_cells) + c];
    const double ax = x < 0.0 ? -x : x, axc = xc < 0.0 ? -xc : xc;
    const double big = ax < axc ? axc : ax;
    const double diff = x - xc;
    const double adiff = diff < 0.0 ? -diff : diff;
    d[j] = adiff <= 64.0 * eps * big ? 0.0 : diff;
  }
}

// The fit's weight of an entry: 1 / |d|^2, or 0 for an entry left out.
AUTAN_HD double inverse_square(const double* d, bool fit) {
  return fit ? 1.0 / (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) : 0.0;
}

// One attempt at cell c's weights: the normal matrix a (row-major) summed over the stencil
// [begin, end), each entry adding s d_u d_v as (s d_u) d_v; a fit is accepted when
// |det a| > 1e-10 |a00 a11 a22|; then w_u = s (row u of a^-1 . d), the inverse by cofactors over
// the determinant. Returns false (nothing written) for a rejected fit.
AUTAN_HD bool lsq_attempt(const MeshView& m, int32_t c, int64_t begin, int64_t end,
                          const int32_t* entries, const uint8_t* bc_kind, bool all_boundaries,
                          double* w, int64_t n_stencil) {
  double a[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t k = begin; k < end; ++k) {
    double d[3];
    bool fit;
    entry_offset(m, c, entries[k], bc_kind, all_boundaries, d, &fit);
    const double s = inverse_square(d, fit);
    for (int u = 0; u < 3; ++u) {
      const double su = s * d[u];
      for (int v = 0; v < 3; ++v) a[3 * u + v] += su * d[v];
    }
  }
  // cofactors of the first row, then the determinant expanded along it
  const double c00 = a[4] * a[8] - a[5] * a[7];
  const double c01 = a[3] * a[8] - a[5] * a[6];
  const double c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 - a[1] * c01 + a[2] * c02;
  const double diag = a[0] * a[4] * a[8];
  const double adet = det < 0.0 ? -det : det, adiag = diag < 0.0 ? -diag : diag;
  if (!(adet > 1e-10 * adiag)) return false;
  double inv[9];
  inv[0] = c00 / det;
  inv[1] = (a[2] * a[7] - a[1] * a[8]) / det;
  inv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
  inv[3] = (a[5] * a[6] - a[3] * a[8]) / det;
  inv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
  inv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
  inv[6] = c02 / det;
  inv[7] = (a[1] * a[6] - a[0] * a[7]) / det;
  inv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
  for (int64_t k = begin; k < end; ++k) {
    double d[3];
    bool fit;
    entry_offset(m, c, entries[k], bc_kind, all_boundaries, d, &fit);
    const double s = inverse_square(d, fit);
    for (int u = 0; u < 3; ++u)
      w[u * n_stencil + k] = s * (inv[3 * u] * d[0] + inv[3 * u + 1] * d[1] + inv[3 * u + 2] * d[2]);
  }
  return true;
}

// Cell c's weights (3 x n_stencil, component-major): the boundary faces of other conditions left
// out of the fit unless the cell's remaining entries do not determine a gradient, in which case
// every boundary face enters. Returns 1 when that retry was needed, 2 when no fit was accepted
// (weights left as they were), 0 otherwise.
AUTAN_HD int lsq_cell_weights(const MeshView& m, int32_t c, const int64_t* offsets,
                              const int32_t* entries, const uint8_t* bc_kind, double* w,
                              int64_t n_stencil) {
  const int64_t begin = offsets[c], end = offsets[c + 1];
  if (lsq_attempt(m, c, begin, end, entries, bc_kind, false, w, n_stencil)) return 0;
  return lsq_attempt(m, c, begin, end, entries, bc_kind, true, w, n_stencil) ? 1 : 2;
}

}  // namespace setup
}  // namespace autan_b200
