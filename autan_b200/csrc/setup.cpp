// Host set-up of the explicit Euler path: face-based mesh assembly, FP64 geometry, face2 stencil
// and BC-aware least-squares weights, in the layouts of Autan's mesh contract
// (docs/contracts/mesh.md). Every function cites the reference function it stands in for.
#include "autan_b200_setup.h"
#include "autan_euler_device.h"
#include "convergence.hpp"
#include "setup_rules.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

namespace setup = autan_b200::setup;
using i32 = std::int32_t;
using i64 = std::int64_t;
using Vec = std::array<double, 3>;

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const char* code, const std::string& what) {
  throw Failure(std::string(code) + ": " + what);
}

// A mesh given cell by cell: each cell a list of outward node loops (CellwiseMesh of
// core/include/autan/core/cellwise.hpp, restricted to what the generators here produce).
struct Cellwise {
  std::vector<double> x, y, z;
  std::vector<i64> cell_face_offsets{0};
  std::vector<i64> face_node_offsets{0};
  std::vector<i32> face_nodes;
  std::vector<i32> face_zone;  // per cell face: boundary zone when unshared, -1 when it must be shared
  std::vector<i32> image;      // per cell: -1 owned, else the owned cell (this numbering) it copies
  std::vector<double> shift;   // 3 per cell: translation of an image
  i32 n_cells() const { return static_cast<i32>(cell_face_offsets.size() - 1); }
};

struct Mesh {
  i32 n_cells = 0, n_owned = 0, n_faces = 0, n_interior = 0, n_owned_interior = 0,
      n_owned_faces = 0, n_zones = 0;
  std::vector<double> points;  // 3 x n_points
  std::vector<i64> face_node_offsets{0};
  std::vector<i32> face_nodes;
  std::vector<i32> owner, neighbour, face_zone;
  std::vector<i64> cell_face_offsets;
  std::vector<i32> cell_faces;
  std::vector<i32> ghost_owner, owned_order;
  std::vector<double> ghost_translation;
  // Geometry (SoA, FP64).
  std::vector<double> face_area, face_area_magnitude, face_normal, face_centroid, face_moment;
  std::vector<double> cell_centroid, cell_volume;
  bool all_planar = true;
  // face2 stencil (codegen/include/autan/kernels/geometry.hpp CellStencil).
  std::vector<i64> stencil_offsets;
  std::vector<i32> stencil;
  i64 n_points() const { return static_cast<i64>(points.size() / 3); }
};

std::uint64_t mix(std::uint64_t h) {
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdULL;
  h ^= h >> 33;
  h *= 0xc4ceb9fe1a85ec53ULL;
  h ^= h >> 33;
  return h;
}

// ------------------------------------------------------------------ reverse Cuthill-McKee

// Reverse Cuthill-McKee order of a graph in CSR form (core/src/renumber.cpp:109 rcm_order):
// breadth-first from a pseudo-peripheral vertex of least degree, neighbours by increasing
// degree, the whole order reversed. Returns new -> old.
std::vector<i32> rcm(i32 n, const std::vector<i64>& off, const std::vector<i32>& adj) {
  std::vector<i32> order;
  order.reserve(static_cast<std::size_t>(n));
  std::vector<char> seen(static_cast<std::size_t>(n), 0);
  std::vector<i32> level(static_cast<std::size_t>(n), -1);
  auto degree = [&](i32 v) { return off[v + 1] - off[v]; };
  std::vector<i32> queue, nb;
  auto bfs_last = [&](i32 s, std::vector<i32>& touched) {
    // Breadth-first levels from s; returns a vertex of the last level of least degree.
    queue.assign(1, s);
    level[s] = 0;
    touched.assign(1, s);
    i32 best = s;
    for (std::size_t h = 0; h < queue.size(); ++h) {
      const i32 v = queue[h];
      if (level[v] > level[best] || (level[v] == level[best] && degree(v) < degree(best)))
        best = v;
      for (i64 k = off[v]; k < off[v + 1]; ++k) {
        const i32 w = adj[k];
        if (level[w] < 0) {
          level[w] = level[v] + 1;
          queue.push_back(w);
          touched.push_back(w);
        }
      }
    }
    for (const i32 v : touched) level[v] = -1;
    return best;
  };
  std::vector<i32> touched;
  for (i32 root = 0; root < n; ++root) {
    if (seen[root]) continue;
    i32 start = root;
    for (int pass = 0; pass < 2; ++pass) start = bfs_last(start, touched);
    const std::size_t first = order.size();
    order.push_back(start);
    seen[start] = 1;
    for (std::size_t h = first; h < order.size(); ++h) {
      const i32 v = order[h];
      nb.clear();
      for (i64 k = off[v]; k < off[v + 1]; ++k) {
        const i32 w = adj[k];
        if (!seen[w]) {
          seen[w] = 1;
          nb.push_back(w);
        }
      }
      std::stable_sort(nb.begin(), nb.end(),
                       [&](i32 a, i32 b) { return degree(a) < degree(b); });
      order.insert(order.end(), nb.begin(), nb.end());
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

// ------------------------------------------------------------------ assembly

struct Instance {
  std::uint64_t hash;
  i64 face;  // cell face index in the Cellwise numbering
};

// to_face_based + assemble (core/src/cellwise.cpp, core/src/mesh.cpp:273): cell faces shared by
// two cells become interior faces, owner the lower cell index, oriented by its loop; unshared
// faces on a boundary zone become boundary faces. With images: owned cells first, then the ghosts
// within two face layers of them; faces that touch an owned cell or a first-layer ghost are kept.
// Interior faces sorted by (owner, neighbour); boundary faces of owned cells, then of ghosts,
// each by (zone, owner); each cell's faces in increasing index.
Mesh assemble(const Cellwise& in, int order) {
  const i32 ncw = in.n_cells();
  const i64 ncf = static_cast<i64>(in.face_node_offsets.size()) - 1;
  std::vector<i32> face_cell(static_cast<std::size_t>(ncf));
  for (i32 c = 0; c < ncw; ++c)
    for (i64 f = in.cell_face_offsets[c]; f < in.cell_face_offsets[c + 1]; ++f) face_cell[f] = c;

  // Match cell faces by node set.
  auto sorted_nodes = [&](i64 f, std::array<i32, 16>& out) {
    const i64 b = in.face_node_offsets[f], e = in.face_node_offsets[f + 1];
    const i64 n = e - b;
    if (n < 3 || n > 16) fail("E0113", "a face has fewer than 3 or more than 16 nodes");
    for (i64 i = 0; i < n; ++i) out[i] = in.face_nodes[b + i];
    std::sort(out.begin(), out.begin() + n);
    return static_cast<int>(n);
  };
  std::vector<Instance> inst(static_cast<std::size_t>(ncf));
  {
    std::array<i32, 16> s{};
    for (i64 f = 0; f < ncf; ++f) {
      const int n = sorted_nodes(f, s);
      std::uint64_t h = 0x9e3779b97f4a7c15ULL * static_cast<std::uint64_t>(n);
      for (int i = 0; i < n; ++i) h = mix(h ^ (static_cast<std::uint64_t>(s[i]) + 0x632be59bd9b4e019ULL));
      inst[f] = {h, f};
    }
  }
  std::sort(inst.begin(), inst.end(), [](const Instance& a, const Instance& b) {
    return a.hash != b.hash ? a.hash < b.hash : a.face < b.face;
  });
  std::vector<i64> partner(static_cast<std::size_t>(ncf), -1);
  {
    std::array<i32, 16> sa{}, sb{};
    for (std::size_t i = 0; i < inst.size();) {
      std::size_t j = i;
      while (j < inst.size() && inst[j].hash == inst[i].hash) ++j;
      for (std::size_t a = i; a < j; ++a) {
        if (partner[inst[a].face] >= 0) continue;
        const int na = sorted_nodes(inst[a].face, sa);
        for (std::size_t b = a + 1; b < j; ++b) {
          const int nb = sorted_nodes(inst[b].face, sb);
          if (na != nb || !std::equal(sa.begin(), sa.begin() + na, sb.begin())) continue;
          if (partner[inst[b].face] >= 0) fail("E0114", "a face is shared by more than two cells");
          partner[inst[a].face] = inst[b].face;
          partner[inst[b].face] = inst[a].face;
          break;
        }
      }
      i = j;
    }
  }

  // Ghost layers: breadth-first distance from the owned cells over shared faces.
  std::vector<i32> layer(static_cast<std::size_t>(ncw), -1);
  std::vector<i32> queue;
  for (i32 c = 0; c < ncw; ++c)
    if (in.image[c] < 0) {
      layer[c] = 0;
      queue.push_back(c);
    }
  for (std::size_t h = 0; h < queue.size(); ++h) {
    const i32 c = queue[h];
    if (layer[c] >= 2) continue;
    for (i64 f = in.cell_face_offsets[c]; f < in.cell_face_offsets[c + 1]; ++f) {
      if (partner[f] < 0) continue;
      const i32 o = face_cell[partner[f]];
      if (layer[o] < 0) {
        layer[o] = layer[c] + 1;
        queue.push_back(o);
      }
    }
  }
  for (i32 c = 0; c < ncw; ++c) {
    if (in.image[c] >= 0 && in.image[in.image[c]] >= 0)
      fail("E0118", "a periodic image must copy an owned cell");
    if (in.image[c] < 0) {
      for (i64 f = in.cell_face_offsets[c]; f < in.cell_face_offsets[c + 1]; ++f)
        if (partner[f] < 0 && in.face_zone[f] < 0)
          fail("E0115", "owned cell " + std::to_string(c) + " has an open face");
    }
  }

  // Owned cells: generator order or RCM over the owned-to-owned faces.
  std::vector<i32> owned_cw;
  for (i32 c = 0; c < ncw; ++c)
    if (in.image[c] < 0) owned_cw.push_back(c);
  const i32 n_owned = static_cast<i32>(owned_cw.size());
  std::vector<i32> owned_index(static_cast<std::size_t>(ncw), -1);
  for (i32 i = 0; i < n_owned; ++i) owned_index[owned_cw[i]] = i;
  if (order == 2) {
    // Morton (Z-order) of the cells' node means, quantised to 21 bits per axis over the owned
    // cells' bounding box: a warp's 32 consecutive cells form a compact blob whose stencils
    // overlap, so neighbours' records are shared within the warp and stay in cache.
    std::vector<std::array<double, 3>> centre(static_cast<std::size_t>(n_owned));
    std::array<double, 3> lo{1e300, 1e300, 1e300}, hi{-1e300, -1e300, -1e300};
    for (i32 i = 0; i < n_owned; ++i) {
      const i32 c = owned_cw[i];
      std::array<double, 3> m{0.0, 0.0, 0.0};
      i64 count = 0;
      for (i64 f = in.cell_face_offsets[c]; f < in.cell_face_offsets[c + 1]; ++f)
        for (i64 k = in.face_node_offsets[f]; k < in.face_node_offsets[f + 1]; ++k) {
          const i32 p = in.face_nodes[k];
          m[0] += in.x[p];
          m[1] += in.y[p];
          m[2] += in.z[p];
          ++count;
        }
      for (int a = 0; a < 3; ++a) {
        m[a] /= static_cast<double>(count);
        lo[a] = std::min(lo[a], m[a]);
        hi[a] = std::max(hi[a], m[a]);
      }
      centre[i] = m;
    }
    auto spread = [](std::uint64_t v) {
      v &= 0x1fffffULL;
      v = (v | v << 32) & 0x1f00000000ffffULL;
      v = (v | v << 16) & 0x1f0000ff0000ffULL;
      v = (v | v << 8) & 0x100f00f00f00f00fULL;
      v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
      v = (v | v << 2) & 0x1249249249249249ULL;
      return v;
    };
    std::vector<std::pair<std::uint64_t, i32>> key(static_cast<std::size_t>(n_owned));
    // One scale for the three axes, so that the curve's boxes stay cubes on a flat domain.
    double span = 0.0;
    for (int a = 0; a < 3; ++a) span = std::max(span, hi[a] - lo[a]);
    if (!(span > 0.0)) span = 1.0;
    for (i32 i = 0; i < n_owned; ++i) {
      std::uint64_t q[3];
      for (int a = 0; a < 3; ++a)
        q[a] = static_cast<std::uint64_t>((centre[i][a] - lo[a]) / span * 2097151.0);
      key[i] = {spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2, owned_cw[i]};
    }
    std::stable_sort(key.begin(), key.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (i32 i = 0; i < n_owned; ++i) owned_cw[i] = key[i].second;
  } else if (order == 1) {
    std::vector<i64> off(static_cast<std::size_t>(n_owned) + 1, 0);
    std::vector<i32> adj;
    for (i32 i = 0; i < n_owned; ++i) {
      const i32 c = owned_cw[i];
      for (i64 f = in.cell_face_offsets[c]; f < in.cell_face_offsets[c + 1]; ++f) {
        if (partner[f] < 0) continue;
        const i32 o = owned_index[face_cell[partner[f]]];
        if (o >= 0) adj.push_back(o);
      }
      off[i + 1] = static_cast<i64>(adj.size());
    }
    const auto order = rcm(n_owned, off, adj);
    std::vector<i32> reordered(static_cast<std::size_t>(n_owned));
    for (i32 i = 0; i < n_owned; ++i) reordered[i] = owned_cw[order[i]];
    owned_cw.swap(reordered);
  }
  std::vector<i32> ghosts_cw;
  for (i32 c = 0; c < ncw; ++c)
    if (in.image[c] >= 0 && layer[c] >= 1 && layer[c] <= 2) ghosts_cw.push_back(c);
  std::stable_sort(ghosts_cw.begin(), ghosts_cw.end(),
                   [&](i32 a, i32 b) { return layer[a] < layer[b]; });

  Mesh m;
  m.n_owned = n_owned;
  m.n_cells = n_owned + static_cast<i32>(ghosts_cw.size());
  std::vector<i32> new_index(static_cast<std::size_t>(ncw), -1);
  for (i32 i = 0; i < n_owned; ++i) new_index[owned_cw[i]] = i;
  for (std::size_t g = 0; g < ghosts_cw.size(); ++g)
    new_index[ghosts_cw[g]] = n_owned + static_cast<i32>(g);
  m.owned_order = owned_cw;
  for (const i32 c : ghosts_cw) {
    m.ghost_owner.push_back(new_index[in.image[c]]);
    if (m.ghost_owner.back() < 0) fail("E0118", "an image copies a cell outside the mesh");
  }
  m.ghost_translation.assign(3 * ghosts_cw.size(), 0.0);
  for (std::size_t g = 0; g < ghosts_cw.size(); ++g)
    for (int a = 0; a < 3; ++a)
      m.ghost_translation[a * ghosts_cw.size() + g] = in.shift[3 * ghosts_cw[g] + a];

  // Faces.
  struct FaceRec {
    i32 owner, neighbour, zone;
    i64 loop;  // cell face whose node loop (the owner's) the face takes
  };
  std::vector<FaceRec> interior, boundary;
  for (i64 f = 0; f < ncf; ++f) {
    const i32 c = face_cell[f];
    const i32 nc = new_index[c];
    if (nc < 0) continue;
    if (partner[f] >= 0) {
      const i64 p = partner[f];
      const i32 no = new_index[face_cell[p]];
      if (no < 0 || nc > no) continue;  // recorded once, from the lower cell
      if (std::min(layer[c], layer[face_cell[p]]) > 1) continue;
      interior.push_back({nc, no, -1, f});
    } else if (in.face_zone[f] >= 0 && layer[c] <= 1) {
      boundary.push_back({nc, -1, in.face_zone[f], f});
    }
  }
  std::sort(interior.begin(), interior.end(), [](const FaceRec& a, const FaceRec& b) {
    return a.owner != b.owner ? a.owner < b.owner
                              : (a.neighbour != b.neighbour ? a.neighbour < b.neighbour
                                                            : a.loop < b.loop);
  });
  std::sort(boundary.begin(), boundary.end(), [&](const FaceRec& a, const FaceRec& b) {
    const bool ga = a.owner >= n_owned, gb = b.owner >= n_owned;
    if (ga != gb) return gb;
    if (a.zone != b.zone) return a.zone < b.zone;
    if (a.owner != b.owner) return a.owner < b.owner;
    return a.loop < b.loop;
  });
  m.n_interior = static_cast<i32>(interior.size());
  m.n_faces = m.n_interior + static_cast<i32>(boundary.size());
  m.n_owned_interior = 0;
  for (const auto& r : interior)
    if (r.owner < n_owned) ++m.n_owned_interior;
  m.n_owned_faces = m.n_interior;
  for (const auto& r : boundary)
    if (r.owner < n_owned) ++m.n_owned_faces;
  for (const auto& r : boundary) m.n_zones = std::max(m.n_zones, r.zone + 1);

  // Points: only those some face uses, in first-use order.
  std::vector<i32> point_index(in.x.size(), -1);
  std::vector<i32> used;
  auto add_face = [&](const FaceRec& r) {
    m.owner.push_back(r.owner);
    if (r.neighbour >= 0) m.neighbour.push_back(r.neighbour);
    m.face_zone.push_back(r.zone);
    for (i64 k = in.face_node_offsets[r.loop]; k < in.face_node_offsets[r.loop + 1]; ++k) {
      const i32 p = in.face_nodes[k];
      if (point_index[p] < 0) {
        point_index[p] = static_cast<i32>(used.size());
        used.push_back(p);
      }
      m.face_nodes.push_back(point_index[p]);
    }
    m.face_node_offsets.push_back(static_cast<i64>(m.face_nodes.size()));
  };
  for (const auto& r : interior) add_face(r);
  for (const auto& r : boundary) add_face(r);
  m.points.resize(3 * used.size());
  for (std::size_t i = 0; i < used.size(); ++i) {
    m.points[i] = in.x[used[i]];
    m.points[used.size() + i] = in.y[used[i]];
    m.points[2 * used.size() + i] = in.z[used[i]];
  }

  // Cell -> face CSR, faces of each cell in increasing index (faces are visited in order).
  m.cell_face_offsets.assign(static_cast<std::size_t>(m.n_cells) + 1, 0);
  for (i32 f = 0; f < m.n_faces; ++f) {
    ++m.cell_face_offsets[m.owner[f] + 1];
    if (f < m.n_interior) ++m.cell_face_offsets[m.neighbour[f] + 1];
  }
  for (i32 c = 0; c < m.n_cells; ++c) m.cell_face_offsets[c + 1] += m.cell_face_offsets[c];
  m.cell_faces.resize(static_cast<std::size_t>(m.cell_face_offsets[m.n_cells]));
  {
    std::vector<i64> next(m.cell_face_offsets.begin(), m.cell_face_offsets.end() - 1);
    for (i32 f = 0; f < m.n_faces; ++f) {
      m.cell_faces[next[m.owner[f]]++] = f;
      if (f < m.n_interior) m.cell_faces[next[m.neighbour[f]]++] = f;
    }
  }
  for (i32 c = 0; c < n_owned; ++c)
    if (m.cell_face_offsets[c + 1] - m.cell_face_offsets[c] < 4)
      fail("E0116", "owned cell " + std::to_string(c) + " has fewer than 4 faces");
  return m;
}

// ------------------------------------------------------------------ geometry

Vec sub(const Vec& a, const Vec& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
Vec add(const Vec& a, const Vec& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
Vec scale(double s, const Vec& a) { return {s * a[0], s * a[1], s * a[2]}; }
double dot(const Vec& a, const Vec& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec cross(const Vec& a, const Vec& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

// compute_geometry (core/src/geometry.cpp:44-100,120-176): fan triangles about the node mean;
// face centroid weighted by projected fan areas; cell volume and centroid from tetrahedra
// (apex, m, p_i, p_i+1), apex the mean of the face centroids, in units of the cell size. Ghost
// cells take their image's volume and its centroid shifted by the translation
// (partition/src/self_exchange.cpp:32-49).
void compute_geometry(Mesh& m) {
  const auto nf = static_cast<std::size_t>(m.n_faces);
  const auto nc = static_cast<std::size_t>(m.n_cells);
  const auto np = static_cast<std::size_t>(m.n_points());
  auto point = [&](i32 p) { return Vec{m.points[p], m.points[np + p], m.points[2 * np + p]}; };
  m.face_area.assign(3 * nf, 0.0);
  m.face_area_magnitude.assign(nf, 0.0);
  m.face_normal.assign(3 * nf, 0.0);
  m.face_centroid.assign(3 * nf, 0.0);
  for (std::size_t f = 0; f < nf; ++f) {
    const i64 b = m.face_node_offsets[f];
    const i64 n = m.face_node_offsets[f + 1] - b;
    const Vec origin = point(m.face_nodes[b]);
    Vec sum{0.0, 0.0, 0.0};
    for (i64 i = 0; i < n; ++i) sum = add(sum, sub(point(m.face_nodes[b + i]), origin));
    const Vec mean = add(origin, scale(1.0 / static_cast<double>(n), sum));
    Vec area{0.0, 0.0, 0.0};
    for (i64 i = 0; i < n; ++i) {
      const Vec a = sub(point(m.face_nodes[b + i]), mean);
      const Vec c = sub(point(m.face_nodes[b + (i + 1) % n]), mean);
      area = add(area, scale(0.5, cross(a, c)));
    }
    const double mag = std::hypot(area[0], area[1], area[2]);
    if (!(mag > 0.0) || !std::isfinite(mag))
      fail("E0120", "face " + std::to_string(f) + " has zero or non-finite area");
    const Vec normal = scale(1.0 / mag, area);
    Vec moment{0.0, 0.0, 0.0};
    double weight = 0.0;
    for (i64 i = 0; i < n; ++i) {
      const Vec a = sub(point(m.face_nodes[b + i]), mean);
      const Vec c = sub(point(m.face_nodes[b + (i + 1) % n]), mean);
      const double w = dot(scale(0.5, cross(a, c)), normal);
      moment = add(moment, scale(w / 3.0, add(a, c)));
      weight += w;
    }
    const Vec centroid = add(mean, scale(1.0 / weight, moment));
    for (int a = 0; a < 3; ++a) {
      m.face_area[a * nf + f] = area[a];
      m.face_centroid[a * nf + f] = centroid[a];
      m.face_normal[a * nf + f] = area[a] / mag;  // pack_geometry: S / |S|
    }
    m.face_area_magnitude[f] = mag;
  }
  m.cell_volume.assign(nc, std::numeric_limits<double>::quiet_NaN());
  m.cell_centroid.assign(3 * nc, std::numeric_limits<double>::quiet_NaN());
  for (i32 c = 0; c < m.n_owned; ++c) {
    const i64 b = m.cell_face_offsets[c], e = m.cell_face_offsets[c + 1];
    Vec apex{0.0, 0.0, 0.0};
    double length = 0.0;
    for (i64 k = b; k < e; ++k) {
      const i32 f = m.cell_faces[k];
      apex = add(apex, Vec{m.face_centroid[f], m.face_centroid[nf + f], m.face_centroid[2 * nf + f]});
      length = std::max(length, std::sqrt(m.face_area_magnitude[f]));
    }
    apex = scale(1.0 / static_cast<double>(e - b), apex);
    const double inv = 1.0 / length;
    double volume = 0.0;
    Vec moment{0.0, 0.0, 0.0};
    for (i64 k = b; k < e; ++k) {
      const i32 f = m.cell_faces[k];
      const double sign = m.owner[f] == c ? 1.0 : -1.0;
      const i64 fb = m.face_node_offsets[f];
      const i64 n = m.face_node_offsets[f + 1] - fb;
      const Vec origin = point(m.face_nodes[fb]);
      Vec sum{0.0, 0.0, 0.0};
      for (i64 i = 0; i < n; ++i) sum = add(sum, sub(point(m.face_nodes[fb + i]), origin));
      const Vec mean = add(origin, scale(1.0 / static_cast<double>(n), sum));
      const Vec mm = scale(inv, sub(mean, apex));
      for (i64 i = 0; i < n; ++i) {
        const Vec a = scale(inv, sub(point(m.face_nodes[fb + i]), apex));
        const Vec d = scale(inv, sub(point(m.face_nodes[fb + (i + 1) % n]), apex));
        const double v = sign * dot(scale(0.5, cross(sub(a, mm), sub(d, mm))), mm) / 3.0;
        volume += v;
        moment = add(moment, scale(v / 4.0, add(add(mm, a), d)));
      }
    }
    const double vol = volume * length * length * length;
    if (!(volume > 0.0) || !std::isfinite(vol) || !(vol > 0.0))
      fail("E0121", "cell " + std::to_string(c) + " has non-positive or non-finite volume");
    m.cell_volume[c] = vol;
    const Vec centroid = add(apex, scale(length / volume, moment));
    for (int a = 0; a < 3; ++a) m.cell_centroid[a * nc + c] = centroid[a];
  }
  const std::size_t ng = m.ghost_owner.size();
  for (std::size_t g = 0; g < ng; ++g) {
    const auto c = static_cast<std::size_t>(m.n_owned) + g;
    const auto o = static_cast<std::size_t>(m.ghost_owner[g]);
    m.cell_volume[c] = m.cell_volume[o];
    for (int a = 0; a < 3; ++a)
      m.cell_centroid[a * nc + c] = m.cell_centroid[a * nc + o] + m.ghost_translation[a * ng + g];
  }

  // Face moments (codegen/cpp/geometry.cpp:208-272): an exact signed zero where the face is proven
  // planar (a triangle, nodes sharing one coordinate, or two parallel lines along an axis), else
  // the fan sum from the node of smallest (x, y, z).
  m.face_moment.assign(9 * nf, 0.0);
  m.all_planar = true;
  for (std::size_t f = 0; f < nf; ++f) {
    const i64 b = m.face_node_offsets[f];
    const std::size_t nn = static_cast<std::size_t>(m.face_node_offsets[f + 1] - b);
    auto pt = [&](std::size_t i) { return point(m.face_nodes[b + static_cast<i64>(i)]); };
    bool planar = nn == 3;
    const Vec p0 = pt(0);
    for (std::size_t a = 0; a < 3 && !planar; ++a) {
      const std::size_t bb = (a + 1) % 3, cc = (a + 2) % 3;
      bool shared = true, two_lines = true;
      std::size_t second = 0;
      for (std::size_t i = 1; i < nn && (shared || two_lines); ++i) {
        const Vec q = pt(i);
        shared = shared && q[a] == p0[a];
        if (q[bb] == p0[bb] && q[cc] == p0[cc]) continue;
        if (second == 0) {
          second = i;
        } else {
          const Vec s = pt(second);
          two_lines = two_lines && q[bb] == s[bb] && q[cc] == s[cc];
        }
      }
      planar = shared || two_lines;
    }
    if (planar) continue;
    m.all_planar = false;
    std::size_t start = 0;
    for (std::size_t i = 1; i < nn; ++i)
      if (pt(i) < pt(start)) start = i;
    auto at = [&](std::size_t i) { return pt((start + i) % nn); };
    Vec mean{0.0, 0.0, 0.0};
    for (std::size_t i = 0; i < nn; ++i) mean = add(mean, at(i));
    const double k = static_cast<double>(nn);
    mean = {mean[0] / k, mean[1] / k, mean[2] / k};
    const Vec xf{m.face_centroid[f], m.face_centroid[nf + f], m.face_centroid[2 * nf + f]};
    std::array<double, 9> mo{};
    for (std::size_t i = 0; i < nn; ++i) {
      const Vec a = at(i), c = at(i + 1);
      const Vec s = cross(sub(a, mean), sub(c, mean));
      const Vec tc{(mean[0] + a[0] + c[0]) / 3.0, (mean[1] + a[1] + c[1]) / 3.0,
                   (mean[2] + a[2] + c[2]) / 3.0};
      const Vec r = sub(tc, xf);
      for (int u = 0; u < 3; ++u)
        for (int v = 0; v < 3; ++v) mo[3 * u + v] += 0.5 * r[u] * s[v];
    }
    for (int j = 0; j < 9; ++j) m.face_moment[j * nf + f] = mo[j];
  }
}

// The face2 stencil of every cell (owned and ghost) with the shared rule of setup_rules.cuh
// (codegen/cpp/geometry.cpp:432, StencilKind::face2): one pass, each cell's entries appended.
setup::MeshView view_of(const Mesh& m) {
  return {m.n_cells, m.n_owned, m.n_faces, m.n_interior, m.cell_face_offsets.data(),
          m.cell_faces.data(), m.owner.data(), m.neighbour.data(), m.cell_centroid.data(),
          m.face_centroid.data()};
}

void face2_stencil(Mesh& m) {
  const setup::MeshView v = view_of(m);
  m.stencil_offsets.assign(static_cast<std::size_t>(m.n_cells) + 1, 0);
  m.stencil.clear();
  std::vector<i32> buf(setup::kMaxCandidates), row(setup::kMaxCandidates);
  for (i32 c = 0; c < m.n_cells; ++c) {
    const int len = setup::face2_entries(v, c, buf.data(), setup::kMaxCandidates, row.data());
    if (len < 0) fail("E1102", "a cell's face2 stencil has more than 512 candidates");
    m.stencil.insert(m.stencil.end(), row.begin(), row.begin() + len);
    m.stencil_offsets[static_cast<std::size_t>(c) + 1] = static_cast<i64>(m.stencil.size());
  }
}

void finish(Mesh& m) {
  compute_geometry(m);
  face2_stencil(m);
}

// ------------------------------------------------------------------ lattice generator

Mesh lattice(const autan_lattice& s) {
  const int n[3] = {s.nx, s.ny, s.nz};
  for (int a = 0; a < 3; ++a) {
    if (n[a] < 1) fail("E1101", "lattice sizes must be positive");
    if (!(s.extent[a] > 0.0)) fail("E1101", "lattice extents must be positive");
    if (s.periodic[a] && n[a] < 3) fail("E1101", "a periodic axis needs at least 3 boxes");
  }
  if (s.fill != AUTAN_FILL_HEXA && s.fill != AUTAN_FILL_TETRA) fail("E1101", "unknown fill");
  const int pad[3] = {s.periodic[0] ? 2 : 0, s.periodic[1] ? 2 : 0, s.periodic[2] ? 2 : 0};
  // Extended lattice: box index b in [-pad, n + pad), node index in [-pad, n + pad].
  const int ne[3] = {n[0] + 2 * pad[0] + 1, n[1] + 2 * pad[1] + 1, n[2] + 2 * pad[2] + 1};
  const double h[3] = {s.extent[0] / n[0], s.extent[1] / n[1], s.extent[2] / n[2]};
  Cellwise cw;
  const std::size_t nn = static_cast<std::size_t>(ne[0]) * ne[1] * ne[2];
  cw.x.resize(nn);
  cw.y.resize(nn);
  cw.z.resize(nn);
  auto node = [&](int i, int j, int k) {
    return static_cast<i32>((i + pad[0]) + ne[0] * ((j + pad[1]) + ne[1] * (k + pad[2])));
  };
  auto wrap = [&](int a, int i, int& q) {
    // Base index along axis a and how many periods away the node lies.
    q = 0;
    if (!s.periodic[a]) return i;
    while (i < 0) {
      i += n[a];
      --q;
    }
    while (i >= n[a]) {
      i -= n[a];
      ++q;
    }
    return i;
  };
  for (int k = -pad[2]; k <= n[2] + pad[2]; ++k)
    for (int j = -pad[1]; j <= n[1] + pad[1]; ++j)
      for (int i = -pad[0]; i <= n[0] + pad[0]; ++i) {
        int q[3];
        const int b[3] = {wrap(0, i, q[0]), wrap(1, j, q[1]), wrap(2, k, q[2])};
        double p[3];
        for (int a = 0; a < 3; ++a) {
          p[a] = s.origin[a] + b[a] * h[a];
          if (s.displacement != nullptr) {
            const std::size_t di = static_cast<std::size_t>(b[0]) +
                                   static_cast<std::size_t>(n[0] + 1) *
                                       (static_cast<std::size_t>(b[1]) +
                                        static_cast<std::size_t>(n[1] + 1) * b[2]);
            p[a] += s.displacement[a * static_cast<std::size_t>(n[0] + 1) * (n[1] + 1) * (n[2] + 1) + di];
          }
        }
        // Images: one addition of the translation per period, so that x_b = x_a + T.
        for (int a = 0; a < 3; ++a)
          for (int r = 0; r < std::abs(q[a]); ++r) p[a] += q[a] > 0 ? s.extent[a] : -s.extent[a];
        const i32 id = node(i, j, k);
        cw.x[id] = p[0];
        cw.y[id] = p[1];
        cw.z[id] = p[2];
      }
  // Boundary zone of a face whose nodes all lie on one lattice plane of a non-periodic side.
  auto face_zone = [&](const int (*idx)[3], int count) {
    for (int a = 0; a < 3; ++a) {
      if (s.periodic[a]) continue;
      for (int side = 0; side < 2; ++side) {
        const int plane = side == 0 ? 0 : n[a];
        bool all = true;
        for (int v = 0; v < count && all; ++v) all = idx[v][a] == plane;
        if (all) return s.zone[2 * a + side];
      }
    }
    return -1;
  };
  auto add_face = [&](std::initializer_list<std::array<int, 3>> loop) {
    int idx[16][3];
    int cnt = 0;
    for (const auto& v : loop) {
      idx[cnt][0] = v[0];
      idx[cnt][1] = v[1];
      idx[cnt][2] = v[2];
      cw.face_nodes.push_back(node(v[0], v[1], v[2]));
      ++cnt;
    }
    cw.face_node_offsets.push_back(static_cast<i64>(cw.face_nodes.size()));
    cw.face_zone.push_back(face_zone(idx, cnt));
  };
  // Owned boxes first in lattice order, so that images index them directly.
  auto box_id = [&](int i, int j, int k) {
    return static_cast<i64>(i) + static_cast<i64>(n[0]) * (j + static_cast<i64>(n[1]) * k);
  };
  const int per_box = s.fill == AUTAN_FILL_HEXA ? 1 : 6;
  std::vector<std::array<int, 3>> boxes;
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) boxes.push_back({i, j, k});
  for (int k = -pad[2]; k < n[2] + pad[2]; ++k)
    for (int j = -pad[1]; j < n[1] + pad[1]; ++j)
      for (int i = -pad[0]; i < n[0] + pad[0]; ++i)
        if (i < 0 || i >= n[0] || j < 0 || j >= n[1] || k < 0 || k >= n[2]) boxes.push_back({i, j, k});
  static constexpr int orders[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  for (const auto& bx : boxes) {
    const int i = bx[0], j = bx[1], k = bx[2];
    int q[3];
    const int bi = wrap(0, i, q[0]), bj = wrap(1, j, q[1]), bk = wrap(2, k, q[2]);
    const bool owned = q[0] == 0 && q[1] == 0 && q[2] == 0;
    const i64 base = box_id(bi, bj, bk) * per_box;
    auto v = [&](int di, int dj, int dk) { return std::array<int, 3>{i + di, j + dj, k + dk}; };
    for (int t = 0; t < per_box; ++t) {
      cw.image.push_back(owned ? -1 : static_cast<i32>(base + t));
      for (int a = 0; a < 3; ++a) cw.shift.push_back(q[a] * s.extent[a]);
      if (s.fill == AUTAN_FILL_HEXA) {
        add_face({v(0, 0, 0), v(0, 0, 1), v(0, 1, 1), v(0, 1, 0)});
        add_face({v(1, 0, 0), v(1, 1, 0), v(1, 1, 1), v(1, 0, 1)});
        add_face({v(0, 0, 0), v(1, 0, 0), v(1, 0, 1), v(0, 0, 1)});
        add_face({v(0, 1, 0), v(0, 1, 1), v(1, 1, 1), v(1, 1, 0)});
        add_face({v(0, 0, 0), v(0, 1, 0), v(1, 1, 0), v(1, 0, 0)});
        add_face({v(0, 0, 1), v(1, 0, 1), v(1, 1, 1), v(0, 1, 1)});
      } else {
        // Kuhn subdivision: the tetrahedron of axis-step order `orders[t]` from v000 to v111,
        // odd orders mirrored (tests/core/fixtures.cpp BoxFill::tetra).
        std::array<std::array<int, 3>, 4> tet{};
        int st[3] = {0, 0, 0};
        tet[0] = v(0, 0, 0);
        for (int sidx = 0; sidx < 3; ++sidx) {
          st[orders[t][sidx]] = 1;
          tet[sidx + 1] = v(st[0], st[1], st[2]);
        }
        if (t >= 3) std::swap(tet[1], tet[2]);
        const auto &a = tet[0], &b = tet[1], &c = tet[2], &d = tet[3];
        add_face({a, c, b});
        add_face({a, b, d});
        add_face({a, d, c});
        add_face({b, c, d});
      }
      cw.cell_face_offsets.push_back(static_cast<i64>(cw.face_node_offsets.size()) - 1);
    }
  }
  Mesh m = assemble(cw, s.rcm);
  finish(m);
  return m;
}

// ------------------------------------------------------------------ bump channel generator

// The hybrid channel over a Gaussian bump (a steady subsonic test case of the path): nodes on
// x_i = L_x i / nx, z_k = L_z k / nz and, in each column, y from the wall
// y_w(x) = h exp(-25 (x - 1.5)^2) to L_y with wall-normal spacings growing by `ratio` per layer up
// to layer `stretched`, constant above. Rows of hexahedra, a band of triangular prisms (each hex
// split along its x-y diagonal), and a block of polyhedra: 2 x 1 "bricks" staggered from row to
// row, so that each brick meets two half-faces above and below and has hexagonal z faces. Every
// face is an extrusion along z, hence planar. Zones: 0 inlet (x = 0), 1 outlet (x = L_x), 2 the
// bump wall, 3 the top, 4 z = 0, 5 z = L_z.
Mesh bump_channel(const autan_bump_channel& s) {
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  if (nx < 2 || ny < 2 || nz < 1) fail("E1101", "channel sizes too small");
  if (!(s.extent[0] > 0.0 && s.extent[1] > 0.0 && s.extent[2] > 0.0))
    fail("E1101", "channel extents must be positive");
  if (!(s.ratio >= 1.0)) fail("E1101", "the stretching ratio must be at least 1");
  if (s.prism_rows[0] < 0 || s.prism_rows[1] < s.prism_rows[0] || s.prism_rows[1] > ny)
    fail("E1101", "prism rows out of range");
  const int bi0 = s.brick_cols[0], bi1 = s.brick_cols[1], bj0 = s.brick_rows[0], bj1 = s.brick_rows[1];
  if (bi0 < 0 || bi1 < bi0 || bi1 > nx || bj0 < 0 || bj1 < bj0 || bj1 > ny)
    fail("E1101", "brick block out of range");
  if (bj1 > bj0 && !(bj0 >= s.prism_rows[1] || bj1 <= s.prism_rows[0]))
    fail("E1101", "the brick block overlaps the prism band");
  // Wall-normal distribution on [0, 1].
  std::vector<double> sy(static_cast<std::size_t>(ny) + 1, 0.0);
  {
    std::vector<double> d(static_cast<std::size_t>(ny));
    double step = 1.0;
    for (int j = 0; j < ny; ++j) {
      d[j] = step;
      if (j + 1 < s.stretched) step *= s.ratio;
    }
    double total = 0.0;
    for (int j = 0; j < ny; ++j) total += d[j];
    for (int j = 0; j < ny; ++j) sy[j + 1] = sy[j] + d[j] / total;
    sy[ny] = 1.0;
  }
  Cellwise cw;
  const std::size_t nn = static_cast<std::size_t>(nx + 1) * (ny + 1) * (nz + 1);
  cw.x.resize(nn);
  cw.y.resize(nn);
  cw.z.resize(nn);
  auto node = [&](int i, int j, int k) {
    return static_cast<i32>(i + (nx + 1) * (j + (ny + 1) * static_cast<i64>(k)));
  };
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const double x = s.extent[0] * i / nx;
        const double xc = x - 1.5;
        const double yw = s.bump * std::exp(-25.0 * xc * xc);
        const i32 id = node(i, j, k);
        cw.x[id] = x;
        cw.y[id] = yw + (s.extent[1] - yw) * sy[j];
        cw.z[id] = s.extent[2] * k / nz;
      }
  using Ijk = std::array<int, 3>;
  auto zone_of = [&](const std::vector<Ijk>& loop) {
    auto all = [&](int a, int v) {
      for (const auto& p : loop)
        if (p[a] != v) return false;
      return true;
    };
    if (all(0, 0)) return 0;
    if (all(0, nx)) return 1;
    if (all(1, 0)) return 2;
    if (all(1, ny)) return 3;
    if (all(2, 0)) return 4;
    if (all(2, nz)) return 5;
    return -1;
  };
  auto pos = [&](const Ijk& p) {
    const i32 id = node(p[0], p[1], p[2]);
    return Vec{cw.x[id], cw.y[id], cw.z[id]};
  };
  // A cell from its face loops, each turned outward: its area vector (Newell's sum) points away
  // from the cell's node mean.
  auto add_cell = [&](std::vector<std::vector<Ijk>> faces) {
    Vec mid{0.0, 0.0, 0.0};
    int cnt = 0;
    for (const auto& f : faces)
      for (const auto& p : f) {
        mid = add(mid, pos(p));
        ++cnt;
      }
    mid = scale(1.0 / cnt, mid);
    for (auto& f : faces) {
      Vec area{0.0, 0.0, 0.0}, fc{0.0, 0.0, 0.0};
      for (std::size_t a = 0; a < f.size(); ++a) {
        const Vec p = pos(f[a]), q = pos(f[(a + 1) % f.size()]);
        area = add(area, cross(p, q));
        fc = add(fc, p);
      }
      fc = scale(1.0 / static_cast<double>(f.size()), fc);
      if (dot(area, sub(fc, mid)) < 0.0) std::reverse(f.begin(), f.end());
      for (const auto& p : f) cw.face_nodes.push_back(node(p[0], p[1], p[2]));
      cw.face_node_offsets.push_back(static_cast<i64>(cw.face_nodes.size()));
      cw.face_zone.push_back(zone_of(f));
    }
    cw.cell_face_offsets.push_back(static_cast<i64>(cw.face_node_offsets.size()) - 1);
    cw.image.push_back(-1);
    for (int a = 0; a < 3; ++a) cw.shift.push_back(0.0);
  };
  auto quad = [](Ijk a, Ijk b, Ijk c, Ijk d) { return std::vector<Ijk>{a, b, c, d}; };
  auto hex = [&](int i, int j, int k) {
    auto v = [&](int di, int dj, int dk) { return Ijk{i + di, j + dj, k + dk}; };
    add_cell({quad(v(0, 0, 0), v(0, 1, 0), v(0, 1, 1), v(0, 0, 1)),
              quad(v(1, 0, 0), v(1, 1, 0), v(1, 1, 1), v(1, 0, 1)),
              quad(v(0, 0, 0), v(1, 0, 0), v(1, 0, 1), v(0, 0, 1)),
              quad(v(0, 1, 0), v(1, 1, 0), v(1, 1, 1), v(0, 1, 1)),
              quad(v(0, 0, 0), v(1, 0, 0), v(1, 1, 0), v(0, 1, 0)),
              quad(v(0, 0, 1), v(1, 0, 1), v(1, 1, 1), v(0, 1, 1))});
  };
  // The two prisms of box (i, j, k) split along the diagonal (i, j) - (i + 1, j + 1).
  auto prisms = [&](int i, int j, int k) {
    auto v = [&](int di, int dj, int dk) { return Ijk{i + di, j + dj, k + dk}; };
    add_cell({{v(0, 0, 0), v(1, 0, 0), v(1, 1, 0)}, {v(0, 0, 1), v(1, 0, 1), v(1, 1, 1)},
              quad(v(0, 0, 0), v(1, 0, 0), v(1, 0, 1), v(0, 0, 1)),
              quad(v(1, 0, 0), v(1, 1, 0), v(1, 1, 1), v(1, 0, 1)),
              quad(v(0, 0, 0), v(1, 1, 0), v(1, 1, 1), v(0, 0, 1))});
    add_cell({{v(0, 0, 0), v(1, 1, 0), v(0, 1, 0)}, {v(0, 0, 1), v(1, 1, 1), v(0, 1, 1)},
              quad(v(0, 0, 0), v(1, 1, 0), v(1, 1, 1), v(0, 0, 1)),
              quad(v(0, 1, 0), v(1, 1, 0), v(1, 1, 1), v(0, 1, 1)),
              quad(v(0, 0, 0), v(0, 1, 0), v(0, 1, 1), v(0, 0, 1))});
  };
  // A brick over columns i and i + 1 of row j.
  auto brick = [&](int i, int j, int k) {
    auto v = [&](int di, int dj, int dk) { return Ijk{i + di, j + dj, k + dk}; };
    add_cell({quad(v(0, 0, 0), v(0, 1, 0), v(0, 1, 1), v(0, 0, 1)),
              quad(v(2, 0, 0), v(2, 1, 0), v(2, 1, 1), v(2, 0, 1)),
              quad(v(0, 0, 0), v(1, 0, 0), v(1, 0, 1), v(0, 0, 1)),
              quad(v(1, 0, 0), v(2, 0, 0), v(2, 0, 1), v(1, 0, 1)),
              quad(v(0, 1, 0), v(1, 1, 0), v(1, 1, 1), v(0, 1, 1)),
              quad(v(1, 1, 0), v(2, 1, 0), v(2, 1, 1), v(1, 1, 1)),
              {v(0, 0, 0), v(1, 0, 0), v(2, 0, 0), v(2, 1, 0), v(1, 1, 0), v(0, 1, 0)},
              {v(0, 0, 1), v(1, 0, 1), v(2, 0, 1), v(2, 1, 1), v(1, 1, 1), v(0, 1, 1)}});
  };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      const bool prism_row = j >= s.prism_rows[0] && j < s.prism_rows[1];
      const bool brick_row = j >= bj0 && j < bj1;
      for (int i = 0; i < nx;) {
        if (prism_row) {
          prisms(i, j, k);
          ++i;
        } else if (brick_row && i >= bi0 && i < bi1) {
          // bricks start at bi0 on even rows of the block, at bi0 + 1 on odd ones
          const int off = (i - bi0 - ((j - bj0) & 1)) & 1;
          if (off == 0 && i + 1 < bi1 && !((j - bj0) & 1 && i == bi0)) {
            brick(i, j, k);
            i += 2;
          } else {
            hex(i, j, k);
            ++i;
          }
        } else {
          hex(i, j, k);
          ++i;
        }
      }
    }
  Mesh m = assemble(cw, s.order);
  finish(m);
  return m;
}

// ------------------------------------------------------------------ gradient weights

// The least-squares weights of the owned cells (physics/src/euler.cpp:340-416), one cell at a
// time with the shared rule of setup_rules.cuh; ghost cells' weights stay 0.
void gradient_weights(const Mesh& m, const std::uint8_t* kind, double* w) {
  const setup::MeshView v = view_of(m);
  const auto nst = static_cast<i64>(m.stencil.size());
  std::fill(w, w + 3 * nst, 0.0);
  for (i32 c = 0; c < m.n_owned; ++c)
    setup::lsq_cell_weights(v, c, m.stencil_offsets.data(), m.stencil.data(), kind, w, nst);
}

int fail_to(char* err, std::size_t len, const std::string& what) {
  if (err != nullptr && len > 0) {
    std::strncpy(err, what.c_str(), len - 1);
    err[len - 1] = '\0';
  }
  return 1;
}

template <class F>
int guarded(char* err, std::size_t len, F&& body) {
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

}  // namespace

extern "C" {

int autan_mesh_build_lattice(const autan_lattice* spec, void** mesh, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (spec == nullptr || mesh == nullptr) fail("E1101", "null argument");
    *mesh = new Mesh(lattice(*spec));
  });
}

int autan_mesh_build_cells(int64_t n_points, const double* points, int64_t n_cells,
                           const int64_t* cell_face_offsets, const int64_t* face_node_offsets,
                           const int32_t* face_nodes, const int32_t* face_zone, int32_t rcm_flag,
                           void** mesh, char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if (n_points < 4 || n_cells < 1 || points == nullptr || mesh == nullptr)
      fail("E1101", "empty or null mesh arrays");
    Cellwise cw;
    const auto np = static_cast<std::size_t>(n_points);
    cw.x.assign(points, points + np);
    cw.y.assign(points + np, points + 2 * np);
    cw.z.assign(points + 2 * np, points + 3 * np);
    cw.cell_face_offsets.assign(cell_face_offsets, cell_face_offsets + n_cells + 1);
    const i64 nfaces = cw.cell_face_offsets.back();
    cw.face_node_offsets.assign(face_node_offsets, face_node_offsets + nfaces + 1);
    cw.face_nodes.assign(face_nodes, face_nodes + cw.face_node_offsets.back());
    cw.face_zone.assign(face_zone, face_zone + nfaces);
    for (const i32 p : cw.face_nodes)
      if (p < 0 || p >= n_points) fail("E1101", "a face node is out of range");
    cw.image.assign(static_cast<std::size_t>(n_cells), -1);
    cw.shift.assign(3 * static_cast<std::size_t>(n_cells), 0.0);
    Mesh m = assemble(cw, rcm_flag);
    finish(m);
    *mesh = new Mesh(std::move(m));
  });
}

int autan_mesh_build_bump_channel(const autan_bump_channel* spec, void** mesh, char* err,
                                  size_t err_len) {
  return guarded(err, err_len, [&] {
    if (spec == nullptr || mesh == nullptr) fail("E1101", "null argument");
    *mesh = new Mesh(bump_channel(*spec));
  });
}

void autan_mesh_free(void* mesh) { delete static_cast<Mesh*>(mesh); }

int autan_convergence_iteration(const double* residuals, int64_t n, double orders,
                                const double* floors, int64_t* iteration, int32_t* plateau_mask,
                                char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    if ((residuals == nullptr && n > 0) || iteration == nullptr) fail("E1101", "null argument");
    autan_b200::Convergence conv(orders, floors);
    *iteration = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (conv.add(residuals + 5 * i)) {
        *iteration = i + 1;
        if (plateau_mask != nullptr) *plateau_mask = conv.plateau_mask();
        return;
      }
    }
    if (plateau_mask != nullptr) *plateau_mask = 0;
  });
}

void autan_mesh_counts(const void* mesh, int64_t* counts) {
  const auto& m = *static_cast<const Mesh*>(mesh);
  counts[0] = m.n_points();
  counts[1] = m.n_cells;
  counts[2] = m.n_owned;
  counts[3] = m.n_faces;
  counts[4] = m.n_interior;
  counts[5] = m.n_owned_interior;
  counts[6] = m.n_owned_faces;
  counts[7] = static_cast<int64_t>(m.cell_faces.size());
  counts[8] = static_cast<int64_t>(m.stencil.size());
  counts[9] = m.all_planar ? 1 : 0;
  counts[10] = static_cast<int64_t>(m.ghost_owner.size());
  counts[11] = m.n_zones;
}

int autan_mesh_array(const void* mesh, const char* name, const void** ptr, int64_t* count,
                     int32_t* elem_size) {
  const auto& m = *static_cast<const Mesh*>(mesh);
  const std::string n(name);
  auto give = [&](const auto& v) {
    *ptr = v.data();
    *count = static_cast<int64_t>(v.size());
    *elem_size = static_cast<int32_t>(sizeof(v[0]));
    return 0;
  };
  if (n == "owner") return give(m.owner);
  if (n == "neighbour") return give(m.neighbour);
  if (n == "cell_faces") return give(m.cell_faces);
  if (n == "face_zone") return give(m.face_zone);
  if (n == "stencil") return give(m.stencil);
  if (n == "ghost_owner") return give(m.ghost_owner);
  if (n == "face_nodes") return give(m.face_nodes);
  if (n == "owned_order") return give(m.owned_order);
  if (n == "cell_face_offsets") return give(m.cell_face_offsets);
  if (n == "stencil_offsets") return give(m.stencil_offsets);
  if (n == "face_node_offsets") return give(m.face_node_offsets);
  if (n == "points") return give(m.points);
  if (n == "face_area") return give(m.face_area);
  if (n == "face_area_magnitude") return give(m.face_area_magnitude);
  if (n == "face_normal") return give(m.face_normal);
  if (n == "face_centroid") return give(m.face_centroid);
  if (n == "face_moment") return give(m.face_moment);
  if (n == "cell_centroid") return give(m.cell_centroid);
  if (n == "cell_volume") return give(m.cell_volume);
  if (n == "ghost_translation") return give(m.ghost_translation);
  return 1;
}

int autan_mesh_gradient_weights(const void* mesh, const uint8_t* bc_kind, double* weights,
                                char* err, size_t err_len) {
  return guarded(err, err_len, [&] {
    const auto& m = *static_cast<const Mesh*>(mesh);
    const i32 nb = m.n_faces - m.n_interior;
    for (i32 b = 0; b < nb; ++b)
      if (bc_kind[b] > 5) fail("E1101", "boundary code out of range");
    gradient_weights(m, bc_kind, weights);
  });
}

}  // extern "C"
