// Test infrastructure, not product code: a C entry point over the reference's own set-up chain,
// compiled from the reference's sources (oracle/Makefile, target ref) into oracle/_ref/. It lets
// the tests check the product's mesh assembly, FP64 geometry and face2 stencil against the
// reference's code run on the same mesh:
//   core/src/mesh.cpp:273 assemble            face order and orientation, cell faces
//   core/src/geometry.cpp:120 compute_geometry face areas and centroids, cell volumes and centroids
//   codegen/cpp/geometry.cpp:166 pack_geometry unit normals, area magnitudes, face moments
//   codegen/cpp/geometry.cpp:432 cell_stencil  the face2 stencil and its least-squares weights
//                                              (every boundary face in the fit)
// Only tests/ load the library; it is never part of the product path.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <string>
#include <vector>

#include "autan/core/geometry.hpp"
#include "autan/core/mesh.hpp"
#include "autan/kernels/geometry.hpp"

namespace {

struct Result {
  autan::AssemblyMap map;
  autan::Mesh mesh;
  std::map<std::string, std::vector<double>> f64;
  std::map<std::string, std::vector<std::int64_t>> i64;
};

void put(Result& r, const char* name, const std::vector<double>& v) { r.f64[name] = v; }

template <class T>
void put_int(Result& r, const char* name, const T& v) {
  r.i64[name] = std::vector<std::int64_t>(v.begin(), v.end());
}

}  // namespace

extern "C" {

// A mesh given face by face: points (3 x n_points, component-major), each face's node loop,
// cell0 / cell1 the cells on either side (cell1 -1 on a boundary face, the loop outward from
// cell0), face_zone the boundary zone of each boundary face (interior faces: ignored), the last
// n_ghost cells periodic images. ghost_centroid (3 x n_ghost, or NULL): the images' centroids,
// which the reference's partitioner supplies (its compute_geometry leaves ghosts at NaN), used by
// cell_stencil's weights of owned cells next to them.
int ref_setup(int64_t n_points, const double* points, int64_t n_faces,
              const int64_t* face_node_offsets, const int32_t* face_nodes, const int32_t* cell0,
              const int32_t* cell1, const int32_t* face_zone, int32_t n_zones, int32_t n_cells,
              int32_t n_ghost, const double* ghost_centroid, void** out, char* err,
              size_t err_len) {
  try {
    autan::MeshInput in;
    in.x.assign(points, points + n_points);
    in.y.assign(points + n_points, points + 2 * n_points);
    in.z.assign(points + 2 * n_points, points + 3 * n_points);
    in.face_node_offsets.assign(face_node_offsets, face_node_offsets + n_faces + 1);
    in.face_nodes.assign(face_nodes, face_nodes + face_node_offsets[n_faces]);
    in.face_cell0.assign(cell0, cell0 + n_faces);
    in.face_cell1.assign(cell1, cell1 + n_faces);
    in.face_zone.resize(static_cast<std::size_t>(n_faces));
    // zones 0 .. n_zones-1 hold boundary faces, zone n_zones the interior faces
    for (int64_t f = 0; f < n_faces; ++f) in.face_zone[f] = cell1[f] < 0 ? face_zone[f] : n_zones;
    for (int32_t z = 0; z <= n_zones; ++z) {
      autan::FaceZone fz;
      fz.name = "zone" + std::to_string(z);
      fz.boundary = z < n_zones;
      in.face_zones.push_back(fz);
    }
    in.cell_zones.push_back(autan::CellZone{"fluid", "", autan::CellKind::fluid, {}});
    in.cell_zone.assign(static_cast<std::size_t>(n_cells), 0);
    in.n_ghost_cells = n_ghost;
    auto* r = new Result();
    r->mesh = autan::assemble(std::move(in), &r->map);
    const autan::Mesh& m = r->mesh;
    put_int(*r, "face_source", r->map.face_source);
    put_int(*r, "face_reversed", r->map.face_reversed);
    put_int(*r, "owner", m.owner());
    put_int(*r, "neighbour", m.neighbour());
    put_int(*r, "cell_face_offsets", m.cell_face_offsets());
    put_int(*r, "cell_faces", m.cell_faces());
    put_int(*r, "counts", std::vector<std::int64_t>{m.n_cells(), m.n_owned_cells(), m.n_faces(),
                                                   m.n_interior_faces(),
                                                   m.n_owned_interior_faces(), m.n_owned_faces()});
    const autan::Geometry g = autan::compute_geometry(m);
    auto soa = [](const std::vector<double>& a, const std::vector<double>& b,
                  const std::vector<double>& c) {
      std::vector<double> v(a);
      v.insert(v.end(), b.begin(), b.end());
      v.insert(v.end(), c.begin(), c.end());
      return v;
    };
    put(*r, "face_area", soa(g.face_area_x, g.face_area_y, g.face_area_z));
    put(*r, "face_area_magnitude", g.face_area);
    put(*r, "face_centroid", soa(g.face_centroid_x, g.face_centroid_y, g.face_centroid_z));
    put(*r, "cell_volume", g.cell_volume);
    put(*r, "cell_centroid", soa(g.cell_centroid_x, g.cell_centroid_y, g.cell_centroid_z));
    autan::kernels::PackedGeometry pg = autan::kernels::pack_geometry(m, g, nullptr);
    put(*r, "face_normal", pg.face_normal);
    put(*r, "face_moment", pg.face_moment);
    const std::size_t nc = static_cast<std::size_t>(m.n_cells());
    const std::size_t owned = static_cast<std::size_t>(m.n_owned_cells());
    if (ghost_centroid != nullptr)
      for (std::size_t gi = 0; gi < nc - owned; ++gi)
        for (std::size_t a = 0; a < 3; ++a)
          pg.cell_centroid[a * nc + owned + gi] = ghost_centroid[a * (nc - owned) + gi];
    const autan::kernels::CellStencil st =
        autan::kernels::cell_stencil(m, pg, autan::kernels::StencilKind::face2, nullptr);
    put_int(*r, "stencil_offsets", st.offsets);
    put_int(*r, "stencil", st.entries);
    put(*r, "stencil_lsq_weight", st.lsq_weight);
    *out = r;
    return 0;
  } catch (const std::exception& e) {
    if (err != nullptr && err_len > 0) std::snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// Element count of array `name` (-1: unknown); is_int receives 1 for an int64 array.
int64_t ref_count(void* h, const char* name, int32_t* is_int) {
  auto* r = static_cast<Result*>(h);
  if (auto it = r->f64.find(name); it != r->f64.end()) {
    *is_int = 0;
    return static_cast<int64_t>(it->second.size());
  }
  if (auto it = r->i64.find(name); it != r->i64.end()) {
    *is_int = 1;
    return static_cast<int64_t>(it->second.size());
  }
  return -1;
}

// Copies array `name` (doubles or int64) into dst.
int ref_copy(void* h, const char* name, void* dst) {
  auto* r = static_cast<Result*>(h);
  if (auto it = r->f64.find(name); it != r->f64.end()) {
    std::memcpy(dst, it->second.data(), it->second.size() * sizeof(double));
    return 0;
  }
  if (auto it = r->i64.find(name); it != r->i64.end()) {
    std::memcpy(dst, it->second.data(), it->second.size() * sizeof(std::int64_t));
    return 0;
  }
  return 1;
}

void ref_free(void* h) { delete static_cast<Result*>(h); }

}  // extern "C"
