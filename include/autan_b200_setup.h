/* Host-side mesh set-up for the explicit Euler path: the inputs the residual reads, built in the
 * layouts of Autan's face-based mesh contract (docs/contracts/mesh.md).
 *
 * These entry points replace, for callers that have no Autan mesh of their own (tests, the
 * benchmark), the reference's set-up chain:
 *   core/src/cellwise.cpp  to_face_based + core/src/mesh.cpp assemble  -> autan_mesh_build_*
 *   core/src/renumber.cpp:109 rcm_order                                  -> spec.rcm = 1
 *   (a Morton order of the cell centres, spec.rcm = 2, has no counterpart in the reference)
 *   core/src/geometry.cpp:120 compute_geometry                           -> built with the mesh
 *   codegen/cpp/geometry.cpp:166 pack_geometry (normals, moments)        -> built with the mesh
 *   codegen/cpp/geometry.cpp:432 cell_stencil (face2)                    -> built with the mesh
 *   physics/src/euler.cpp:340 Euler::Impl::compute_gradient_weights      -> autan_mesh_gradient_weights
 * A caller that holds an assembled Autan mesh passes its own arrays to autan_euler_device_create
 * (autan_euler_device.h) instead.
 *
 * Conventions of the reference's C ABI (physics/mms/capi.cpp:42-60): int return, 0 on success,
 * 1 on failure with "Exxxx: message" written into err (err_len bytes, NUL-terminated); no C++
 * exception crosses the boundary. Arrays are structure of arrays: component c of entity i at
 * c * n + i. */
#ifndef AUTAN_B200_SETUP_H
#define AUTAN_B200_SETUP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cell shapes of a lattice mesh. */
enum autan_lattice_fill { AUTAN_FILL_HEXA = 0, AUTAN_FILL_TETRA = 1 };

/* A structured lattice of nx x ny x nz boxes on [origin, origin + extent], each box one hexahedron
 * or six Kuhn tetrahedra (tests/core/fixtures.cpp BoxFill::tetra). An axis with periodic[a] != 0
 * is periodic with translation extent[a]: the cells across it are periodic images (ghost cells,
 * two face layers deep, as a one-rank partition with self-exchange holds them), each the copy of
 * an owned cell shifted by the translation. The two sides of a non-periodic axis are boundary
 * zones zone[2a] (low) and zone[2a + 1] (high); the zone index is the value the caller maps to a
 * boundary condition. `displacement`, when not NULL, moves the lattice nodes: 3 x (nx+1)(ny+1)(nz+1)
 * values, node (i, j, k) at i + (nx+1) (j + (ny+1) k); along a periodic axis the node at index n
 * takes the displacement of index 0 so that the images match (the caller keeps it periodic). */
struct autan_lattice {
  int32_t fill;
  int32_t nx, ny, nz;
  double origin[3];
  double extent[3];
  int32_t periodic[3];
  int32_t zone[6];
  const double* displacement;
  int32_t rcm; /* owned cell order: 0 generator's, 1 reverse Cuthill-McKee, 2 Morton (Z-order) */
};

/* Builds an assembled mesh with its geometry and face2 stencil. */
int autan_mesh_build_lattice(const struct autan_lattice* spec, void** mesh, char* err,
                             size_t err_len);

/* A general mesh from cells given by their faces (outward node loops), for meshes a lattice does
 * not describe (hybrid hex/prism/polyhedral channels):
 *   points: 3 x n_points; cell_face_offsets: n_cells + 1; face_node_offsets: one more than the
 *   total number of cell faces; face_nodes: the node loops; face_zone: per cell face, the boundary
 *   zone it lies on when no other cell shares it (-1: it must be shared).
 * No ghost cells (no periodic axis). */
int autan_mesh_build_cells(int64_t n_points, const double* points, int64_t n_cells,
                           const int64_t* cell_face_offsets, const int64_t* face_node_offsets,
                           const int32_t* face_nodes, const int32_t* face_zone, int32_t order,
                           void** mesh, char* err, size_t err_len);

/* The hybrid channel over a Gaussian bump, y_w(x) = bump exp(-25 (x - 1.5)^2), on
 * [0, extent[0]] x [y_w, extent[1]] x [0, extent[2]] (no counterpart in the reference, whose
 * meshes come from files; its V&V bump meshes come from gmsh): nx x ny x nz boxes with wall-normal
 * spacings growing by `ratio` per layer up to layer `stretched`, constant above; rows
 * [prism_rows[0], prism_rows[1]) split into two triangular prisms per box; in rows
 * [brick_rows[0], brick_rows[1]) and columns [brick_cols[0], brick_cols[1]), polyhedral 2 x 1
 * bricks staggered row to row (two half-faces above and below, hexagonal z faces); hexahedra
 * elsewhere. All faces planar. Zones: 0 inlet (x = 0), 1 outlet, 2 bump wall, 3 top, 4 z = 0,
 * 5 z = extent[2]. order: owned cell order as autan_lattice.rcm. */
struct autan_bump_channel {
  int32_t nx, ny, nz;
  double extent[3];
  double bump;
  double ratio;
  int32_t stretched;
  int32_t prism_rows[2];
  int32_t brick_rows[2];
  int32_t brick_cols[2];
  int32_t order;
};
int autan_mesh_build_bump_channel(const struct autan_bump_channel* spec, void** mesh, char* err,
                                  size_t err_len);

void autan_mesh_free(void* mesh);

/* counts[0..11]: n_points, n_cells, n_owned_cells, n_faces, n_interior_faces,
 * n_owned_interior_faces, n_owned_faces, n_incidences (cell_faces entries), n_stencil,
 * all_planar (1 when every face moment is an exact zero), n_ghost_cells, n_zones. */
void autan_mesh_counts(const void* mesh, int64_t* counts);

/* Borrowed pointer to one of the mesh's arrays and its number of elements, by name:
 *   int32: "owner" (n_faces), "neighbour" (n_interior_faces), "cell_faces", "face_zone" (n_faces,
 *          -1 on interior faces), "stencil" (entries: a cell, or -(f + 1) for boundary face f),
 *          "ghost_owner" (per ghost: the owned cell it images), "face_nodes", "owned_order"
 *          (per owned cell: its index in the generator's numbering)
 *   int64: "cell_face_offsets" (n_cells + 1), "stencil_offsets" (n_cells + 1), "face_node_offsets"
 *   double: "points" (3 x n_points), "face_area" (3 x n_faces, the area vector S_f),
 *          "face_area_magnitude", "face_normal" (3 x n_faces), "face_centroid" (3 x n_faces),
 *          "face_moment" (9 x n_faces, row-major per face), "cell_centroid" (3 x n_cells),
 *          "cell_volume" (n_cells), "ghost_translation" (3 x n_ghost_cells)
 * Returns 1 for an unknown name. *elem_size receives the element size in bytes. */
int autan_mesh_array(const void* mesh, const char* name, const void** ptr, int64_t* count,
                     int32_t* elem_size);

/* Least-squares weights of the gradient over the face2 stencil (3 x n_stencil, FP64), as
 * Euler<P>::gradient_weights returns them once set_boundary has run (physics/src/euler.cpp:340-416):
 * a boundary face enters a cell's fit only where its condition gives the state there
 * (bc_kind == 0, "state"), unless the cell's other entries do not determine a gradient; offsets
 * within 64 ulps of the coordinates count as zero. bc_kind: one code per boundary face
 * (n_faces - n_interior_faces), the codes of autan_euler_device.h. Weights of ghost cells are 0. */
int autan_mesh_gradient_weights(const void* mesh, const uint8_t* bc_kind, double* weights,
                                char* err, size_t err_len);

/* ---- the gradient set-up on the GPU -------------------------------------------------------
 * The face2 stencil of every cell (codegen/cpp/geometry.cpp:432, StencilKind::face2) and the
 * least-squares weights of the owned cells (physics/src/euler.cpp:340-416) computed by kernels, one
 * thread per cell, with the same per-cell rules as the host set-up above: the stencil and weights
 * equal those of autan_mesh_build_* and autan_mesh_gradient_weights bit for bit. For meshes whose
 * host set-up would dominate (millions of cells, large batches of cases). The mesh is given by its
 * arrays (host pointers, the mesh contract's layouts), as autan_euler_device_create takes it. */
struct autan_setup_mesh {
  int32_t n_cells, n_owned_cells, n_faces, n_interior_faces;
  const int64_t* cell_face_offsets; /* n_cells + 1 */
  const int32_t* cell_faces;
  const int32_t* owner;         /* n_faces */
  const int32_t* neighbour;     /* n_interior_faces */
  const double* cell_centroid;  /* 3 x n_cells (ghost cells: their images' centroids) */
  const double* face_centroid;  /* 3 x n_faces */
};
/* Copies the mesh arrays to `device` and computes the stencil there; *n_stencil receives its
 * length. E1102 when a cell gathers more than 512 stencil candidates. */
int autan_setup_device_create(const struct autan_setup_mesh* mesh, int32_t device, void** handle,
                              int64_t* n_stencil, char* err, size_t err_len);
/* The weights for the boundary codes bc_kind (n_faces - n_interior_faces, the codes of
 * autan_euler_device.h); *retried (may be NULL) receives the number of cells that needed every
 * boundary face in their fit. */
int autan_setup_device_weights(void* handle, const uint8_t* bc_kind, int64_t* retried, char* err,
                               size_t err_len);
/* Copies the stencil offsets (n_cells + 1), entries (n_stencil) and weights (3 x n_stencil, after
 * autan_setup_device_weights) to host arrays; any may be NULL. */
int autan_setup_device_download(void* handle, int64_t* stencil_offsets, int32_t* stencil,
                                double* weights, char* err, size_t err_len);
/* Device times in ms (CUDA events on the handle's stream): [0] copying the mesh arrays, [1] the
 * stencil, [2] the last weights. */
void autan_setup_device_times(void* handle, double* ms);
void autan_setup_device_free(void* handle);

#ifdef __cplusplus
}
#endif

#endif
