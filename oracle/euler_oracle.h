/* CPU oracle of the explicit Euler residual-and-update path: a plain-C restatement of the
 * reference's host algorithm, used ONLY as the checker by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py. It is never linked into, called by or shipped with the product.
 *
 * It follows the reference operation for operation:
 *   residual       physics/src/euler.cpp:934-941 (Euler<P>::residual), the loops of
 *                  kernels/euler.py as the generator emits them (codegen/src/autan_codegen/
 *                  emit_cpp.py, emit_cpu.py): bodies in the compute type, inputs converted on
 *                  first use, rel() in FP64 then converted, Sum accumulators in FP64, Min/Max in
 *                  the compute type, face loops scattered in face order;
 *   ghost fills    physics/src/euler.cpp:96-136 (a one-rank partition's periodic images);
 *   SSP-RK3 step   physics/src/euler_physics.cpp:1362-1393; local steps device_stepper.cuh:84-104;
 *   norms          physics/src/euler_physics.cpp:1040-1054 with runtime/src/exact_sum.cpp;
 *   divergence     physics/src/euler_physics.cpp:1399-1435.
 * Classical RK4 is not in the reference; its form here is stated in oracle_step().
 * Parity pin: tests/golden/ holds outputs of the reference's own kernels/euler.py bodies evaluated
 * in Python (tests/golden/make_golden.py), which this restatement must reproduce bit for bit. */
#ifndef AUTAN_ORACLE_H
#define AUTAN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The same layout as struct autan_euler_mesh (include/autan_euler_device.h). */
typedef struct oracle_mesh {
  int32_t n_cells, n_owned_cells, n_faces, n_interior_faces, n_owned_interior_faces, n_owned_faces;
  const int32_t* owner;
  const int32_t* neighbour;
  const int64_t* cell_face_offsets;
  const int32_t* cell_faces;
  const int32_t* ghost_owner;
  const double* face_normal;
  const double* face_area_magnitude;
  const double* face_centroid;
  const double* face_moment;
  const double* cell_centroid;
  const double* cell_volume;
  const int64_t* stencil_offsets;
  const int32_t* stencil;
  const double* stencil_lsq_weight;
} oracle_mesh;

/* The same layout as struct autan_euler_scheme. flux 0 Roe, 1 HLLC, 2 AUSM+-up; precision 0 fp64,
 * 1 fp32+acc64; planar: the *_planar loops. */
typedef struct oracle_scheme {
  int32_t flux, second_order, limiter, precision, planar;
  double gamma, gas_constant, venkat_k, length, mach_ref;
  double scale[5];
  double reference[5];
} oracle_scheme;

typedef struct oracle oracle;

/* The ranks of a partitioned mesh, for the oracle's steps (test infrastructure: the checker of the
 * partitioned device path). halo: at each ghost fill (kind 0 primitives, 1 gradients, 2 limiter
 * values), `send` holds this rank's owned values (comps x owned cells) and the callee writes the
 * external ghosts' values into `recv` (comps x ghost cells, ghost order; images' entries unused).
 * min: the minimum over the ranks, in place (the global CFL step). */
typedef void (*oracle_halo_fn)(void* user, int32_t kind, int32_t comps, const double* send,
                               double* recv);
typedef void (*oracle_min_fn)(void* user, double* value);

oracle* oracle_create(const oracle_mesh* mesh, const oracle_scheme* scheme, const uint8_t* bc_kind,
                      const double* bc, const double* source);
void oracle_free(oracle* o);
void oracle_set_second_order(oracle* o, int32_t on);
/* R(state(u)): u, res 5 x n_cells FP64 (owned cells meaningful). */
void oracle_residual(oracle* o, const double* u, double* res);
/* The arrays of the last evaluation, as FP64: prim 5 x nc, grad 15 x nc, phi 5 x nc, wmin/wmax
 * 5 x nc, prim_b 5 x nf (any may be NULL). */
/* A rank's external ghosts (ghost_owner -1): their primitives, gradients and limiter values
 * (5, 15 and 5 x ghosts in ghost order) for the ghost fills of the following residuals. */
void oracle_set_external(oracle* o, const double* prim, const double* grad, const double* phi);
/* A rank of a partitioned mesh: its exchange and minimum over the ranks (NULL: one rank). */
void oracle_set_ranks(oracle* o, oracle_halo_fn halo, oracle_min_fn min, void* user);
void oracle_arrays(const oracle* o, double* prim, double* grad, double* phi, double* wmin,
                   double* wmax, double* prim_b);
/* After a residual: the spectral radius of each cell (n_cells, FP64 of the stored value). */
void oracle_spectral_radius(oracle* o, double* lambda);
/* One explicit step of u (5 x n_cells FP64, in place): rk 3 (SSP-RK3) or 4 (classical RK4);
 * dt > 0 fixed, else CFL; local != 0: each cell its own CFL step. norms[5]: RMS of R(u) before the
 * step; *dt_out: the global step. Returns the least invalid cell after the step, or -1. */
int64_t oracle_step(oracle* o, double* u, int32_t rk, double cfl, double dt, int32_t local,
                    double* norms, double* dt_out);
/* Euler<P>::face_parts (physics/src/euler.cpp:944-965) of state(u): res_faces (5 x n_cells) the
 * residual's face part (no sources, from zero), face_flux (5 x n_faces) each owned interior and
 * owned boundary face's flux (kernels/euler.py:1059-1085); other entries zero. */
void oracle_face_parts(oracle* o, const double* u, double* res_faces, double* face_flux);
/* Euler<P>::boundary_pressure (physics/src/euler.cpp:1182-1223) of the last evaluation's arrays:
 * p (n_faces - n_interior_faces), force (3 x that, or NULL). */
void oracle_boundary_pressure(const oracle* o, double* p, double* force);
/* RMS over the owned cells of each residual component, exact sums. */
void oracle_norms(const double* res, int32_t n_owned, int32_t n_cells, double* rms);
/* ExactSum (runtime/src/exact_sum.cpp) of n terms, rounded once to the nearest double. */
double oracle_exact_sum(const double* terms, int64_t n);
/* Euler::Impl::compute_gradient_weights (physics/src/euler.cpp:340-416): the least-squares
 * gradient weights of the owned cells over mesh->stencil (w: 3 x n_stencil, written; ghost cells
 * 0) for the boundary codes bc_kind (n_faces - n_interior_faces). Reads the mesh's stencil and
 * centroids only (mesh->stencil_lsq_weight is not read). */
void oracle_gradient_weights(const oracle_mesh* mesh, const uint8_t* bc_kind, double* w);
/* First invalid cell of a state and residual (euler_physics.cpp:1399-1435), or -1. */
int64_t oracle_first_invalid(const oracle* o, const double* u, const double* res);

/* Pointwise bodies, for the golden vectors (compute in the scheme's precision; FP64 I/O):
 * flux of two face states (W gauge, 5 each) through n, times area; boundary state of kind. */
void oracle_flux(const oracle_scheme* s, const double* wl, const double* wr, const double* n,
                 double* out);
void oracle_boundary_value(const oracle_scheme* s, const double* wg, double kind,
                           const double* data, const double* n, double* out);
void oracle_to_primitive(const oracle_scheme* s, const double* dq, double* out);

#ifdef __cplusplus
}
#endif

#endif
