/* C ABI of the B200-native explicit Euler residual-and-update path.
 *
 * It replaces, for one rank on one GPU, the reference's device stepper and host residual:
 *   physics/include/autan/physics/euler_device.hpp:22-41   DeviceStepper<P>::{step, evaluate,
 *                                                           residual, set_second_order, upload,
 *                                                           download}
 *   physics/include/autan/physics/euler_device.hpp:49-54   make_device_stepper<P>(...)
 *   physics/include/autan/physics/euler.hpp:127-184        Euler<P>::{set_boundary,
 *                                                           set_boundary_data, set_source,
 *                                                           residual}
 * with the conventions of the reference's own C ABI (physics/mms/capi.cpp:42-60,126-347): opaque
 * handles, int return (0 success, 1 failure with "Exxxx: message" copied into err, err_len bytes,
 * NUL-terminated), no exception across the boundary, caller-owned FP64 host arrays copied at the
 * call, structure of arrays (component c of entity i at c * n + i).
 *
 * Meshes follow Autan's face-based mesh contract (docs/contracts/mesh.md): owned cells then ghost
 * cells; interior faces sorted by (owner, neighbour), owner < neighbour, faces touching an owned
 * cell first; boundary faces after the interior ones; cell_faces per cell in increasing face
 * index. Ghost cells are periodic images of owned cells (a one-rank partition with self-exchange,
 * partition/src/self_exchange.cpp:15-30): ghost g takes the values of owned cell ghost_owner[g].
 * The device reads an image's values at its owned cell, so no ghost fill runs for images. On a
 * rank of a partitioned mesh, a ghost with ghost_owner -1 is external: another rank owns it, and
 * the ranks' exchange fills its records (autan_euler_device_set_ranks).
 *
 * Not thread-safe per handle; distinct handles may run concurrently. Every call is ordered on the
 * handle's stream; calls that return host data synchronise it. */
#ifndef AUTAN_EULER_DEVICE_H
#define AUTAN_EULER_DEVICE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary condition codes (physics/include/autan/physics/euler.hpp:31-38, kernels/euler.py:55-60)
 * and the meaning of each face's five data values. */
enum autan_boundary_kind {
  AUTAN_BC_STATE = 0,    /* W = (rho, u, v, w, p) given */
  AUTAN_BC_FARFIELD = 1, /* freestream W; Riemann invariants normal to the face */
  AUTAN_BC_SLIP = 2,     /* slip wall or symmetry plane; data unused */
  AUTAN_BC_INLET = 3,    /* subsonic inflow normal to the face: (p0, T0, -, -, -) */
  AUTAN_BC_OUTLET = 4,   /* subsonic outflow: (-, -, -, -, p) */
  AUTAN_BC_WALL = 5      /* no-slip wall at rest: (T_wall or 0 when adiabatic, -, -, -, -) */
};

enum autan_flux { AUTAN_FLUX_ROE = 0, AUTAN_FLUX_HLLC = 1, AUTAN_FLUX_AUSM_UP = 2 };
enum autan_precision { AUTAN_FP64 = 0, AUTAN_FP32_ACC64 = 1 };

/* Scheme and gas (physics/include/autan/physics/euler.hpp:40-71, the real[] of
 * autan_mms_euler_create). `planar` selects the loops without warped-face terms
 * (Euler<P>::set_planar): refused unless every face moment is zero. */
struct autan_euler_scheme {
  int32_t flux;
  int32_t second_order;
  int32_t limiter;
  int32_t precision;
  int32_t planar;
  double gamma;
  double gas_constant;
  double venkat_k;
  double length;
  double mach_ref;
  double scale[5];
  double reference[5]; /* conserved reference state U_ref; density > 0 */
};

/* The mesh, its FP64 geometry and gradient stencil, in the layouts of kernels::Topology
 * (codegen/include/autan/kernels/runtime.hpp:167-216) and kernels::PackedGeometry
 * (codegen/include/autan/kernels/geometry.hpp:16-42). face_moment may be NULL (all planar).
 * stencil_lsq_weight: Euler<P>::gradient_weights() for the boundary kinds set_boundary will give. */
struct autan_euler_mesh {
  int32_t n_cells, n_owned_cells, n_faces, n_interior_faces, n_owned_interior_faces, n_owned_faces;
  const int32_t* owner;             /* n_faces */
  const int32_t* neighbour;         /* n_interior_faces */
  const int64_t* cell_face_offsets; /* n_cells + 1 */
  const int32_t* cell_faces;
  const int32_t* ghost_owner;        /* n_cells - n_owned_cells */
  const double* face_normal;         /* 3 x n_faces, unit, owner -> neighbour */
  const double* face_area_magnitude; /* n_faces */
  const double* face_centroid;       /* 3 x n_faces */
  const double* face_moment;         /* 9 x n_faces, row-major per face, or NULL */
  const double* cell_centroid;       /* 3 x n_cells, ghosts at their shifted positions */
  const double* cell_volume;         /* n_cells */
  const int64_t* stencil_offsets;    /* n_cells + 1 */
  const int32_t* stencil;            /* cell, or -(f + 1) for boundary face f */
  const double* stencil_lsq_weight;  /* 3 x stencil entries */
};

/* What one explicit step reports (DeviceStepper<P>::Result, euler_device.hpp:25-29). */
struct autan_euler_step_result {
  double residuals[5]; /* RMS of each residual component at the start of the last step */
  double time_step;    /* the global step of the last step (the least, with local steps) */
  int64_t invalid_cell; /* least owned cell with a non-finite or non-positive state or a
                           non-finite residual after the last step, -1 if none */
  int64_t steps;       /* steps taken */
};

/* make_device_stepper (euler_device.hpp:49-54, physics/src/euler_device.cu:8-23): copies the
 * mesh, geometry and stencil to `device` (an ordinal; -1: the current device) and runs on
 * `stream` (a cudaStream_t; NULL: a stream of the handle's own). Boundary kinds default to slip
 * with zero data, the source to zero. */
int autan_euler_device_create(const struct autan_euler_mesh* mesh,
                              const struct autan_euler_scheme* scheme, int32_t device,
                              void* stream, void** handle, char* err, size_t err_len);
void autan_euler_device_destroy(void* handle);

/* Euler<P>::set_boundary (euler.hpp:126-127): one code per boundary face (n_faces -
 * n_interior_faces) and 5 x n_boundary data values. */
int autan_euler_device_set_boundary(void* handle, const uint8_t* kind, const double* data,
                                    int64_t n_boundary, char* err, size_t err_len);
/* Euler<P>::set_boundary_data (euler.hpp:128-129). */
int autan_euler_device_set_boundary_data(void* handle, const double* data, int64_t n_boundary,
                                         char* err, size_t err_len);
/* Euler<P>::set_source (euler.hpp:178-179): 5 x n_cells, per unit volume. */
int autan_euler_device_set_source(void* handle, const double* source, char* err, size_t err_len);
/* DeviceStepper<P>::set_second_order (euler_device.hpp:38). */
int autan_euler_device_set_second_order(void* handle, int32_t on, char* err, size_t err_len);

/* DeviceStepper<P>::upload / download (euler_device.hpp:39-40): the FP64 conserved state,
 * 5 x n_cells (ghost entries ignored on upload; on download an image's written as its owned
 * cell's, an external ghost's left as they are). */
int autan_euler_device_upload(void* handle, const double* u, char* err, size_t err_len);
int autan_euler_device_download(void* handle, double* u, char* err, size_t err_len);

/* DeviceStepper<P>::residual (euler_device.hpp:37): R(state(u)) of a host FP64 state into a host
 * FP64 residual, both 5 x n_cells (ghost entries of res set to zero). The device state is
 * unchanged. */
int autan_euler_device_residual(void* handle, const double* u, double* res, char* err,
                                size_t err_len);

/* DeviceStepper<P>::step (euler_device.hpp:33), `n_steps` times on the device state:
 *   rk 3: SSP-RK3 (Shu and Osher 1988, eq. 2.18) as CudaStepper::step (device_stepper.cuh:313-345);
 *   rk 4: classical RK4, stage_s = u - ((c_s dt) / V) R with c = (1/2, 1/2, 1), then
 *         u - ((dt / 6) / V) (R_0 + 2 R_1 + 2 R_2 + R_3) (not in the reference);
 *   dt > 0: that global step; else CFL: dt = min over owned cells of (cfl V) / lambda, lambda the
 *   convective spectral radius (kernels/euler.py:1091-1112); `local` != 0: each cell its own.
 * use_graph != 0 captures one step in a CUDA graph and replays it. The host reads nothing until
 * the last step; *out describes the last step. */
int autan_euler_device_step(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                            int64_t n_steps, int32_t use_graph,
                            struct autan_euler_step_result* out, char* err, size_t err_len);
/* DeviceStepper<P>::evaluate (euler_device.hpp:35): residual norms and validity of the state. */
int autan_euler_device_evaluate(void* handle, struct autan_euler_step_result* out, char* err,
                                size_t err_len);
/* Per-step history of the last autan_euler_device_step call: for step i < min(steps, 4096),
 * 5 RMS values at rms[5 i], the global step at dt[i]; either pointer may be NULL. */
int autan_euler_device_history(void* handle, int64_t count, double* rms, double* dt, char* err,
                               size_t err_len);

/* After a residual or step: the reconstruction gradients (15 x n_owned_cells, row-major per cell
 * (3 i + j) as Euler<P>::Arrays::grad) and limiter (5 x n_owned_cells) of the last evaluation, as
 * FP64; either pointer may be NULL. */
int autan_euler_device_gradients(void* handle, double* grad, double* phi, char* err,
                                 size_t err_len);
/* The CFL time step of each owned cell for the device state, (cfl V) / lambda (n_owned_cells). */
int autan_euler_device_time_steps(void* handle, double cfl, double* dt, char* err, size_t err_len);

/* Runs n_steps steps as autan_euler_device_step does, launching without a graph and recording a
 * CUDA event pair around every kernel on the handle's stream; per kernel kind, ms[k] receives the
 * summed durations and launches[k] the launches: 0 boundary states, 1 gradients and limiter,
 * 2 spectral radius and time step, 3 faces and RK update, 4 residual norms, 5 step control. */
int autan_euler_device_kernel_times(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                    int64_t n_steps, double* ms, int64_t* launches, char* err,
                                    size_t err_len);
/* Launch choices of the hot kernels (10 values; set_tuning also takes the first 6 alone, the rest
 * then keep their values): [0] stencil entries the gradient kernel loads
 * together (1, 2 or 4, where 2 takes at most 128 threads per block; 2, 4 or 8 when staged), [1]
 * its threads per block, [2] face strategy (0 gather-recompute: each cell recomputes its faces'
 * fluxes; 1 store-gather: each face's flux once into a face scratch, then summed per cell; 2 as 1,
 * with a step's stage-0 residual norms summed inside the gather instead of a pass over a stored
 * residual, without batched cases), [3]
 * threads per block of the face kernel, [4] of the store-gather sum, [5] gradient staging (0:
 * each thread loads its stencil rows; 1: each block's rows staged into shared memory by TMA bulk
 * copies, at most 128 threads per block; 2: as 0, software-pipelined: the next entry's gather and
 * the row after it in flight while an entry is added; 3: each thread's next [0] neighbour records
 * and 2 x [0] rows in a shared-memory ring filled by asynchronous copies (cp.async), [0] = 2, 4
 * or 8, at most 128 threads per block; 4, fp32+acc64 only: as 0 with [0] entries loaded together,
 * 128 threads per block, and [6] 0, 1 or 2: none, the x and y, or all of each entry's 15 products
 * widened to FP64 on the integer pipe, exactly (2^-896-scaled bit moves) instead of by cvt; [7]
 * 1: neighbours gathered as 16 + 4 bytes instead of one 32-byte load; [8] the blocks of 128
 * threads per SM the registers are bounded for: 7 or 6 with [0] = 2, 5 with [0] = 4; 5,
 * fp32+acc64 only: each warp's
 * stencil rows streamed by TMA bulk copies into a ring of [9] (4 or 8) shared-memory slots ahead of
 * the warp, [0] (2 or 3) gathers in flight, [7] as for 4, 128 threads per block).
 * Every choice gives the same bits. No counterpart in the reference beyond its Strategy enum
 * (codegen/include/autan/kernels/strategy.hpp:14-21). */
int autan_euler_device_set_tuning(void* handle, const int32_t* params, int32_t count, char* err,
                                  size_t err_len);
int autan_euler_device_get_tuning(void* handle, int32_t* params, int32_t count, char* err,
                                  size_t err_len);
/* The autotuner: times candidate launch choices on `trial_steps` steps each of this handle's own
 * case (the device state is restored after every trial), keeps the fastest and returns it in
 * params (10 values, or NULL) with its ms per step. */
int autan_euler_device_autotune(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                int32_t trial_steps, int32_t* params, double* ms_per_step,
                                char* err, size_t err_len);
/* Euler<P>::face_parts (physics/src/euler.cpp:944-965) of the host state u (5 x n_cells) or, with
 * u NULL, of the device state: res_faces (5 x n_cells) the residual's face part R^F, no sources,
 * summed from zero in each cell's face order (ghost entries 0); face_flux (5 x n_faces) the flux of
 * every owned interior and owned boundary face as the write-only loops give it
 * (kernels/euler.py:1059-1085), other entries 0. Either output may be NULL. */
int autan_euler_device_face_parts(void* handle, const double* u, double* res_faces,
                                  double* face_flux, char* err, size_t err_len);
/* Euler<P>::boundary_pressure (physics/src/euler.cpp:1182-1223) after evaluating the host state u
 * or, with u NULL, the device state (EulerPhysics::face_pressure, euler_physics.cpp:1478-1492): p
 * (n_faces - n_interior_faces) the reconstructed face pressure of every boundary face, force
 * (3 x that, or NULL) p_f S + phi_p M^T grad p. */
int autan_euler_device_boundary_pressure(void* handle, const double* u, double* p, double* force,
                                         char* err, size_t err_len);
/* The sums of EulerPhysics::check_conservation (physics/src/euler_physics.cpp:1740-1779) on the
 * device state, one rank: sums[20] = E[5], D[5], boundary[5], faces[5], each an exact sum over the
 * owned cells and faces (E = sum R^F - sum boundary fluxes; D = sum |flux| per incidence of an
 * owned cell); *max_faces (may be NULL) the most faces of an owned cell, the d of the bound
 * tau = max(64 2^-52, 2 gamma_(d+2)) (docs/validation/acceptance.md, D2 gate 7). */
int autan_euler_device_conservation(void* handle, double* sums, int32_t* max_faces, char* err,
                                    size_t err_len);
/* The result of a march to convergence. */
struct autan_march_result {
  int64_t iterations;   /* the iteration at which the rule held, or the steps taken if it never did */
  int64_t steps;        /* steps taken: up to batch - 1 more than `iterations` (the last batch) */
  int32_t converged;    /* 1 when the rule held */
  int32_t plateau_mask; /* bit e: equation e converged on a round-off plateau */
  double first[5];      /* the residual RMS of iteration 1 */
  double last[5];       /* the residual RMS of iteration `iterations` */
  double time_step;     /* that iteration's global step */
  double gpu_ms;        /* device time of the march (CUDA events on the handle's stream) */
  int64_t invalid_cell; /* as autan_euler_step_result, -1 if none; the march stops at one */
};

/* A steady march (runtime/src/run.cpp:2351-2389): steps of autan_euler_device_step, `batch` per
 * captured-graph call, until every equation's RMS residual has dropped `orders` decades from its
 * reference or, with `floors` (round_off_floor * Phi_k, 5 values; NULL: no plateau rule), sits on
 * a round-off plateau at most 10 floors high (runtime/include/autan/runtime/round_off.hpp), or
 * until max_steps. The rule as autan_convergence_iteration. */
int autan_euler_device_march(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                             int64_t max_steps, int32_t batch, double orders, const double* floors,
                             struct autan_march_result* out, char* err, size_t err_len);
/* The convergence rule alone, on a residual history (n iterations x 5, row-major): *iteration the
 * first (1-based) at which it holds, 0 if none; *plateau_mask (may be NULL) as above. Host only. */
int autan_convergence_iteration(const double* residuals, int64_t n, double orders,
                                const double* floors, int64_t* iteration, int32_t* plateau_mask,
                                char* err, size_t err_len);
/* Batched cases (many steady cases advanced together; no counterpart in the reference, which runs
 * one case per process): the handle's mesh is the disjoint union of the cases' meshes, case k's
 * owned cells [cell_offsets[k], cell_offsets[k + 1]) (n_cases + 1 offsets from 0 to
 * n_owned_cells). Every kernel of a stage runs once over all cases; with local time steps the
 * cases do not interact. Each step then also records each case's RMS residual (exact sums over its
 * cells), and a case whose active flag is 0 is skipped: its state no longer changes. */
int autan_euler_device_set_cases(void* handle, int32_t n_cases, const int64_t* cell_offsets,
                                 char* err, size_t err_len);
/* One flag per case, nonzero: the case steps. */
int autan_euler_device_set_active(void* handle, const uint8_t* active, char* err, size_t err_len);
/* Per case (n_cases values, each positive), the AUSM+-up cut-off Mach number M_co
 * (Scheme::mach_ref, kernels/euler.py:268-303) of the faces whose owner cell is in the case, in
 * place of the scheme's one value: each case then steps as its own run with its own mach_ref
 * would. Reset by autan_euler_device_set_cases. No other flux uses it. */
int autan_euler_device_set_case_mach_ref(void* handle, const double* mach_ref, char* err,
                                         size_t err_len);
/* The per-case RMS of the last `count` steps of the last step call: count x n_cases x 5, oldest
 * first. */
int autan_euler_device_case_history(void* handle, int64_t count, double* rms, char* err,
                                    size_t err_len);
/* The batched march: steps (`batch` per captured-graph call) until every case has met the
 * convergence rule of autan_euler_device_march (floors: 5 per case or NULL; reference: 5 per case,
 * the residuals each case's drop is measured from, as a continued run's start.residual_reference,
 * or NULL for each case's first iteration), each case stopping at the end of the batch in which it
 * converged, or until max_steps. iterations[k] (n_cases): the iteration at which case k converged,
 * or the steps taken; converged[k]: 1 if it did; first (5 per case, may be NULL): the reference
 * used; *steps: steps taken; *gpu_ms: device time; stop_ms (n_cases, may be NULL): the device
 * time from the march's start to the end of the batch in which each case converged (the whole
 * march's time for a case that did not). Once cases stop, the stage kernels are launched over the
 * 32-item tiles of the cases still stepping only. Every case steps again afterwards. */
int autan_euler_device_march_cases(void* handle, double cfl, double dt, int32_t local, int32_t rk,
                                   int64_t max_steps, int32_t batch, double orders,
                                   const double* floors, const double* reference,
                                   int64_t* iterations, int32_t* converged, double* first,
                                   int64_t* steps, double* gpu_ms, double* stop_ms, char* err,
                                   size_t err_len);
/* Test hook of the failure detection (no counterpart in the reference): with polls > 0 every warp
 * of the mode-5 gradient kernel also waits, at most `polls` polls, on an mbarrier that nothing
 * arrives on; the bounded wait runs out, the warp marks the fault word, waits (up to 2^20 polls)
 * for the copies it has issued and stores nothing, and the step call returns E1201. 0 turns the
 * hook off; the handle stays usable either way. */
int autan_euler_device_set_stall_test(void* handle, int32_t polls, char* err, size_t err_len);

/* One rank's share of a partitioned mesh (the reference's GhostFill / HaloExchange forward and
 * Ranks::sum / min, partition/include/autan/partition/halo_exchange.hpp:14-66,
 * physics/src/euler.cpp:96-136). The handle's mesh then holds external ghosts: ghost cells whose
 * ghost_owner is -1, whose values another rank owns. Their records are filled by `exchange` at
 * the start of every RK stage (primitives: what 0, 8 words a cell) and, second order, after its
 * gradient loop (phi then grad: what 1, 24 words a cell; words of the precision's storage type,
 * 4 bytes in fp32+acc64, 8 in fp64). Before each call the library has enqueued on `stream` the
 * packing of the records of send_cells[0 .. n_send) into `send`, record after record; the
 * callee leaves in `recv`, for the work the library enqueues on `stream` after the call returns,
 * the records of the external ghosts in their order in the mesh. `reduce` combines `count` words
 * at `words` over the ranks in place, for the work enqueued after it returns: op 0 the sum
 * modulo 2^64 (the 5 x 71 exact-sum words of the stage-0 residual norms), op 1 the minimum as
 * signed 64-bit integers (the bits of the CFL step, a positive double). The RMS norms divide by
 * global_cells. Every rank makes the same calls in the same order. A callback's nonzero return
 * fails the step call with E1301.
 *
 * With ranks set, step runs eagerly (no graph); step, evaluate, kernel_times, march and autotune
 * make the exchanges, so every rank calls them together (autotune's trials are the same on every
 * rank; each rank keeps its own fastest choices, which change no result). residual, time_steps,
 * face_parts, boundary_pressure, conservation and batched cases are refused (E1101) on a mesh
 * with external ghosts, and every entry that steps is refused there until ranks are set.
 * invalid_cell stays a local cell; the Python driver (autan_b200/partition.py) reduces it to the
 * least global id. A march stops on every rank when any rank meets an invalid cell (one more
 * minimum over the ranks after each batch). NULL detaches the ranks. */
struct autan_euler_ranks {
  void* user;
  int32_t (*exchange)(void* user, int32_t what, int64_t record_bytes, void* stream);
  int32_t (*reduce)(void* user, int32_t op, int64_t count, void* stream);
  void* send;                /* device, n_send x 24 words */
  void* recv;                /* device, external ghosts x 24 words */
  uint64_t* words;           /* device, at least 5 x 71 words */
  int64_t n_send;
  const int32_t* send_cells; /* n_send owned cells (host; copied), repeats allowed */
  double global_cells;       /* owned cells over all ranks */
};
int autan_euler_device_set_ranks(void* handle, const struct autan_euler_ranks* ranks, char* err,
                                 size_t err_len);
/* The number of external ghosts of the handle's mesh. */
int autan_euler_device_external_ghosts(void* handle, int64_t* count, char* err, size_t err_len);

/* Waits for the handle's stream. */
int autan_euler_device_sync(void* handle, char* err, size_t err_len);
/* The handle's cudaStream_t. */
void* autan_euler_device_stream(void* handle);
/* Counters of the handle since creation: [0] kernels launched by the library, [1] steps taken,
 * [2] residual evaluations, [3] device bytes held. */
int autan_euler_device_counters(void* handle, int64_t* counters, char* err, size_t err_len);

/* Exact-sum RMS of device arrays that allocates no device memory: rms[k] = sqrt(sum_i
 * values[k * stride + i]^2 / n) for k < components, each sum exact and rounded once (the norms of
 * autan_euler_device_evaluate, bit for bit on the same residual). No counterpart in the reference.
 *   values: device pointer; rms: device pointer to `components` doubles, written on `stream`
 *   (a cudaStream_t, NULL for the default stream) of the calling thread's current device.
 * Limits: components 1 to 8, n 1 to 2^30 (a sum's words cannot overflow), device index < 64;
 * anything beyond is refused with E1101 before any device work.
 * Scratch: 4544 bytes of module-level device memory per device, found with cudaGetSymbolAddress
 * on the first call for each device (make that first call before any stream capture) and kept
 * for the process: the device's primary context must live as long (no cudaDeviceReset between
 * calls, which would reload the module elsewhere); each call
 * clears the words it uses on `stream` first. Calls that overlap in time on one device share the
 * scratch and race: order them on one stream or wait between them. For callers that cannot
 * allocate at the point of the call (a pool allocator holding all device memory, a path where
 * cudaFree's device-wide wait is not acceptable). */
int autan_exact_rms_static(const double* values, int64_t n, int64_t stride, int32_t components,
                           double* rms, void* stream, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif
