/* C ABI of the learned warm start of the steady bump-channel cases: a small MLP that predicts each
 * cell's conserved-variable offsets from the freestream out of the cell's geometry and its case's
 * parameters, trained and evaluated on the GPU by this library's own BF16 tensor-core kernels
 * (BF16 weights and activations, FP32 accumulation), and the wall distance it takes as an input.
 * No counterpart in the reference (its wall distance: core/src/wall_distance.cpp,
 * core/src/wall_distance_device.cu, WallSurface::distance).
 *
 * Conventions as include/autan_euler_device.h: int return, 0 on success, 1 with "Exxxx: message"
 * in err; arrays are row-major [rows x columns] unless stated; host pointers unless stated. */
#ifndef AUTAN_MLP_H
#define AUTAN_MLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The network: `inputs` features -> `layers` hidden layers of `width` (GELU, the erf form) ->
 * `outputs`, each layer y = W x + b with W stored [out x in]. width a multiple of 16 (at most 128);
 * inputs and outputs at most width. Inputs are standardised (x - mean) / std and outputs
 * de-standardised y std + mean with the statistics of autan_mlp_set_scaling. Weights: Glorot
 * uniform from `seed`, biases zero. */
int autan_mlp_create(int32_t inputs, int32_t width, int32_t layers, int32_t outputs, uint64_t seed,
                     int32_t device, void** handle, char* err, size_t err_len);
void autan_mlp_destroy(void* handle);
/* The GEMM engine: 0 warp-level mma.sync m16n8k16, a kernel per layer; 1 tcgen05.mma with the
 * accumulator in tensor memory, a kernel per layer (128-row tiles, operands staged in shared
 * memory); 2 (width 128 only; the default there, else 0) fused tcgen05: one kernel takes each
 * 128-row tile through every layer's forward and, for training, backward GEMMs (weights staged by
 * TMA bulk copies, accumulators in tensor memory), a second sums the tiles' gradients and applies
 * the Adam step. All take BF16 operands and accumulate in FP32. E1101 for engine 2 at another
 * width. */
int autan_mlp_set_engine(void* handle, int32_t engine, char* err, size_t err_len);
/* Test hook of the failure detection (0, the default, in normal use): with polls > 0 every launch
 * of the fused engine first waits, `polls` polls at most, on an mbarrier that nothing arrives on;
 * the wait runs out, the kernel records a fault and leaves without stores, and the call fails with
 * E1201. Setting 0 again restores normal work on the same handle. */
int autan_mlp_set_stall_test(void* handle, int32_t polls, char* err, size_t err_len);
/* The standardisation: in_mean, in_std (inputs values each), out_mean, out_std (outputs each). */
int autan_mlp_set_scaling(void* handle, const float* in_mean, const float* in_std,
                          const float* out_mean, const float* out_std, char* err, size_t err_len);
/* FP32 master weights and biases, layer by layer: W (out x in) then b (out). count: the number of
 * floats (autan_mlp_parameter_count). get copies out, set copies in (and refreshes the BF16
 * weights). */
int64_t autan_mlp_parameter_count(void* handle);
int autan_mlp_get_parameters(void* handle, float* params, int64_t count, char* err, size_t err_len);
int autan_mlp_set_parameters(void* handle, const float* params, int64_t count, char* err,
                             size_t err_len);

/* The training set, copied to the device: x (n x inputs), y (n x outputs), raw (unscaled). */
int autan_mlp_set_data(void* handle, const float* x, const float* y, int64_t n, char* err,
                       size_t err_len);
/* Training: `epochs` passes over the data in shuffled minibatches of `batch` rows (a multiple of
 * 128), Adam (beta1 0.9, beta2 0.999, eps 1e-8) at learning rate lr, decayed along a half cosine
 * over the call's steps, on the mean squared error of the standardised outputs. loss (epochs
 * values, may be NULL): each epoch's mean minibatch loss. */
int autan_mlp_train(void* handle, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                    float* loss, char* err, size_t err_len);
/* One forward and backward pass on n rows (host x, y as set_data's), no update: *loss and the
 * gradient of the loss with respect to every parameter (parameter_count floats, as
 * get_parameters); n from 1 to 2^20. For checks against a CPU restatement. */
int autan_mlp_gradient(void* handle, const float* x, const float* y, int64_t n, float* loss,
                       float* grad, char* err, size_t err_len);
/* Prediction of n rows: x (n x inputs) to y (n x outputs), raw units. device_ptrs != 0: x and y
 * are device pointers, the work ordered on the library's stream of the handle. */
int autan_mlp_predict(void* handle, const float* x, int64_t n, float* y, int32_t device_ptrs,
                      char* err, size_t err_len);

/* Wall distance, exact in FP64 (the point-triangle projection of WallSurface::distance,
 * core/include/autan/core/wall_distance.hpp:28-31): for every point i of case k (points
 * [point_offsets[k], point_offsets[k + 1])), the distance to the nearest of that case's wall
 * triangles [tri_offsets[k], tri_offsets[k + 1]); triangles as (a, b, c) corner triples, 9 doubles
 * each; points 3 x n_points (x row, y row, z row). +infinity for a case without triangles. On the
 * current device; host arrays. */
int autan_wall_distance(const double* triangles, const int64_t* tri_offsets, const double* points,
                        const int64_t* point_offsets, int32_t n_cases, int64_t n_points,
                        double* distance, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif
