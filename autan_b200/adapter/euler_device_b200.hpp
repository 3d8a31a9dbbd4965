// Declarations shared by the reference-side adapter files (euler_device_b200.cpp, which needs
// only the reference's headers, and euler_device_b200_data.cpp, which also needs the generated
// euler_cpu.hpp of the reference's build).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "autan/core/geometry.hpp"
#include "autan/core/mesh.hpp"
#include "autan/kernels/geometry.hpp"
#include "autan/physics/euler.hpp"
#include "autan/physics/euler_device.hpp"
#include "autan/runtime/ranks.hpp"

namespace autan::physics {

// What the device takes from the host residual beyond its stencil, weights and scheme: each
// boundary face's condition as the codes of autan_euler_device.h and its five data values
// (5 x n_boundary_faces), and the source (5 x n_cells; empty: none). Euler<P> keeps these in its
// generated dataset (Euler<P>::data(), kernels::euler::Data<P>: bc_kind, bc and source, the arrays
// physics/src/device_stepper.cuh:250-253 uploads), whose definition only the generated
// euler_cpu.hpp holds, so b200_host_inputs is defined beside that header.
struct B200HostInputs {
  std::vector<std::uint8_t> kind;
  std::vector<double> data;
  std::vector<double> source;
};
template <class P>
B200HostInputs b200_host_inputs(const Euler<P>& host, const Mesh& mesh);

// The B200 stepper of `host` when the case is in scope (one rank, no global keys, the linear face2
// gradient), else null: make_device_stepper then builds its device::CudaStepper. The arguments are
// make_device_stepper's (physics/include/autan/physics/euler_device.hpp:49-54), with the gas
// constant of the case's Gas beside gamma.
template <class P>
std::unique_ptr<DeviceStepper<P>> make_b200_stepper(const Mesh& mesh, const Geometry& geometry,
                                                    const Euler<P>& host, double gamma,
                                                    double gas_constant, bool second_order,
                                                    runtime::Ranks& ranks, void* stream,
                                                    const kernels::GlobalKeys* keys);

}  // namespace autan::physics
