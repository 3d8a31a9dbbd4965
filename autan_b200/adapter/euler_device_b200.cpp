// The reference-side adapter of the B200 path: a physics::DeviceStepper<P>
// (physics/include/autan/physics/euler_device.hpp:22-41) over the C ABI of
// include/autan_euler_device.h, for make_device_stepper (physics/src/euler_device.cu:8-23) to
// return when a case is in the library's scope. It is compiled inside the reference's build
// (with the reference's include directories and this repository's include/) and linked with
// libautan_b200.so; EulerPhysics (physics/src/euler_physics.cpp:307, 1539-1576) is unchanged.
//
// Scope (make_b200_stepper returns null otherwise, and the caller keeps device::CudaStepper):
// one rank; no global keys (the mesh's own face order); the linear face2 gradient; ghost cells,
// if any, periodic images of owned cells (a one-rank partition with self-exchange), recognised by
// their global id.
#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "autan/core/geometry.hpp"
#include "autan/core/mesh.hpp"
#include "autan/kernels/geometry.hpp"
#include "autan/kernels/runtime.hpp"
#include "autan/physics/euler.hpp"
#include "autan/physics/euler_device.hpp"
#include "autan/runtime/ranks.hpp"
#include "autan_euler_device.h"
#include "euler_device_b200.hpp"

namespace autan::physics {

namespace b200 {

// x, y, z arrays as one structure-of-arrays buffer (component c of entity i at c n + i).
inline std::vector<double> soa3(std::span<const double> x, std::span<const double> y,
                                std::span<const double> z) {
  std::vector<double> v(x.begin(), x.end());
  v.insert(v.end(), y.begin(), y.end());
  v.insert(v.end(), z.begin(), z.end());
  return v;
}

// Per ghost cell, the owned cell it is an image of: the owned cell with its global id (a periodic
// image shares its owner's id). Throws for a ghost with no owned cell of that id (another rank's
// cell: out of scope).
inline std::vector<std::int32_t> ghost_owners(const Mesh& mesh) {
  const auto ids = mesh.cell_global_id();
  const auto owned = static_cast<std::size_t>(mesh.n_owned_cells());
  std::unordered_map<std::int64_t, std::int32_t> of_id;
  of_id.reserve(owned);
  for (std::size_t c = 0; c < owned; ++c) of_id.emplace(ids[c], static_cast<std::int32_t>(c));
  std::vector<std::int32_t> g;
  g.reserve(static_cast<std::size_t>(mesh.n_cells()) - owned);
  for (std::size_t c = owned; c < static_cast<std::size_t>(mesh.n_cells()); ++c) {
    const auto it = of_id.find(ids[c]);
    if (it == of_id.end()) throw std::runtime_error("E1101: a ghost cell that is not an image");
    g.push_back(it->second);
  }
  return g;
}

inline autan_euler_scheme scheme_of(const Scheme& s, double gamma, double gas_constant,
                                    bool second_order, bool planar, bool fp64) {
  autan_euler_scheme out{};
  out.flux = s.flux == Flux::roe ? AUTAN_FLUX_ROE : s.flux == Flux::hllc ? AUTAN_FLUX_HLLC
                                                                          : AUTAN_FLUX_AUSM_UP;
  out.second_order = second_order ? 1 : 0;
  out.limiter = s.limiter ? 1 : 0;
  out.precision = fp64 ? AUTAN_FP64 : AUTAN_FP32_ACC64;
  out.planar = planar ? 1 : 0;
  out.gamma = gamma;
  out.gas_constant = gas_constant;
  out.venkat_k = s.venkat_k;
  out.length = s.length;
  out.mach_ref = s.mach_ref;
  for (int k = 0; k < 5; ++k) {
    out.scale[k] = s.scale[static_cast<std::size_t>(k)];
    out.reference[k] = s.reference[static_cast<std::size_t>(k)];
  }
  return out;
}

inline void check(int rc, const char* err) {
  if (rc != 0) throw std::runtime_error(err);  // "Exxxx: message"
}

}  // namespace b200

template <class P>
class B200Stepper final : public DeviceStepper<P> {
 public:
  using Result = typename DeviceStepper<P>::Result;

  B200Stepper(const Mesh& mesh, const Geometry& geometry, const Euler<P>& host, double gamma,
              double gas_constant, bool second_order, void* stream) {
    const kernels::PackedGeometry packed = kernels::pack_geometry(mesh, geometry);
    const kernels::CellStencil& st = host.stencil();
    weights_ = host.gradient_weights();
    ghost_owner_ = b200::ghost_owners(mesh);
    cell_centroid_ = b200::soa3(geometry.cell_centroid_x, geometry.cell_centroid_y,
                                geometry.cell_centroid_z);
    autan_euler_mesh m{};
    m.n_cells = mesh.n_cells();
    m.n_owned_cells = mesh.n_owned_cells();
    m.n_faces = mesh.n_faces();
    m.n_interior_faces = mesh.n_interior_faces();
    m.n_owned_interior_faces = mesh.n_owned_interior_faces();
    m.n_owned_faces = mesh.n_owned_faces();
    m.owner = mesh.owner().data();
    m.neighbour = mesh.neighbour().data();
    m.cell_face_offsets = mesh.cell_face_offsets().data();
    m.cell_faces = mesh.cell_faces().data();
    m.ghost_owner = ghost_owner_.empty() ? nullptr : ghost_owner_.data();
    m.face_normal = packed.face_normal.data();
    m.face_area_magnitude = packed.face_area_magnitude.data();
    m.face_centroid = packed.face_centroid.data();
    m.face_moment = packed.all_planar ? nullptr : packed.face_moment.data();
    m.cell_centroid = cell_centroid_.data();
    m.cell_volume = geometry.cell_volume.data();
    m.stencil_offsets = st.offsets.data();
    m.stencil = st.entries.data();
    m.stencil_lsq_weight = weights_.data();
    const autan_euler_scheme s =
        b200::scheme_of(host.scheme(), gamma, gas_constant, second_order, host.planar(),
                        std::is_same_v<P, kernels::fp64>);
    char err[256];
    b200::check(autan_euler_device_create(&m, &s, -1, stream, &h_, err, sizeof err), err);
    try {
      const B200HostInputs in = b200_host_inputs(host, mesh);
      b200::check(autan_euler_device_set_boundary(h_, in.kind.data(), in.data.data(),
                                                  static_cast<std::int64_t>(in.kind.size()), err,
                                                  sizeof err),
                  err);
      if (!in.source.empty())
        b200::check(autan_euler_device_set_source(h_, in.source.data(), err, sizeof err), err);
    } catch (...) {
      autan_euler_device_destroy(h_);
      throw;
    }
  }
  B200Stepper(const B200Stepper&) = delete;
  B200Stepper& operator=(const B200Stepper&) = delete;
  ~B200Stepper() override { autan_euler_device_destroy(h_); }

  Result step(double cfl, std::optional<double> dt, bool local) override {
    autan_euler_step_result r{};
    char err[256];
    b200::check(autan_euler_device_step(h_, cfl, dt.value_or(0.0), local ? 1 : 0, /*rk=*/3,
                                        /*n_steps=*/1, /*use_graph=*/1, &r, err, sizeof err),
                err);
    return result_of(r);
  }
  Result evaluate() override {
    autan_euler_step_result r{};
    char err[256];
    b200::check(autan_euler_device_evaluate(h_, &r, err, sizeof err), err);
    return result_of(r);
  }
  void residual(std::span<const double> u, std::span<double> res) override {
    char err[256];
    b200::check(autan_euler_device_residual(h_, u.data(), res.data(), err, sizeof err), err);
  }
  void set_second_order(bool on) override {
    char err[256];
    b200::check(autan_euler_device_set_second_order(h_, on ? 1 : 0, err, sizeof err), err);
  }
  void upload(std::span<const double> u) override {
    char err[256];
    b200::check(autan_euler_device_upload(h_, u.data(), err, sizeof err), err);
  }
  void download(std::span<double> u) override {
    char err[256];
    b200::check(autan_euler_device_download(h_, u.data(), err, sizeof err), err);
  }

 private:
  static Result result_of(const autan_euler_step_result& r) {
    Result out;
    out.residuals.assign(r.residuals, r.residuals + 5);
    out.time_step = r.time_step;
    if (r.invalid_cell >= 0) out.invalid = static_cast<index_t>(r.invalid_cell);
    return out;
  }
  void* h_ = nullptr;
  std::vector<double> weights_, cell_centroid_;
  std::vector<std::int32_t> ghost_owner_;
};

template <class P>
std::unique_ptr<DeviceStepper<P>> make_b200_stepper(const Mesh& mesh, const Geometry& geometry,
                                                    const Euler<P>& host, double gamma,
                                                    double gas_constant, bool second_order,
                                                    runtime::Ranks& ranks, void* stream,
                                                    const kernels::GlobalKeys* keys) {
  const Scheme& s = host.scheme();
  if (ranks.size() != 1 || keys != nullptr || s.gradient != GradientStencil::face2 ||
      s.gradient_fit != GradientFit::linear)
    return nullptr;
  return std::make_unique<B200Stepper<P>>(mesh, geometry, host, gamma, gas_constant,
                                          second_order, stream);
}

template std::unique_ptr<DeviceStepper<kernels::fp64>> make_b200_stepper(
    const Mesh&, const Geometry&, const Euler<kernels::fp64>&, double, double, bool,
    runtime::Ranks&, void*, const kernels::GlobalKeys*);
template std::unique_ptr<DeviceStepper<kernels::fp32_acc64>> make_b200_stepper(
    const Mesh&, const Geometry&, const Euler<kernels::fp32_acc64>&, double, double, bool,
    runtime::Ranks&, void*, const kernels::GlobalKeys*);

}  // namespace autan::physics
