// The convergence decision of a steady run, host side: runtime/src/run.cpp:2351-2389 with the
// round-off exemption and plateau of runtime/include/autan/runtime/round_off.hpp.
//
// Fed one iteration's residual RMS at a time (equations: mass, momentum x, y, z, energy), it
// reports converged once every equation has either dropped `orders` decades below its reference
// or, when floors are given (fp32+acc64 steady runs, run.cpp:1874-1897), sits on a round-off
// plateau at most 10 floors high. References (RoundOffExemption): the first iteration's residuals;
// a momentum component drops from the largest first momentum residual; an equation below 1e-12
// of the largest first residual is exempt while it stays at or below that floor and, once above,
// drops from its woken reference. A residual's plateau (ResidualPlateau): the median of its last
// 100 values has not fallen below 0.9 of its reference for 100 values.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <limits>

namespace autan_b200 {

class Convergence {
 public:
  static constexpr int kEquations = 5;
  static constexpr std::size_t kWindow = 100;  // plateau_window
  static constexpr std::size_t kSteps = 100;   // plateau_steps
  static constexpr double kRatio = 0.9;        // plateau_ratio
  static constexpr double kBand = 10.0;        // round_off_band

  // floors: round_off_floor * Phi_k per equation, or nullptr for no plateau rule. reference: the
  // residuals the drops are taken from (a continued run's `start.residual_reference`,
  // run.cpp:2351-2356), or nullptr for the first iteration's.
  Convergence(double orders, const double* floors, const double* reference = nullptr)
      : drop_(std::pow(10.0, -orders)) {
    if (floors != nullptr) {
      use_floor_ = true;
      for (int e = 0; e < kEquations; ++e) floor_[e] = floors[e];
    }
    if (reference != nullptr) set_first(reference);
  }

  // This iteration's residuals; true once converged. plateau_mask(): the equations that
  // converged on a plateau rather than by their drop.
  bool add(const double* r) {
    if (!have_first_) set_first(r);
    for (int e = 0; e < kEquations; ++e)
      if (exempt_[e] && r[e] > zero_floor_) exempt_[e] = false;
    bool converged = true;
    int mask = 0;
    for (int e = 0; e < kEquations; ++e) {
      const bool flat = plateau_[e].add(r[e]);
      const bool woken = zero_[e] && !exempt_[e];
      const double ref = woken ? woken_reference(e) : drop_reference(e);
      const bool met = exempt_[e] || r[e] <= ref * drop_;
      const bool plateau = use_floor_ && flat && r[e] <= kBand * floor_[e];
      if (!met && plateau) mask |= 1 << e;
      converged = converged && (met || plateau);
    }
    if (converged) mask_ = mask;
    return converged;
  }

  int plateau_mask() const { return mask_; }

  void set_first(const double* r) {
    have_first_ = true;
    for (int e = 0; e < kEquations; ++e) first_[e] = r[e];
    zero_floor_ = 1e-12 * *std::max_element(first_.begin(), first_.end());
    for (int e = 0; e < kEquations; ++e) {
      zero_[e] = first_[e] < zero_floor_;
      exempt_[e] = zero_[e];
    }
  }
  const std::array<double, kEquations>& first() const { return first_; }

 private:
  static bool momentum(int e) { return e >= 1 && e <= 3; }
  double drop_reference(int e) const {
    if (!momentum(e)) return first_[e];
    return std::max(std::max(first_[1], first_[2]), first_[3]);
  }
  double woken_reference(int e) const {
    if (momentum(e)) return drop_reference(e);
    return *std::max_element(first_.begin(), first_.end());
  }

  // The median of the last kWindow values kept by a window in arrival order and the same values
  // sorted (one removal and one insertion per value): the level (sorted[49] + sorted[50]) / 2 is
  // the one the reference takes from nth_element on a copy of the window.
  struct Plateau {
    std::array<double, kWindow> window{}, sorted{};
    double reference = std::numeric_limits<double>::infinity();
    std::size_t count = 0, since = 0;
    bool add(double value) {
      std::size_t filled = std::min(count, kWindow);
      double* const s = sorted.data();
      if (count >= kWindow) {
        double* at = std::lower_bound(s, s + filled, window[count % kWindow]);
        if (at == s + filled) at = s + filled - 1;  // not found (a NaN left the window)
        std::move(at + 1, s + filled, at);
        --filled;
      }
      window[count % kWindow] = value;
      double* const pos = std::upper_bound(s, s + filled, value);
      std::move_backward(pos, s + filled, s + filled + 1);
      *pos = value;
      ++count;
      if (count >= kWindow) {
        const double level = (s[kWindow / 2 - 1] + s[kWindow / 2]) / 2;
        if (level < kRatio * reference) {
          reference = level;
          since = count;
        }
      }
      return since > 0 && count - since >= kSteps;
    }
  };

  double drop_;
  bool use_floor_ = false, have_first_ = false;
  std::array<double, kEquations> floor_{}, first_{};
  std::array<bool, kEquations> zero_{}, exempt_{};
  double zero_floor_ = 0.0;
  std::array<Plateau, kEquations> plateau_{};
  int mask_ = 0;
};

}  // namespace autan_b200
