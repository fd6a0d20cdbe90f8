// Ideal pulses (reference: include/spinsim/core/Gate.hpp:15-93).
#pragma once

#include <array>
#include <complex>
#include <string_view>
#include <vector>

#include "spinsim/core/Bits.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

struct Axis3 {
  double x = 0.0;
  double y = 0.0;
  double z = 1.0;
  [[nodiscard]] Axis3 normalized() const;
};

class SpinRotation {
 public:
  SpinRotation(Axis3 axis, double angle, std::vector<SpinIndex> targets);
  static SpinRotation onAllSpins(Axis3 axis, double angle, std::size_t nspins);
  void apply(StateVector& psi) const;
  [[nodiscard]] const std::vector<SpinIndex>& targets() const noexcept { return targets_; }
  [[nodiscard]] double angle() const noexcept { return angle_; }
  [[nodiscard]] Axis3 axis() const noexcept { return axis_; }

 private:
  Axis3 axis_;
  double angle_;
  std::vector<SpinIndex> targets_;
};

class TwoSpinGate {
 public:
  using Matrix = std::array<std::complex<double>, 16>;
  TwoSpinGate(Matrix matrix, SpinPair pair);
  void apply(StateVector& psi) const;
  [[nodiscard]] double unitarityDefect() const;

 private:
  Matrix matrix_;
  SpinPair pair_;
};

[[nodiscard]] SpinRotation makeRotation(std::string_view spec, std::size_t nspins);

}  // namespace spinsim
