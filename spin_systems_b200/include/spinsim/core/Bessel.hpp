// Bessel sequences J_n, I_n (reference: include/spinsim/core/Bessel.hpp:9-45).
#pragma once

#include <cstddef>
#include <vector>

namespace spinsim {

struct BesselSequence {
  std::vector<double> values;
  std::size_t nonzero = 0;
};

[[nodiscard]] BesselSequence besselJ(double x, std::size_t count);
[[nodiscard]] BesselSequence besselI(double x, std::size_t count);

}  // namespace spinsim
