// Chebyshev propagation on the device (reference: include/spinsim/core/Propagator.hpp:21-55).
#pragma once

#include <cstddef>

#include "spinsim/core/Chebyshev.hpp"
#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

class Propagator {
 public:
  explicit Propagator(std::size_t nspins, double epsilon = 1.0e-7);
  void evolve(const Hamiltonian& hamiltonian, TimeMode mode, StateVector& psi, double tau,
              std::size_t nsteps, bool autonormalize = false);
  [[nodiscard]] std::size_t lastOrder() const noexcept { return lastOrder_; }
  [[nodiscard]] double epsilon() const noexcept { return epsilon_; }

 private:
  std::size_t nspins_;
  double epsilon_;
  std::size_t lastOrder_ = 0;
};

}  // namespace spinsim
