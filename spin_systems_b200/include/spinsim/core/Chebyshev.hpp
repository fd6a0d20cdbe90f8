// Chebyshev expansion of one step (reference: include/spinsim/core/Chebyshev.hpp:11-89).
#pragma once

#include <cstddef>
#include <span>
#include <stdexcept>
#include <vector>

namespace spinsim {

enum class TimeMode { Real, Imaginary };

class ChebyshevConvergenceError : public std::runtime_error {
 public:
  ChebyshevConvergenceError(double spectralBound, double tau, double epsilon,
                            std::size_t attemptedOrder);
  ChebyshevConvergenceError(const char* message, double spectralBound, double tau,
                            double epsilon, std::size_t attemptedOrder);
  [[nodiscard]] double spectralBound() const noexcept { return bound_; }
  [[nodiscard]] double tau() const noexcept { return tau_; }
  [[nodiscard]] double epsilon() const noexcept { return epsilon_; }
  [[nodiscard]] std::size_t attemptedOrder() const noexcept { return order_; }

 private:
  double bound_, tau_, epsilon_;
  std::size_t order_;
};

class ChebyshevExpansion {
 public:
  static ChebyshevExpansion build(TimeMode mode, double spectralBound, double tau,
                                  double epsilon, std::size_t maxOrder = 6000);
  [[nodiscard]] std::size_t order() const noexcept {
    return coefficients_.empty() ? 0 : coefficients_.size() - 1;
  }
  [[nodiscard]] std::span<const double> coefficients() const noexcept { return coefficients_; }
  [[nodiscard]] double effectiveBound() const noexcept { return bound_; }
  [[nodiscard]] bool isIdentity() const noexcept { return order() == 0; }

 private:
  std::vector<double> coefficients_;
  double bound_ = 1.0;
};

}  // namespace spinsim
