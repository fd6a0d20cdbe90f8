// Realisation assembly and statistics (reference: include/spinsim/ensemble/Ensemble.hpp:14-96).
#pragma once

#include <cstddef>
#include <span>
#include <string_view>
#include <vector>

#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/Observable.hpp"
#include "spinsim/core/StateVector.hpp"
#include "spinsim/ensemble/Rng.hpp"

namespace spinsim {

enum class InitialStateKind { Random, AllUp, AllDown, BasisState, RandomProduct };

[[nodiscard]] InitialStateKind parseInitialStateKind(std::string_view name);
void prepareInitialState(StateVector& psi, InitialStateKind kind, Rng& rng,
                         std::size_t basisIndex = 0);
void prepareReferenceState(const StateVector& psi, Axis axis, StateVector& reference);
[[nodiscard]] std::vector<Coupling> generateDipolarLattice2D(std::size_t nspins, Rng& rng,
                                                             double scale = 1.0,
                                                             double minSeparation = 5.0e-2);
void applyFieldDisorder(Hamiltonian& hamiltonian, Rng& rng, double sigma);

class Accumulator {
 public:
  explicit Accumulator(std::size_t width);
  void add(std::span<const double> sample);
  void merge(const Accumulator& other);
  [[nodiscard]] std::size_t count() const noexcept { return count_; }
  [[nodiscard]] std::size_t width() const noexcept { return mean_.size(); }
  [[nodiscard]] const std::vector<double>& mean() const noexcept { return mean_; }
  [[nodiscard]] std::vector<double> standardDeviation() const;
  [[nodiscard]] std::vector<double> standardError() const;

 private:
  std::size_t count_ = 0;
  std::vector<double> mean_;
  std::vector<double> m2_;
};

}  // namespace spinsim
