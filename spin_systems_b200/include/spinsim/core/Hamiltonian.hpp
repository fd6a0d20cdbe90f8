// H = sum_i h_i . S_i + sum_<ij> (Jx SxSx + Jy SySy + Jz SzSz), S = sigma/2
// (reference: include/spinsim/core/Hamiltonian.hpp:12-110).  Terms are kept on
// the host; a device copy (ss_ham) is refreshed lazily when they change.
#pragma once

#include <vector>

#include "spinsim/core/Bits.hpp"
#include "spinsim/core/StateVector.hpp"
#include "spinsim_b200.h"

namespace spinsim {

struct Field {
  double x = 0.0;
  double y = 0.0;
  double z = 0.0;
};

struct Coupling {
  SpinPair pair;
  double jx = 0.0;
  double jy = 0.0;
  double jz = 0.0;
};

class Hamiltonian {
 public:
  explicit Hamiltonian(std::size_t nspins);
  Hamiltonian(const Hamiltonian& other);
  Hamiltonian& operator=(const Hamiltonian& other);
  ~Hamiltonian();

  [[nodiscard]] std::size_t nspins() const noexcept { return nspins_; }
  void setField(SpinIndex spin, Field field);
  [[nodiscard]] const Field& field(SpinIndex spin) const;
  void setCoupling(SpinPair pair, double jx, double jy, double jz);
  [[nodiscard]] const std::vector<Coupling>& couplings() const noexcept { return couplings_; }
  [[nodiscard]] const std::vector<Field>& fields() const noexcept { return fields_; }
  [[nodiscard]] double spectralBound() const noexcept;

  void applyPhysical(const StateVector& in, StateVector& out) const;
  void applyTwiceNormalized(double bound, const StateVector& in, StateVector& out) const;
  void accumulateTwiceNormalized(double bound, const StateVector& in, StateVector& out) const;

  /// The device Hamiltonian, refreshed if the terms changed.
  [[nodiscard]] ss_ham* device() const;

 private:
  std::size_t nspins_;
  std::vector<Field> fields_;
  std::vector<Coupling> couplings_;
  mutable ss_ham* dev_ = nullptr;
  mutable bool dirty_ = true;
};

}  // namespace spinsim
