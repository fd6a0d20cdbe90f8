// Pulse programs (reference: include/spinsim/sequence/Sequence.hpp:17-104).
#pragma once

#include <cstddef>
#include <memory>
#include <span>
#include <string>
#include <variant>
#include <vector>

#include "spinsim/core/Chebyshev.hpp"
#include "spinsim/core/Gate.hpp"
#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/Observable.hpp"
#include "spinsim/core/Propagator.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

struct Evolve {
  double tau = 0.0;
  std::size_t nsteps = 1;
  TimeMode mode = TimeMode::Real;
  bool autonormalize = false;
  std::vector<Field> fields;
  /// Additive: use the realisation's drawn tau times `tau` (0/1).
  bool tauFromDraw = false;
};

struct Pulse {
  SpinRotation rotation;
};

struct Measure {};

struct Repeat;

using Step = std::variant<Evolve, Pulse, Measure, Repeat>;

struct Repeat {
  std::size_t count = 1;
  std::vector<Step> body;
};

class Recorder {
 public:
  virtual ~Recorder() = default;
  virtual void record(double time, std::span<const double> values) = 0;
};

struct RunContext {
  Hamiltonian* hamiltonian = nullptr;
  StateVector* state = nullptr;
  StateVector* reference = nullptr;
  Propagator* propagator = nullptr;
  std::span<const std::unique_ptr<Observable>> observables;
  Recorder* recorder = nullptr;
  std::size_t subsystemSize = 0;
  double time = 0.0;
  double tauDraw = 1.0;  ///< additive: the realisation's drawn tau
};

class Sequence {
 public:
  explicit Sequence(std::vector<Step> steps) : steps_(std::move(steps)) {}
  [[nodiscard]] const std::vector<Step>& steps() const noexcept { return steps_; }
  void run(RunContext& ctx) const;
  [[nodiscard]] std::size_t measurementCount() const;

 private:
  std::vector<Step> steps_;
};

[[nodiscard]] std::vector<std::string> resultColumns(
    std::span<const std::unique_ptr<Observable>> observables);

}  // namespace spinsim
