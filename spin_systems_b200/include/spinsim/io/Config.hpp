// TOML configuration (reference: include/spinsim/io/Config.hpp:14-65), parsed
// by the project's own TOML reader; additive keys are documented in
// docs of RunConfig below and default to the reference's behaviour.
#pragma once

#include <cstdint>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "spinsim/ensemble/Ensemble.hpp"
#include "spinsim/sequence/Sequence.hpp"

namespace spinsim {

class ConfigError : public std::runtime_error {
 public:
  ConfigError(std::string_view file, std::string_view key, std::string_view problem);
};

struct RunConfig {
  std::size_t nspins = 0;
  std::vector<Field> baseFields;
  InitialStateKind initialState = InitialStateKind::Random;
  std::size_t basisIndex = 0;
  std::size_t realizations = 1;
  std::uint64_t seed = 0;
  bool generateGeometry = true;
  double dipolarScale = 1.0;
  double fieldDisorder = 0.0;
  Axis referenceAxis = Axis::Z;
  std::vector<std::string> observables;
  double epsilon = 1.0e-7;
  Sequence sequence{{}};
  // additive keys ([ensemble] draw_seed, disorder_range, tau_range, spin_choices)
  std::uint64_t drawSeed = 0;
  double disorderRange[2] = {0.0, 0.0};
  double tauRange[2] = {0.0, 0.0};
  std::vector<int> spinChoices;

  void validate(std::string_view origin = "<config>") const;
};

[[nodiscard]] RunConfig loadConfig(const std::filesystem::path& path);
[[nodiscard]] RunConfig parseConfig(std::string_view text, std::string_view origin);

}  // namespace spinsim
