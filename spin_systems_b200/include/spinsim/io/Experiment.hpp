// Experiments (reference: include/spinsim/io/Experiment.hpp:11-31).
#pragma once

#include <filesystem>
#include <iosfwd>

#include "spinsim/ensemble/EnsembleRunner.hpp"
#include "spinsim/io/Config.hpp"
#include "spinsim_b200.h"

namespace spinsim {

/// One realisation on the device through the reference's call structure
/// (Sequence::run with one Propagator::evolve per step and vector).
void runRealization(const RunConfig& config, std::size_t index, VectorRecorder& out);

/// The ensemble through `runner` (the plain FP64 path per realisation).
[[nodiscard]] EnsembleResult runExperiment(const RunConfig& config, EnsembleRunner& runner);

/// The ensemble through the batched engine in one persistent launch per size
/// (precision SS_PRECISION_FP64 or SS_PRECISION_MIXED).
[[nodiscard]] EnsembleResult runExperimentBatched(const RunConfig& config, int precision);

/// The C view of a RunConfig; `storage` keeps the arrays it points into.
struct ConfigView {
  ss_run_config config{};
  std::vector<double> baseFields;
  std::vector<ss_step> steps;
  std::vector<double> stepFields;
  std::vector<ss_observable> observables;
};
void toConfigView(const RunConfig& config, ConfigView& view);

void writeCsv(const EnsembleResult& result, std::ostream& out);
void writeCsv(const EnsembleResult& result, const std::filesystem::path& path);

}  // namespace spinsim
