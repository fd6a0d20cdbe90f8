// Ensemble averaging (reference: include/spinsim/ensemble/EnsembleRunner.hpp:16-82).
#pragma once

#include <cstddef>
#include <functional>
#include <span>
#include <string>
#include <vector>

#include "spinsim/ensemble/Ensemble.hpp"
#include "spinsim/sequence/Sequence.hpp"

namespace spinsim {

class VectorRecorder final : public Recorder {
 public:
  void record(double time, std::span<const double> values) override;
  [[nodiscard]] const std::vector<double>& times() const noexcept { return times_; }
  [[nodiscard]] const std::vector<double>& values() const noexcept { return values_; }
  [[nodiscard]] std::size_t rows() const noexcept { return times_.size(); }
  void clear();

 private:
  std::vector<double> times_;
  std::vector<double> values_;
};

struct EnsembleResult {
  std::vector<double> times;
  std::vector<std::string> columns;
  Accumulator statistics{0};
};

using RealizationJob = std::function<void(std::size_t index, VectorRecorder&)>;

class EnsembleRunner {
 public:
  virtual ~EnsembleRunner() = default;
  virtual EnsembleResult run(std::size_t realizations, std::span<const std::string> columns,
                             const RealizationJob& job) = 0;
};

/// Runs realisations over host threads, each thread with its own engine and
/// stream on the GPU; folds rows in index order (bitwise thread-count
/// independent, as the reference's LocalRunner).
class LocalRunner final : public EnsembleRunner {
 public:
  explicit LocalRunner(std::size_t threads = 0);
  EnsembleResult run(std::size_t realizations, std::span<const std::string> columns,
                     const RealizationJob& job) override;
  [[nodiscard]] std::size_t threads() const noexcept { return threads_; }

 private:
  std::size_t threads_;
};

/// Folds rows (realisations x points x width) in index order.
EnsembleResult foldRows(std::size_t realizations, const std::vector<double>& times,
                        std::span<const std::string> columns, const std::vector<double>& rows);

}  // namespace spinsim
