// Measurement registry (reference: include/spinsim/core/Observable.hpp:12-134).
#pragma once

#include <memory>
#include <span>
#include <string>
#include <string_view>
#include <vector>

#include "spinsim/core/Bits.hpp"
#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

enum class Axis { X, Y, Z };
[[nodiscard]] Axis parseAxis(std::string_view name);
[[nodiscard]] std::string_view axisName(Axis axis);

struct MeasureContext {
  double time = 0.0;
  const StateVector* state = nullptr;
  const StateVector* reference = nullptr;
  const Hamiltonian* hamiltonian = nullptr;
  std::size_t subsystemSize = 0;
};

class Observable {
 public:
  virtual ~Observable() = default;
  [[nodiscard]] virtual std::string name() const = 0;
  [[nodiscard]] virtual std::vector<std::string> columns() const = 0;
  virtual void measure(const MeasureContext& ctx, std::span<double> out) const = 0;
  [[nodiscard]] std::size_t width() const { return columns().size(); }
};

class TotalSpinCorrelator final : public Observable {
 public:
  explicit TotalSpinCorrelator(Axis axis) : axis_(axis) {}
  [[nodiscard]] std::string name() const override;
  [[nodiscard]] std::vector<std::string> columns() const override;
  void measure(const MeasureContext& ctx, std::span<double> out) const override;
  [[nodiscard]] Axis axis() const noexcept { return axis_; }

 private:
  Axis axis_;
};

class SingleSpinMagnetization final : public Observable {
 public:
  SingleSpinMagnetization(SpinIndex spin, Axis axis) : spin_(spin), axis_(axis) {}
  [[nodiscard]] std::string name() const override;
  [[nodiscard]] std::vector<std::string> columns() const override;
  void measure(const MeasureContext& ctx, std::span<double> out) const override;
  [[nodiscard]] SpinIndex spin() const noexcept { return spin_; }
  [[nodiscard]] Axis axis() const noexcept { return axis_; }

 private:
  SpinIndex spin_;
  Axis axis_;
};

class StateNorms final : public Observable {
 public:
  [[nodiscard]] std::string name() const override { return "norm"; }
  [[nodiscard]] std::vector<std::string> columns() const override;
  void measure(const MeasureContext& ctx, std::span<double> out) const override;
};

class Energy final : public Observable {
 public:
  [[nodiscard]] std::string name() const override { return "energy"; }
  [[nodiscard]] std::vector<std::string> columns() const override;
  void measure(const MeasureContext& ctx, std::span<double> out) const override;
};

[[nodiscard]] std::unique_ptr<Observable> makeObservable(std::string_view spec);

}  // namespace spinsim
