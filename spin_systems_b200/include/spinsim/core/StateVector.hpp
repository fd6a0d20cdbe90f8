// A many-spin pure state (reference: include/spinsim/core/StateVector.hpp:82-140).
//
// The amplitudes live in device memory (ss_state); a host mirror serves the
// element accessors.  Whichever side was written last is authoritative, and
// the other is brought up to date on first use, so code written against the
// reference's StateVector keeps working while every operation runs on the GPU.
#pragma once

#include <cstddef>
#include <span>
#include <utility>
#include <vector>

#include "spinsim/core/Bits.hpp"
#include "spinsim_b200.h"

namespace spinsim {

class StateVector {
 public:
  StateVector() = default;
  explicit StateVector(std::size_t nspins);
  StateVector(const StateVector& other);
  StateVector& operator=(const StateVector& other);
  StateVector(StateVector&& other) noexcept;
  StateVector& operator=(StateVector&& other) noexcept;
  ~StateVector();

  [[nodiscard]] std::size_t nspins() const noexcept { return nspins_; }
  [[nodiscard]] std::size_t size() const noexcept { return nspins_ ? stateCount(nspins_) : 0; }

  /// Interleaved re/im host view, 2 * size() doubles.
  [[nodiscard]] double* data();
  [[nodiscard]] const double* data() const;
  [[nodiscard]] std::span<double> amplitudes() { return {data(), 2 * size()}; }
  [[nodiscard]] std::span<const double> amplitudes() const { return {data(), 2 * size()}; }

  [[nodiscard]] double& re(std::size_t k) { return data()[2 * k]; }
  [[nodiscard]] double& im(std::size_t k) { return data()[2 * k + 1]; }
  [[nodiscard]] double re(std::size_t k) const { return data()[2 * k]; }
  [[nodiscard]] double im(std::size_t k) const { return data()[2 * k + 1]; }

  void setZero();
  void scale(double factor);
  void negate();
  void addScaled(double cr, double ci, const StateVector& other);
  void setBasisState(std::size_t index);
  [[nodiscard]] double norm() const;
  double normalize();
  [[nodiscard]] std::pair<double, double> innerProduct(const StateVector& other) const;
  void swap(StateVector& other) noexcept;

  /// The device state, brought up to date with any host writes.
  [[nodiscard]] ss_state* device() const;
  /// Marks the device copy as the authoritative one (after a kernel wrote it).
  void deviceWritten() const { where_ = Where::Device; }

 private:
  enum class Where { Both, Host, Device };
  std::size_t nspins_ = 0;
  mutable ss_state* dev_ = nullptr;
  mutable std::vector<double> host_;
  mutable Where where_ = Where::Both;
};

}  // namespace spinsim
