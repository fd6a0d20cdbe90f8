// Spin indices and masks (reference: include/spinsim/core/Bits.hpp:13-55).
#pragma once

#include <cassert>
#include <cstddef>
#include <cstdint>

namespace spinsim {

/// Largest supported number of spins (a sanity bound, not an allocation).
inline constexpr std::size_t kMaxSpins = 30;

/// Spin s owns bit s of a basis index; a set bit means "up".
using SpinIndex = std::size_t;

[[nodiscard]] constexpr std::uint64_t spinMask(SpinIndex spin) noexcept {
  return std::uint64_t{1} << spin;
}

[[nodiscard]] constexpr std::size_t stateCount(std::size_t nspins) noexcept {
  return std::size_t{1} << nspins;
}

/// An unordered pair of distinct spins, stored with low < high.
class SpinPair {
 public:
  constexpr SpinPair(SpinIndex a, SpinIndex b) noexcept
      : low_(a < b ? a : b), high_(a < b ? b : a) {
    assert(a != b && "a spin cannot couple to itself");
  }
  [[nodiscard]] constexpr SpinIndex low() const noexcept { return low_; }
  [[nodiscard]] constexpr SpinIndex high() const noexcept { return high_; }
  friend constexpr bool operator==(SpinPair, SpinPair) noexcept = default;

 private:
  SpinIndex low_;
  SpinIndex high_;
};

}  // namespace spinsim
