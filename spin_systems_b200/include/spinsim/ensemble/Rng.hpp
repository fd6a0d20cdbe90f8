// Per-realisation random streams (reference: include/spinsim/ensemble/Rng.hpp:25-58).
#pragma once

#include <cstddef>
#include <cstdint>
#include <random>

namespace spinsim {

class Rng {
 public:
  explicit Rng(std::uint64_t seed) : engine_(mix(seed)) {}
  [[nodiscard]] static Rng forRealization(std::uint64_t baseSeed, std::size_t index) {
    return Rng(mix(baseSeed ^ (mix(index + 1) * 0x9E3779B97F4A7C15ULL)));
  }
  [[nodiscard]] double uniform() { return static_cast<double>(engine_() >> 11) * 0x1.0p-53; }
  [[nodiscard]] double gaussian();

 private:
  [[nodiscard]] static std::uint64_t mix(std::uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  std::mt19937_64 engine_;
  double spare_ = 0.0;
  bool hasSpare_ = false;
};

}  // namespace spinsim
