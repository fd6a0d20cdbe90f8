// Host-side FP64 numerics of the echo path: the realisation random streams,
// dipolar geometry and disorder, initial states, Bessel sequences and the
// Chebyshev order rule.  These must agree bit for bit with the reference
// (BekturMur/Spin_Systems) so that geometries, fields and expansion orders
// match; they run on the host because glibc's log/sin/cos are part of that
// contract (src/ensemble/Rng.cpp:8-23).
#pragma once

#include <cstddef>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "../../include/spinsim_b200.h"

namespace ss {

// One realisation's random source (ensemble/Rng.hpp:25-58).
class Stream {
 public:
  explicit Stream(uint64_t seed) : engine_(finalize(seed)) {}
  static Stream for_realization(uint64_t base, uint64_t index) {
    return Stream(finalize(base ^ (finalize(index + 1) * 0x9E3779B97F4A7C15ULL)));
  }
  double uniform() { return static_cast<double>(engine_() >> 11) * 0x1.0p-53; }
  double gaussian();

 private:
  static uint64_t finalize(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  std::mt19937_64 engine_;
  double spare_ = 0.0;
  bool has_spare_ = false;
};

struct PairTerm {
  int lo = 0, hi = 0;
  double jx = 0.0, jy = 0.0, jz = 0.0;
};

// generateDipolarLattice2D (src/ensemble/Ensemble.cpp:60-104).
std::vector<PairTerm> dipolar_lattice_2d(int nspins, Stream& rng, double scale,
                                         double min_separation = 5.0e-2);

// Per-realisation draws of the additive keys (L, sigma, tau) from the
// harness stream (draw_seed, index); defaults when the keys are off.
struct Draws {
  int nspins;
  double sigma;
  double tau;
};
Draws realization_draws(const ss_run_config& cfg, uint64_t index);

// The assembled realisation (io/Experiment.cpp:10-35).
struct Realization {
  int nspins = 0;
  double tau_draw = 1.0;
  std::vector<double> fields;  // 3L
  std::vector<PairTerm> pairs;
  std::vector<double> psi0;    // 2 * 2^L, interleaved
};
Realization assemble_realization(const ss_run_config& cfg, uint64_t index);

// Bessel J (kind 0) or I (kind 1), orders 0..count-1 (src/core/Bessel.cpp).
std::vector<double> bessel(int kind, double x, size_t count, size_t* nonzero);

// The Chebyshev expansion of one step (src/core/Chebyshev.cpp:54-107).
struct Expansion {
  std::vector<double> a;  // a_0 .. a_order
  double bound = 1.0;     // effective bound
  size_t order() const { return a.empty() ? 0 : a.size() - 1; }
};
Expansion chebyshev(int mode, double spectral_bound, double tau, double epsilon,
                    size_t max_order = 6000);

// Sum of term norms (src/core/Hamiltonian.cpp:82-93).
double spectral_bound(int nspins, const double* fields, const std::vector<PairTerm>& pairs);

// Series weights c_n = 2 a_n w_n (and c_0 = a_0), w_n = (-i)^n or (-1)^n
// (src/core/Propagator.cpp:14-35, 58-72), as (re, im) pairs.
std::vector<double> series_weights(const Expansion& e, int mode);

// Measurement points of a pre-order program and values per point.
int64_t measurement_count(const ss_step* steps, int begin, int end);
int64_t observable_width(const ss_observable* obs, int n);

}  // namespace ss
