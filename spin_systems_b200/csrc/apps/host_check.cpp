// The engine's host layer under AddressSanitizer and UndefinedBehaviorSanitizer,
// with no GPU: the TOML reader and config validation on every file named on
// the command line, then the realisation assembly (random streams, dipolar
// placement, field disorder, initial states), the Bessel sequences and the
// Chebyshev expansions over a range of sizes and arguments.
//
//   host_check [--expect-errors] config.toml ...
//   host_check --csv rows.txt
//
// Every file must load and validate, or with --expect-errors every file must
// be rejected with a ConfigError (malformed input).  Prints one summary line
// and exits 0; a sanitizer finding aborts the process with its own report.
//
// With --csv the checker instead folds measurement rows through the C++ API's
// Accumulator in index order and prints writeCsv's output.  rows.txt holds
// "points columns realisations", the column names, the times, then one line
// of points x columns values per realisation (decimal, round-tripping every
// double).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../host_numerics.hpp"
#include "spinsim/io/Config.hpp"
#include "spinsim/io/Experiment.hpp"

namespace {

int checkConfigs(const std::vector<std::string>& paths, bool expectErrors) {
  int failures = 0;
  for (const std::string& p : paths) {
    bool rejected = false;
    try {
      spinsim::RunConfig c = spinsim::loadConfig(p);
      c.validate(p);
    } catch (const spinsim::ConfigError& e) {
      rejected = true;
      if (!expectErrors) std::fprintf(stderr, "%s: unexpected ConfigError: %s\n", p.c_str(), e.what());
    } catch (const std::exception& e) {
      std::fprintf(stderr, "%s: unexpected exception: %s\n", p.c_str(), e.what());
      ++failures;
      continue;
    }
    if (rejected != expectErrors) ++failures;
  }
  return failures;
}

int rejected_steps = 0;

// Assembles realisations of every size with disorder, initial states and the
// harness draws switched on, and expands their steps.
int checkNumerics() {
  int failures = 0;
  for (int L = 2; L <= 16; ++L) {
    std::vector<double> base(3 * static_cast<size_t>(L), 0.0);
    for (int s = 0; s < L; ++s) base[3 * s + 2] = 0.1 * s;
    for (int kind = 0; kind < 5; ++kind) {
      ss_run_config c{};
      c.nspins = L;
      c.initial_state = kind;
      c.basis_index = (1ull << L) - 1;
      c.realizations = 4;
      c.seed = 20240726u + static_cast<uint64_t>(L);
      c.generate_geometry = 1;
      c.reference_axis = kind % 3;
      c.dipolar_scale = 1.0;
      c.field_disorder = 0.5;
      c.epsilon = 1e-7;
      c.base_fields = base.data();
      c.draw_seed = 7;
      c.disorder_range[0] = 0.1;
      c.disorder_range[1] = 1.0;
      c.tau_range[0] = 0.1;
      c.tau_range[1] = 1.0;
      for (uint64_t i = 0; i < 4; ++i) {
        const ss::Realization r = ss::assemble_realization(c, i);
        if (r.nspins != L || r.fields.size() != 3u * L ||
            r.psi0.size() != (2ull << L) ||
            r.pairs.size() != static_cast<size_t>(L) * (L - 1) / 2) {
          ++failures;
          continue;
        }
        const double bound = ss::spectral_bound(L, r.fields.data(), r.pairs);
        for (double tau : {1e-3, 0.05, 0.5, 2.0}) {
          for (int mode = 0; mode < 2; ++mode) {
            try {
              const ss::Expansion e = ss::chebyshev(mode, bound, tau, c.epsilon);
              const std::vector<double> w = ss::series_weights(e, mode);
              if (w.size() != 2 * (e.order() + 1) || !std::isfinite(w[0])) ++failures;
            } catch (const std::exception&) {
              // a rejected step (the unscaled I_n overflows in imaginary
              // time at large bound * tau; an over-long expansion), as the
              // reference rejects it
              ++rejected_steps;
            }
          }
        }
      }
    }
  }
  for (int kind = 0; kind < 2; ++kind) {
    for (double x : {0.0, 1e-300, 1e-8, 0.5, 7.0, 123.4, 4096.0}) {
      try {
        size_t nz = 0;
        const std::vector<double> v = ss::bessel(kind, x, 64, &nz);
        if (v.size() != 64 || nz > v.size()) ++failures;
      } catch (const std::exception&) {
        ++rejected_steps;  // the reference rejects the same arguments (1e-300; I_n at 4096)
      }
    }
  }
  return failures;
}

// Rows -> Accumulator (index order) -> writeCsv on standard output.
int foldRows(const char* path) {
  std::ifstream in(path);
  std::size_t points = 0, ncols = 0, count = 0;
  if (!(in >> points >> ncols >> count) || points == 0 || ncols == 0 || count == 0) {
    std::fprintf(stderr, "%s: bad header\n", path);
    return 1;
  }
  spinsim::EnsembleResult result;
  result.columns.resize(ncols);
  for (std::string& c : result.columns) in >> c;
  result.times.resize(points);
  for (double& t : result.times) in >> t;
  result.statistics = spinsim::Accumulator(points * ncols);
  std::vector<double> row(points * ncols);
  for (std::size_t r = 0; r < count; ++r) {
    for (double& v : row) in >> v;
    if (!in) {
      std::fprintf(stderr, "%s: short row %zu\n", path, r);
      return 1;
    }
    result.statistics.add(row);
  }
  spinsim::writeCsv(result, std::cout);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 3 && std::strcmp(argv[1], "--csv") == 0) return foldRows(argv[2]);
  bool expectErrors = false;
  std::vector<std::string> paths;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--expect-errors") == 0) {
      expectErrors = true;
    } else {
      paths.emplace_back(argv[i]);
    }
  }
  const int bad = checkConfigs(paths, expectErrors) + checkNumerics();
  std::printf("host_check: %zu config(s)%s, numerics over L = 2..16 (%d steps rejected): "
              "%d failure(s)\n",
              paths.size(), expectErrors ? " rejected as expected" : " loaded", rejected_steps, bad);
  return bad == 0 ? 0 : 1;
}
