// Test infrastructure, not product code: a C-ABI shim over the reference
// spinsim library, compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/libspinsim_ref.so.  Only tests/, the smoke
// check and bench.py's CPU-baseline leg load it.
//
// Every function drives the reference through its public C++ API
// (include/spinsim/**); nothing here reimplements its numerics.

#include <cstring>
#include <exception>
#include <memory>
#include <numbers>
#include <span>
#include <string>
#include <thread>
#include <vector>
#include <atomic>
#include <chrono>
#include <mutex>
#include <random>
#include <sstream>

#include "spinsim/core/Bessel.hpp"
#include "spinsim/core/Chebyshev.hpp"
#include "spinsim/core/Gate.hpp"
#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/Observable.hpp"
#include "spinsim/core/Propagator.hpp"
#include "spinsim/core/SpinOperators.hpp"
#include "spinsim/ensemble/Ensemble.hpp"
#include "spinsim/ensemble/EnsembleRunner.hpp"
#include "spinsim/ensemble/Rng.hpp"
#include "spinsim/io/Experiment.hpp"

#include "../include/spinsim_b200.h"

using namespace spinsim;

namespace {

thread_local std::string g_error;

int fail(const std::exception& e, int code) {
  g_error = e.what();
  return code;
}

template <typename F>
int guarded(F&& body) {
  try {
    body();
    return 0;
  } catch (const ChebyshevConvergenceError& e) {
    return fail(e, SS_ERR_CONVERGENCE);
  } catch (const std::invalid_argument& e) {
    return fail(e, SS_ERR_INVALID_ARGUMENT);
  } catch (const std::out_of_range& e) {
    return fail(e, SS_ERR_OUT_OF_RANGE);
  } catch (const std::domain_error& e) {
    return fail(e, SS_ERR_DOMAIN);
  } catch (const std::overflow_error& e) {
    return fail(e, SS_ERR_OVERFLOW);
  } catch (const std::exception& e) {
    return fail(e, SS_ERR_RUNTIME);
  }
}

Hamiltonian makeHamiltonian(int nspins, const double* fields, int npairs,
                            const int32_t* pairs, const double* J) {
  Hamiltonian h(static_cast<std::size_t>(nspins));
  for (int s = 0; s < nspins; ++s) {
    h.setField(static_cast<SpinIndex>(s),
               Field{fields[3 * s], fields[3 * s + 1], fields[3 * s + 2]});
  }
  for (int p = 0; p < npairs; ++p) {
    h.setCoupling(SpinPair{static_cast<SpinIndex>(pairs[2 * p]),
                           static_cast<SpinIndex>(pairs[2 * p + 1])},
                  J[3 * p], J[3 * p + 1], J[3 * p + 2]);
  }
  return h;
}

StateVector makeState(int nspins, const double* data) {
  StateVector psi(static_cast<std::size_t>(nspins));
  std::memcpy(psi.data(), data, sizeof(double) * 2 * psi.size());
  return psi;
}

void storeState(const StateVector& psi, double* data) {
  std::memcpy(data, psi.data(), sizeof(double) * 2 * psi.size());
}

Axis toAxis(int a) {
  return a == SS_AXIS_X ? Axis::X : a == SS_AXIS_Y ? Axis::Y : Axis::Z;
}

std::string axisChar(int a) {
  return a == SS_AXIS_X ? "x" : a == SS_AXIS_Y ? "y" : "z";
}

// Rebuilds the reference's Step tree from the pre-order node array.
std::vector<Step> buildSteps(const ss_run_config& cfg, int begin, int end);

Step buildOne(const ss_run_config& cfg, int at, int* next) {
  const ss_step& n = cfg.steps[at];
  const auto nspins = static_cast<std::size_t>(cfg.nspins);
  switch (n.kind) {
    case SS_STEP_EVOLVE: {
      if (n.tau_from_draw) {
        throw std::invalid_argument("drawn tau is not expressible in the reference");
      }
      Evolve e;
      e.tau = n.tau;
      e.nsteps = static_cast<std::size_t>(n.count);
      e.mode = n.mode == SS_TIME_IMAGINARY ? TimeMode::Imaginary : TimeMode::Real;
      e.autonormalize = n.autonormalize != 0;
      if (n.field_table >= 0) {
        const double* t = cfg.step_fields + 3 * nspins * static_cast<std::size_t>(n.field_table);
        e.fields.resize(nspins);
        for (std::size_t s = 0; s < nspins; ++s) {
          e.fields[s] = Field{t[3 * s], t[3 * s + 1], t[3 * s + 2]};
        }
      }
      *next = at + 1;
      return e;
    }
    case SS_STEP_PULSE: {
      const Axis3 axis{n.axis[0], n.axis[1], n.axis[2]};
      *next = at + 1;
      if (n.target < 0) return Pulse{SpinRotation::onAllSpins(axis, n.angle, nspins)};
      return Pulse{SpinRotation(axis, n.angle, {static_cast<SpinIndex>(n.target)})};
    }
    case SS_STEP_MEASURE:
      *next = at + 1;
      return Measure{};
    case SS_STEP_REPEAT: {
      Repeat r;
      r.count = static_cast<std::size_t>(n.count);
      r.body = buildSteps(cfg, at + 1, at + 1 + n.body_len);
      *next = at + 1 + n.body_len;
      return r;
    }
    default:
      throw std::invalid_argument("unknown step kind");
  }
}

std::vector<Step> buildSteps(const ss_run_config& cfg, int begin, int end) {
  std::vector<Step> out;
  int at = begin;
  while (at < end) {
    int next = at;
    out.push_back(buildOne(cfg, at, &next));
    at = next;
  }
  return out;
}

std::string observableSpec(const ss_observable& o) {
  switch (o.kind) {
    case SS_OBS_CORR: return "corr:" + axisChar(o.axis);
    case SS_OBS_MAG: return "mag:" + std::to_string(o.spin + 1) + ":" + axisChar(o.axis);
    case SS_OBS_NORM: return "norm";
    case SS_OBS_ENERGY: return "energy";
    default: throw std::invalid_argument("unknown observable kind");
  }
}

RunConfig toRunConfig(const ss_run_config& c) {
  if (c.initial_state == SS_INIT_RANDOM_PRODUCT || c.n_spin_choices > 0 ||
      c.disorder_range[1] > c.disorder_range[0] || c.tau_range[1] > c.tau_range[0]) {
    throw std::invalid_argument("additive config keys are not expressible in the reference");
  }
  RunConfig cfg;
  cfg.nspins = static_cast<std::size_t>(c.nspins);
  cfg.baseFields.resize(cfg.nspins);
  for (std::size_t s = 0; s < cfg.nspins; ++s) {
    cfg.baseFields[s] = Field{c.base_fields[3 * s], c.base_fields[3 * s + 1],
                              c.base_fields[3 * s + 2]};
  }
  cfg.initialState = c.initial_state == SS_INIT_UP     ? InitialStateKind::AllUp
                     : c.initial_state == SS_INIT_DOWN ? InitialStateKind::AllDown
                     : c.initial_state == SS_INIT_BASIS ? InitialStateKind::BasisState
                                                        : InitialStateKind::Random;
  cfg.basisIndex = static_cast<std::size_t>(c.basis_index);
  cfg.realizations = static_cast<std::size_t>(c.realizations);
  cfg.seed = c.seed;
  cfg.generateGeometry = c.generate_geometry != 0;
  cfg.dipolarScale = c.dipolar_scale;
  cfg.fieldDisorder = c.field_disorder;
  cfg.referenceAxis = toAxis(c.reference_axis);
  for (int i = 0; i < c.n_observables; ++i) cfg.observables.push_back(observableSpec(c.observables[i]));
  cfg.epsilon = c.epsilon;
  cfg.sequence = Sequence(buildSteps(c, 0, c.n_steps));
  return cfg;
}

}  // namespace

extern "C" {

const char* refd_last_error(void) { return g_error.c_str(); }

int refd_bessel(int kind, double x, int64_t count, double* out, int64_t* nonzero) {
  return guarded([&] {
    const BesselSequence s = kind == 0 ? besselJ(x, static_cast<std::size_t>(count))
                                       : besselI(x, static_cast<std::size_t>(count));
    std::memcpy(out, s.values.data(), sizeof(double) * s.values.size());
    *nonzero = static_cast<int64_t>(s.nonzero);
  });
}

int refd_chebyshev(int mode, double bound, double tau, double eps, int64_t maxOrder,
                   double* coeffs, int64_t cap, int64_t* order, double* effBound) {
  return guarded([&] {
    const ChebyshevExpansion e = ChebyshevExpansion::build(
        mode == SS_TIME_IMAGINARY ? TimeMode::Imaginary : TimeMode::Real, bound, tau,
        eps, static_cast<std::size_t>(maxOrder));
    const auto a = e.coefficients();
    if (static_cast<int64_t>(a.size()) > cap) throw std::runtime_error("capacity");
    std::memcpy(coeffs, a.data(), sizeof(double) * a.size());
    *order = static_cast<int64_t>(e.order());
    *effBound = e.effectiveBound();
  });
}

// kind 0: uniform, 1: gaussian.
int refd_rng(uint64_t seed, uint64_t index, int kind, int64_t n, double* out) {
  return guarded([&] {
    Rng rng = Rng::forRealization(seed, static_cast<std::size_t>(index));
    for (int64_t i = 0; i < n; ++i) out[i] = kind == 0 ? rng.uniform() : rng.gaussian();
  });
}

int refd_geometry(int nspins, uint64_t seed, uint64_t index, double scale,
                  int32_t* pairs, double* J) {
  return guarded([&] {
    Rng rng = Rng::forRealization(seed, static_cast<std::size_t>(index));
    const auto cs = generateDipolarLattice2D(static_cast<std::size_t>(nspins), rng, scale);
    for (std::size_t p = 0; p < cs.size(); ++p) {
      pairs[2 * p] = static_cast<int32_t>(cs[p].pair.low());
      pairs[2 * p + 1] = static_cast<int32_t>(cs[p].pair.high());
      J[3 * p] = cs[p].jx;
      J[3 * p + 1] = cs[p].jy;
      J[3 * p + 2] = cs[p].jz;
    }
  });
}

// The realisation's Hamiltonian and initial/reference states, assembled in the
// order io/Experiment.cpp:10-35 uses.
int refd_setup(const ss_run_config* c, uint64_t index, double* fields, int32_t* pairs,
               double* J, int32_t* npairs, double* psi0, double* ref0) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    Rng rng = Rng::forRealization(cfg.seed, static_cast<std::size_t>(index));
    Hamiltonian h(cfg.nspins);
    for (SpinIndex s = 0; s < cfg.nspins; ++s) h.setField(s, cfg.baseFields[s]);
    if (cfg.generateGeometry) {
      for (const Coupling& cp : generateDipolarLattice2D(cfg.nspins, rng, cfg.dipolarScale)) {
        h.setCoupling(cp.pair, cp.jx, cp.jy, cp.jz);
      }
    }
    if (cfg.fieldDisorder != 0.0) applyFieldDisorder(h, rng, cfg.fieldDisorder);
    StateVector state(cfg.nspins);
    prepareInitialState(state, cfg.initialState, rng, cfg.basisIndex);
    StateVector reference(cfg.nspins);
    prepareReferenceState(state, cfg.referenceAxis, reference);

    for (std::size_t s = 0; s < cfg.nspins; ++s) {
      fields[3 * s] = h.field(s).x;
      fields[3 * s + 1] = h.field(s).y;
      fields[3 * s + 2] = h.field(s).z;
    }
    const auto& cs = h.couplings();
    for (std::size_t p = 0; p < cs.size(); ++p) {
      pairs[2 * p] = static_cast<int32_t>(cs[p].pair.low());
      pairs[2 * p + 1] = static_cast<int32_t>(cs[p].pair.high());
      J[3 * p] = cs[p].jx;
      J[3 * p + 1] = cs[p].jy;
      J[3 * p + 2] = cs[p].jz;
    }
    *npairs = static_cast<int32_t>(cs.size());
    storeState(state, psi0);
    storeState(reference, ref0);
  });
}

int refd_apply(int nspins, const double* fields, int npairs, const int32_t* pairs,
               const double* J, const double* in, double* out, int variant, double bound) {
  // variant 0: applyPhysical; 1: applyTwiceNormalized(bound); 2: accumulate
  // twice-normalized into the existing `out`.
  return guarded([&] {
    const Hamiltonian h = makeHamiltonian(nspins, fields, npairs, pairs, J);
    const StateVector a = makeState(nspins, in);
    StateVector b = makeState(nspins, out);
    if (variant == 0) h.applyPhysical(a, b);
    else if (variant == 1) h.applyTwiceNormalized(bound, a, b);
    else h.accumulateTwiceNormalized(bound, a, b);
    storeState(b, out);
  });
}

int refd_spectral_bound(int nspins, const double* fields, int npairs,
                        const int32_t* pairs, const double* J, double* out) {
  return guarded([&] {
    *out = makeHamiltonian(nspins, fields, npairs, pairs, J).spectralBound();
  });
}

int refd_evolve(int nspins, const double* fields, int npairs, const int32_t* pairs,
                const double* J, double* psi, int mode, double tau, int64_t nsteps,
                int autonorm, double eps, int64_t* order) {
  return guarded([&] {
    const Hamiltonian h = makeHamiltonian(nspins, fields, npairs, pairs, J);
    StateVector s = makeState(nspins, psi);
    Propagator prop(static_cast<std::size_t>(nspins), eps);
    prop.evolve(h, mode == SS_TIME_IMAGINARY ? TimeMode::Imaginary : TimeMode::Real, s, tau,
                static_cast<std::size_t>(nsteps), autonorm != 0);
    *order = static_cast<int64_t>(prop.lastOrder());
    storeState(s, psi);
  });
}

int refd_rotate(int nspins, double* psi, const double* axis, double angle,
                const int32_t* targets, int ntargets) {
  return guarded([&] {
    std::vector<SpinIndex> t;
    for (int i = 0; i < ntargets; ++i) t.push_back(static_cast<SpinIndex>(targets[i]));
    StateVector s = makeState(nspins, psi);
    SpinRotation(Axis3{axis[0], axis[1], axis[2]}, angle, t).apply(s);
    storeState(s, psi);
  });
}

int refd_two_spin_gate(int nspins, double* psi, const double* m, int a, int b) {
  return guarded([&] {
    TwoSpinGate::Matrix mat{};
    for (int i = 0; i < 16; ++i) mat[static_cast<std::size_t>(i)] = {m[2 * i], m[2 * i + 1]};
    StateVector s = makeState(nspins, psi);
    TwoSpinGate(mat, SpinPair{static_cast<SpinIndex>(a), static_cast<SpinIndex>(b)}).apply(s);
    storeState(s, psi);
  });
}

// Pauli kernels: op 0 axpySigma(axis), 1 applySigma(axis), 2 axpyCoupling.
int refd_pauli(int nspins, int op, int axis, double c, int spin, int spin_b,
               const double* jxyz, const double* in, double* out) {
  return guarded([&] {
    const StateVector a = makeState(nspins, in);
    StateVector b = makeState(nspins, out);
    const auto s = static_cast<SpinIndex>(spin);
    if (op == 0) {
      if (axis == 0) axpySigmaX(c, a, s, b);
      else if (axis == 1) axpySigmaY(c, a, s, b);
      else axpySigmaZ(c, a, s, b);
    } else if (op == 1) {
      if (axis == 0) applySigmaX(a, s, b);
      else if (axis == 1) applySigmaY(a, s, b);
      else applySigmaZ(a, s, b);
    } else {
      axpyCoupling(jxyz[0], jxyz[1], jxyz[2], a,
                   SpinPair{s, static_cast<SpinIndex>(spin_b)}, b);
    }
    storeState(b, out);
  });
}

// Observable::measure through the reference registry, on given states.
int refd_measure(int nspins, const ss_observable* obs, const double* psi, const double* ref,
                 const double* fields, int npairs, const int32_t* pairs, const double* J,
                 double* out) {
  return guarded([&] {
    const StateVector s = makeState(nspins, psi);
    const StateVector r = makeState(nspins, ref);
    const Hamiltonian h = makeHamiltonian(nspins, fields, npairs, pairs, J);
    MeasureContext ctx;
    ctx.state = &s;
    ctx.reference = &r;
    ctx.hamiltonian = &h;
    const auto o = makeObservable(observableSpec(*obs));
    std::vector<double> v(o->width());
    o->measure(ctx, v);
    std::memcpy(out, v.data(), sizeof(double) * v.size());
  });
}

int refd_measurement_count(const ss_run_config* c, int64_t* points, int64_t* width) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    *points = static_cast<int64_t>(cfg.sequence.measurementCount());
    int64_t w = 0;
    for (const auto& spec : cfg.observables) w += static_cast<int64_t>(makeObservable(spec)->width());
    *width = w;
  });
}

// runRealization (io/Experiment.cpp:10-55) for one index.
int refd_run_realization(const ss_run_config* c, uint64_t index, double* times,
                         double* values) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    VectorRecorder rec;
    runRealization(cfg, static_cast<std::size_t>(index), rec);
    std::memcpy(times, rec.times().data(), sizeof(double) * rec.times().size());
    std::memcpy(values, rec.values().data(), sizeof(double) * rec.values().size());
  });
}

// runRealization for the `count` realisation indices `indices` on `threads`
// host threads taking the next index as they finish (the dynamic schedule of
// the reference's LocalRunner, EnsembleRunner.cpp:27-88), rows stored in list
// order.  Wall-clock seconds of the parallel region go to *seconds.
int refd_run_indices(const ss_run_config* c, const uint64_t* indices, int64_t count, int threads,
                     double* times, double* values, double* seconds) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    std::vector<VectorRecorder> recs(static_cast<std::size_t>(count));
    std::atomic<int64_t> next{0};
    std::exception_ptr failure;
    std::mutex m;
    const auto t0 = std::chrono::steady_clock::now();
    {
      std::vector<std::jthread> pool;
      const int workers = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
      for (int w = 0; w < workers; ++w) {
        pool.emplace_back([&] {
          for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= count) return;
            try {
              runRealization(cfg, static_cast<std::size_t>(indices[i]),
                             recs[static_cast<std::size_t>(i)]);
            } catch (...) {
              std::lock_guard lock(m);
              if (!failure) failure = std::current_exception();
              next.store(count);
              return;
            }
          }
        });
      }
    }
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (failure) std::rethrow_exception(failure);
    const auto& t = recs.front().times();
    std::memcpy(times, t.data(), sizeof(double) * t.size());
    std::size_t at = 0;
    for (const auto& r : recs) {
      std::memcpy(values + at, r.values().data(), sizeof(double) * r.values().size());
      at += r.values().size();
    }
  });
}

// The same for indices [first, first+count).
int refd_run_range(const ss_run_config* c, uint64_t first, int64_t count, int threads,
                   double* times, double* values, double* seconds) {
  std::vector<uint64_t> idx(static_cast<std::size_t>(count > 0 ? count : 0));
  for (std::size_t i = 0; i < idx.size(); ++i) idx[i] = first + i;
  return refd_run_indices(c, idx.data(), count, threads, times, values, seconds);
}

// runExperiment (io/Experiment.cpp:57-72) with LocalRunner(threads): mean,
// sd and stderr per (point, column), and the wall-clock seconds it took.
int refd_run_experiment(const ss_run_config* c, int threads, double* times, double* mean,
                        double* sd, double* se, double* seconds) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    LocalRunner runner(static_cast<std::size_t>(threads));
    const auto t0 = std::chrono::steady_clock::now();
    const EnsembleResult r = runExperiment(cfg, runner);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::memcpy(times, r.times.data(), sizeof(double) * r.times.size());
    const auto& m = r.statistics.mean();
    const auto s = r.statistics.standardDeviation();
    const auto e = r.statistics.standardError();
    std::memcpy(mean, m.data(), sizeof(double) * m.size());
    std::memcpy(sd, s.data(), sizeof(double) * s.size());
    std::memcpy(se, e.data(), sizeof(double) * e.size());
  });
}

// runExperiment with LocalRunner(threads), written by the reference's own
// writeCsv (io/Experiment.cpp:74-97): the bytes `spinsim run` prints.
// `needed` receives the length; the text goes to buf when cap allows.
int refd_experiment_csv(const ss_run_config* c, int threads, char* buf, size_t cap,
                        size_t* needed) {
  return guarded([&] {
    const RunConfig cfg = toRunConfig(*c);
    LocalRunner runner(static_cast<std::size_t>(threads));
    std::ostringstream out;
    writeCsv(runExperiment(cfg, runner), out);
    const std::string text = out.str();
    *needed = text.size();
    if (buf != nullptr && cap >= text.size()) std::memcpy(buf, text.data(), text.size());
  });
}

// The test-state recipe of the reference's tests/DenseReference.cpp:204-214
// (mt19937_64 seeded directly, standard normal re then im, normalised), so
// the reference's own propagator cases can be replayed on the same states.
int refd_random_state(int nspins, uint64_t seed, double* out) {
  return guarded([&] {
    StateVector psi(static_cast<std::size_t>(nspins));
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    for (std::size_t k = 0; k < psi.size(); ++k) {
      psi.re(k) = gauss(rng);
      psi.im(k) = gauss(rng);
    }
    psi.normalize();
    storeState(psi, out);
  });
}

}  // extern "C"
