// The plain path for one realisation: runRealization (io/Experiment.cpp:10-55)
// driving Sequence::run (src/sequence/Sequence.cpp) on the device, one
// Propagator::evolve per Evolve step for the state and again for the
// reference, exactly the reference's call structure (FP64 by default; the
// _ex entry point takes the propagator's precision and kernel family).
#include <cmath>
#include <memory>

#include "hamiltonian.cuh"

namespace ss {

void evolve(ss_ham* h, ss_state* psi, const std::vector<double>& weights, double bound,
            int64_t nsteps, bool autonormalize, int precision, int kernel);
int resolve_kernel(int nspins, int precision, int kernel);
void rotation_matrix(const double axis[3], double angle, double u[8]);
void rotate(ss_state* psi, const double u[8], const int32_t* targets, int ntargets);
void total_spin(int axis, const ss_state* in, ss_state* out);
void corr_async(const ss_state* psi, const ss_state* ref, int axis, int slot);
void mag_async(const ss_state* psi, int spin, int axis, int slot);
void energy_async(ss_ham* h, const ss_state* psi, int slot);
void state_norm2_async(const ss_state* s, int slot);

namespace {

struct StateDeleter {
  void operator()(ss_state* s) const { ss_state_destroy(s); }
};
struct HamDeleter {
  void operator()(ss_ham* h) const { ss_ham_destroy(h); }
};
using StatePtr = std::unique_ptr<ss_state, StateDeleter>;
using HamPtr = std::unique_ptr<ss_ham, HamDeleter>;

StatePtr make_state(ss_engine* e, int L) {
  ss_state* s = nullptr;
  if (int rc = ss_state_create(e, L, &s)) fail(rc, ss_last_error());
  return StatePtr(s);
}

HamPtr make_ham(ss_engine* e, int L, const double* fields, const std::vector<PairTerm>& pairs) {
  ss_ham* h = nullptr;
  if (int rc = ss_ham_create(e, L, &h)) fail(rc, ss_last_error());
  HamPtr out(h);
  h->fields.assign(fields, fields + 3 * L);
  h->pairs = pairs;
  return out;
}

struct Runner {
  const ss_run_config& cfg;
  ss_engine* e;
  Realization r;
  std::vector<HamPtr> hams;  // [0] = the realisation's fields, [1+t] = step table t
  StatePtr psi, ref;
  double time = 0.0;
  int64_t row = 0;
  int64_t width = 0;
  double* times;
  double* values;
  int precision = SS_PRECISION_FP64;
  int kernel = SS_KERNEL_AUTO;

  ss_ham* ham_for(int table) {
    const size_t slot = static_cast<size_t>(table + 1);
    if (!hams[slot]) {
      const double* f = cfg.step_fields + static_cast<size_t>(3) * cfg.nspins * table;
      hams[slot] = make_ham(e, r.nspins, f, r.pairs);
    }
    return hams[slot].get();
  }

  void evolve(const ss_step& s) {
    ss_ham* h = s.field_table >= 0 ? ham_for(s.field_table) : hams[0].get();
    const double tau = s.tau_from_draw ? s.tau * r.tau_draw : s.tau;
    if (s.count > 0) {
      const Expansion ex = chebyshev(s.mode, spectral_bound(r.nspins, h->fields.data(), h->pairs),
                                     tau, cfg.epsilon);
      if (ex.order() > 0) {
        const std::vector<double> w = series_weights(ex, s.mode);
        ss::evolve(h, psi.get(), w, ex.bound, s.count, s.autonormalize != 0, precision, kernel);
        ss::evolve(h, ref.get(), w, ex.bound, s.count, s.autonormalize != 0, precision, kernel);
      }
    }
    time += tau * static_cast<double>(s.count);
  }

  void pulse(const ss_step& s) {
    double u[8];
    rotation_matrix(s.axis, s.angle, u);
    std::vector<int32_t> targets;
    if (s.target < 0) {
      for (int q = 0; q < r.nspins; ++q) targets.push_back(q);
    } else {
      require(s.target < r.nspins, SS_ERR_OUT_OF_RANGE, "rotation names a spin outside the system");
      targets.push_back(s.target);
    }
    rotate(psi.get(), u, targets.data(), static_cast<int>(targets.size()));
    rotate(ref.get(), u, targets.data(), static_cast<int>(targets.size()));
  }

  void measure() {
    // Every observable is queued into its own result slots, then one read.
    require(width <= 64, SS_ERR_CONFIG, "too many observables (at most 64 values per point)");
    int slot = 0;
    for (int i = 0; i < cfg.n_observables; ++i) {
      const ss_observable& o = cfg.observables[i];
      switch (o.kind) {
        case SS_OBS_CORR: corr_async(psi.get(), ref.get(), o.axis, slot++); break;
        case SS_OBS_MAG:
          require(o.spin >= 0 && o.spin < r.nspins, SS_ERR_OUT_OF_RANGE,
                  "observable names a spin outside the system");
          mag_async(psi.get(), o.spin, o.axis, slot++);
          break;
        case SS_OBS_NORM:
          state_norm2_async(psi.get(), slot++);
          state_norm2_async(ref.get(), slot++);
          break;
        case SS_OBS_ENERGY: energy_async(hams[0].get(), psi.get(), slot++); break;
        default: fail(SS_ERR_INVALID_ARGUMENT, "unknown observable");
      }
    }
    read_results(e, slot);
    double* out = values + row * width;
    slot = 0;
    for (int i = 0; i < cfg.n_observables; ++i) {
      const ss_observable& o = cfg.observables[i];
      if (o.kind == SS_OBS_CORR) {
        *out++ = e->host_result[slot].x;
        *out++ = e->host_result[slot++].y;
      } else if (o.kind == SS_OBS_NORM) {
        *out++ = std::sqrt(e->host_result[slot++].x);
        *out++ = std::sqrt(e->host_result[slot++].x);
      } else {
        *out++ = e->host_result[slot++].x;
      }
    }
    times[row++] = time;
  }

  void run(int begin, int end) {
    for (int at = begin; at < end;) {
      const ss_step& s = cfg.steps[at];
      switch (s.kind) {
        case SS_STEP_EVOLVE: evolve(s); ++at; break;
        case SS_STEP_PULSE: pulse(s); ++at; break;
        case SS_STEP_MEASURE: measure(); ++at; break;
        case SS_STEP_REPEAT:
          for (int64_t i = 0; i < s.count; ++i) run(at + 1, at + 1 + s.body_len);
          at += 1 + s.body_len;
          break;
        default: fail(SS_ERR_INVALID_ARGUMENT, "unknown step kind");
      }
    }
  }
};

}  // namespace

void validate_config(const ss_run_config& c) {
  require(c.nspins >= 1 && c.nspins <= kMaxSpins, SS_ERR_CONFIG,
          "system.spins must be between 1 and 30");
  require(c.base_fields != nullptr, SS_ERR_CONFIG, "field does not cover every spin");
  require(c.epsilon > 0.0, SS_ERR_CONFIG, "numerics.epsilon must be positive");
  require(c.n_observables > 0 && c.observables != nullptr, SS_ERR_CONFIG,
          "measurement.observables must not be empty");
  require(c.n_steps >= 0 && (c.n_steps == 0 || c.steps != nullptr), SS_ERR_CONFIG, "bad program");
  require(measurement_count(c.steps, 0, c.n_steps) > 0, SS_ERR_CONFIG,
          "the sequence records nothing; add a measure step");
  for (int i = 0; i < c.n_steps; ++i) {
    const ss_step& s = c.steps[i];
    if (s.kind == SS_STEP_EVOLVE && s.field_table >= 0) {
      require(s.field_table < c.n_step_fields && c.step_fields != nullptr, SS_ERR_CONFIG,
              "step field table index out of range");
    }
    if (s.kind == SS_STEP_REPEAT) {
      require(s.body_len >= 0 && i + s.body_len < c.n_steps, SS_ERR_CONFIG,
              "repeat body runs past the program");
    }
    if (s.kind == SS_STEP_PULSE) {
      const double len = std::sqrt(s.axis[0] * s.axis[0] + s.axis[1] * s.axis[1] +
                                   s.axis[2] * s.axis[2]);
      require(len > 0.0, SS_ERR_INVALID_ARGUMENT, "rotation axis must have non-zero length");
    }
    require(s.kind >= 0 && s.kind <= 3, SS_ERR_CONFIG, "unknown step kind");
  }
}

void run_realization_plain(ss_engine* e, const ss_run_config& cfg, uint64_t index, double* times,
                           double* values, int precision, int kernel) {
  validate_config(cfg);
  Runner x{cfg, e, assemble_realization(cfg, index), {}, nullptr, nullptr};
  const int L = x.r.nspins;
  resolve_kernel(L, precision, kernel);  // rejects unknown or too-small choices up front
  x.precision = precision;
  x.kernel = kernel;
  x.hams.resize(static_cast<size_t>(cfg.n_step_fields) + 1);
  x.hams[0] = make_ham(e, L, x.r.fields.data(), x.r.pairs);
  x.psi = make_state(e, L);
  x.ref = make_state(e, L);
  SS_CUDA(cudaMemcpyAsync(x.psi->data, x.r.psi0.data(), sizeof(double) * x.r.psi0.size(),
                          cudaMemcpyHostToDevice, e->stream));
  total_spin(cfg.reference_axis, x.psi.get(), x.ref.get());  // Ensemble.cpp:47-58
  x.width = observable_width(cfg.observables, cfg.n_observables);
  x.times = times;
  x.values = values;
  x.run(0, cfg.n_steps);
  sync(e);
}

}  // namespace ss

using namespace ss;

extern "C" int ss_run_realization(ss_engine* engine, const ss_run_config* config, uint64_t index,
                                  double* times, double* values) {
  return guarded([&] {
    TraceRange trace("ss_run_realization");
    require(engine != nullptr && config != nullptr && times != nullptr && values != nullptr,
            SS_ERR_INVALID_ARGUMENT, "null argument");
    run_realization_plain(engine, *config, index, times, values, SS_PRECISION_FP64,
                          SS_KERNEL_AUTO);
  });
}

extern "C" int ss_run_realization_ex(ss_engine* engine, const ss_run_config* config,
                                     uint64_t index, int precision, int kernel, double* times,
                                     double* values) {
  return guarded([&] {
    TraceRange trace("ss_run_realization");
    require(engine != nullptr && config != nullptr && times != nullptr && values != nullptr,
            SS_ERR_INVALID_ARGUMENT, "null argument");
    run_realization_plain(engine, *config, index, times, values, precision, kernel);
  });
}
