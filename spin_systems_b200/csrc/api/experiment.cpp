// Experiments (reference: src/io/Experiment.cpp:10-110): one realisation
// through the C++ API (plain FP64 device path), whole ensembles through a
// runner or the batched engine, and the CSV writer.
#include <cmath>
#include <format>
#include <fstream>
#include <ostream>
#include <stdexcept>

#include "spinsim/core/Device.hpp"
#include "spinsim/io/Experiment.hpp"

namespace spinsim {
namespace {

struct Draws {
  std::size_t nspins;
  double sigma;
  double tau;
};

// Additive per-realisation draws from the harness stream (drawSeed, index):
// L first, then sigma, then tau; the (seed, index) stream is untouched.
Draws drawFor(const RunConfig& c, std::size_t index) {
  Draws d{c.nspins, c.fieldDisorder, 1.0};
  const bool any = !c.spinChoices.empty() || c.disorderRange[1] > c.disorderRange[0] ||
                   c.tauRange[1] > c.tauRange[0];
  if (!any) return d;
  Rng r = Rng::forRealization(c.drawSeed, index);
  if (!c.spinChoices.empty()) {
    std::size_t k = static_cast<std::size_t>(r.uniform() * static_cast<double>(c.spinChoices.size()));
    if (k >= c.spinChoices.size()) k = c.spinChoices.size() - 1;
    d.nspins = static_cast<std::size_t>(c.spinChoices[k]);
  }
  if (c.disorderRange[1] > c.disorderRange[0]) {
    d.sigma = c.disorderRange[0] + (c.disorderRange[1] - c.disorderRange[0]) * r.uniform();
  }
  if (c.tauRange[1] > c.tauRange[0]) {
    d.tau = c.tauRange[0] + (c.tauRange[1] - c.tauRange[0]) * r.uniform();
  }
  return d;
}

std::vector<std::string> observableColumns(const RunConfig& config) {
  std::vector<std::unique_ptr<Observable>> probes;
  for (const std::string& spec : config.observables) probes.push_back(makeObservable(spec));
  std::vector<std::string> columns = resultColumns(probes);
  columns.erase(columns.begin());
  return columns;
}

int axisCode(Axis a) { return a == Axis::X ? SS_AXIS_X : a == Axis::Y ? SS_AXIS_Y : SS_AXIS_Z; }

void flatten(const std::vector<Step>& steps, std::size_t nspins, ConfigView& v) {
  for (const Step& step : steps) {
    ss_step s{};
    s.field_table = -1;
    s.target = -1;
    if (const auto* e = std::get_if<Evolve>(&step)) {
      s.kind = SS_STEP_EVOLVE;
      s.mode = e->mode == TimeMode::Real ? SS_TIME_REAL : SS_TIME_IMAGINARY;
      s.autonormalize = e->autonormalize ? 1 : 0;
      s.count = static_cast<int64_t>(e->nsteps);
      s.tau = e->tau;
      s.tau_from_draw = e->tauFromDraw ? 1 : 0;
      if (!e->fields.empty()) {
        s.field_table = static_cast<int32_t>(v.stepFields.size() / (3 * nspins));
        for (const Field& f : e->fields) v.stepFields.insert(v.stepFields.end(), {f.x, f.y, f.z});
      }
      v.steps.push_back(s);
    } else if (const auto* p = std::get_if<Pulse>(&step)) {
      s.kind = SS_STEP_PULSE;
      s.angle = p->rotation.angle();
      s.axis[0] = p->rotation.axis().x;
      s.axis[1] = p->rotation.axis().y;
      s.axis[2] = p->rotation.axis().z;
      const auto& t = p->rotation.targets();
      bool all = t.size() == nspins;
      for (std::size_t i = 0; all && i < t.size(); ++i) all = t[i] == i;
      if (all) {
        s.target = -1;
      } else if (t.size() == 1) {
        s.target = static_cast<int32_t>(t[0]);
      } else {
        throw std::invalid_argument("a pulse on several but not all spins has no batched form");
      }
      v.steps.push_back(s);
    } else if (std::holds_alternative<Measure>(step)) {
      s.kind = SS_STEP_MEASURE;
      v.steps.push_back(s);
    } else {
      const auto& r = std::get<Repeat>(step);
      s.kind = SS_STEP_REPEAT;
      s.count = static_cast<int64_t>(r.count);
      const std::size_t at = v.steps.size();
      v.steps.push_back(s);
      flatten(r.body, nspins, v);
      v.steps[at].body_len = static_cast<int32_t>(v.steps.size() - at - 1);
    }
  }
}

}  // namespace

void toConfigView(const RunConfig& c, ConfigView& v) {
  v = ConfigView{};
  for (const Field& f : c.baseFields) v.baseFields.insert(v.baseFields.end(), {f.x, f.y, f.z});
  flatten(c.sequence.steps(), c.nspins, v);
  for (const std::string& spec : c.observables) {
    const auto o = makeObservable(spec);
    ss_observable so{};
    if (const auto* corr = dynamic_cast<const TotalSpinCorrelator*>(o.get())) {
      so.kind = SS_OBS_CORR;
      so.axis = axisCode(corr->axis());
    } else if (const auto* mag = dynamic_cast<const SingleSpinMagnetization*>(o.get())) {
      so.kind = SS_OBS_MAG;
      so.axis = axisCode(mag->axis());
      so.spin = static_cast<int32_t>(mag->spin());
    } else if (dynamic_cast<const StateNorms*>(o.get())) {
      so.kind = SS_OBS_NORM;
    } else {
      so.kind = SS_OBS_ENERGY;
    }
    v.observables.push_back(so);
  }
  ss_run_config& x = v.config;
  x.nspins = static_cast<int32_t>(c.nspins);
  x.initial_state = c.initialState == InitialStateKind::AllUp        ? SS_INIT_UP
                    : c.initialState == InitialStateKind::AllDown    ? SS_INIT_DOWN
                    : c.initialState == InitialStateKind::BasisState ? SS_INIT_BASIS
                    : c.initialState == InitialStateKind::RandomProduct ? SS_INIT_RANDOM_PRODUCT
                                                                        : SS_INIT_RANDOM;
  x.basis_index = c.basisIndex;
  x.realizations = c.realizations;
  x.seed = c.seed;
  x.generate_geometry = c.generateGeometry ? 1 : 0;
  x.reference_axis = axisCode(c.referenceAxis);
  x.dipolar_scale = c.dipolarScale;
  x.field_disorder = c.fieldDisorder;
  x.epsilon = c.epsilon;
  x.base_fields = v.baseFields.data();
  x.n_observables = static_cast<int32_t>(v.observables.size());
  x.n_steps = static_cast<int32_t>(v.steps.size());
  x.observables = v.observables.data();
  x.steps = v.steps.data();
  x.n_step_fields = static_cast<int32_t>(v.stepFields.size() / (3 * c.nspins));
  x.step_fields = v.stepFields.data();
  x.draw_seed = c.drawSeed;
  x.disorder_range[0] = c.disorderRange[0];
  x.disorder_range[1] = c.disorderRange[1];
  x.tau_range[0] = c.tauRange[0];
  x.tau_range[1] = c.tauRange[1];
  x.n_spin_choices = static_cast<int32_t>(c.spinChoices.size());
  for (std::size_t i = 0; i < c.spinChoices.size() && i < 8; ++i) x.spin_choices[i] = c.spinChoices[i];
}

void runRealization(const RunConfig& config, std::size_t index, VectorRecorder& out) {
  const Draws d = drawFor(config, index);
  const std::size_t L = d.nspins;
  Rng rng = Rng::forRealization(config.seed, index);
  Hamiltonian hamiltonian(L);
  for (SpinIndex s = 0; s < L; ++s) hamiltonian.setField(s, config.baseFields[s]);
  // Order matters: geometry, then disorder, then the initial state.
  if (config.generateGeometry) {
    for (const Coupling& c : generateDipolarLattice2D(L, rng, config.dipolarScale)) {
      hamiltonian.setCoupling(c.pair, c.jx, c.jy, c.jz);
    }
  }
  if (d.sigma != 0.0) applyFieldDisorder(hamiltonian, rng, d.sigma);
  StateVector state(L);
  prepareInitialState(state, config.initialState, rng, config.basisIndex);
  StateVector reference(L);
  prepareReferenceState(state, config.referenceAxis, reference);

  std::vector<std::unique_ptr<Observable>> observables;
  for (const std::string& spec : config.observables) observables.push_back(makeObservable(spec));
  Propagator propagator(L, config.epsilon);
  RunContext ctx;
  ctx.hamiltonian = &hamiltonian;
  ctx.state = &state;
  ctx.reference = &reference;
  ctx.propagator = &propagator;
  ctx.observables = observables;
  ctx.recorder = &out;
  ctx.tauDraw = d.tau;
  config.sequence.run(ctx);
}

EnsembleResult runExperiment(const RunConfig& config, EnsembleRunner& runner) {
  const std::vector<std::string> columns = observableColumns(config);
  return runner.run(config.realizations, columns,
                    [&config](std::size_t index, VectorRecorder& out) {
                      runRealization(config, index, out);
                    });
}

EnsembleResult runExperimentBatched(const RunConfig& config, int precision) {
  ConfigView view;
  toConfigView(config, view);
  ss_batch* b = nullptr;
  checkStatus(ss_batch_create(threadEngine(), &view.config, 0,
                              static_cast<int64_t>(config.realizations), precision, &b));
  int64_t points = 0, width = 0;
  ss_batch_shape(b, &points, &width);
  std::vector<double> rows(config.realizations * static_cast<std::size_t>(points * width));
  std::vector<double> times(static_cast<std::size_t>(points));
  const int rc = ss_batch_run(b, rows.data(), times.data());
  ss_batch_destroy(b);
  checkStatus(rc);
  return foldRows(config.realizations, times, observableColumns(config), rows);
}

void writeCsv(const EnsembleResult& result, std::ostream& out) {
  const std::size_t ncols = result.columns.size();
  if (result.statistics.width() != result.times.size() * ncols) {
    throw std::runtime_error("result shape does not match its column names");
  }
  out << "time";
  for (const std::string& name : result.columns) {
    out << ',' << name << "_mean," << name << "_sd," << name << "_stderr";
  }
  out << '\n';
  const std::vector<double>& mean = result.statistics.mean();
  const std::vector<double> sd = result.statistics.standardDeviation();
  const std::vector<double> se = result.statistics.standardError();
  for (std::size_t point = 0; point < result.times.size(); ++point) {
    out << std::format("{:.10g}", result.times[point]);
    for (std::size_t c = 0; c < ncols; ++c) {
      const std::size_t k = point * ncols + c;
      out << std::format(",{:.12g},{:.12g},{:.12g}", mean[k], sd[k], se[k]);
    }
    out << '\n';
  }
}

void writeCsv(const EnsembleResult& result, const std::filesystem::path& path) {
  if (path.has_parent_path()) std::filesystem::create_directories(path.parent_path());
  std::ofstream out(path);
  if (!out) throw std::runtime_error(std::format("cannot open '{}' for writing", path.string()));
  writeCsv(result, out);
}

}  // namespace spinsim
