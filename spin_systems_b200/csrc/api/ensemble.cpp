// Ensemble layer of the C++ API: random streams, geometry and disorder on the
// host, states and their operators on the device, statistics on the host.
//
// Restated for bit-exact parity with the reference (their arithmetic and the
// order of their random draws define geometries, fields and initial states,
// so those are kept; the code around them is this library's own):
//   Rng::gaussian              src/ensemble/Rng.cpp:8-23 (Box-Muller, u floored at 1e-15)
//   prepareInitialState        src/ensemble/Ensemble.cpp:20-45 (re then im per k, then
//                              one normalisation in index order)
//   generateDipolarLattice2D   src/ensemble/Ensemble.cpp:60-104 (draw order, rejection
//                              rule, coupling order and r^3 arithmetic)
//   Accumulator                src/ensemble/Ensemble.cpp:114-166 (Welford in index
//                              order, Chan's merge)
#include <atomic>
#include <cmath>
#include <exception>
#include <format>
#include <numbers>
#include <optional>
#include <stdexcept>
#include <thread>
#include <utility>

#include "spinsim/core/Device.hpp"
#include "spinsim/core/SpinOperators.hpp"
#include "spinsim/ensemble/Ensemble.hpp"
#include "spinsim/ensemble/EnsembleRunner.hpp"
#include "spinsim_b200.h"

namespace spinsim {
namespace {

// Box-Muller on two uniforms: (r cos, r sin) with r = sqrt(-2 ln u).
std::pair<double, double> boxMuller(double u, double v) {
  const double r = std::sqrt(-2.0 * std::log(u));
  const double phase = 2.0 * std::numbers::pi * v;
  return {r * std::cos(phase), r * std::sin(phase)};
}

// Scales v to unit norm, the squares summed in index order.
void normalizeInIndexOrder(double* v, std::size_t n) {
  double sum = 0.0;
  for (std::size_t i = 0; i < n; ++i) sum += v[i] * v[i];
  const double norm = std::sqrt(sum);
  if (norm == 0.0) throw std::domain_error("cannot normalize a zero state");
  const double inv = 1.0 / norm;
  for (std::size_t i = 0; i < n; ++i) v[i] *= inv;
}

// Product of single-spin states cos(th/2)|up> + e^{i ph} sin(th/2)|down>
// with th, ph drawn per spin (additive initial state, not in the reference).
void fillRandomProduct(StateVector& psi, Rng& rng) {
  const std::size_t L = psi.nspins();
  std::vector<double> theta(L), phi(L);
  for (std::size_t s = 0; s < L; ++s) {
    theta[s] = std::acos(1.0 - 2.0 * rng.uniform());
    phi[s] = 2.0 * std::numbers::pi * rng.uniform();
  }
  double* d = psi.data();
  for (std::size_t k = 0; k < psi.size(); ++k) {
    double re = 1.0, im = 0.0;
    for (std::size_t s = 0; s < L; ++s) {
      const bool up = (k >> s) & 1u;
      const double half = 0.5 * theta[s];
      const double fr = up ? std::cos(half) : std::sin(half) * std::cos(phi[s]);
      const double fi = up ? 0.0 : std::sin(half) * std::sin(phi[s]);
      const double nr = re * fr - im * fi;
      im = re * fi + im * fr;
      re = nr;
    }
    d[2 * k] = re;
    d[2 * k + 1] = im;
  }
  normalizeInIndexOrder(d, 2 * psi.size());
}

struct Point {
  double x = 0.0, y = 0.0;
};

// A spin position uniform in the square [-h, h]^2, redrawn while it lies
// within `minSep` of an earlier spin in both coordinates.
Point drawPosition(Rng& rng, double h, double minSep, const std::vector<Point>& placed) {
  for (;;) {
    Point p;
    p.x = h * (2.0 * rng.uniform() - 1.0);
    p.y = h * (2.0 * rng.uniform() - 1.0);
    bool clear = true;
    for (const Point& q : placed) {
      if (std::abs(p.x - q.x) < minSep && std::abs(p.y - q.y) < minSep) {
        clear = false;
        break;
      }
    }
    if (clear) return p;
  }
}

}  // namespace

double Rng::gaussian() {
  if (hasSpare_) {
    hasSpare_ = false;
    return spare_;
  }
  constexpr double kEdge = 1.0e-15;  // keeps u away from 0 and 1
  const double u = kEdge + (1.0 - 2.0 * kEdge) * uniform();
  const double v = uniform();
  const auto [first, second] = boxMuller(u, v);
  spare_ = second;
  hasSpare_ = true;
  return first;
}

InitialStateKind parseInitialStateKind(std::string_view name) {
  static constexpr std::pair<std::string_view, InitialStateKind> kNames[] = {
      {"random", InitialStateKind::Random},
      {"up", InitialStateKind::AllUp},
      {"down", InitialStateKind::AllDown},
      {"basis", InitialStateKind::BasisState},
      {"random_product", InitialStateKind::RandomProduct},
  };
  for (const auto& [text, kind] : kNames) {
    if (text == name) return kind;
  }
  throw std::invalid_argument(std::format(
      "unknown initial state '{}'; expected random, up, down, basis or random_product", name));
}

void prepareInitialState(StateVector& psi, InitialStateKind kind, Rng& rng,
                         std::size_t basisIndex) {
  switch (kind) {
    case InitialStateKind::AllUp: psi.setBasisState(psi.size() - 1); break;
    case InitialStateKind::AllDown: psi.setBasisState(0); break;
    case InitialStateKind::BasisState: psi.setBasisState(basisIndex); break;
    case InitialStateKind::RandomProduct: fillRandomProduct(psi, rng); break;
    case InitialStateKind::Random: {
      // Complex Gaussian amplitudes, real part first, in index order.
      double* d = psi.data();
      for (std::size_t i = 0; i < 2 * psi.size(); ++i) d[i] = rng.gaussian();
      normalizeInIndexOrder(d, 2 * psi.size());
      break;
    }
  }
}

void prepareReferenceState(const StateVector& psi, Axis axis, StateVector& reference) {
  if (reference.size() != psi.size()) reference = StateVector(psi.nspins());
  const int code = axis == Axis::X ? SS_AXIS_X : axis == Axis::Y ? SS_AXIS_Y : SS_AXIS_Z;
  checkStatus(ss_apply_total_spin(code, psi.device(), reference.device()));
  reference.deviceWritten();
}

std::vector<Coupling> generateDipolarLattice2D(std::size_t nspins, Rng& rng, double scale,
                                               double minSeparation) {
  if (nspins == 0) throw std::invalid_argument("need at least one spin");
  // Placement first: spin 0 at the origin, the others drawn in turn (the
  // draws are the only use of the stream); then every pair (j, i), j < i,
  // in order of i, with Jz = scale / r^3 and Jx = Jy = -Jz / 2.
  const double h = 0.5 * std::sqrt(static_cast<double>(nspins));
  std::vector<Point> placed(1);
  placed.reserve(nspins);
  while (placed.size() < nspins) placed.push_back(drawPosition(rng, h, minSeparation, placed));
  std::vector<Coupling> out;
  out.reserve(nspins * (nspins - 1) / 2);
  for (std::size_t i = 1; i < nspins; ++i) {
    for (std::size_t j = 0; j < i; ++j) {
      const double dx = placed[i].x - placed[j].x;
      const double dy = placed[i].y - placed[j].y;
      const double r2 = dx * dx + dy * dy;
      const double jz = scale / (r2 * std::sqrt(r2));
      out.push_back(Coupling{SpinPair{j, i}, -0.5 * jz, -0.5 * jz, jz});
    }
  }
  return out;
}

void applyFieldDisorder(Hamiltonian& hamiltonian, Rng& rng, double sigma) {
  for (SpinIndex s = 0; s < hamiltonian.nspins(); ++s) {
    Field f = hamiltonian.field(s);
    f.z += sigma * rng.gaussian();
    hamiltonian.setField(s, f);
  }
}

// ------------------------------------------------------------- statistics

Accumulator::Accumulator(std::size_t width) : mean_(width, 0.0), m2_(width, 0.0) {}

void Accumulator::add(std::span<const double> sample) {
  if (sample.size() != mean_.size()) {
    throw std::invalid_argument("sample width does not match the accumulator");
  }
  const double n = static_cast<double>(++count_);
  for (std::size_t k = 0; k < sample.size(); ++k) {  // Welford per column
    const double before = mean_[k];
    mean_[k] = before + (sample[k] - before) / n;
    m2_[k] += (sample[k] - before) * (sample[k] - mean_[k]);
  }
}

void Accumulator::merge(const Accumulator& other) {
  if (other.mean_.size() != mean_.size()) {
    throw std::invalid_argument("cannot merge accumulators of different width");
  }
  if (other.count_ == 0) return;
  if (count_ == 0) {
    *this = other;
    return;
  }
  const double na = static_cast<double>(count_), nb = static_cast<double>(other.count_);
  const double n = na + nb;
  for (std::size_t k = 0; k < mean_.size(); ++k) {  // Chan et al. pairwise update
    const double gap = other.mean_[k] - mean_[k];
    mean_[k] += gap * nb / n;
    m2_[k] += other.m2_[k] + gap * gap * na * nb / n;
  }
  count_ += other.count_;
}

std::vector<double> Accumulator::standardDeviation() const {
  std::vector<double> sd(mean_.size(), 0.0);
  if (count_ > 1) {
    const double dof = static_cast<double>(count_ - 1);
    for (std::size_t k = 0; k < sd.size(); ++k) sd[k] = std::sqrt(m2_[k] / dof);
  }
  return sd;
}

std::vector<double> Accumulator::standardError() const {
  std::vector<double> se = standardDeviation();
  if (count_ > 1) {
    const double f = 1.0 / std::sqrt(static_cast<double>(count_));
    for (double& v : se) v *= f;
  }
  return se;
}

void VectorRecorder::record(double time, std::span<const double> values) {
  times_.push_back(time);
  values_.insert(values_.end(), values.begin(), values.end());
}

void VectorRecorder::clear() {
  times_.clear();
  values_.clear();
}

// ---------------------------------------------------------------- runners

namespace {

// Realisation indices handed out in increasing order to whichever worker
// asks next; cancel() hands out nothing more.
class JobQueue {
 public:
  explicit JobQueue(std::size_t n) : n_(n) {}
  std::optional<std::size_t> next() {
    const std::size_t i = cursor_.fetch_add(1, std::memory_order_relaxed);
    if (i >= n_ || cancelled_.load(std::memory_order_relaxed)) return std::nullopt;
    return i;
  }
  void cancel() { cancelled_.store(true, std::memory_order_relaxed); }

 private:
  std::size_t n_;
  std::atomic<std::size_t> cursor_{0};
  std::atomic<bool> cancelled_{false};
};

// Every realisation's rows folded into one Accumulator in index order, so the
// statistics do not depend on how the realisations were spread over workers.
EnsembleResult foldInIndexOrder(std::size_t realizations, std::vector<double> times,
                                std::span<const std::string> columns,
                                const std::function<std::span<const double>(std::size_t)>& row) {
  EnsembleResult result;
  result.times = std::move(times);
  result.columns.assign(columns.begin(), columns.end());
  const std::size_t width = result.times.size() * result.columns.size();
  result.statistics = Accumulator(width);
  for (std::size_t i = 0; i < realizations; ++i) result.statistics.add(row(i));
  return result;
}

}  // namespace

LocalRunner::LocalRunner(std::size_t threads)
    : threads_(threads > 0 ? threads : std::max(1u, std::thread::hardware_concurrency())) {}

EnsembleResult LocalRunner::run(std::size_t realizations, std::span<const std::string> columns,
                                const RealizationJob& job) {
  if (realizations == 0) throw std::invalid_argument("an ensemble needs at least one realisation");
  // Each worker thread drives the device through its own engine and stream
  // (the core API's per-thread engine).  A failing realisation stops the
  // hand-out; of the failures, the lowest realisation index is reported, so
  // the error does not depend on thread timing.
  std::vector<VectorRecorder> recorders(realizations);
  std::vector<std::exception_ptr> errors(realizations);
  JobQueue queue(realizations);
  {
    std::vector<std::jthread> workers;
    const std::size_t n = std::min(threads_, realizations);
    workers.reserve(n);
    for (std::size_t w = 0; w < n; ++w) {
      workers.emplace_back([&] {
        while (const auto index = queue.next()) {
          try {
            job(*index, recorders[*index]);
          } catch (...) {
            errors[*index] = std::current_exception();
            queue.cancel();
          }
        }
      });
    }
  }
  for (const std::exception_ptr& e : errors) {
    if (e) std::rethrow_exception(e);
  }
  const std::size_t points = recorders.front().rows();
  const std::size_t width = points * columns.size();
  for (std::size_t i = 0; i < realizations; ++i) {
    if (recorders[i].rows() != points || recorders[i].values().size() != width) {
      throw std::runtime_error(std::format(
          "realisation {} recorded {} points and {} values; expected {} and {}", i,
          recorders[i].rows(), recorders[i].values().size(), points, width));
    }
  }
  return foldInIndexOrder(realizations, recorders.front().times(), columns,
                          [&](std::size_t i) { return std::span<const double>(recorders[i].values()); });
}

EnsembleResult foldRows(std::size_t realizations, const std::vector<double>& times,
                        std::span<const std::string> columns, const std::vector<double>& rows) {
  const std::size_t width = times.size() * columns.size();
  if (rows.size() != realizations * width) {
    throw std::runtime_error("batched rows do not match the measurement shape");
  }
  return foldInIndexOrder(realizations, times, columns, [&](std::size_t i) {
    return std::span<const double>(rows.data() + i * width, width);
  });
}

}  // namespace spinsim
