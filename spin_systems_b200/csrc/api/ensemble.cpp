// Ensemble layer of the C++ API (reference: src/ensemble/*.cpp): random
// streams and geometry on the host (bit-for-bit with the reference, since
// glibc's log/sin/cos and mt19937_64 define the streams), states and their
// operators on the device, statistics on the host.
#include <atomic>
#include <cmath>
#include <exception>
#include <format>
#include <mutex>
#include <numbers>
#include <stdexcept>
#include <thread>

#include "spinsim/core/Device.hpp"
#include "spinsim/core/SpinOperators.hpp"
#include "spinsim/ensemble/Ensemble.hpp"
#include "spinsim/ensemble/EnsembleRunner.hpp"
#include "spinsim_b200.h"

namespace spinsim {

double Rng::gaussian() {
  if (hasSpare_) {
    hasSpare_ = false;
    return spare_;
  }
  constexpr double kFloor = 1.0e-15;
  const double u = kFloor + (1.0 - 2.0 * kFloor) * uniform();
  const double v = uniform();
  const double radius = std::sqrt(-2.0 * std::log(u));
  const double phase = 2.0 * std::numbers::pi * v;
  spare_ = radius * std::sin(phase);
  hasSpare_ = true;
  return radius * std::cos(phase);
}

InitialStateKind parseInitialStateKind(std::string_view name) {
  if (name == "random") return InitialStateKind::Random;
  if (name == "up") return InitialStateKind::AllUp;
  if (name == "down") return InitialStateKind::AllDown;
  if (name == "basis") return InitialStateKind::BasisState;
  if (name == "random_product") return InitialStateKind::RandomProduct;
  throw std::invalid_argument(std::format(
      "unknown initial state '{}'; expected random, up, down, basis or random_product", name));
}

namespace {

// Host normalisation in the reference's summation order, so psi0 is
// bit-identical to the reference's (StateVector.cpp:43-56).
void normalizeHost(double* v, std::size_t n) {
  double sum = 0.0;
  for (std::size_t i = 0; i < n; ++i) sum += v[i] * v[i];
  const double nrm = std::sqrt(sum);
  if (nrm == 0.0) throw std::domain_error("cannot normalize a zero state");
  const double f = 1.0 / nrm;
  for (std::size_t i = 0; i < n; ++i) v[i] *= f;
}

}  // namespace

void prepareInitialState(StateVector& psi, InitialStateKind kind, Rng& rng,
                         std::size_t basisIndex) {
  switch (kind) {
    case InitialStateKind::AllUp: psi.setBasisState(psi.size() - 1); return;
    case InitialStateKind::AllDown: psi.setBasisState(0); return;
    case InitialStateKind::BasisState: psi.setBasisState(basisIndex); return;
    case InitialStateKind::RandomProduct: {
      const std::size_t L = psi.nspins();
      std::vector<double> th(L), ph(L);
      for (std::size_t s = 0; s < L; ++s) {
        th[s] = std::acos(1.0 - 2.0 * rng.uniform());
        ph[s] = 2.0 * std::numbers::pi * rng.uniform();
      }
      double* d = psi.data();
      for (std::size_t k = 0; k < psi.size(); ++k) {
        double ar = 1.0, ai = 0.0;
        for (std::size_t s = 0; s < L; ++s) {
          double fr, fi;
          if (k & (std::size_t{1} << s)) {
            fr = std::cos(0.5 * th[s]);
            fi = 0.0;
          } else {
            const double sn = std::sin(0.5 * th[s]);
            fr = sn * std::cos(ph[s]);
            fi = sn * std::sin(ph[s]);
          }
          const double nr = ar * fr - ai * fi;
          ai = ar * fi + ai * fr;
          ar = nr;
        }
        d[2 * k] = ar;
        d[2 * k + 1] = ai;
      }
      normalizeHost(d, 2 * psi.size());
      return;
    }
    case InitialStateKind::Random: break;
  }
  double* d = psi.data();
  for (std::size_t k = 0; k < psi.size(); ++k) {
    d[2 * k] = rng.gaussian();
    d[2 * k + 1] = rng.gaussian();
  }
  normalizeHost(d, 2 * psi.size());
}

void prepareReferenceState(const StateVector& psi, Axis axis, StateVector& reference) {
  if (reference.size() != psi.size()) reference = StateVector(psi.nspins());
  const int a = axis == Axis::X ? SS_AXIS_X : axis == Axis::Y ? SS_AXIS_Y : SS_AXIS_Z;
  ss_state* out = reference.device();
  checkStatus(ss_apply_total_spin(a, psi.device(), out));
  reference.deviceWritten();
}

std::vector<Coupling> generateDipolarLattice2D(std::size_t nspins, Rng& rng, double scale,
                                               double minSeparation) {
  if (nspins == 0) throw std::invalid_argument("need at least one spin");
  const double halfWidth = 0.5 * std::sqrt(static_cast<double>(nspins));
  std::vector<double> x(nspins, 0.0), y(nspins, 0.0);
  std::vector<Coupling> couplings;
  couplings.reserve(nspins * (nspins - 1) / 2);
  for (std::size_t i = 1; i < nspins; ++i) {
    double px = 0.0, py = 0.0;
    for (bool placed = false; !placed;) {
      px = halfWidth * (2.0 * rng.uniform() - 1.0);
      py = halfWidth * (2.0 * rng.uniform() - 1.0);
      placed = true;
      for (std::size_t j = 0; j < i; ++j) {
        if (std::abs(px - x[j]) < minSeparation && std::abs(py - y[j]) < minSeparation) {
          placed = false;
          break;
        }
      }
    }
    x[i] = px;
    y[i] = py;
    for (std::size_t j = 0; j < i; ++j) {
      const double dx = px - x[j];
      const double dy = py - y[j];
      const double r2 = dx * dx + dy * dy;
      const double jz = scale / (r2 * std::sqrt(r2));
      couplings.push_back(Coupling{SpinPair{j, i}, -0.5 * jz, -0.5 * jz, jz});
    }
  }
  return couplings;
}

void applyFieldDisorder(Hamiltonian& hamiltonian, Rng& rng, double sigma) {
  for (SpinIndex s = 0; s < hamiltonian.nspins(); ++s) {
    Field f = hamiltonian.field(s);
    f.z += sigma * rng.gaussian();
    hamiltonian.setField(s, f);
  }
}

Accumulator::Accumulator(std::size_t width) : mean_(width, 0.0), m2_(width, 0.0) {}

void Accumulator::add(std::span<const double> sample) {
  if (sample.size() != mean_.size()) {
    throw std::invalid_argument("sample width does not match the accumulator");
  }
  ++count_;
  const double n = static_cast<double>(count_);
  for (std::size_t k = 0; k < sample.size(); ++k) {
    const double delta = sample[k] - mean_[k];
    mean_[k] += delta / n;
    m2_[k] += delta * (sample[k] - mean_[k]);
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
  const double total = na + nb;
  for (std::size_t k = 0; k < mean_.size(); ++k) {
    const double delta = other.mean_[k] - mean_[k];
    mean_[k] += delta * nb / total;
    m2_[k] += other.m2_[k] + delta * delta * na * nb / total;
  }
  count_ += other.count_;
}

std::vector<double> Accumulator::standardDeviation() const {
  std::vector<double> out(mean_.size(), 0.0);
  if (count_ < 2) return out;
  const double denom = static_cast<double>(count_ - 1);
  for (std::size_t k = 0; k < out.size(); ++k) out[k] = std::sqrt(m2_[k] / denom);
  return out;
}

std::vector<double> Accumulator::standardError() const {
  std::vector<double> out = standardDeviation();
  if (count_ < 2) return out;
  const double scale = 1.0 / std::sqrt(static_cast<double>(count_));
  for (double& v : out) v *= scale;
  return out;
}

void VectorRecorder::record(double time, std::span<const double> values) {
  times_.push_back(time);
  values_.insert(values_.end(), values.begin(), values.end());
}

void VectorRecorder::clear() {
  times_.clear();
  values_.clear();
}

LocalRunner::LocalRunner(std::size_t threads)
    : threads_(threads > 0 ? threads : std::thread::hardware_concurrency()) {
  if (threads_ == 0) threads_ = 1;
}

EnsembleResult LocalRunner::run(std::size_t realizations, std::span<const std::string> columns,
                                const RealizationJob& job) {
  if (realizations == 0) throw std::invalid_argument("an ensemble needs at least one realisation");
  std::vector<VectorRecorder> per(realizations);
  std::atomic<std::size_t> next{0};
  std::mutex failureMutex;
  std::exception_ptr failure;
  const std::size_t workers = std::min(threads_, realizations);
  {
    std::vector<std::jthread> pool;
    for (std::size_t w = 0; w < workers; ++w) {
      pool.emplace_back([&] {
        for (;;) {
          const std::size_t index = next.fetch_add(1);
          if (index >= realizations) return;
          try {
            job(index, per[index]);
          } catch (...) {
            const std::lock_guard lock(failureMutex);
            if (!failure) failure = std::current_exception();
            next.store(realizations);
            return;
          }
        }
      });
    }
  }
  if (failure) std::rethrow_exception(failure);
  EnsembleResult result;
  result.times = per.front().times();
  result.columns.assign(columns.begin(), columns.end());
  const std::size_t points = result.times.size();
  const std::size_t width = points * result.columns.size();
  result.statistics = Accumulator(width);
  for (std::size_t i = 0; i < realizations; ++i) {
    const VectorRecorder& r = per[i];
    if (r.rows() != points || r.values().size() != width) {
      throw std::runtime_error(std::format(
          "realisation {} recorded {} points and {} values; expected {} and {}", i, r.rows(),
          r.values().size(), points, width));
    }
    result.statistics.add(r.values());
  }
  return result;
}

EnsembleResult foldRows(std::size_t realizations, const std::vector<double>& times,
                        std::span<const std::string> columns, const std::vector<double>& rows) {
  EnsembleResult result;
  result.times = times;
  result.columns.assign(columns.begin(), columns.end());
  const std::size_t width = times.size() * result.columns.size();
  if (rows.size() != realizations * width) {
    throw std::runtime_error("batched rows do not match the measurement shape");
  }
  result.statistics = Accumulator(width);
  for (std::size_t i = 0; i < realizations; ++i) {
    result.statistics.add(std::span<const double>(rows.data() + i * width, width));
  }
  return result;
}

}  // namespace spinsim
