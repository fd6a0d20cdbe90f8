// The spinsim C++ core API over the device C ABI: StateVector, Pauli kernels,
// Hamiltonian, Bessel, Chebyshev, Propagator, gates and observables.  Every
// numerical operation runs on the GPU through include/spinsim_b200.h; this
// layer only keeps host mirrors coherent and maps statuses to exceptions.
#include <cmath>
#include <cstdlib>
#include <format>
#include <numbers>
#include <stdexcept>
#include <string>

#include "spinsim/core/Bessel.hpp"
#include "spinsim/core/Chebyshev.hpp"
#include "spinsim/core/Device.hpp"
#include "spinsim/core/Gate.hpp"
#include "spinsim/core/Hamiltonian.hpp"
#include "spinsim/core/Observable.hpp"
#include "spinsim/core/Propagator.hpp"
#include "spinsim/core/SpinOperators.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

// ------------------------------------------------------------------ device
namespace {

struct EngineHolder {
  ss_engine* engine = nullptr;
  ~EngineHolder() {
    if (engine) ss_engine_destroy(engine);
  }
};

}  // namespace

ss_engine* threadEngine() {
  thread_local EngineHolder holder;
  if (!holder.engine) {
    const char* dev = std::getenv("SPINSIM_DEVICE");
    checkStatus(ss_engine_create(dev ? std::atoi(dev) : 0, &holder.engine));
  }
  return holder.engine;
}

void checkStatus(int status) {
  if (status == SS_OK) return;
  const std::string msg = ss_last_error();
  switch (status) {
    case SS_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case SS_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
    case SS_ERR_DOMAIN: throw std::domain_error(msg);
    case SS_ERR_OVERFLOW: throw std::overflow_error(msg);
    case SS_ERR_CONVERGENCE: throw ChebyshevConvergenceError(msg.c_str(), 0.0, 0.0, 0.0, 0);
    default: throw std::runtime_error(msg);
  }
}

// ------------------------------------------------------------- StateVector
StateVector::StateVector(std::size_t nspins) : nspins_(nspins) {
  if (nspins == 0 || nspins > kMaxSpins) {
    throw std::out_of_range("number of spins must be in [1, kMaxSpins]");
  }
  host_.assign(2 * size(), 0.0);
  checkStatus(ss_state_create(threadEngine(), static_cast<int>(nspins), &dev_));
  where_ = Where::Both;
}

StateVector::StateVector(const StateVector& other) : nspins_(other.nspins_) {
  if (!nspins_) return;
  checkStatus(ss_state_create(threadEngine(), static_cast<int>(nspins_), &dev_));
  if (other.where_ == Where::Host) {
    host_ = other.host_;
    where_ = Where::Host;
  } else {
    checkStatus(ss_state_copy(dev_, other.dev_));
    host_ = other.host_;
    where_ = other.where_ == Where::Both ? Where::Both : Where::Device;
  }
}

StateVector& StateVector::operator=(const StateVector& other) {
  if (this == &other) return *this;
  StateVector tmp(other);
  swap(tmp);
  return *this;
}

StateVector::StateVector(StateVector&& other) noexcept
    : nspins_(other.nspins_), dev_(other.dev_), host_(std::move(other.host_)),
      where_(other.where_) {
  other.dev_ = nullptr;
  other.nspins_ = 0;
}

StateVector& StateVector::operator=(StateVector&& other) noexcept {
  swap(other);
  return *this;
}

StateVector::~StateVector() {
  if (dev_) ss_state_destroy(dev_);
}

double* StateVector::data() {
  if (where_ == Where::Device) checkStatus(ss_state_download(dev_, host_.data()));
  where_ = Where::Host;
  return host_.data();
}

const double* StateVector::data() const {
  if (where_ == Where::Device) {
    checkStatus(ss_state_download(dev_, host_.data()));
    where_ = Where::Both;
  }
  return host_.data();
}

ss_state* StateVector::device() const {
  if (!dev_) throw std::invalid_argument("empty state vector");
  if (where_ == Where::Host) {
    checkStatus(ss_state_upload(dev_, host_.data()));
    where_ = Where::Both;
  }
  return dev_;
}

void StateVector::setZero() {
  checkStatus(ss_state_set_zero(device()));
  deviceWritten();
}

void StateVector::scale(double factor) {
  checkStatus(ss_state_scale(device(), factor));
  deviceWritten();
}

void StateVector::negate() {
  checkStatus(ss_state_negate(device()));
  deviceWritten();
}

void StateVector::addScaled(double cr, double ci, const StateVector& other) {
  checkStatus(ss_state_add_scaled(device(), cr, ci, other.device()));
  deviceWritten();
}

void StateVector::setBasisState(std::size_t index) {
  checkStatus(ss_state_set_basis(device(), index));
  deviceWritten();
}

double StateVector::norm() const {
  double n = 0.0;
  checkStatus(ss_state_norm(device(), &n));
  return n;
}

double StateVector::normalize() {
  double n = 0.0;
  checkStatus(ss_state_normalize(device(), &n));
  deviceWritten();
  return n;
}

std::pair<double, double> StateVector::innerProduct(const StateVector& other) const {
  double out[2];
  checkStatus(ss_state_inner_product(device(), other.device(), out));
  return {out[0], out[1]};
}

void StateVector::swap(StateVector& other) noexcept {
  std::swap(nspins_, other.nspins_);
  std::swap(dev_, other.dev_);
  host_.swap(other.host_);
  std::swap(where_, other.where_);
}

// ----------------------------------------------------------- Pauli kernels
namespace {

void sigma(double c, const StateVector& in, SpinIndex spin, StateVector& out, int axis,
           bool accumulate) {
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  if (accumulate) {
    checkStatus(ss_axpy_sigma(c, in.device(), static_cast<int>(spin), axis, o));
  } else {
    checkStatus(ss_apply_sigma(in.device(), static_cast<int>(spin), axis, o));
  }
  out.deviceWritten();
}

}  // namespace

void axpySigmaX(double c, const StateVector& in, SpinIndex s, StateVector& out) { sigma(c, in, s, out, SS_AXIS_X, true); }
void axpySigmaY(double c, const StateVector& in, SpinIndex s, StateVector& out) { sigma(c, in, s, out, SS_AXIS_Y, true); }
void axpySigmaZ(double c, const StateVector& in, SpinIndex s, StateVector& out) { sigma(c, in, s, out, SS_AXIS_Z, true); }
void applySigmaX(const StateVector& in, SpinIndex s, StateVector& out) { sigma(0.0, in, s, out, SS_AXIS_X, false); }
void applySigmaY(const StateVector& in, SpinIndex s, StateVector& out) { sigma(0.0, in, s, out, SS_AXIS_Y, false); }
void applySigmaZ(const StateVector& in, SpinIndex s, StateVector& out) { sigma(0.0, in, s, out, SS_AXIS_Z, false); }

void axpyCoupling(double jx, double jy, double jz, const StateVector& in, SpinPair pair,
                  StateVector& out) {
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  checkStatus(ss_axpy_coupling(jx, jy, jz, in.device(), static_cast<int>(pair.low()),
                               static_cast<int>(pair.high()), o));
  out.deviceWritten();
}

void axpyDiagonal(double c, std::span<const double> diagonal, const StateVector& in,
                  StateVector& out) {
  if (diagonal.size() != in.size()) throw std::invalid_argument("diagonal does not match the space");
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  checkStatus(ss_axpy_diagonal(c, diagonal.data(), in.device(), o));
  out.deviceWritten();
}

void axpyTransverse(double cx, double cy, const StateVector& in, SpinIndex spin,
                    StateVector& out) {
  // (cx sx + cy sy) in one operator: the x part, then the y part.
  axpySigmaX(cx, in, spin, out);
  axpySigmaY(cy, in, spin, out);
}

void axpyFlipFlop(double c, const StateVector& in, SpinPair pair, StateVector& out) {
  // |ud> <-> |du| with weight c: the coupling kernel with jx = jy = c/2, jz = 0.
  axpyCoupling(0.5 * c, 0.5 * c, 0.0, in, pair, out);
}

void axpyFlipBoth(double c, const StateVector& in, SpinPair pair, StateVector& out) {
  // |dd> <-> |uu| with weight c: jx = c/2, jy = -c/2.
  axpyCoupling(0.5 * c, -0.5 * c, 0.0, in, pair, out);
}

// ------------------------------------------------------------- Hamiltonian
Hamiltonian::Hamiltonian(std::size_t nspins) : nspins_(nspins), fields_(nspins) {
  if (nspins == 0 || nspins > kMaxSpins) {
    throw std::out_of_range("number of spins must be in [1, kMaxSpins]");
  }
}

Hamiltonian::Hamiltonian(const Hamiltonian& other)
    : nspins_(other.nspins_), fields_(other.fields_), couplings_(other.couplings_) {}

Hamiltonian& Hamiltonian::operator=(const Hamiltonian& other) {
  if (this != &other) {
    nspins_ = other.nspins_;
    fields_ = other.fields_;
    couplings_ = other.couplings_;
    if (dev_) ss_ham_destroy(dev_);
    dev_ = nullptr;
    dirty_ = true;
  }
  return *this;
}

Hamiltonian::~Hamiltonian() {
  if (dev_) ss_ham_destroy(dev_);
}

void Hamiltonian::setField(SpinIndex spin, Field field) {
  if (spin >= nspins_) throw std::out_of_range("spin index out of range");
  fields_[spin] = field;
  dirty_ = true;
}

const Field& Hamiltonian::field(SpinIndex spin) const {
  if (spin >= nspins_) throw std::out_of_range("spin index out of range");
  return fields_[spin];
}

void Hamiltonian::setCoupling(SpinPair pair, double jx, double jy, double jz) {
  if (pair.high() >= nspins_) throw std::out_of_range("coupled spin index out of range");
  for (Coupling& c : couplings_) {
    if (c.pair == pair) {
      c.jx = jx;
      c.jy = jy;
      c.jz = jz;
      dirty_ = true;
      return;
    }
  }
  couplings_.push_back(Coupling{pair, jx, jy, jz});
  dirty_ = true;
}

double Hamiltonian::spectralBound() const noexcept {
  double bound = 0.0;
  for (const Field& f : fields_) bound += 0.5 * (std::abs(f.x) + std::abs(f.y) + std::abs(f.z));
  for (const Coupling& c : couplings_) {
    bound += 0.25 * (std::abs(c.jx) + std::abs(c.jy) + std::abs(c.jz));
  }
  return bound;
}

ss_ham* Hamiltonian::device() const {
  if (!dev_) checkStatus(ss_ham_create(threadEngine(), static_cast<int>(nspins_), &dev_));
  if (dirty_) {
    std::vector<double> f(3 * nspins_);
    for (std::size_t s = 0; s < nspins_; ++s) {
      f[3 * s] = fields_[s].x;
      f[3 * s + 1] = fields_[s].y;
      f[3 * s + 2] = fields_[s].z;
    }
    std::vector<int32_t> pairs;
    std::vector<double> J;
    for (const Coupling& c : couplings_) {
      pairs.push_back(static_cast<int32_t>(c.pair.low()));
      pairs.push_back(static_cast<int32_t>(c.pair.high()));
      J.insert(J.end(), {c.jx, c.jy, c.jz});
    }
    checkStatus(ss_ham_set_terms(dev_, f.data(), static_cast<int>(couplings_.size()),
                                 pairs.data(), J.data()));
    dirty_ = false;
  }
  return dev_;
}

void Hamiltonian::applyPhysical(const StateVector& in, StateVector& out) const {
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  checkStatus(ss_ham_apply(device(), 1.0, in.device(), o, 0));
  out.deviceWritten();
}

void Hamiltonian::applyTwiceNormalized(double bound, const StateVector& in, StateVector& out) const {
  if (!(bound > 0.0)) throw std::domain_error("spectral bound must be positive");
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  checkStatus(ss_ham_apply(device(), -2.0 / bound, in.device(), o, 0));
  out.deviceWritten();
}

void Hamiltonian::accumulateTwiceNormalized(double bound, const StateVector& in,
                                            StateVector& out) const {
  if (!(bound > 0.0)) throw std::domain_error("spectral bound must be positive");
  if (&in == &out) throw std::invalid_argument("kernels require distinct input and output");
  ss_state* o = out.device();
  checkStatus(ss_ham_apply(device(), -2.0 / bound, in.device(), o, 1));
  out.deviceWritten();
}

// ----------------------------------------------------------------- Bessel
namespace {

BesselSequence bessel(int kind, double x, std::size_t count) {
  BesselSequence out;
  out.values.assign(count, 0.0);
  int64_t nz = 0;
  checkStatus(ss_bessel(kind, x, static_cast<int64_t>(count), out.values.data(), &nz));
  out.nonzero = static_cast<std::size_t>(nz);
  return out;
}

}  // namespace

BesselSequence besselJ(double x, std::size_t count) { return bessel(0, x, count); }
BesselSequence besselI(double x, std::size_t count) { return bessel(1, x, count); }

// -------------------------------------------------------------- Chebyshev
ChebyshevConvergenceError::ChebyshevConvergenceError(double spectralBound, double tau,
                                                     double epsilon, std::size_t attemptedOrder)
    : std::runtime_error(std::format(
          "Chebyshev expansion did not converge: |H| <= {:g}, tau = {:g}, alpha = {:g}, "
          "epsilon = {:g}, order tried = {}. Shorten the time step or raise epsilon.",
          spectralBound, tau, spectralBound * std::abs(tau), epsilon, attemptedOrder)),
      bound_(spectralBound), tau_(tau), epsilon_(epsilon), order_(attemptedOrder) {}

ChebyshevConvergenceError::ChebyshevConvergenceError(const char* message, double spectralBound,
                                                     double tau, double epsilon,
                                                     std::size_t attemptedOrder)
    : std::runtime_error(message), bound_(spectralBound), tau_(tau), epsilon_(epsilon),
      order_(attemptedOrder) {}

ChebyshevExpansion ChebyshevExpansion::build(TimeMode mode, double spectralBound, double tau,
                                             double epsilon, std::size_t maxOrder) {
  std::vector<double> a(maxOrder + 8);
  int64_t order = 0;
  double bound = 1.0;
  const int rc = ss_chebyshev_build(mode == TimeMode::Real ? SS_TIME_REAL : SS_TIME_IMAGINARY,
                                    spectralBound, tau, epsilon, static_cast<int64_t>(maxOrder),
                                    a.data(), static_cast<int64_t>(a.size()), &order, &bound);
  if (rc == SS_ERR_CONVERGENCE) {
    const double alpha = spectralBound * std::abs(tau);
    throw ChebyshevConvergenceError(
        spectralBound, tau, epsilon,
        std::min(static_cast<std::size_t>(1.5 * alpha) + 64, maxOrder + 4));
  }
  checkStatus(rc);
  ChebyshevExpansion out;
  out.coefficients_.assign(a.begin(), a.begin() + order + 1);
  out.bound_ = bound;
  return out;
}

// ------------------------------------------------------------- Propagator
Propagator::Propagator(std::size_t nspins, double epsilon) : nspins_(nspins), epsilon_(epsilon) {
  if (!(epsilon > 0.0)) throw std::invalid_argument("epsilon must be positive");
}

void Propagator::evolve(const Hamiltonian& hamiltonian, TimeMode mode, StateVector& psi,
                        double tau, std::size_t nsteps, bool autonormalize) {
  if (psi.nspins() != hamiltonian.nspins()) {
    throw std::invalid_argument("state and Hamiltonian disagree on spin count");
  }
  if (psi.nspins() != nspins_) {
    throw std::invalid_argument("state does not match the propagator's size");
  }
  if (nsteps == 0) return;
  const ChebyshevExpansion e =
      ChebyshevExpansion::build(mode, hamiltonian.spectralBound(), tau, epsilon_);
  lastOrder_ = e.order();
  if (e.isIdentity()) return;
  ss_state* d = psi.device();
  checkStatus(ss_evolve(hamiltonian.device(), d, e.coefficients().data(),
                        static_cast<int64_t>(e.coefficients().size()), e.effectiveBound(),
                        mode == TimeMode::Real ? SS_TIME_REAL : SS_TIME_IMAGINARY,
                        static_cast<int64_t>(nsteps), autonormalize ? 1 : 0));
  psi.deviceWritten();
}

// ------------------------------------------------------------------ gates
Axis3 Axis3::normalized() const {
  const double length = std::sqrt(x * x + y * y + z * z);
  if (!(length > 0.0)) throw std::invalid_argument("rotation axis must have non-zero length");
  return Axis3{x / length, y / length, z / length};
}

SpinRotation::SpinRotation(Axis3 axis, double angle, std::vector<SpinIndex> targets)
    : axis_(axis.normalized()), angle_(angle), targets_(std::move(targets)) {
  if (targets_.empty()) throw std::invalid_argument("a rotation must name at least one spin");
}

SpinRotation SpinRotation::onAllSpins(Axis3 axis, double angle, std::size_t nspins) {
  std::vector<SpinIndex> all(nspins);
  for (std::size_t s = 0; s < nspins; ++s) all[s] = s;
  return SpinRotation(axis, angle, std::move(all));
}

void SpinRotation::apply(StateVector& psi) const {
  const double ax[3] = {axis_.x, axis_.y, axis_.z};
  double u[8];
  checkStatus(ss_rotation_matrix(ax, angle_, u));
  std::vector<int32_t> t;
  for (const SpinIndex s : targets_) {
    if (s >= psi.nspins()) throw std::out_of_range("rotation names a spin outside the system");
    t.push_back(static_cast<int32_t>(s));
  }
  checkStatus(ss_rotate(psi.device(), u, t.data(), static_cast<int32_t>(t.size())));
  psi.deviceWritten();
}

TwoSpinGate::TwoSpinGate(Matrix matrix, SpinPair pair) : matrix_(matrix), pair_(pair) {}

void TwoSpinGate::apply(StateVector& psi) const {
  if (pair_.high() >= psi.nspins()) throw std::out_of_range("gate names a spin outside the system");
  double m[32];
  for (int i = 0; i < 16; ++i) {
    m[2 * i] = matrix_[static_cast<std::size_t>(i)].real();
    m[2 * i + 1] = matrix_[static_cast<std::size_t>(i)].imag();
  }
  checkStatus(ss_two_spin_gate(psi.device(), m, static_cast<int>(pair_.low()),
                               static_cast<int>(pair_.high())));
  psi.deviceWritten();
}

double TwoSpinGate::unitarityDefect() const {
  double worst = 0.0;
  for (std::size_t r = 0; r < 4; ++r) {
    for (std::size_t c = 0; c < 4; ++c) {
      std::complex<double> acc{0.0, 0.0};
      for (std::size_t k = 0; k < 4; ++k) acc += std::conj(matrix_[k * 4 + r]) * matrix_[k * 4 + c];
      const std::complex<double> want = r == c ? 1.0 : 0.0;
      worst = std::max(worst, std::abs(acc - want));
    }
  }
  return worst;
}

namespace {

std::vector<std::string_view> splitColon(std::string_view spec) {
  std::vector<std::string_view> parts;
  std::size_t start = 0;
  for (;;) {
    const std::size_t sep = spec.find(':', start);
    if (sep == std::string_view::npos) {
      parts.push_back(spec.substr(start));
      return parts;
    }
    parts.push_back(spec.substr(start, sep - start));
    start = sep + 1;
  }
}

bool parseIndex(std::string_view text, unsigned long& out) {
  if (text.empty()) return false;
  out = 0;
  for (const char ch : text) {
    if (ch < '0' || ch > '9') return false;
    out = out * 10 + static_cast<unsigned long>(ch - '0');
  }
  return true;
}

}  // namespace

SpinRotation makeRotation(std::string_view spec, std::size_t nspins) {
  const auto parts = splitColon(spec);
  if (parts.size() != 2 && parts.size() != 3) {
    throw std::invalid_argument(std::format(
        "malformed pulse '{}'; expected <angle>:<axis> or <angle>:<axis>:<spin>", spec));
  }
  double angle = 0.0;
  if (parts[0] == "pi") angle = std::numbers::pi;
  else if (parts[0] == "pi/2") angle = 0.5 * std::numbers::pi;
  else if (parts[0] == "pi/4") angle = 0.25 * std::numbers::pi;
  else throw std::invalid_argument(std::format("unknown pulse angle '{}'; expected pi, pi/2 or pi/4", parts[0]));
  Axis3 axis;
  if (parts[1] == "x") axis = Axis3{1.0, 0.0, 0.0};
  else if (parts[1] == "y") axis = Axis3{0.0, 1.0, 0.0};
  else if (parts[1] == "z") axis = Axis3{0.0, 0.0, 1.0};
  else throw std::invalid_argument(std::format("unknown rotation axis '{}'; expected x, y or z", parts[1]));
  if (parts.size() == 2) return SpinRotation::onAllSpins(axis, angle, nspins);
  unsigned long index = 0;
  if (!parseIndex(parts[2], index) || index == 0 || index > nspins) {
    throw std::invalid_argument(std::format("pulse '{}': spin must be between 1 and {}", spec, nspins));
  }
  return SpinRotation(axis, angle, {static_cast<SpinIndex>(index - 1)});
}

// ------------------------------------------------------------ observables
Axis parseAxis(std::string_view name) {
  if (name == "x" || name == "X") return Axis::X;
  if (name == "y" || name == "Y") return Axis::Y;
  if (name == "z" || name == "Z") return Axis::Z;
  throw std::invalid_argument(std::format("unknown axis '{}'; expected x, y or z", name));
}

std::string_view axisName(Axis axis) {
  switch (axis) {
    case Axis::X: return "x";
    case Axis::Y: return "y";
    case Axis::Z: return "z";
  }
  return "?";
}

namespace {

int axisCode(Axis a) { return a == Axis::X ? SS_AXIS_X : a == Axis::Y ? SS_AXIS_Y : SS_AXIS_Z; }

void requireStates(const MeasureContext& ctx, bool needsReference) {
  if (ctx.state == nullptr) throw std::invalid_argument("measurement context has no state");
  if (needsReference && ctx.reference == nullptr) {
    throw std::invalid_argument("this observable needs a reference state");
  }
}

}  // namespace

std::string TotalSpinCorrelator::name() const { return std::format("corr:{}", axisName(axis_)); }

std::vector<std::string> TotalSpinCorrelator::columns() const {
  return {std::format("corr_{}_re", axisName(axis_)), std::format("corr_{}_im", axisName(axis_))};
}

void TotalSpinCorrelator::measure(const MeasureContext& ctx, std::span<double> out) const {
  requireStates(ctx, true);
  double v[2];
  checkStatus(ss_measure_corr(ctx.state->device(), ctx.reference->device(), axisCode(axis_), v));
  out[0] = v[0];
  out[1] = v[1];
}

std::string SingleSpinMagnetization::name() const {
  return std::format("mag:{}:{}", spin_ + 1, axisName(axis_));
}

std::vector<std::string> SingleSpinMagnetization::columns() const {
  return {std::format("mag_{}_{}", spin_ + 1, axisName(axis_))};
}

void SingleSpinMagnetization::measure(const MeasureContext& ctx, std::span<double> out) const {
  requireStates(ctx, false);
  if (spin_ >= ctx.state->nspins()) {
    throw std::out_of_range("observable names a spin outside the system");
  }
  checkStatus(ss_measure_mag(ctx.state->device(), static_cast<int>(spin_), axisCode(axis_), &out[0]));
}

std::vector<std::string> StateNorms::columns() const { return {"norm_state", "norm_reference"}; }

void StateNorms::measure(const MeasureContext& ctx, std::span<double> out) const {
  requireStates(ctx, true);
  out[0] = ctx.state->norm();
  out[1] = ctx.reference->norm();
}

std::vector<std::string> Energy::columns() const { return {"energy"}; }

void Energy::measure(const MeasureContext& ctx, std::span<double> out) const {
  requireStates(ctx, false);
  if (ctx.hamiltonian == nullptr) throw std::invalid_argument("energy needs a Hamiltonian in the context");
  checkStatus(ss_measure_energy(ctx.hamiltonian->device(), ctx.state->device(), &out[0]));
}

std::unique_ptr<Observable> makeObservable(std::string_view spec) {
  const auto parts = splitColon(spec);
  const auto reject = [&]() -> std::unique_ptr<Observable> {
    throw std::invalid_argument(std::format(
        "unknown observable '{}'; expected one of corr:<axis>, mag:<spin>:<axis>, norm, energy", spec));
  };
  if (parts[0] == "norm" && parts.size() == 1) return std::make_unique<StateNorms>();
  if (parts[0] == "energy" && parts.size() == 1) return std::make_unique<Energy>();
  if (parts[0] == "corr" && parts.size() == 2) {
    return std::make_unique<TotalSpinCorrelator>(parseAxis(parts[1]));
  }
  if (parts[0] == "mag" && parts.size() == 3) {
    unsigned long index = 0;
    if (!parseIndex(parts[1], index) || index == 0) {
      throw std::invalid_argument(std::format("observable '{}': spin must be a positive integer", spec));
    }
    return std::make_unique<SingleSpinMagnetization>(static_cast<SpinIndex>(index - 1),
                                                     parseAxis(parts[2]));
  }
  return reject();
}

}  // namespace spinsim
