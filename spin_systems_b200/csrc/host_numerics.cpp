// Host FP64 numerics; see host_numerics.hpp.  Compiled with
// -ffp-contract=off so no multiply-add is fused and every value matches the
// reference's build bit for bit.
#include "host_numerics.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numbers>
#include <string>

#include "common_host.hpp"

namespace ss {

double Stream::gaussian() {
  if (has_spare_) {
    has_spare_ = false;
    return spare_;
  }
  constexpr double kFloor = 1.0e-15;
  const double u = kFloor + (1.0 - 2.0 * kFloor) * uniform();
  const double v = uniform();
  const double radius = std::sqrt(-2.0 * std::log(u));
  const double phase = 2.0 * std::numbers::pi * v;
  spare_ = radius * std::sin(phase);
  has_spare_ = true;
  return radius * std::cos(phase);
}

std::vector<PairTerm> dipolar_lattice_2d(int nspins, Stream& rng, double scale,
                                         double min_separation) {
  host_require(nspins >= 1, SS_ERR_INVALID_ARGUMENT, "need at least one spin");
  const double half = 0.5 * std::sqrt(static_cast<double>(nspins));
  std::vector<double> x(static_cast<size_t>(nspins), 0.0), y(static_cast<size_t>(nspins), 0.0);
  std::vector<PairTerm> out;
  out.reserve(static_cast<size_t>(nspins) * static_cast<size_t>(nspins - 1) / 2);
  for (int i = 1; i < nspins; ++i) {
    double px = 0.0, py = 0.0;
    for (bool placed = false; !placed;) {
      px = half * (2.0 * rng.uniform() - 1.0);
      py = half * (2.0 * rng.uniform() - 1.0);
      placed = true;
      for (int j = 0; j < i; ++j) {
        // Close in both coordinates at once: the loose test of the original.
        if (std::abs(px - x[j]) < min_separation && std::abs(py - y[j]) < min_separation) {
          placed = false;
          break;
        }
      }
    }
    x[i] = px;
    y[i] = py;
    for (int j = 0; j < i; ++j) {
      const double dx = px - x[j];
      const double dy = py - y[j];
      const double r2 = dx * dx + dy * dy;
      const double jz = scale / (r2 * std::sqrt(r2));
      out.push_back(PairTerm{j, i, -0.5 * jz, -0.5 * jz, jz});
    }
  }
  return out;
}

Draws realization_draws(const ss_run_config& c, uint64_t index) {
  Draws d{c.nspins, c.field_disorder, 1.0};
  const bool any = c.n_spin_choices > 0 || c.disorder_range[1] > c.disorder_range[0] ||
                   c.tau_range[1] > c.tau_range[0];
  if (!any) return d;
  Stream r = Stream::for_realization(c.draw_seed, index);
  if (c.n_spin_choices > 0) {
    int k = static_cast<int>(r.uniform() * static_cast<double>(c.n_spin_choices));
    if (k >= c.n_spin_choices) k = c.n_spin_choices - 1;
    d.nspins = c.spin_choices[k];
  }
  if (c.disorder_range[1] > c.disorder_range[0]) {
    d.sigma = c.disorder_range[0] + (c.disorder_range[1] - c.disorder_range[0]) * r.uniform();
  }
  if (c.tau_range[1] > c.tau_range[0]) {
    d.tau = c.tau_range[0] + (c.tau_range[1] - c.tau_range[0]) * r.uniform();
  }
  return d;
}

namespace {

void normalize_host(std::vector<double>& v) {
  double sum = 0.0;
  for (const double x : v) sum += x * x;
  const double n = std::sqrt(sum);
  host_require(n != 0.0, SS_ERR_DOMAIN, "cannot normalize a zero state");
  const double f = 1.0 / n;
  for (double& x : v) x *= f;
}

}  // namespace

Realization assemble_realization(const ss_run_config& c, uint64_t index) {
  host_require(c.nspins >= 1 && c.nspins <= 30, SS_ERR_OUT_OF_RANGE,
               "number of spins must be in [1, kMaxSpins]");
  const Draws d = realization_draws(c, index);
  host_require(d.nspins >= 1 && d.nspins <= c.nspins, SS_ERR_CONFIG,
               "a drawn spin count exceeds system.spins");
  Realization r;
  r.nspins = d.nspins;
  r.tau_draw = d.tau;
  const int L = d.nspins;
  Stream rng = Stream::for_realization(c.seed, index);
  r.fields.assign(c.base_fields, c.base_fields + 3 * L);
  if (c.generate_geometry) r.pairs = dipolar_lattice_2d(L, rng, c.dipolar_scale);
  if (d.sigma != 0.0) {
    for (int s = 0; s < L; ++s) r.fields[3 * s + 2] += d.sigma * rng.gaussian();
  }
  const size_t n = size_t{1} << L;
  r.psi0.assign(2 * n, 0.0);
  switch (c.initial_state) {
    case SS_INIT_UP:
      r.psi0[2 * (n - 1)] = 1.0;
      break;
    case SS_INIT_DOWN:
      r.psi0[0] = 1.0;
      break;
    case SS_INIT_BASIS:
      host_require(c.basis_index < n, SS_ERR_OUT_OF_RANGE,
                   "basis state index outside the 2^L state space");
      r.psi0[2 * c.basis_index] = 1.0;
      break;
    case SS_INIT_RANDOM_PRODUCT: {
      // Additive: per spin a uniform point on the Bloch sphere, drawn after
      // geometry and fields, cos(t/2)|up> + e^{ip} sin(t/2)|down>.
      std::vector<double> th(static_cast<size_t>(L)), ph(static_cast<size_t>(L));
      for (int s = 0; s < L; ++s) {
        th[s] = std::acos(1.0 - 2.0 * rng.uniform());
        ph[s] = 2.0 * std::numbers::pi * rng.uniform();
      }
      for (size_t k = 0; k < n; ++k) {
        double ar = 1.0, ai = 0.0;
        for (int s = 0; s < L; ++s) {
          double fr, fi;
          if (k & (size_t{1} << s)) {
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
        r.psi0[2 * k] = ar;
        r.psi0[2 * k + 1] = ai;
      }
      normalize_host(r.psi0);
      break;
    }
    default:  // random typical state (Ensemble.cpp:40-44)
      for (size_t k = 0; k < n; ++k) {
        r.psi0[2 * k] = rng.gaussian();
        r.psi0[2 * k + 1] = rng.gaussian();
      }
      normalize_host(r.psi0);
      break;
  }
  return r;
}

std::vector<double> bessel(int kind, double x, size_t count, size_t* nonzero) {
  host_require(count > 0, SS_ERR_INVALID_ARGUMENT, "Bessel sequence length must be positive");
  host_require(x >= 0.0, SS_ERR_INVALID_ARGUMENT, "Bessel argument must be non-negative");
  std::vector<double> v(count, 0.0);
  if (x == 0.0) {
    v[0] = 1.0;
    if (nonzero) *nonzero = 1;
    return v;
  }
  host_require(!(kind == 1 && x > 709.0), SS_ERR_OVERFLOW, "unscaled modified Bessel I overflows");
  // Miller's backward recurrence from far above both the order and the
  // argument, rescaled near the top of the double range, normalised by
  // J0 + 2(J2 + J4 + ...) = 1 or I0 + 2(I1 + I2 + ...) = e^x.
  const double top = std::max(static_cast<double>(count), std::ceil(x));
  const auto s0 = static_cast<size_t>(top + (40.0 + 6.0 * std::sqrt(top)));
  const size_t start = s0 + (s0 % 2);
  constexpr double kBig = 1.0e250, kInvBig = 1.0e-250;
  double higher = 0.0, current = 1.0e-30, norm = 0.0;
  for (size_t k = start; k >= 1; --k) {
    const double ratio = 2.0 * static_cast<double>(k) / x;
    const double lower = kind == 0 ? ratio * current - higher : ratio * current + higher;
    higher = current;
    current = lower;
    if (kind == 0) {
      if (k % 2 == 1) norm += 2.0 * current;
    } else {
      norm += 2.0 * current;
    }
    if (std::abs(current) > kBig) {
      current *= kInvBig;
      higher *= kInvBig;
      norm *= kInvBig;
      for (double& e : v) e *= kInvBig;
    }
    if (k - 1 < count) v[k - 1] = current;
  }
  norm -= current;
  host_require(norm != 0.0 && std::isfinite(norm), SS_ERR_RUNTIME,
               "Bessel recurrence failed to normalise");
  const double scale = kind == 0 ? 1.0 / norm : std::exp(x) / norm;
  for (double& e : v) e *= scale;
  if (nonzero) {
    size_t n = count;
    while (n > 0 && v[n - 1] == 0.0) --n;
    *nonzero = n;
  }
  return v;
}

Expansion chebyshev(int mode, double bound, double tau, double eps, size_t max_order) {
  host_require(bound >= 0.0, SS_ERR_INVALID_ARGUMENT, "spectral bound must be non-negative");
  host_require(eps > 0.0, SS_ERR_INVALID_ARGUMENT, "epsilon must be positive");
  Expansion out;
  const double alpha = bound * std::abs(tau);
  if (alpha < 2.0 * eps) {  // identity to the requested accuracy
    out.a = {1.0};
    out.bound = 1.0;
    return out;
  }
  const size_t want = static_cast<size_t>(1.5 * alpha) + 64;
  const size_t count = std::min(want, max_order + 3 + 1);
  const std::vector<double> seq = bessel(mode == SS_TIME_IMAGINARY ? 1 : 0, alpha, count, nullptr);
  // First i >= 1 with a_i, a_i+1, a_i+2 all <= eps and strictly decreasing.
  size_t tail = std::string::npos;
  if (seq.size() >= 4) {
    for (size_t i = 1; i + 2 < seq.size(); ++i) {
      const double p = std::abs(seq[i]), q = std::abs(seq[i + 1]), r = std::abs(seq[i + 2]);
      if (p <= eps && q <= eps && r <= eps && q < p && r < q) {
        tail = i;
        break;
      }
    }
  }
  if (tail == std::string::npos || tail - 1 > max_order) {
    char msg[320];
    std::snprintf(msg, sizeof msg,
                  "Chebyshev expansion did not converge: |H| <= %g, tau = %g, alpha = %g, "
                  "epsilon = %g, order tried = %zu. Shorten the time step or raise epsilon.",
                  bound, tau, alpha, eps, count);
    host_fail(SS_ERR_CONVERGENCE, msg);
  }
  out.a.assign(seq.begin(), seq.begin() + static_cast<std::ptrdiff_t>(tail));
  out.bound = bound;
  if (tau < 0.0) {  // J_n(-a) = (-1)^n J_n(a)
    for (size_t n = 1; n < out.a.size(); n += 2) out.a[n] = -out.a[n];
  }
  return out;
}

double spectral_bound(int nspins, const double* f, const std::vector<PairTerm>& pairs) {
  double b = 0.0;
  for (int s = 0; s < nspins; ++s) {
    b += 0.5 * (std::abs(f[3 * s]) + std::abs(f[3 * s + 1]) + std::abs(f[3 * s + 2]));
  }
  for (const PairTerm& p : pairs) b += 0.25 * (std::abs(p.jx) + std::abs(p.jy) + std::abs(p.jz));
  return b;
}

std::vector<double> series_weights(const Expansion& e, int mode) {
  std::vector<double> c(2 * e.a.size(), 0.0);
  c[0] = e.a[0];
  double wr = mode == SS_TIME_REAL ? 0.0 : -1.0;
  double wi = mode == SS_TIME_REAL ? -1.0 : 0.0;
  for (size_t n = 1; n < e.a.size(); ++n) {
    c[2 * n] = 2.0 * e.a[n] * wr;
    c[2 * n + 1] = 2.0 * e.a[n] * wi;
    if (mode == SS_TIME_REAL) {  // multiply by -i
      const double r0 = wr;
      wr = wi;
      wi = -r0;
    } else {
      wr = -wr;
      wi = -wi;
    }
  }
  return c;
}

int64_t measurement_count(const ss_step* steps, int begin, int end) {
  int64_t total = 0;
  for (int at = begin; at < end;) {
    if (steps[at].kind == SS_STEP_MEASURE) {
      ++total;
      ++at;
    } else if (steps[at].kind == SS_STEP_REPEAT) {
      total += steps[at].count * measurement_count(steps, at + 1, at + 1 + steps[at].body_len);
      at += 1 + steps[at].body_len;
    } else {
      ++at;
    }
  }
  return total;
}

int64_t observable_width(const ss_observable* obs, int n) {
  int64_t w = 0;
  for (int i = 0; i < n; ++i) w += (obs[i].kind == SS_OBS_CORR || obs[i].kind == SS_OBS_NORM) ? 2 : 1;
  return w;
}

}  // namespace ss
