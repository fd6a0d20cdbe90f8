/*
 * Test infrastructure -- CPU oracle for the spinsim echo path.  See
 * spinsim_oracle.h.  Never linked into the product.
 *
 * The arithmetic follows the reference operation by operation where the
 * result must agree bit for bit (random streams, geometry, disorder, initial
 * states, Bessel coefficients, expansion order) and pass by pass elsewhere
 * (Hamiltonian application, recurrence, reductions).  Build flags match the
 * reference's (-O2 -ffp-contract=off): no fused multiply-add anywhere.
 */
#define _GNU_SOURCE
#include "spinsim_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static _Thread_local char g_err[512];

static int set_err(int code, const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

const char* orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------ RNG */
/* mt19937_64 (Matsumoto & Nishimura, 2000) as std::mt19937_64 defines it. */
enum { MT_N = 312, MT_M = 156 };
#define MT_MATRIX 0xB5026F5AA96619E9ULL
#define MT_UPPER 0xFFFFFFFF80000000ULL
#define MT_LOWER 0x000000007FFFFFFFULL

void orc_rng_seed(orc_rng* r, uint64_t seed) {
  /* Rng(seed) : engine_(mix(seed))  -- ensemble/Rng.hpp:27 */
  uint64_t z = seed + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  r->mt[0] = z;
  for (int i = 1; i < MT_N; ++i) {
    r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
  }
  r->index = MT_N;
  r->spare = 0.0;
  r->has_spare = 0;
}

static uint64_t splitmix_finalize(uint64_t z) {
  /* ensemble/Rng.hpp:51-56 mix() */
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void orc_rng_for_realization(orc_rng* r, uint64_t base, uint64_t index) {
  /* ensemble/Rng.hpp:30-35 */
  orc_rng_seed(r, splitmix_finalize(base ^ (splitmix_finalize(index + 1) * 0x9E3779B97F4A7C15ULL)));
}

static void mt_twist(orc_rng* r) {
  for (int i = 0; i < MT_N; ++i) {
    const uint64_t x = (r->mt[i] & MT_UPPER) | (r->mt[(i + 1) % MT_N] & MT_LOWER);
    uint64_t xa = x >> 1;
    if (x & 1ULL) xa ^= MT_MATRIX;
    r->mt[i] = r->mt[(i + MT_M) % MT_N] ^ xa;
  }
  r->index = 0;
}

uint64_t orc_rng_next(orc_rng* r) {
  if (r->index >= MT_N) mt_twist(r);
  uint64_t y = r->mt[r->index++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}

double orc_rng_uniform(orc_rng* r) {
  /* ensemble/Rng.hpp:38-41: 53 significant bits */
  return (double)(orc_rng_next(r) >> 11) * 0x1.0p-53;
}

double orc_rng_gaussian(orc_rng* r) {
  /* src/ensemble/Rng.cpp:8-23: Box-Muller, cos returned, sin kept. */
  if (r->has_spare) {
    r->has_spare = 0;
    return r->spare;
  }
  const double floor_ = 1.0e-15;
  const double u = floor_ + (1.0 - 2.0 * floor_) * orc_rng_uniform(r);
  const double v = orc_rng_uniform(r);
  const double radius = sqrt(-2.0 * log(u));
  const double phase = 2.0 * M_PI * v;
  r->spare = radius * sin(phase);
  r->has_spare = 1;
  return radius * cos(phase);
}

void orc_rng_draws(uint64_t seed, uint64_t index, int kind, int64_t n, double* out) {
  orc_rng r;
  orc_rng_for_realization(&r, seed, index);
  for (int64_t i = 0; i < n; ++i) out[i] = kind == 0 ? orc_rng_uniform(&r) : orc_rng_gaussian(&r);
}

/* ------------------------------------------------------------- geometry */
void orc_geometry(int nspins, orc_rng* r, double scale, double min_sep, int32_t* pairs,
                  double* J) {
  /* src/ensemble/Ensemble.cpp:60-104 */
  const double half = 0.5 * sqrt((double)nspins);
  double* x = calloc((size_t)nspins, sizeof(double));
  double* y = calloc((size_t)nspins, sizeof(double));
  int64_t p = 0;
  for (int i = 1; i < nspins; ++i) {
    double px = 0.0, py = 0.0;
    int placed = 0;
    while (!placed) {
      px = half * (2.0 * orc_rng_uniform(r) - 1.0);
      py = half * (2.0 * orc_rng_uniform(r) - 1.0);
      placed = 1;
      for (int j = 0; j < i; ++j) {
        if (fabs(px - x[j]) < min_sep && fabs(py - y[j]) < min_sep) {
          placed = 0;
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
      const double jz = scale / (r2 * sqrt(r2));
      pairs[2 * p] = j;
      pairs[2 * p + 1] = i;
      J[3 * p] = -0.5 * jz;
      J[3 * p + 1] = -0.5 * jz;
      J[3 * p + 2] = jz;
      ++p;
    }
  }
  free(x);
  free(y);
}

/* --------------------------------------------------------------- Bessel */
/* src/core/Bessel.cpp:13-25 start index, :45-96 J, :98-149 I. */
static int64_t bessel_start(double x, int64_t count) {
  const double top = fmax((double)count, ceil(x));
  const double margin = 40.0 + 6.0 * sqrt(top);
  const int64_t start = (int64_t)(top + margin);
  return start + (start % 2);
}

int orc_bessel(int kind, double x, int64_t count, double* out, int64_t* nonzero) {
  if (count == 0) return set_err(SS_ERR_INVALID_ARGUMENT, "Bessel sequence length must be positive");
  if (!(x >= 0.0)) return set_err(SS_ERR_INVALID_ARGUMENT, "Bessel argument must be non-negative");
  for (int64_t i = 0; i < count; ++i) out[i] = 0.0;
  if (x == 0.0) {
    out[0] = 1.0;
    *nonzero = 1;
    return 0;
  }
  if (kind == 1 && x > 709.0) return set_err(SS_ERR_OVERFLOW, "unscaled modified Bessel I overflows");
  const double big = 1.0e250, inv_big = 1.0e-250;
  const int64_t start = bessel_start(x, count);
  double higher = 0.0, current = 1.0e-30, norm = 0.0;
  for (int64_t k = start; k >= 1; --k) {
    const double lower = kind == 0 ? (2.0 * (double)k / x) * current - higher
                                   : (2.0 * (double)k / x) * current + higher;
    higher = current;
    current = lower;
    if (kind == 0) {
      if (k % 2 == 1) norm += 2.0 * current;
    } else {
      norm += 2.0 * current;
    }
    if (fabs(current) > big) {
      current *= inv_big;
      higher *= inv_big;
      norm *= inv_big;
      for (int64_t i = 0; i < count; ++i) out[i] *= inv_big;
    }
    if (k - 1 < count) out[k - 1] = current;
  }
  norm -= current;
  if (norm == 0.0 || !isfinite(norm)) return set_err(SS_ERR_RUNTIME, "Bessel recurrence failed to normalise");
  const double scale = kind == 0 ? 1.0 / norm : exp(x) / norm;
  for (int64_t i = 0; i < count; ++i) out[i] *= scale;
  int64_t n = count;
  while (n > 0 && out[n - 1] == 0.0) --n;
  *nonzero = n;
  return 0;
}

/* ------------------------------------------------------------ Chebyshev */
/* src/core/Chebyshev.cpp:24-35 tail rule, :54-107 build. */
int orc_chebyshev(int mode, double bound, double tau, double eps, int64_t max_order,
                  double* coeffs, int64_t cap, int64_t* order, double* eff_bound) {
  if (!(bound >= 0.0)) return set_err(SS_ERR_INVALID_ARGUMENT, "spectral bound must be non-negative");
  if (!(eps > 0.0)) return set_err(SS_ERR_INVALID_ARGUMENT, "epsilon must be positive");
  const double alpha = bound * fabs(tau);
  if (alpha < 2.0 * eps) {
    if (cap < 1) return set_err(SS_ERR_RUNTIME, "coefficient capacity");
    coeffs[0] = 1.0;
    *order = 0;
    *eff_bound = 1.0;
    return 0;
  }
  const int64_t want = (int64_t)(1.5 * alpha) + 64;
  const int64_t limit = max_order + 3 + 1;
  const int64_t count = want < limit ? want : limit;
  double* seq = malloc(sizeof(double) * (size_t)count);
  int64_t nz = 0;
  const int rc = orc_bessel(mode == SS_TIME_IMAGINARY ? 1 : 0, alpha, count, seq, &nz);
  if (rc) {
    free(seq);
    return rc;
  }
  int64_t tail = -1;
  if (count >= 4) {
    for (int64_t i = 1; i + 2 < count; ++i) {
      const double a = fabs(seq[i]), b = fabs(seq[i + 1]), c = fabs(seq[i + 2]);
      if (a <= eps && b <= eps && c <= eps && b < a && c < b) {
        tail = i;
        break;
      }
    }
  }
  if (tail < 0 || tail - 1 > max_order) {
    free(seq);
    char msg[256];
    snprintf(msg, sizeof msg,
             "Chebyshev expansion did not converge: |H| <= %g, tau = %g, alpha = %g, "
             "epsilon = %g, order tried = %lld.",
             bound, tau, alpha, eps, (long long)count);
    return set_err(SS_ERR_CONVERGENCE, msg);
  }
  if (tail > cap) {
    free(seq);
    return set_err(SS_ERR_RUNTIME, "coefficient capacity");
  }
  for (int64_t i = 0; i < tail; ++i) coeffs[i] = seq[i];
  if (tau < 0.0) {
    for (int64_t i = 1; i < tail; i += 2) coeffs[i] = -coeffs[i];
  }
  *order = tail - 1;
  *eff_bound = bound;
  free(seq);
  return 0;
}

/* ---------------------------------------------------------- Hamiltonian */
double orc_spectral_bound(int nspins, const double* f, int npairs, const double* J) {
  /* src/core/Hamiltonian.cpp:82-93 */
  double b = 0.0;
  for (int s = 0; s < nspins; ++s) b += 0.5 * (fabs(f[3 * s]) + fabs(f[3 * s + 1]) + fabs(f[3 * s + 2]));
  for (int p = 0; p < npairs; ++p) b += 0.25 * (fabs(J[3 * p]) + fabs(J[3 * p + 1]) + fabs(J[3 * p + 2]));
  return b;
}

static const double kNegligible = 1.0e-14; /* Hamiltonian.cpp:16 */

static void build_diagonal(int nspins, const double* f, int npairs, const int32_t* pairs,
                           const double* J, double* d) {
  /* src/core/Hamiltonian.cpp:54-80 */
  const size_t n = (size_t)1 << nspins;
  for (size_t k = 0; k < n; ++k) d[k] = 0.0;
  for (int s = 0; s < nspins; ++s) {
    const double c = 0.5 * f[3 * s + 2];
    if (fabs(c) <= kNegligible) continue;
    const size_t m = (size_t)1 << s;
    for (size_t k = 0; k < n; ++k) d[k] += (k & m) ? c : -c;
  }
  for (int p = 0; p < npairs; ++p) {
    const double c = 0.25 * J[3 * p + 2];
    if (fabs(c) <= kNegligible) continue;
    const size_t mh = (size_t)1 << pairs[2 * p + 1], ml = (size_t)1 << pairs[2 * p];
    for (size_t k = 0; k < n; ++k) {
      const int aligned = ((k & mh) != 0) == ((k & ml) != 0);
      d[k] += aligned ? c : -c;
    }
  }
}

/* out += c * (|first> <-> |second>) over every block of a pair, indices as in
   src/core/SpinOperators.cpp:54-69 (forEachCouplingChannel). */
static void channel(size_t n, int lo, int hi, size_t off1, size_t off2, double c,
                    const double* in, double* out) {
  const size_t mh = (size_t)1 << hi, ml = (size_t)1 << lo;
  for (size_t outer = 0; outer < n; outer += mh << 1) {
    for (size_t mid = outer; mid < outer + mh; mid += ml << 1) {
      for (size_t dd = mid; dd < mid + ml; ++dd) {
        const size_t a = 2 * (dd + off1), b = 2 * (dd + off2);
        out[a] += c * in[b];
        out[a + 1] += c * in[b + 1];
        out[b] += c * in[a];
        out[b + 1] += c * in[a + 1];
      }
    }
  }
}

/* Hamiltonian::accumulate with the diagonal already built (the reference
   caches it, Hamiltonian.hpp:91-109). */
static void ham_accumulate(int nspins, const double* f, int npairs, const int32_t* pairs,
                           const double* J, const double* d, double scale, const double* in,
                           double* out) {
  const size_t n = (size_t)1 << nspins;
  for (size_t k = 0; k < n; ++k) { /* SpinOperators.cpp:211-226 */
    const double g = scale * d[k];
    out[2 * k] += g * in[2 * k];
    out[2 * k + 1] += g * in[2 * k + 1];
  }
  for (int s = 0; s < nspins; ++s) { /* SpinOperators.cpp:228-252 */
    const double cx = scale * 0.5 * f[3 * s];
    const double cy = scale * 0.5 * f[3 * s + 1];
    if (!(fabs(cx) > kNegligible || fabs(cy) > kNegligible)) continue;
    const size_t stride = (size_t)1 << s;
    for (size_t base = 0; base < n; base += stride << 1) {
      for (size_t lo = base; lo < base + stride; ++lo) {
        const size_t l = 2 * lo, h = 2 * (lo + stride);
        const double ar = in[l], ai = in[l + 1], br = in[h], bi = in[h + 1];
        out[l] += cx * br - cy * bi;
        out[l + 1] += cx * bi + cy * br;
        out[h] += cx * ar + cy * ai;
        out[h + 1] += cx * ai - cy * ar;
      }
    }
  }
  for (int p = 0; p < npairs; ++p) { /* Hamiltonian.cpp:115-126 */
    const double quarter = scale * 0.25;
    const double ff = quarter * (J[3 * p] + J[3 * p + 1]);
    const double fb = quarter * (J[3 * p] - J[3 * p + 1]);
    const int lo = pairs[2 * p] < pairs[2 * p + 1] ? pairs[2 * p] : pairs[2 * p + 1];
    const int hi = pairs[2 * p] < pairs[2 * p + 1] ? pairs[2 * p + 1] : pairs[2 * p];
    if (fabs(ff) > kNegligible) channel(n, lo, hi, (size_t)1 << hi, (size_t)1 << lo, ff, in, out);
    if (fabs(fb) > kNegligible) channel(n, lo, hi, 0, ((size_t)1 << hi) + ((size_t)1 << lo), fb, in, out);
  }
}

void orc_ham_apply(int nspins, const double* f, int npairs, const int32_t* pairs,
                   const double* J, double scale, const double* in, double* out,
                   int accumulate) {
  /* src/core/Hamiltonian.cpp:95-127 accumulate; :129-132 applyPhysical */
  const size_t n = (size_t)1 << nspins;
  if (!accumulate) memset(out, 0, sizeof(double) * 2 * n);
  double* d = malloc(sizeof(double) * n);
  build_diagonal(nspins, f, npairs, pairs, J, d);
  ham_accumulate(nspins, f, npairs, pairs, J, d, scale, in, out);
  free(d);
}

/* ----------------------------------------------------------- Propagator */
double orc_norm(int nspins, const double* psi) {
  /* StateVector.cpp:43-49 */
  const size_t n = (size_t)2 << nspins;
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) sum += psi[i] * psi[i];
  return sqrt(sum);
}

void orc_inner(int nspins, const double* a, const double* b, double out[2]) {
  /* StateVector.cpp:58-70: <b|a> */
  const size_t n = (size_t)2 << nspins;
  double re = 0.0, im = 0.0;
  for (size_t k = 0; k < n; k += 2) {
    re += b[k] * a[k] + b[k + 1] * a[k + 1];
    im += b[k] * a[k + 1] - b[k + 1] * a[k];
  }
  out[0] = re;
  out[1] = im;
}

static int normalize(int nspins, double* psi) {
  const double nrm = orc_norm(nspins, psi);
  if (nrm == 0.0) return set_err(SS_ERR_DOMAIN, "cannot normalize a zero state");
  const double f = 1.0 / nrm;
  const size_t n = (size_t)2 << nspins;
  for (size_t i = 0; i < n; ++i) psi[i] *= f;
  return 0;
}

int orc_evolve(int nspins, const double* f, int npairs, const int32_t* pairs,
               const double* J, double* psi, int mode, double tau, int64_t nsteps,
               int autonorm, double eps, int64_t* order_out) {
  /* src/core/Propagator.cpp:46-100 */
  if (!(eps > 0.0)) return set_err(SS_ERR_INVALID_ARGUMENT, "epsilon must be positive");
  if (nsteps == 0) return 0;
  const double bound_h = orc_spectral_bound(nspins, f, npairs, J);
  const int64_t cap = 6000 + 8;
  double* a = malloc(sizeof(double) * (size_t)cap);
  int64_t order = 0;
  double bound = 1.0;
  int rc = orc_chebyshev(mode, bound_h, tau, eps, 6000, a, cap, &order, &bound);
  if (rc) {
    free(a);
    return rc;
  }
  *order_out = order;
  if (order == 0) {
    free(a);
    return 0;
  }
  const size_t n = (size_t)1 << nspins;
  double* cur = malloc(sizeof(double) * 2 * n);
  double* prev = malloc(sizeof(double) * 2 * n);
  double* diag = malloc(sizeof(double) * n);
  build_diagonal(nspins, f, npairs, pairs, J, diag);
  for (int64_t step = 0; step < nsteps; ++step) {
    memcpy(cur, psi, sizeof(double) * 2 * n);
    for (size_t i = 0; i < 2 * n; ++i) psi[i] *= a[0];
    memset(prev, 0, sizeof(double) * 2 * n);
    double wre = mode == SS_TIME_REAL ? 0.0 : -1.0;
    double wim = mode == SS_TIME_REAL ? -1.0 : 0.0;
    for (int64_t k = 1; k <= order; ++k) {
      for (size_t i = 0; i < 2 * n; ++i) prev[i] = -prev[i];
      if (!(bound > 0.0)) {
        rc = set_err(SS_ERR_DOMAIN, "spectral bound must be positive");
        goto done;
      }
      ham_accumulate(nspins, f, npairs, pairs, J, diag, -2.0 / bound, cur, prev);
      if (k == 1) {
        for (size_t i = 0; i < 2 * n; ++i) prev[i] *= 0.5;
      }
      double* t = prev;
      prev = cur;
      cur = t;
      const double cr = 2.0 * a[k] * wre, ci = 2.0 * a[k] * wim;
      for (size_t i = 0; i < 2 * n; i += 2) { /* StateVector.cpp:20-31 */
        const double orr = cur[i], oi = cur[i + 1];
        psi[i] += cr * orr - ci * oi;
        psi[i + 1] += cr * oi + ci * orr;
      }
      if (mode == SS_TIME_REAL) {
        const double r0 = wre;
        wre = wim;
        wim = -r0;
      } else {
        wre = -wre;
        wim = -wim;
      }
    }
    if (autonorm) {
      rc = normalize(nspins, psi);
      if (rc) goto done;
    }
  }
done:
  free(cur);
  free(prev);
  free(diag);
  free(a);
  return rc;
}

/* ----------------------------------------------------------------- gates */
void orc_rotation_matrix(const double axis[3], double angle, double u[8]) {
  /* src/core/Gate.cpp:20-33 (after Axis3::normalized, :35-42) */
  const double len = sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
  const double nx = axis[0] / len, ny = axis[1] / len, nz = axis[2] / len;
  const double c = cos(0.5 * angle), s = sin(0.5 * angle);
  u[0] = c;       u[1] = s * nz;   /* ll */
  u[2] = s * ny;  u[3] = -s * nx;  /* lh */
  u[4] = -s * ny; u[5] = -s * nx;  /* hl */
  u[6] = c;       u[7] = -s * nz;  /* hh */
}

int orc_rotate(int nspins, double* psi, const double axis[3], double angle,
               const int32_t* targets, int ntargets) {
  /* src/core/Gate.cpp:60-85 */
  const double len = sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
  if (!(len > 0.0)) return set_err(SS_ERR_INVALID_ARGUMENT, "rotation axis must have non-zero length");
  if (ntargets <= 0) return set_err(SS_ERR_INVALID_ARGUMENT, "a rotation must name at least one spin");
  double u[8];
  orc_rotation_matrix(axis, angle, u);
  const size_t n = (size_t)1 << nspins;
  for (int t = 0; t < ntargets; ++t) {
    if (targets[t] < 0 || targets[t] >= nspins) return set_err(SS_ERR_OUT_OF_RANGE, "rotation names a spin outside the system");
    const size_t stride = (size_t)1 << targets[t];
    for (size_t base = 0; base < n; base += stride << 1) {
      for (size_t lo = base; lo < base + stride; ++lo) {
        const size_t hi = lo + stride;
        const double ar = psi[2 * lo], ai = psi[2 * lo + 1];
        const double br = psi[2 * hi], bi = psi[2 * hi + 1];
        const double lr = (u[0] * ar - u[1] * ai) + (u[2] * br - u[3] * bi);
        const double li = (u[0] * ai + u[1] * ar) + (u[2] * bi + u[3] * br);
        const double hr = (u[4] * ar - u[5] * ai) + (u[6] * br - u[7] * bi);
        const double hi_ = (u[4] * ai + u[5] * ar) + (u[6] * bi + u[7] * br);
        psi[2 * lo] = lr;
        psi[2 * lo + 1] = li;
        psi[2 * hi] = hr;
        psi[2 * hi + 1] = hi_;
      }
    }
  }
  return 0;
}

int orc_two_spin_gate(int nspins, double* psi, const double m[32], int a, int b) {
  /* src/core/Gate.cpp:90-121, basis (dd, low-up, high-up, uu) */
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  if (hi >= nspins) return set_err(SS_ERR_OUT_OF_RANGE, "gate names a spin outside the system");
  const size_t n = (size_t)1 << nspins, mh = (size_t)1 << hi, ml = (size_t)1 << lo;
  for (size_t outer = 0; outer < n; outer += mh << 1) {
    for (size_t mid = outer; mid < outer + mh; mid += ml << 1) {
      for (size_t dd = mid; dd < mid + ml; ++dd) {
        const size_t idx[4] = {dd, dd + ml, dd + mh, dd + mh + ml};
        double vr[4], vi[4];
        for (int k = 0; k < 4; ++k) {
          vr[k] = psi[2 * idx[k]];
          vi[k] = psi[2 * idx[k] + 1];
        }
        for (int r = 0; r < 4; ++r) {
          double accr = 0.0, acci = 0.0;
          for (int c = 0; c < 4; ++c) {
            const double mr = m[2 * (r * 4 + c)], mi = m[2 * (r * 4 + c) + 1];
            accr += mr * vr[c] - mi * vi[c];
            acci += mr * vi[c] + mi * vr[c];
          }
          psi[2 * idx[r]] = accr;
          psi[2 * idx[r] + 1] = acci;
        }
      }
    }
  }
  return 0;
}

/* --------------------------------------------------------- Pauli kernels */
void orc_pauli(int nspins, int op, int axis, double c, int spin, int spin_b,
               const double* jxyz, const double* in, double* out) {
  /* src/core/SpinOperators.cpp:90-209 */
  const size_t n = (size_t)1 << nspins;
  if (op == 2) {
    const int lo = spin < spin_b ? spin : spin_b, hi = spin < spin_b ? spin_b : spin;
    const double fboth = jxyz[0] - jxyz[1], fone = jxyz[0] + jxyz[1], jz = jxyz[2];
    const size_t mh = (size_t)1 << hi, ml = (size_t)1 << lo;
    for (size_t outer = 0; outer < n; outer += mh << 1) {
      for (size_t mid = outer; mid < outer + mh; mid += ml << 1) {
        for (size_t dd = mid; dd < mid + ml; ++dd) {
          const size_t d = 2 * dd, a = 2 * (dd + mh), b = 2 * (dd + ml), u = 2 * (dd + mh + ml);
          out[u] += fboth * in[d] + jz * in[u];
          out[u + 1] += fboth * in[d + 1] + jz * in[u + 1];
          out[d] += fboth * in[u] + jz * in[d];
          out[d + 1] += fboth * in[u + 1] + jz * in[d + 1];
          out[a] += fone * in[b] - jz * in[a];
          out[a + 1] += fone * in[b + 1] - jz * in[a + 1];
          out[b] += fone * in[a] - jz * in[b];
          out[b + 1] += fone * in[a + 1] - jz * in[b + 1];
        }
      }
    }
    return;
  }
  const size_t stride = (size_t)1 << spin;
  for (size_t base = 0; base < n; base += stride << 1) {
    for (size_t lo = base; lo < base + stride; ++lo) {
      const size_t l = 2 * lo, h = 2 * (lo + stride);
      if (op == 0) {
        if (axis == 0) {
          out[h] += c * in[l];
          out[h + 1] += c * in[l + 1];
          out[l] += c * in[h];
          out[l + 1] += c * in[h + 1];
        } else if (axis == 1) {
          out[h] += c * in[l + 1];
          out[h + 1] -= c * in[l];
          out[l] -= c * in[h + 1];
          out[l + 1] += c * in[h];
        } else {
          out[h] += c * in[h];
          out[h + 1] += c * in[h + 1];
          out[l] -= c * in[l];
          out[l + 1] -= c * in[l + 1];
        }
      } else {
        if (axis == 0) {
          out[h] = in[l];
          out[h + 1] = in[l + 1];
          out[l] = in[h];
          out[l + 1] = in[h + 1];
        } else if (axis == 1) {
          out[h] = in[l + 1];
          out[h + 1] = -in[l];
          out[l] = -in[h + 1];
          out[l + 1] = in[h];
        } else {
          out[h] = in[h];
          out[h + 1] = in[h + 1];
          out[l] = -in[l];
          out[l + 1] = -in[l + 1];
        }
      }
    }
  }
}

/* ---------------------------------------------------------- observables */
static int obs_width(const ss_observable* o) {
  return o->kind == SS_OBS_CORR || o->kind == SS_OBS_NORM ? 2 : 1;
}

int orc_measure(int nspins, const ss_observable* o, const double* psi, const double* ref,
                const double* f, int npairs, const int32_t* pairs, const double* J,
                double* out) {
  /* src/core/Observable.cpp:66-120 */
  const size_t n = (size_t)1 << nspins;
  double* scratch = calloc(2 * n, sizeof(double));
  double ip[2];
  switch (o->kind) {
    case SS_OBS_CORR:
      for (int s = 0; s < nspins; ++s) orc_pauli(nspins, 0, o->axis, 1.0, s, 0, NULL, psi, scratch);
      orc_inner(nspins, scratch, ref, ip);
      out[0] = ip[0];
      out[1] = ip[1];
      break;
    case SS_OBS_MAG:
      if (o->spin < 0 || o->spin >= nspins) {
        free(scratch);
        return set_err(SS_ERR_OUT_OF_RANGE, "observable names a spin outside the system");
      }
      orc_pauli(nspins, 1, o->axis, 0.0, o->spin, 0, NULL, psi, scratch);
      orc_inner(nspins, scratch, psi, ip);
      out[0] = ip[0];
      break;
    case SS_OBS_NORM:
      out[0] = orc_norm(nspins, psi);
      out[1] = orc_norm(nspins, ref);
      break;
    case SS_OBS_ENERGY:
      orc_ham_apply(nspins, f, npairs, pairs, J, 1.0, psi, scratch, 0);
      orc_inner(nspins, psi, scratch, ip);
      out[0] = ip[0];
      break;
    default:
      free(scratch);
      return set_err(SS_ERR_INVALID_ARGUMENT, "unknown observable");
  }
  free(scratch);
  return 0;
}

/* ------------------------------------------------------ sequence program */
static int64_t count_measures(const ss_step* s, int begin, int end) {
  /* src/sequence/Sequence.cpp:89-100 */
  int64_t total = 0;
  int at = begin;
  while (at < end) {
    if (s[at].kind == SS_STEP_MEASURE) {
      ++total;
      ++at;
    } else if (s[at].kind == SS_STEP_REPEAT) {
      total += s[at].count * count_measures(s, at + 1, at + 1 + s[at].body_len);
      at += 1 + s[at].body_len;
    } else {
      ++at;
    }
  }
  return total;
}

int orc_shape(const ss_run_config* cfg, int64_t* points, int64_t* width) {
  *points = count_measures(cfg->steps, 0, cfg->n_steps);
  int64_t w = 0;
  for (int i = 0; i < cfg->n_observables; ++i) w += obs_width(&cfg->observables[i]);
  *width = w;
  return 0;
}

/* Per-realisation additive draws from the harness stream (draw_seed, index):
   L first (if a list is given), then sigma, then tau. */
typedef struct draws {
  int nspins;
  double sigma;
  double tau;
} draws;

static draws realization_draws(const ss_run_config* c, uint64_t index) {
  draws d = {c->nspins, c->field_disorder, 1.0};
  const int any = c->n_spin_choices > 0 || c->disorder_range[1] > c->disorder_range[0] ||
                  c->tau_range[1] > c->tau_range[0];
  if (!any) return d;
  orc_rng r;
  orc_rng_for_realization(&r, c->draw_seed, index);
  if (c->n_spin_choices > 0) {
    int k = (int)(orc_rng_uniform(&r) * (double)c->n_spin_choices);
    if (k >= c->n_spin_choices) k = c->n_spin_choices - 1;
    d.nspins = c->spin_choices[k];
  }
  if (c->disorder_range[1] > c->disorder_range[0]) {
    d.sigma = c->disorder_range[0] + (c->disorder_range[1] - c->disorder_range[0]) * orc_rng_uniform(&r);
  }
  if (c->tau_range[1] > c->tau_range[0]) {
    d.tau = c->tau_range[0] + (c->tau_range[1] - c->tau_range[0]) * orc_rng_uniform(&r);
  }
  return d;
}

int orc_setup(const ss_run_config* c, uint64_t index, int32_t* nspins_out, double* f,
              int32_t* pairs, double* J, int32_t* npairs, double* psi0, double* ref0) {
  /* io/Experiment.cpp:10-35 */
  const draws d = realization_draws(c, index);
  const int L = d.nspins;
  *nspins_out = L;
  orc_rng r;
  orc_rng_for_realization(&r, c->seed, index);
  for (int s = 0; s < L; ++s) {
    f[3 * s] = c->base_fields[3 * s];
    f[3 * s + 1] = c->base_fields[3 * s + 1];
    f[3 * s + 2] = c->base_fields[3 * s + 2];
  }
  int P = 0;
  if (c->generate_geometry) {
    orc_geometry(L, &r, c->dipolar_scale, 5.0e-2, pairs, J);
    P = L * (L - 1) / 2;
  }
  *npairs = P;
  if (d.sigma != 0.0) { /* Ensemble.cpp:106-112 */
    for (int s = 0; s < L; ++s) f[3 * s + 2] += d.sigma * orc_rng_gaussian(&r);
  }
  const size_t n = (size_t)1 << L;
  memset(psi0, 0, sizeof(double) * 2 * n);
  switch (c->initial_state) { /* Ensemble.cpp:20-45 */
    case SS_INIT_UP: psi0[2 * (n - 1)] = 1.0; break;
    case SS_INIT_DOWN: psi0[0] = 1.0; break;
    case SS_INIT_BASIS:
      if (c->basis_index >= n) return set_err(SS_ERR_OUT_OF_RANGE, "basis state index outside the 2^L state space");
      psi0[2 * c->basis_index] = 1.0;
      break;
    case SS_INIT_RANDOM_PRODUCT: {
      /* additive: per spin a uniform Bloch vector, cos(t/2)|up> +
         e^{i p} sin(t/2)|down>, drawn after geometry and fields */
      double* th = malloc(sizeof(double) * (size_t)L);
      double* ph = malloc(sizeof(double) * (size_t)L);
      for (int s = 0; s < L; ++s) {
        th[s] = acos(1.0 - 2.0 * orc_rng_uniform(&r));
        ph[s] = 2.0 * M_PI * orc_rng_uniform(&r);
      }
      for (size_t k = 0; k < n; ++k) {
        double ar = 1.0, ai = 0.0;
        for (int s = 0; s < L; ++s) {
          double fr, fi;
          if (k & ((size_t)1 << s)) {
            fr = cos(0.5 * th[s]);
            fi = 0.0;
          } else {
            const double sn = sin(0.5 * th[s]);
            fr = sn * cos(ph[s]);
            fi = sn * sin(ph[s]);
          }
          const double nr = ar * fr - ai * fi;
          ai = ar * fi + ai * fr;
          ar = nr;
        }
        psi0[2 * k] = ar;
        psi0[2 * k + 1] = ai;
      }
      free(th);
      free(ph);
      if (normalize(L, psi0)) return SS_ERR_DOMAIN;
      break;
    }
    default:
      for (size_t k = 0; k < n; ++k) {
        psi0[2 * k] = orc_rng_gaussian(&r);
        psi0[2 * k + 1] = orc_rng_gaussian(&r);
      }
      if (normalize(L, psi0)) return SS_ERR_DOMAIN;
      break;
  }
  if (ref0) { /* Ensemble.cpp:47-58 */
    memset(ref0, 0, sizeof(double) * 2 * n);
    for (int s = 0; s < L; ++s) orc_pauli(L, 0, c->reference_axis, 1.0, s, 0, NULL, psi0, ref0);
  }
  return 0;
}

typedef struct run_ctx {
  const ss_run_config* cfg;
  int L;
  double tau_draw;
  double* fields;      /* the realisation's fields */
  double* active;      /* fields in force for the current step */
  int32_t* pairs;
  double* J;
  int npairs;
  double* psi;
  double* ref;
  double time;
  double* times;
  double* values;
  int64_t row;
  int64_t width;
} run_ctx;

static int run_steps(run_ctx* x, int begin, int end) {
  /* src/sequence/Sequence.cpp:35-87 */
  const ss_run_config* c = x->cfg;
  const int L = x->L;
  int at = begin;
  while (at < end) {
    const ss_step* s = &c->steps[at];
    int rc = 0;
    if (s->kind == SS_STEP_EVOLVE) {
      if (s->field_table >= 0) {
        const double* t = c->step_fields + (size_t)3 * (size_t)c->nspins * (size_t)s->field_table;
        memcpy(x->active, t, sizeof(double) * 3 * (size_t)L);
      } else {
        memcpy(x->active, x->fields, sizeof(double) * 3 * (size_t)L);
      }
      const double tau = s->tau_from_draw ? s->tau * x->tau_draw : s->tau;
      int64_t ord = 0;
      rc = orc_evolve(L, x->active, x->npairs, x->pairs, x->J, x->psi, s->mode, tau, s->count,
                      s->autonormalize, c->epsilon, &ord);
      if (!rc) rc = orc_evolve(L, x->active, x->npairs, x->pairs, x->J, x->ref, s->mode, tau,
                               s->count, s->autonormalize, c->epsilon, &ord);
      x->time += tau * (double)s->count;
      ++at;
    } else if (s->kind == SS_STEP_PULSE) {
      int32_t* targets = malloc(sizeof(int32_t) * (size_t)L);
      int nt = 0;
      if (s->target < 0) {
        for (int q = 0; q < L; ++q) targets[nt++] = q;
      } else {
        targets[nt++] = s->target;
      }
      rc = orc_rotate(L, x->psi, s->axis, s->angle, targets, nt);
      if (!rc) rc = orc_rotate(L, x->ref, s->axis, s->angle, targets, nt);
      free(targets);
      ++at;
    } else if (s->kind == SS_STEP_MEASURE) {
      double* row = x->values + x->row * x->width;
      int64_t col = 0;
      for (int i = 0; i < c->n_observables; ++i) {
        rc = orc_measure(L, &c->observables[i], x->psi, x->ref, x->fields, x->npairs,
                         x->pairs, x->J, row + col);
        if (rc) break;
        col += obs_width(&c->observables[i]);
      }
      x->times[x->row] = x->time;
      ++x->row;
      ++at;
    } else if (s->kind == SS_STEP_REPEAT) {
      for (int64_t i = 0; i < s->count && !rc; ++i) rc = run_steps(x, at + 1, at + 1 + s->body_len);
      at += 1 + s->body_len;
    } else {
      rc = set_err(SS_ERR_INVALID_ARGUMENT, "unknown step kind");
    }
    if (rc) return rc;
  }
  return 0;
}

int orc_run_realization(const ss_run_config* c, uint64_t index, double* times, double* values) {
  const int Lmax = c->nspins;
  const size_t nmax = (size_t)1 << Lmax;
  run_ctx x;
  memset(&x, 0, sizeof x);
  x.cfg = c;
  x.fields = malloc(sizeof(double) * 3 * (size_t)Lmax);
  x.active = malloc(sizeof(double) * 3 * (size_t)Lmax);
  x.pairs = malloc(sizeof(int32_t) * (size_t)(Lmax * (Lmax - 1) + 2));
  x.J = malloc(sizeof(double) * (size_t)(3 * Lmax * (Lmax - 1) / 2 + 3));
  x.psi = malloc(sizeof(double) * 2 * nmax);
  x.ref = malloc(sizeof(double) * 2 * nmax);
  int32_t L = 0, P = 0;
  int rc = orc_setup(c, index, &L, x.fields, x.pairs, x.J, &P, x.psi, x.ref);
  if (!rc) {
    x.L = L;
    x.npairs = P;
    x.tau_draw = realization_draws(c, index).tau;
    int64_t points = 0;
    orc_shape(c, &points, &x.width);
    x.times = times;
    x.values = values;
    rc = run_steps(&x, 0, c->n_steps);
  }
  free(x.fields);
  free(x.active);
  free(x.pairs);
  free(x.J);
  free(x.psi);
  free(x.ref);
  return rc;
}

typedef struct range_job {
  const ss_run_config* cfg;
  const uint64_t* indices; /* NULL: first + i */
  uint64_t first;
  int64_t count;
  int64_t points, width;
  double* times;
  double* values;
  int64_t next;
  int rc;
  pthread_mutex_t lock;
} range_job;

static void* range_worker(void* arg) {
  range_job* j = arg;
  double* t = malloc(sizeof(double) * (size_t)(j->points > 0 ? j->points : 1));
  for (;;) {
    pthread_mutex_lock(&j->lock);
    const int64_t i = j->next++;
    const int stop = j->rc != 0;
    pthread_mutex_unlock(&j->lock);
    if (i >= j->count || stop) break;
    const uint64_t index = j->indices ? j->indices[i] : j->first + (uint64_t)i;
    const int rc = orc_run_realization(j->cfg, index, t,
                                       j->values + i * j->points * j->width);
    if (rc) {
      pthread_mutex_lock(&j->lock);
      if (!j->rc) j->rc = rc;
      pthread_mutex_unlock(&j->lock);
      break;
    }
    if (i == 0) memcpy(j->times, t, sizeof(double) * (size_t)j->points);
  }
  free(t);
  return NULL;
}

static int run_job(range_job* j, int threads, double* seconds) {
  orc_shape(j->cfg, &j->points, &j->width);
  pthread_mutex_init(&j->lock, NULL);
  if (threads <= 0) threads = 1;
  pthread_t* pool = malloc(sizeof(pthread_t) * (size_t)threads);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int i = 0; i < threads; ++i) pthread_create(&pool[i], NULL, range_worker, j);
  for (int i = 0; i < threads; ++i) pthread_join(pool[i], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  free(pool);
  pthread_mutex_destroy(&j->lock);
  return j->rc;
}

int orc_run_range(const ss_run_config* c, uint64_t first, int64_t count, int threads,
                  double* times, double* values, double* seconds) {
  range_job j;
  memset(&j, 0, sizeof j);
  j.cfg = c;
  j.first = first;
  j.count = count;
  j.times = times;
  j.values = values;
  return run_job(&j, threads, seconds);
}

int orc_run_indices(const ss_run_config* c, const uint64_t* indices, int64_t count, int threads,
                    double* times, double* values, double* seconds) {
  range_job j;
  memset(&j, 0, sizeof j);
  j.cfg = c;
  j.indices = indices;
  j.count = count;
  j.times = times;
  j.values = values;
  return run_job(&j, threads, seconds);
}

void orc_accumulate(int64_t n, int64_t width, const double* rows, double* mean, double* sd,
                    double* se) {
  /* src/ensemble/Ensemble.cpp:116-166 (Welford, index order) */
  double* m2 = calloc((size_t)width, sizeof(double));
  for (int64_t k = 0; k < width; ++k) mean[k] = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double cnt = (double)(i + 1);
    for (int64_t k = 0; k < width; ++k) {
      const double x = rows[i * width + k];
      const double delta = x - mean[k];
      mean[k] += delta / cnt;
      m2[k] += delta * (x - mean[k]);
    }
  }
  for (int64_t k = 0; k < width; ++k) {
    sd[k] = n < 2 ? 0.0 : sqrt(m2[k] / (double)(n - 1));
    se[k] = n < 2 ? sd[k] : sd[k] * (1.0 / sqrt((double)n));
  }
  free(m2);
}
