/*
 * Test infrastructure -- the CPU oracle for the spinsim echo path.
 *
 * A plain-C restatement of the reference algorithm (BekturMur/Spin_Systems,
 * `spinsim`), written to check the CUDA engine against.  It is never linked
 * into the product: only tests/, the smoke check and bench.py's CPU-baseline
 * leg load liboracle_port.so.  Each function names the reference file:line it
 * follows.  Parity of this port with the reference itself is pinned by
 * tests/test_oracle_pins.py against the reference compiled from its sources
 * (oracle/_ref) and against the reference's golden Bessel tables.
 */
#ifndef SPINSIM_ORACLE_H
#define SPINSIM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/spinsim_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Random stream of one realisation: mt19937_64 + Box-Muller with a spare. */
typedef struct orc_rng {
  uint64_t mt[312];
  int index;
  double spare;
  int has_spare;
} orc_rng;

void orc_rng_seed(orc_rng* r, uint64_t seed);                      /* Rng(seed)            */
void orc_rng_for_realization(orc_rng* r, uint64_t base, uint64_t index);
uint64_t orc_rng_next(orc_rng* r);                                 /* engine_()            */
double orc_rng_uniform(orc_rng* r);
double orc_rng_gaussian(orc_rng* r);
/* kind 0 uniform, 1 gaussian: n draws of realisation (seed, index). */
void orc_rng_draws(uint64_t seed, uint64_t index, int kind, int64_t n, double* out);

/* Dipolar couplings, L(L-1)/2 pairs (low, high) and (jx, jy, jz). */
void orc_geometry(int nspins, orc_rng* r, double scale, double min_sep,
                  int32_t* pairs, double* J);

/* Bessel J / I sequences; returns 0 or an ss_status; *nonzero as in the ref. */
int orc_bessel(int kind, double x, int64_t count, double* out, int64_t* nonzero);

/* ChebyshevExpansion::build; writes order+1 coefficients. */
int orc_chebyshev(int mode, double bound, double tau, double eps, int64_t max_order,
                  double* coeffs, int64_t cap, int64_t* order, double* eff_bound);

double orc_spectral_bound(int nspins, const double* fields, int npairs,
                          const double* J);

/* out = H in (accumulate=0) or out += scale * H in (accumulate=1). */
void orc_ham_apply(int nspins, const double* fields, int npairs, const int32_t* pairs,
                   const double* J, double scale, const double* in, double* out,
                   int accumulate);

/* Propagator::evolve with its own expansion; returns 0 or an ss_status. */
int orc_evolve(int nspins, const double* fields, int npairs, const int32_t* pairs,
               const double* J, double* psi, int mode, double tau, int64_t nsteps,
               int autonorm, double eps, int64_t* order);

/* SpinRotation::apply for an axis (normalised here) and angle. */
int orc_rotate(int nspins, double* psi, const double axis[3], double angle,
               const int32_t* targets, int ntargets);
void orc_rotation_matrix(const double axis[3], double angle, double u[8]);
int orc_two_spin_gate(int nspins, double* psi, const double m[32], int a, int b);

/* Pauli kernels: op 0 axpySigma, 1 applySigma, 2 axpyCoupling. */
void orc_pauli(int nspins, int op, int axis, double c, int spin, int spin_b,
               const double* jxyz, const double* in, double* out);

double orc_norm(int nspins, const double* psi);
void orc_inner(int nspins, const double* self, const double* other, double out[2]);

/* Observable::measure for one observable; writes its width() values. */
int orc_measure(int nspins, const ss_observable* obs, const double* psi,
                const double* ref, const double* fields, int npairs,
                const int32_t* pairs, const double* J, double* out);

/* Measurement points and values per point of a configured run. */
int orc_shape(const ss_run_config* cfg, int64_t* points, int64_t* width);

/* Realisation assembly (io/Experiment.cpp:10-35): fields, couplings, psi0,
   ref0 of realisation `index`; *nspins receives its L. */
int orc_setup(const ss_run_config* cfg, uint64_t index, int32_t* nspins,
              double* fields, int32_t* pairs, double* J, int32_t* npairs,
              double* psi0, double* ref0);

/* runRealization: rows of one realisation (points x width) and the times. */
int orc_run_realization(const ss_run_config* cfg, uint64_t index, double* times,
                        double* values);

/* runRealization over [first, first+count) on `threads` POSIX threads;
   rows in index order; wall-clock seconds of the parallel part. */
int orc_run_range(const ss_run_config* cfg, uint64_t first, int64_t count,
                  int threads, double* times, double* values, double* seconds);
/* The same over an explicit list of realisation indices (rows in list order). */
int orc_run_indices(const ss_run_config* cfg, const uint64_t* indices, int64_t count,
                    int threads, double* times, double* values, double* seconds);

/* Welford / Chan accumulator over rows (Ensemble.cpp:116-166): folds `n`
   rows of `width` in order and writes mean, sd, stderr. */
void orc_accumulate(int64_t n, int64_t width, const double* rows, double* mean,
                    double* sd, double* se);

const char* orc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
