// The plain FP64 propagator: Propagator::evolve of src/core/Propagator.cpp
// as one fused kernel per Chebyshev order.  Each order reads T_{n-1} (its own
// amplitude and its partners), T_{n-2} and psi, and writes T_n over T_{n-2}
// and psi += c_n T_n -- the recurrence, the Hamiltonian and the series update
// in a single pass instead of the reference's 1 + L + P + 3 passes.
#include <cmath>

#include "hamiltonian.cuh"

namespace ss {

void state_normalize_async(ss_state* s, int slot);
void check_flags(ss_engine* e);

namespace {

constexpr int kThreads = 256;

inline unsigned int blocks_for(size_t n) {
  return static_cast<unsigned int>((n + kThreads - 1) / kThreads);
}

// T_0 = psi, psi *= a_0  (Propagator.cpp:53-55)
__global__ void k_cheb_init(double2* psi, double2* t0, size_t n, double a0) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 p = psi[k];
  t0[k] = p;
  psi[k] = make_double2(p.x * a0, p.y * a0);
}

// One order: T_n = 2H^ T_{n-1} - T_{n-2} (T_1 = H^ T_0), written over T_{n-2};
// psi += (cr + i ci) T_n  (Propagator.cpp:58-72).  The table is prescaled by
// -2/bound, so the gather already is 2H^ T_{n-1}.
__global__ void k_cheb_order(const HamTerms* __restrict__ t, const double* __restrict__ diag,
                             const double2* __restrict__ cur, double2* prev, double2* psi,
                             size_t n, int first, double cr, double ci) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 h = ham_gather(t, diag, cur, k);
  double2 tn;
  if (first) {
    tn = make_double2(0.5 * h.x, 0.5 * h.y);
  } else {
    const double2 q = prev[k];
    tn = make_double2(h.x - q.x, h.y - q.y);
  }
  prev[k] = tn;
  double2 p = psi[k];
  p.x += cr * tn.x - ci * tn.y;
  p.y += cr * tn.y + ci * tn.x;
  psi[k] = p;
}

}  // namespace

// The propagator's two work vectors live with the engine, sized for the
// largest L it has propagated; the reference's Propagator owns the same two
// (Propagator.hpp:53-54).
void ensure_evolve_scratch(ss_engine* e, int nspins) {
  if (e->evolve_nspins >= nspins) return;
  sync(e);
  cudaFree(e->evolve_t[0]);
  cudaFree(e->evolve_t[1]);
  e->evolve_t[0] = e->evolve_t[1] = nullptr;
  e->evolve_nspins = 0;
  SS_CUDA(cudaMalloc(&e->evolve_t[0], sizeof(double2) << nspins));
  SS_CUDA(cudaMalloc(&e->evolve_t[1], sizeof(double2) << nspins));
  e->evolve_nspins = nspins;
}

// Applies a built expansion `nsteps` times; `weights` are the series weights
// c_n as (re, im) pairs (c_0 real).
void evolve_fp64(ss_ham* h, ss_state* psi, const std::vector<double>& weights, double bound,
                 int64_t nsteps, bool autonormalize) {
  const size_t ncoef = weights.size() / 2;
  if (nsteps <= 0 || ncoef <= 1) return;  // the identity leaves psi alone
  require(bound > 0.0, SS_ERR_DOMAIN, "spectral bound must be positive");
  ss_engine* e = h->engine;
  ham_prepare(h, -2.0 / bound);
  ensure_evolve_scratch(e, h->nspins);
  const size_t n = h->size();
  const unsigned int grid = blocks_for(n);
  for (int64_t step = 0; step < nsteps; ++step) {
    double2* cur = e->evolve_t[0];
    double2* prev = e->evolve_t[1];
    launch(e, k_cheb_init, grid, kThreads, 0, psi->data, cur, n, weights[0]);
    for (size_t order = 1; order < ncoef; ++order) {
      launch(e, k_cheb_order, grid, kThreads, 0, h->dev_terms, h->diag, cur, prev, psi->data, n,
             order == 1 ? 1 : 0, weights[2 * order], weights[2 * order + 1]);
      std::swap(cur, prev);
    }
    if (autonormalize) state_normalize_async(psi, 1);
  }
  if (autonormalize) check_flags(e);
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_bessel(int kind, double x, int64_t count, double* values, int64_t* nonzero) {
  return guarded([&] {
    require(values != nullptr && count >= 0, SS_ERR_INVALID_ARGUMENT, "bad output buffer");
    require(kind == 0 || kind == 1, SS_ERR_INVALID_ARGUMENT, "kind must be 0 (J) or 1 (I)");
    size_t nz = 0;
    const std::vector<double> v = bessel(kind, x, static_cast<size_t>(count), &nz);
    std::memcpy(values, v.data(), sizeof(double) * v.size());
    if (nonzero) *nonzero = static_cast<int64_t>(nz);
  });
}

int ss_chebyshev_build(int mode, double spectral_bound_, double tau, double epsilon,
                       int64_t max_order, double* coeffs, int64_t cap, int64_t* order,
                       double* effective_bound) {
  return guarded([&] {
    require(coeffs != nullptr && order != nullptr && effective_bound != nullptr,
            SS_ERR_INVALID_ARGUMENT, "null output");
    require(max_order >= 0, SS_ERR_INVALID_ARGUMENT, "max_order must be non-negative");
    const Expansion ex = chebyshev(mode, spectral_bound_, tau, epsilon,
                                   static_cast<size_t>(max_order));
    require(static_cast<int64_t>(ex.a.size()) <= cap, SS_ERR_INVALID_ARGUMENT,
            "coefficient buffer too small");
    std::memcpy(coeffs, ex.a.data(), sizeof(double) * ex.a.size());
    *order = static_cast<int64_t>(ex.order());
    *effective_bound = ex.bound;
  });
}

int ss_evolve(const ss_ham* hc, ss_state* psi, const double* coeffs, int64_t ncoeffs,
              double bound, int mode, int64_t nsteps, int autonormalize) {
  return guarded([&] {
    auto* h = const_cast<ss_ham*>(hc);
    check_ham(h);
    check_state(psi);
    require(psi->nspins == h->nspins, SS_ERR_INVALID_ARGUMENT,
            "state and Hamiltonian disagree on spin count");
    require(coeffs != nullptr && ncoeffs >= 1, SS_ERR_INVALID_ARGUMENT, "empty expansion");
    require(nsteps >= 0, SS_ERR_INVALID_ARGUMENT, "negative step count");
    Expansion ex;
    ex.a.assign(coeffs, coeffs + ncoeffs);
    ex.bound = bound;
    evolve_fp64(h, psi, series_weights(ex, mode), bound, nsteps, autonormalize != 0);
  });
}

int ss_propagate(const ss_ham* hc, ss_state* psi, int mode, double tau, int64_t nsteps,
                 int autonormalize, double epsilon, int64_t* order_used) {
  return guarded([&] {
    auto* h = const_cast<ss_ham*>(hc);
    check_ham(h);
    check_state(psi);
    require(psi->nspins == h->nspins, SS_ERR_INVALID_ARGUMENT,
            "state and Hamiltonian disagree on spin count");
    require(epsilon > 0.0, SS_ERR_INVALID_ARGUMENT, "epsilon must be positive");
    if (nsteps == 0) return;
    const Expansion ex =
        chebyshev(mode, spectral_bound(h->nspins, h->fields.data(), h->pairs), tau, epsilon);
    if (order_used) *order_used = static_cast<int64_t>(ex.order());
    if (ex.order() == 0) return;
    evolve_fp64(h, psi, series_weights(ex, mode), ex.bound, nsteps, autonormalize != 0);
  });
}

}  // extern "C"
