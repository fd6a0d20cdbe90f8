// The plain propagator: Propagator::evolve of src/core/Propagator.cpp.  The
// gather family is one fused kernel per Chebyshev order: each order reads
// T_{n-1} (its own amplitude and its partners), T_{n-2} and psi, and writes
// T_n over T_{n-2} and psi += c_n T_n -- the recurrence, the Hamiltonian and
// the series update in a single pass instead of the reference's 1 + L + P + 3
// passes.  Large vectors take the tiled family (tiled.cu) instead.  Both run
// in FP64 or in mixed precision (FP32 T vectors, FP64 psi and weights).
#include <algorithm>
#include <cmath>

#include "hamiltonian.cuh"
#include "tiled.hpp"

namespace ss {

void state_normalize_async(ss_state* s, int slot);
void check_flags(ss_engine* e);

namespace {

constexpr int kThreads = 256;

// From this many spins up SS_KERNEL_AUTO takes the tiled kernel (measured on
// B200: below it the gather kernel's partners stay in L1/L2 and its single
// launch per order wins).
constexpr int kTiledFromSpins = 18;

inline unsigned int blocks_for(size_t n) {
  return static_cast<unsigned int>((n + kThreads - 1) / kThreads);
}

template <typename C2>
__device__ __forceinline__ C2 narrow(double x, double y) {
  C2 v;
  v.x = static_cast<decltype(v.x)>(x);
  v.y = static_cast<decltype(v.y)>(y);
  return v;
}

// T_0 = psi, psi *= a_0  (Propagator.cpp:53-55); T_0 is FP32 in mixed precision.
template <typename C2>
__global__ void k_cheb_init(double2* psi, C2* t0, size_t n, double a0) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 p = psi[k];
  t0[k] = narrow<C2>(p.x, p.y);
  psi[k] = make_double2(p.x * a0, p.y * a0);
}

// One order: T_n = 2H^ T_{n-1} - T_{n-2} (T_1 = H^ T_0), written over T_{n-2};
// psi += c_n T_n (+ c_{n-1} T_{n-1}: psi is read and written every second
// order, taking both terms at once, as `psi_terms` = 0, 1, 2 says)
// (Propagator.cpp:58-72).  The table is prescaled by -2/bound, so the gather
// already is 2H^ T_{n-1}.  The gather and T_n's formation are FP64;
// C2 = float2 stores the mixed path's T vectors in FP32.
template <typename C2>
__global__ void k_cheb_order(const HamTerms* __restrict__ t, const double* __restrict__ diag,
                             const C2* __restrict__ cur, C2* prev, double2* psi,
                             size_t n, int first, double cr, double ci, int psi_terms, double pr,
                             double pi) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 h = ham_gather(t, diag, cur, k);
  double2 tn;
  if (first) {
    tn = make_double2(0.5 * h.x, 0.5 * h.y);
  } else {
    const C2 q = prev[k];
    tn = make_double2(h.x - q.x, h.y - q.y);
  }
  prev[k] = narrow<C2>(tn.x, tn.y);
  if (psi_terms == 0) return;
  double2 p = psi[k];
  p.x += cr * tn.x - ci * tn.y;
  p.y += cr * tn.y + ci * tn.x;
  if (psi_terms == 2) {
    const C2 o = cur[k];
    p.x += pr * o.x - pi * o.y;
    p.y += pr * o.y + pi * o.x;
  }
  psi[k] = p;
}

}  // namespace

// The propagator's two work vectors live with the engine, sized for the
// largest L it has propagated; the reference's Propagator owns the same two
// (Propagator.hpp:53-54).  The tiled kernel adds a third for its partial sums.
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

static void ensure_part_scratch(ss_engine* e, int nspins) {
  if (e->evolve_part_nspins >= nspins) return;
  sync(e);
  cudaFree(e->evolve_part);
  e->evolve_part = nullptr;
  e->evolve_part_nspins = 0;
  SS_CUDA(cudaMalloc(&e->evolve_part, sizeof(double2) << nspins));
  e->evolve_part_nspins = nspins;
}

// The kernel family a call runs: SS_KERNEL_AUTO resolved by size, and the
// tiled families checked against the vector (one full tile at least).
int resolve_kernel(int nspins, int precision, int kernel) {
  require(precision == SS_PRECISION_FP64 || precision == SS_PRECISION_MIXED,
          SS_ERR_INVALID_ARGUMENT, "unknown precision");
  require(kernel >= SS_KERNEL_AUTO && kernel <= SS_KERNEL_TILED_SMALL, SS_ERR_INVALID_ARGUMENT,
          "unknown kernel family");
  if (kernel == SS_KERNEL_AUTO) {
    return nspins >= kTiledFromSpins ? SS_KERNEL_TILED : SS_KERNEL_GATHER;
  }
  if (kernel != SS_KERNEL_GATHER) {
    require(nspins >= tile_bits_for(precision, kernel), SS_ERR_INVALID_ARGUMENT,
            "the tiled kernel needs at least as many spins as a tile holds");
  }
  return kernel;
}

// Applies a built expansion `nsteps` times; `weights` are the series weights
// c_n as (re, im) pairs (c_0 real).
void evolve(ss_ham* h, ss_state* psi, const std::vector<double>& weights, double bound,
            int64_t nsteps, bool autonormalize, int precision, int kernel) {
  kernel = resolve_kernel(h->nspins, precision, kernel);
  const size_t ncoef = weights.size() / 2;
  if (nsteps <= 0 || ncoef <= 1) return;  // the identity leaves psi alone
  require(bound > 0.0, SS_ERR_DOMAIN, "spectral bound must be positive");
  ss_engine* e = h->engine;
  const double scale = -2.0 / bound;
  ham_prepare(h, scale);
  ensure_evolve_scratch(e, h->nspins);
  const bool tiled = kernel != SS_KERNEL_GATHER;
  const void* passes = nullptr;
  int variant = 0;  // the tiled family's schedule: its kernels differ per variant
  if (tiled) {
    passes = tiled_prepare(h, scale, precision, kernel);
    variant = tile_variant(precision, kernel);
    ensure_part_scratch(e, h->nspins);
  }
  const bool mixed = precision == SS_PRECISION_MIXED;
  const size_t n = h->size();
  const unsigned int grid = blocks_for(n);
  // One step: T_0, every order, the optional renormalisation.
  auto one_step = [&] {
    void* cur = e->evolve_t[0];
    void* prev = e->evolve_t[1];
    if (mixed) {
      launch(e, k_cheb_init<float2>, grid, kThreads, 0, psi->data, static_cast<float2*>(cur), n,
             weights[0]);
    } else {
      launch(e, k_cheb_init<double2>, grid, kThreads, 0, psi->data, static_cast<double2*>(cur),
             n, weights[0]);
    }
    for (size_t order = 1; order < ncoef; ++order) {
      const int first = order == 1 ? 1 : 0;
      const double cr = weights[2 * order], ci = weights[2 * order + 1];
      const double pr = weights[2 * order - 2], pi = weights[2 * order - 1];
      // psi takes c_{n-1} T_{n-1} + c_n T_n on even orders, c_n T_n alone on
      // a final odd order, and nothing on the other odd orders.
      const int psi_terms = order % 2 == 0 ? 2 : (order + 1 == ncoef ? 1 : 0);
      if (tiled) {
        tiled_order(h, precision, kernel, cur, prev, e->evolve_part, psi->data, first, cr, ci,
                    psi_terms, pr, pi);
      } else if (mixed) {
        launch(e, k_cheb_order<float2>, grid, kThreads, 0, h->dev_terms, h->diag,
               static_cast<const float2*>(cur), static_cast<float2*>(prev), psi->data, n, first,
               cr, ci, psi_terms, pr, pi);
      } else {
        launch(e, k_cheb_order<double2>, grid, kThreads, 0, h->dev_terms, h->diag,
               static_cast<const double2*>(cur), static_cast<double2*>(prev), psi->data, n, first,
               cr, ci, psi_terms, pr, pi);
      }
      std::swap(cur, prev);
    }
    if (autonormalize) state_normalize_async(psi, 1);
  };
  // The step is captured once as a CUDA graph per (vectors, tables, weights,
  // precision, kernel family) and replayed: a pulse program repeats a handful
  // of expansions on the same two vectors, and one graph launch replaces
  // ncoef (times the pass count) kernel launches (the launch rate, not the
  // GPU, bounds small L).  The replay issues the same kernels with the same
  // arguments in the same order.
  StepGraph* g = nullptr;
  for (StepGraph& c : e->step_graphs) {
    if (c.terms == h->dev_terms && c.diag == h->diag && c.psi == psi->data &&
        c.t0 == e->evolve_t[0] && c.t1 == e->evolve_t[1] && c.n == n &&
        c.part == (tiled ? e->evolve_part : nullptr) && c.passes == passes &&
        c.precision == precision && c.kernel == kernel * 16 + variant &&
        c.autonormalize == int(autonormalize) && c.weights == weights) {
      g = &c;
      break;
    }
  }
  if (g == nullptr) {
    constexpr size_t kMaxGraphs = 32;
    if (e->step_graphs.size() >= kMaxGraphs) {
      auto old = std::min_element(e->step_graphs.begin(), e->step_graphs.end(),
                                  [](const StepGraph& a, const StepGraph& b) { return a.used < b.used; });
      if (old->exec) cudaGraphExecDestroy(old->exec);
      e->step_graphs.erase(old);
    }
    StepGraph c;
    c.terms = h->dev_terms;
    c.diag = h->diag;
    c.psi = psi->data;
    c.t0 = e->evolve_t[0];
    c.t1 = e->evolve_t[1];
    c.part = tiled ? e->evolve_part : nullptr;
    c.passes = passes;
    c.n = n;
    c.autonormalize = int(autonormalize);
    c.precision = precision;
    c.kernel = kernel * 16 + variant;
    c.weights = weights;
    const int64_t before = e->launches.load();
    cudaGraph_t graph = nullptr;
    SS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    try {
      one_step();
    } catch (...) {
      cudaStreamEndCapture(e->stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      e->launches.store(before);
      throw;
    }
    SS_CUDA(cudaStreamEndCapture(e->stream, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&c.exec, graph, 0);
    cudaGraphDestroy(graph);
    SS_CUDA(ie);
    c.kernels = e->launches.load() - before;
    e->launches.store(before);
    e->step_graphs.push_back(std::move(c));
    g = &e->step_graphs.back();
  }
  g->used = ++e->graph_clock;
  for (int64_t step = 0; step < nsteps; ++step) {
    SS_CUDA(cudaGraphLaunch(g->exec, e->stream));
    e->launches.fetch_add(g->kernels, std::memory_order_relaxed);
  }
  if (autonormalize) check_flags(e);
}

void evolve_fp64(ss_ham* h, ss_state* psi, const std::vector<double>& weights, double bound,
                 int64_t nsteps, bool autonormalize) {
  evolve(h, psi, weights, bound, nsteps, autonormalize, SS_PRECISION_FP64, SS_KERNEL_AUTO);
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

int ss_evolve_ex(const ss_ham* hc, ss_state* psi, const double* coeffs, int64_t ncoeffs,
                 double bound, int mode, int64_t nsteps, int autonormalize, int precision,
                 int kernel) {
  return guarded([&] {
    TraceRange trace("ss_evolve");
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
    evolve(h, psi, series_weights(ex, mode), bound, nsteps, autonormalize != 0, precision,
           kernel);
  });
}

int ss_evolve(const ss_ham* hc, ss_state* psi, const double* coeffs, int64_t ncoeffs,
              double bound, int mode, int64_t nsteps, int autonormalize) {
  return ss_evolve_ex(hc, psi, coeffs, ncoeffs, bound, mode, nsteps, autonormalize,
                      SS_PRECISION_FP64, SS_KERNEL_AUTO);
}

int ss_propagate_ex(const ss_ham* hc, ss_state* psi, int mode, double tau, int64_t nsteps,
                    int autonormalize, double epsilon, int precision, int kernel,
                    int64_t* order_used) {
  return guarded([&] {
    TraceRange trace("ss_propagate");
    auto* h = const_cast<ss_ham*>(hc);
    check_ham(h);
    check_state(psi);
    require(psi->nspins == h->nspins, SS_ERR_INVALID_ARGUMENT,
            "state and Hamiltonian disagree on spin count");
    require(epsilon > 0.0, SS_ERR_INVALID_ARGUMENT, "epsilon must be positive");
    resolve_kernel(h->nspins, precision, kernel);
    if (nsteps == 0) return;
    const Expansion ex =
        chebyshev(mode, spectral_bound(h->nspins, h->fields.data(), h->pairs), tau, epsilon);
    if (order_used) *order_used = static_cast<int64_t>(ex.order());
    if (ex.order() == 0) return;
    evolve(h, psi, series_weights(ex, mode), ex.bound, nsteps, autonormalize != 0, precision,
           kernel);
  });
}

int ss_propagate(const ss_ham* hc, ss_state* psi, int mode, double tau, int64_t nsteps,
                 int autonormalize, double epsilon, int64_t* order_used) {
  return ss_propagate_ex(hc, psi, mode, tau, nsteps, autonormalize, epsilon, SS_PRECISION_FP64,
                         SS_KERNEL_AUTO, order_used);
}

}  // extern "C"
