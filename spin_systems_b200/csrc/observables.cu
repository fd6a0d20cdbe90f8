// Echo observables (src/core/Observable.cpp:66-120) as single fused gather
// reductions: no scratch state vector is materialised.
//   corr:<a>  <ref| sum_s sigma_a(s) |psi>       (re, im)
//   mag:<s:a> <psi| sigma_a(s) |psi>             (re)
//   energy    <psi| H |psi>                      (re)
#include "hamiltonian.cuh"
#include "observables.cuh"

namespace ss {
namespace {

// <ref|A psi> with A = sum_s sigma_axis(s): conj(ref_k) (A psi)_k summed.
__global__ void k_corr(const double2* __restrict__ psi, const double2* __restrict__ ref,
                       int nspins, int axis, size_t n, double2* partials, unsigned int* counter,
                       double2* result) {
  grid_reduce2<kReduceThreads>(corr_thread_sum(psi, ref, nspins, axis, n), partials, counter,
                               result);
}

__global__ void k_mag(const double2* __restrict__ psi, size_t mask, int axis, size_t n,
                      double2* partials, unsigned int* counter, double2* result) {
  double re = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    const double2 t = sigma_at(psi, k, mask, axis);
    const double2 p = psi[k];
    re += p.x * t.x + p.y * t.y;
  }
  grid_reduce2<kReduceThreads>(make_double2(re, 0.0), partials, counter, result);
}

// <Hpsi|psi>.re with H at scale 1 (the physical Hamiltonian).
__global__ void k_energy(const HamTerms* __restrict__ t, const double* __restrict__ diag,
                         const double2* __restrict__ psi, size_t n, double2* partials,
                         unsigned int* counter, double2* result) {
  double re = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    const double2 h = ham_gather(t, diag, psi, k);
    const double2 p = psi[k];
    re += h.x * p.x + h.y * p.y;
  }
  grid_reduce2<kReduceThreads>(make_double2(re, 0.0), partials, counter, result);
}

}  // namespace

// Queue a correlator into result slot `slot` (no synchronisation).
void corr_async(const ss_state* psi, const ss_state* ref, int axis, int slot) {
  ss_engine* e = psi->engine;
  launch(e, k_corr, reduce_blocks(psi->size()), kReduceThreads, 0, psi->data, ref->data,
         psi->nspins, axis, psi->size(), e->red_partials, e->red_counter, e->red_result + slot);
}

void mag_async(const ss_state* psi, int spin, int axis, int slot) {
  ss_engine* e = psi->engine;
  launch(e, k_mag, reduce_blocks(psi->size()), kReduceThreads, 0, psi->data, size_t{1} << spin,
         axis, psi->size(), e->red_partials, e->red_counter, e->red_result + slot);
}

void energy_async(ss_ham* h, const ss_state* psi, int slot) {
  ham_prepare(h, 1.0);
  ss_engine* e = psi->engine;
  launch(e, k_energy, reduce_blocks(psi->size()), kReduceThreads, 0, h->dev_terms, h->diag,
         psi->data, psi->size(), e->red_partials, e->red_counter, e->red_result + slot);
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_measure_corr(const ss_state* psi, const ss_state* ref, int axis, double out[2]) {
  return guarded([&] {
    check_same_space(psi, ref);
    require(axis >= 0 && axis <= 2, SS_ERR_INVALID_ARGUMENT, "unknown axis; expected x, y or z");
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    corr_async(psi, ref, axis, 0);
    read_results(psi->engine, 1);
    out[0] = psi->engine->host_result[0].x;
    out[1] = psi->engine->host_result[0].y;
  });
}

int ss_measure_mag(const ss_state* psi, int spin, int axis, double* out) {
  return guarded([&] {
    check_state(psi);
    require(spin >= 0 && spin < psi->nspins, SS_ERR_OUT_OF_RANGE,
            "observable names a spin outside the system");
    require(axis >= 0 && axis <= 2, SS_ERR_INVALID_ARGUMENT, "unknown axis; expected x, y or z");
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    mag_async(psi, spin, axis, 0);
    read_results(psi->engine, 1);
    *out = psi->engine->host_result[0].x;
  });
}

int ss_measure_energy(const ss_ham* hc, const ss_state* psi, double* out) {
  return guarded([&] {
    auto* h = const_cast<ss_ham*>(hc);
    check_ham(h);
    check_state(psi);
    require(psi->nspins == h->nspins, SS_ERR_INVALID_ARGUMENT,
            "state and Hamiltonian disagree on spin count");
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    energy_async(h, psi, 0);
    read_results(psi->engine, 1);
    *out = psi->engine->host_result[0].x;
  });
}

}  // extern "C"
