// Per-amplitude pieces of the echo observables, shared by the engine's
// correlator (observables.cu) and the no-allocation correlator (noalloc.cu)
// so that both sum the same terms in the same order.
#pragma once

#include "common.cuh"

namespace ss {

// (sigma_axis(s) in)[k] for the spin whose bit is `mask`
// (src/core/SpinOperators.cpp:90-209, Pauli matrices on bit s).
__device__ __forceinline__ double2 sigma_at(const double2* __restrict__ in, size_t k, size_t mask,
                                            int axis) {
  if (axis == SS_AXIS_Z) {
    const double2 a = in[k];
    return (k & mask) ? a : make_double2(-a.x, -a.y);
  }
  const double2 p = in[k ^ mask];
  if (axis == SS_AXIS_X) return p;
  return (k & mask) ? make_double2(p.y, -p.x) : make_double2(-p.y, p.x);
}

// This thread's share of <ref|A psi> with A = sum_s sigma_axis(s)
// (src/core/Observable.cpp:66-73): conj(ref_k) (A psi)_k over a grid-stride
// sweep of the n amplitudes, spins summed in increasing order.
__device__ __forceinline__ double2 corr_thread_sum(const double2* __restrict__ psi,
                                                   const double2* __restrict__ ref, int nspins,
                                                   int axis, size_t n) {
  double re = 0.0, im = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < nspins; ++s) {
      const double2 t = sigma_at(psi, k, size_t{1} << s, axis);
      sr += t.x;
      si += t.y;
    }
    const double2 r = ref[k];
    re += r.x * sr + r.y * si;
    im += r.x * si - r.y * sr;
  }
  return make_double2(re, im);
}

}  // namespace ss
