// The Hamiltonian on the device (core/Hamiltonian.hpp:32-110): host copy of
// the terms, a device table of prescaled coefficients, and the cached sigma_z
// diagonal.
#pragma once

#include <vector>

#include "common.cuh"
#include "host_numerics.hpp"

namespace ss {

// Everything one application of s*H needs, prescaled by s, in device memory.
// Skip rules are those of src/core/Hamiltonian.cpp:54-127: a field or coupling
// component whose (scaled, for the off-diagonal part) coefficient is at most
// 1e-14 in magnitude contributes nothing.
struct HamTerms {
  int nspins;
  int ntrans;      // spins with a transverse field
  int npair;       // pairs with a non-negligible off-diagonal channel
  int nzf;         // sigma_z field terms in the diagonal
  int nzp;         // sigma_z coupling terms in the diagonal
  int pad;
  double scale;    // multiplies the diagonal
  unsigned int trans_mask[kMaxSpins];
  double trans_cx[kMaxSpins];
  double trans_cy[kMaxSpins];
  unsigned int pair_lo[kMaxPairs];
  unsigned int pair_hi[kMaxPairs];
  double pair_ff[kMaxPairs];  // |ud> <-> |du|, scale * (jx + jy) / 4
  double pair_fb[kMaxPairs];  // |dd> <-> |uu|, scale * (jx - jy) / 4
  unsigned int zf_mask[kMaxSpins];
  double zf_c[kMaxSpins];     // hz / 2
  unsigned int zp_lo[kMaxPairs];
  unsigned int zp_hi[kMaxPairs];
  double zp_c[kMaxPairs];     // jz / 4
};

void build_terms(int nspins, const double* fields, const std::vector<PairTerm>& pairs,
                 double scale, HamTerms* out);

// (s*H x)[k] gathered from x's partners: the diagonal, then transverse fields,
// then the off-diagonal channel of every coupling.  x holds double2 (FP64) or
// float2 (the mixed path's FP32 vectors) amplitudes; the sum is FP64 either way.
template <typename C2>
__device__ __forceinline__ double2 ham_gather(const HamTerms* __restrict__ t,
                                              const double* __restrict__ diag,
                                              const C2* __restrict__ x, size_t k) {
  const C2 self = x[k];
  const double g = t->scale * diag[k];
  double re = g * self.x, im = g * self.y;
  for (int i = 0; i < t->ntrans; ++i) {
    const unsigned int m = t->trans_mask[i];
    const C2 p = x[k ^ m];
    const double cx = t->trans_cx[i];
    const double cy = (k & m) ? -t->trans_cy[i] : t->trans_cy[i];
    re += cx * p.x - cy * p.y;
    im += cx * p.y + cy * p.x;
  }
  // Unrolled so that several partner loads are in flight per thread: the
  // loop is bound by their latency, not by the two FMAs each feeds.
#pragma unroll 8
  for (int i = 0; i < t->npair; ++i) {
    const unsigned int lo = t->pair_lo[i], hi = t->pair_hi[i];
    const bool aligned = ((k & lo) != 0) == ((k & hi) != 0);
    const double c = aligned ? t->pair_fb[i] : t->pair_ff[i];
    if (c != 0.0) {
      const C2 p = x[k ^ (lo | hi)];
      re += c * p.x;
      im += c * p.y;
    }
  }
  return make_double2(re, im);
}

struct TiledTables;

}  // namespace ss

struct ss_ham {
  ss_engine* engine = nullptr;
  int nspins = 0;
  std::vector<double> fields;            // 3L
  std::vector<ss::PairTerm> pairs;       // insertion order, unique pairs
  double* diag = nullptr;                // device, 2^L
  bool diag_valid = false;
  ss::HamTerms* dev_terms = nullptr;     // device table for `terms_scale`
  double terms_scale = 0.0;
  bool terms_valid = false;
  ss::TiledTables* tiled = nullptr;      // the tiled kernel's per-pass tables (tiled.cu)
  bool tiled_terms_valid = false;        // false once fields or couplings change
  size_t size() const { return size_t{1} << nspins; }
};

namespace ss {

// Makes the device term table current for `scale` and the diagonal current.
void ham_prepare(ss_ham* h, double scale);
void check_ham(const ss_ham* h);

}  // namespace ss
