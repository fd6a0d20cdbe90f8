// Hamiltonian terms, the cached diagonal and H application
// (src/core/Hamiltonian.cpp:20-147).
#include <cmath>

#include "hamiltonian.cuh"
#include "tiled.hpp"

namespace ss {

void build_terms(int nspins, const double* f, const std::vector<PairTerm>& pairs, double scale,
                 HamTerms* t) {
  std::memset(t, 0, sizeof(HamTerms));
  t->nspins = nspins;
  t->scale = scale;
  for (int s = 0; s < nspins; ++s) {
    const double cx = scale * 0.5 * f[3 * s];
    const double cy = scale * 0.5 * f[3 * s + 1];
    if (std::abs(cx) > kNegligible || std::abs(cy) > kNegligible) {
      t->trans_mask[t->ntrans] = 1u << s;
      t->trans_cx[t->ntrans] = cx;
      t->trans_cy[t->ntrans] = cy;
      ++t->ntrans;
    }
    const double cz = 0.5 * f[3 * s + 2];
    if (std::abs(cz) > kNegligible) {
      t->zf_mask[t->nzf] = 1u << s;
      t->zf_c[t->nzf] = cz;
      ++t->nzf;
    }
  }
  for (const PairTerm& p : pairs) {
    const double quarter = scale * 0.25;
    const double ff = quarter * (p.jx + p.jy);
    const double fb = quarter * (p.jx - p.jy);
    const bool use_ff = std::abs(ff) > kNegligible, use_fb = std::abs(fb) > kNegligible;
    if (use_ff || use_fb) {
      t->pair_lo[t->npair] = 1u << p.lo;
      t->pair_hi[t->npair] = 1u << p.hi;
      t->pair_ff[t->npair] = use_ff ? ff : 0.0;
      t->pair_fb[t->npair] = use_fb ? fb : 0.0;
      ++t->npair;
    }
    const double cz = 0.25 * p.jz;
    if (std::abs(cz) > kNegligible) {
      t->zp_lo[t->nzp] = 1u << p.lo;
      t->zp_hi[t->nzp] = 1u << p.hi;
      t->zp_c[t->nzp] = cz;
      ++t->nzp;
    }
  }
}

namespace {

constexpr int kThreads = 256;

inline unsigned int blocks_for(size_t n) {
  return static_cast<unsigned int>((n + kThreads - 1) / kThreads);
}

// D[k] = sum_s +-hz_s/2 + sum_pairs +-jz/4, accumulated in the reference's
// order (fields by spin, then couplings by insertion), so D is bit-identical.
__global__ void k_build_diag(const HamTerms* __restrict__ t, double* diag, size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  double d = 0.0;
  for (int i = 0; i < t->nzf; ++i) {
    const double c = t->zf_c[i];
    d += (k & t->zf_mask[i]) ? c : -c;
  }
  for (int i = 0; i < t->nzp; ++i) {
    const double c = t->zp_c[i];
    const bool aligned = ((k & t->zp_lo[i]) != 0) == ((k & t->zp_hi[i]) != 0);
    d += aligned ? c : -c;
  }
  diag[k] = d;
}

__global__ void k_ham_apply(const HamTerms* __restrict__ t, const double* __restrict__ diag,
                            const double2* __restrict__ in, double2* out, size_t n,
                            int accumulate) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 h = ham_gather(t, diag, in, k);
  if (accumulate) {
    double2 o = out[k];
    o.x += h.x;
    o.y += h.y;
    out[k] = o;
  } else {
    out[k] = h;
  }
}

}  // namespace

void check_ham(const ss_ham* h) {
  require(h != nullptr && h->engine != nullptr, SS_ERR_INVALID_ARGUMENT, "null Hamiltonian");
}

void ham_prepare(ss_ham* h, double scale) {
  ss_engine* e = h->engine;
  if (!h->dev_terms) SS_CUDA(cudaMalloc(&h->dev_terms, sizeof(HamTerms)));
  if (!h->terms_valid || h->terms_scale != scale) {
    // Pageable source: the copy is staged before the call returns, so the
    // host table may be reused at once.
    HamTerms t;
    build_terms(h->nspins, h->fields.data(), h->pairs, scale, &t);
    SS_CUDA(cudaMemcpyAsync(h->dev_terms, &t, sizeof(HamTerms), cudaMemcpyHostToDevice,
                            e->stream));
    h->terms_scale = scale;
    h->terms_valid = true;
  }
  if (!h->diag_valid) {
    if (!h->diag) SS_CUDA(cudaMalloc(&h->diag, sizeof(double) * h->size()));
    launch(e, k_build_diag, blocks_for(h->size()), kThreads, 0, h->dev_terms, h->diag, h->size());
    h->diag_valid = true;
  }
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_ham_create(ss_engine* e, int nspins, ss_ham** out) {
  return guarded([&] {
    require(e != nullptr && out != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    require(nspins >= 1 && nspins <= kMaxSpins, SS_ERR_OUT_OF_RANGE,
            "number of spins must be in [1, kMaxSpins]");
    auto* h = new ss_ham;
    h->engine = e;
    h->nspins = nspins;
    h->fields.assign(3 * static_cast<size_t>(nspins), 0.0);
    *out = h;
  });
}

int ss_ham_destroy(ss_ham* h) {
  return guarded([&] {
    if (!h) return;
    cudaStreamSynchronize(h->engine->stream);
    cudaFree(h->diag);
    cudaFree(h->dev_terms);
    tiled_release(h);
    delete h;
  });
}

int ss_ham_set_terms(ss_ham* h, const double* fields, int npairs, const int32_t* pairs,
                     const double* couplings) {
  return guarded([&] {
    check_ham(h);
    require(fields != nullptr, SS_ERR_INVALID_ARGUMENT, "null field table");
    require(npairs >= 0 && (npairs == 0 || (pairs && couplings)), SS_ERR_INVALID_ARGUMENT,
            "null coupling arrays");
    std::vector<PairTerm> list;
    for (int i = 0; i < npairs; ++i) {
      const int a = pairs[2 * i], b = pairs[2 * i + 1];
      require(a >= 0 && b >= 0 && a < h->nspins && b < h->nspins, SS_ERR_OUT_OF_RANGE,
              "coupled spin index out of range");
      require(a != b, SS_ERR_INVALID_ARGUMENT, "a spin cannot couple to itself");
      const PairTerm p{a < b ? a : b, a < b ? b : a, couplings[3 * i], couplings[3 * i + 1],
                       couplings[3 * i + 2]};
      bool replaced = false;
      for (PairTerm& q : list) {  // Hamiltonian.cpp:39-52: overwrite in place
        if (q.lo == p.lo && q.hi == p.hi) {
          q = p;
          replaced = true;
          break;
        }
      }
      if (!replaced) list.push_back(p);
    }
    h->fields.assign(fields, fields + 3 * h->nspins);
    h->pairs = std::move(list);
    h->diag_valid = false;
    h->terms_valid = false;
    h->tiled_terms_valid = false;
  });
}

int ss_ham_set_fields(ss_ham* h, const double* fields) {
  return guarded([&] {
    check_ham(h);
    require(fields != nullptr, SS_ERR_INVALID_ARGUMENT, "null field table");
    h->fields.assign(fields, fields + 3 * h->nspins);
    h->diag_valid = false;
    h->terms_valid = false;
    h->tiled_terms_valid = false;
  });
}

int ss_ham_spectral_bound(const ss_ham* h, double* out) {
  return guarded([&] {
    check_ham(h);
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    *out = spectral_bound(h->nspins, h->fields.data(), h->pairs);
  });
}

int ss_ham_apply(const ss_ham* hc, double scale, const ss_state* in, ss_state* out,
                 int accumulate) {
  return guarded([&] {
    auto* h = const_cast<ss_ham*>(hc);
    check_ham(h);
    check_same_space(in, out);
    require(in != out && in->data != out->data, SS_ERR_INVALID_ARGUMENT,
            "kernels require distinct input and output");
    require(in->nspins == h->nspins, SS_ERR_INVALID_ARGUMENT,
            "state and Hamiltonian disagree on spin count");
    ham_prepare(h, scale);
    launch(h->engine, k_ham_apply, blocks_for(h->size()), kThreads, 0, h->dev_terms, h->diag,
           in->data, out->data, h->size(), accumulate);
  });
}

}  // extern "C"
