// The batched echo kernel: one CTA runs one realisation's pulse program
// (state and reference) with both state vectors' Chebyshev recursion held in
// shared memory, then takes the next realisation from a work counter.
//
// Data layout.  A realisation's T_{n-1}, T_{n-2} and the partial H T_{n-1}
// live in three shared buffers of 2^L complex values (FP32 in mixed precision,
// FP64 otherwise), XOR-swizzled so that every access pattern below touches
// each bank once per wavefront.  The FP64 series sum psi lives in registers
// (or, for the largest L, in global memory where the whole CTA streams it).
//
// Register blocking.  Each thread owns 2^R amplitudes that differ in R
// consecutive "register bits" of the basis index.  One application of H is
// split into G passes ("layouts") with different register bits: a coupling
// whose two spins are both register bits of some layout is applied entirely
// in registers there; a coupling (i, j) with only i a register bit is applied
// in the first layout holding i, from the partner block at k ^ (1 << j), which
// serves all R couplings (i, j) of that layout at once.  Fields act in the
// layout holding their spin, the diagonal and the recurrence in the last one.
// For L = 12, R = 4 that is 12 partner-block reads per amplitude per order
// instead of the 66 + 12 single-amplitude gathers of a direct sweep.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace ss {
namespace batch {

enum OpKind { OP_EVOLVE = 0, OP_PULSE = 1, OP_MEASURE = 2 };

// One linearised program step.
//   EVOLVE:  a = step type, b = number of steps, c = autonormalise
//   PULSE:   a = rotation index, b = target spin (-1 = every spin)
//   MEASURE: a = point index
struct Op {
  int kind, a, b, c;
};

// One (realisation, step type): the expansion and its coefficient block.
struct TypeDev {
  double scale;      // -2 / bound; multiplies the diagonal (1 for the energy table)
  long long w_off;   // series weights c_0..c_order (double2) in the weight pool
  long long c_off;   // coefficient block in the coefficient pool, see below
  int order;         // 0 = the step is the identity
  int flags;         // 1: transverse fields present, 2: |dd><uu| channel present
};
// Coefficient block of P pairs and L spins, doubles:
//   [0,P) ff = scale / 4 * (jx + jy)   [P,2P) fb = scale / 4 * (jx - jy)
//   [2P,3P) jz / 4                     [3P,3P+L) hz / 2
//   [3P+L, 3P+2L) scale * hx / 2       [3P+2L, 3P+3L) scale * hy / 2
//   [3P+3L, 3P+3L+4*kCorr) correction terms: (pair index or -1, ff - fl32(ff),
//                                             fb - fl32(fb), 0)
// with the reference's 1e-14 skip rule already applied (zeros).
//
// Mixed precision applies the couplings as FP32 numbers.  Their rounding is a
// fixed perturbation of H, so its error accumulates coherently over every
// step, in proportion to the coupling: for the few strongly coupled pairs of
// the dipolar heavy tail it dominates the whole echo error.  Those pairs'
// rounding residuals (the kCorr largest couplings of each table) are added
// back in FP64 when T_n is formed, and the diagonal is applied in FP64.  The
// heavy tail is one or two close pairs per realisation, so kCorr = 2 takes
// the worst L=10..12 realisations to the level of exact FP64 coefficients.
constexpr int kCorr = 2;

struct RealDev {
  int L, npairs;
  long long pair_off;   // pair list (lo, hi) in the pair pool
  long long state_off;  // 2 * 2^L double2: state, then reference
  long long type_off;   // first TypeDev of this realisation
  long long row_off;    // first value of its measurement rows
  long long rot_off;    // its rotation table in the rotation pool (sweeps)
};

struct Args {
  const Op* ops;
  int op_begin, op_end;
  const double* rots;   // 8 doubles per rotation (ll, lh, hl, hh)
  const RealDev* reals;
  const int* work;      // realisations of this bucket, most expensive first
  int nwork;
  unsigned int* counter;
  const TypeDev* types;
  const double* cpool;
  const double2* wpool;
  const int2* pairs;
  double2* states;
  double* rows;
  const int* obs;       // (kind, axis, spin) per observable
  int nobs, width;
  int measure_type;     // slot of the energy table in each realisation's types
  int* flags;           // [0]: zero norm under autonormalisation
  double2* snap;        // split clusters: both vectors of every work slot at
  int nmeas;            // each of the nmeas measurement points
};

template <typename Real>
struct Cplx;
template <>
struct Cplx<float> {
  using T = float2;
};
template <>
struct Cplx<double> {
  using T = double2;
};

template <int L, int R>
struct Geo {
  static constexpr int NT = 1 << (L - R);  // threads per realisation
  static constexpr int NA = 1 << R;        // amplitudes per thread
  static constexpr int G = (L + R - 1) / R;
  static constexpr int N = 1 << L;
  __host__ __device__ static constexpr int base(int g) {
    return (g + 1) * R <= L ? g * R : L - R;
  }
  __host__ __device__ static constexpr bool holds(int g, int s) {
    return s >= base(g) && s < base(g) + R;
  }
  __host__ __device__ static constexpr int first_layout(int s) {
    for (int g = 0; g < G; ++g) {
      if (holds(g, s)) return g;
    }
    return -1;
  }
  // The layout that applies coupling (i, j), i < j.
  __host__ __device__ static constexpr int pair_layout(int i, int j) {
    for (int g = 0; g < G; ++g) {
      if (holds(g, i) && holds(g, j)) return g;
    }
    return first_layout(i);
  }
  // Whether layout g applies the couplings (base(g) + p, j) for every j above
  // its group.  No earlier layout can hold such a j; the last layout holds
  // both spins exactly when base(g) + p is in it, so this is the same for
  // every j and known at compile time.
  __host__ __device__ static constexpr bool cross_mine(int g, int p) {
    return first_layout(base(g) + p) == g && !(g < G - 1 && base(g) + p >= L - R);
  }
  __host__ __device__ static constexpr bool any_cross(int g) {
    for (int p = 0; p < R; ++p) {
      if (cross_mine(g, p)) return base(g) + R < L;
    }
    return false;
  }
};

// Padded shared-memory index of amplitude k: one spare element after every
// 2^R.  Because a thread's register bits and thread bits never overlap, the
// padded index of (thread base | slot) is padded(base) + padded(slot), so each
// slot is an immediate offset, and every access pattern of the schedules with
// L >= 9 hits each bank once per wavefront.
template <int R>
__device__ __forceinline__ uint32_t pad(uint32_t k) { return k + (k >> R); }

template <int L, int R>
struct Padded {
  static constexpr uint32_t N = (1u << L) + (1u << (L - R));  // elements per buffer
};

template <typename C2>
__device__ __forceinline__ C2 cz() {
  C2 v;
  v.x = 0;
  v.y = 0;
  return v;
}

// Shared-memory workspace of one CTA.
template <typename Real>
struct Smem {
  using C2 = typename Cplx<Real>::T;
  C2* buf[3];   // T_{n-1}, T_{n-2}, partial H T_{n-1}
  Real* cff;    // L x L, upper triangle: flip-flop coefficients
  Real* cfb;    // L x L, upper triangle: flip-both coefficients
  Real* ccx;    // L: scaled hx / 2
  Real* ccy;    // L: scaled hy / 2
  double2* psi; // 2^L FP64 series sum, when it lives in shared memory
  uint2* corr_mask;    // kCorr: (low spin mask, high spin mask) of corrected pairs
  double2* corr_coef;  // kCorr: (ff residual, fb residual)
  int* corr_n;         // number of corrected pairs of the current table
  double2* red; // 32 slots for block reductions
};

// Where a realisation's FP64 series sum psi lives during an Evolve step.
enum PsiHome { PSI_REG = 0, PSI_SMEM = 1, PSI_GLOBAL = 2 };

template <int NT>
__device__ __forceinline__ double2 cta_sum2(double2 v, double2* red) {
  v = warp_sum2(v);
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double2 s = make_double2(0.0, 0.0);
  for (int w = 0; w < NW; ++w) s += red[w];  // every thread, same order
  return s;
}

// The couplings (b + p, j), p < R, from one partner block: slot x of the
// block (amplitude k ^ 2^j with register bits x) feeds the thread's slot
// x ^ 2^p with c1[p] when that slot's bit p is set, c0[p] when it is clear.
// MODE 1 keeps only the clear targets, MODE 2 only the set ones (the other
// half multiplies a zero coefficient), both decided at compile time.
template <int R, int b, int MODE, typename C2, typename Real, int NA>
__device__ __forceinline__ void cross_apply(C2 (&acc)[NA], const C2* partner, const Real (&c0)[R],
                                            const Real (&c1)[R]) {
#pragma unroll
  for (int x = 0; x < NA; ++x) {
    const C2 v = partner[pad<R>(uint32_t(x) << b)];
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const int dst = x ^ (1 << p);
      const bool set = ((dst >> p) & 1) != 0;
      if ((MODE == 1 && set) || (MODE == 2 && !set)) continue;
      const Real c = set ? c1[p] : c0[p];
      acc[dst].x += c * v.x;
      acc[dst].y += c * v.y;
    }
  }
}

// Without a |dd><uu| channel (has_fb false: jx == jy on every pair, as in
// the secular dipolar couplings) a coupling (i, j) acts only on amplitudes
// whose bits i and j differ, so when bit j is the same across the warp only
// half of the targets receive anything: the warp takes the pruned path.
template <int R, int b, typename C2, typename Real, int NA>
__device__ __forceinline__ void cross_block(C2 (&acc)[NA], const C2* partner, const Real (&c0)[R],
                                            const Real (&c1)[R], bool bj, bool has_fb) {
  if (!has_fb) {
    if (__all_sync(0xffffffffu, bj)) {
      cross_apply<R, b, 1>(acc, partner, c0, c1);
      return;
    }
    if (__all_sync(0xffffffffu, !bj)) {
      cross_apply<R, b, 2>(acc, partner, c0, c1);
      return;
    }
  }
  cross_apply<R, b, 0>(acc, partner, c0, c1);
}

// Couplings with a CTA bit from one peer block (bit uniform over the CTA, so
// the MODE pruning of cross_apply always applies without a flip-both
// channel): the register-bit couplings as in cross_apply, and for each of
// the LB lowest spins (lane bits here) the partner from lane ^ 2^q.
template <int R, int b, int MODE, int LB, typename C2, typename Real, int NA>
__device__ __forceinline__ void cta_cross(C2 (&acc)[NA], const C2* partner, const Real (&c0)[R],
                                          const Real (&c1)[R], const Real (&cq)[LB > 0 ? LB : 1]) {
#pragma unroll
  for (int x = 0; x < NA; ++x) {
    const C2 v = partner[pad<R>(uint32_t(x) << b)];
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const int dst = x ^ (1 << p);
      const bool set = ((dst >> p) & 1) != 0;
      if ((MODE == 1 && set) || (MODE == 2 && !set)) continue;
      const Real c = set ? c1[p] : c0[p];
      acc[dst].x += c * v.x;
      acc[dst].y += c * v.y;
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const Real wx = __shfl_xor_sync(0xffffffffu, v.x, 1 << q);
      const Real wy = __shfl_xor_sync(0xffffffffu, v.y, 1 << q);
      acc[x].x += cq[q] * wx;
      acc[x].y += cq[q] * wy;
    }
  }
}

// One layout pass over the register group of layout g: couplings and fields
// assigned to g are applied into acc.  For g > 0 acc is first loaded from the
// partial buffer; own[] receives T_{n-1} of this thread's amplitudes.
//
// A vector spread over 2^CB CTAs of a cluster (see k_batch_dist) runs the same
// layouts over its L local bits; LS is then the whole system's spin count (the
// stride of the coupling tables) and spins L .. LS-1 are CTA bits.  A
// coupling (b + p, j) with j a CTA bit is applied in the first layout holding
// b + p, from the partner block at the same local offsets in the CTA across
// bit j (rcur[j - L], distributed shared memory); `part` is this CTA's value
// of the CTA bits.
template <int L, int R, typename Real, int g, int LS = L, int CB = 0>
__device__ __forceinline__ void layout_pass(const Smem<Real>& sm, const typename Cplx<Real>::T* cur,
                                            typename Cplx<Real>::T (&acc)[Geo<L, R>::NA],
                                            typename Cplx<Real>::T (&own)[Geo<L, R>::NA],
                                            uint32_t t, bool has_trans, bool has_fb,
                                            const typename Cplx<Real>::T* const* rcur = nullptr,
                                            uint32_t part = 0) {
  using Gm = Geo<L, R>;
  using C2 = typename Cplx<Real>::T;
  constexpr int b = Gm::base(g);
  constexpr int NA = Gm::NA;
  const uint32_t kb = ((t >> b) << (b + R)) | (t & ((1u << b) - 1u));

  const C2* mine = cur + pad<R>(kb);
#pragma unroll
  for (int a = 0; a < NA; ++a) own[a] = mine[pad<R>(uint32_t(a) << b)];
  if (g == 0) {
#pragma unroll
    for (int a = 0; a < NA; ++a) acc[a] = cz<C2>();
  } else {
    const C2* part = sm.buf[2] + pad<R>(kb);
#pragma unroll
    for (int a = 0; a < NA; ++a) acc[a] = part[pad<R>(uint32_t(a) << b)];
  }

  // Couplings with both spins in this register group.
#pragma unroll
  for (int p = 0; p < R; ++p) {
#pragma unroll
    for (int q = p + 1; q < R; ++q) {
      if (Gm::pair_layout(b + p, b + q) == g) {
        const Real ff = sm.cff[(b + p) * LS + (b + q)];
        const Real fb = sm.cfb[(b + p) * LS + (b + q)];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const int src = a ^ (1 << p) ^ (1 << q);
          if (((a >> p) & 1) != ((a >> q) & 1)) {
            acc[a].x += ff * own[src].x;
            acc[a].y += ff * own[src].y;
          } else if (has_fb) {
            acc[a].x += fb * own[src].x;
            acc[a].y += fb * own[src].y;
          }
        }
      }
    }
  }

  // Transverse fields of this group's spins: (cx +- i cy) from the partner.
  if (has_trans) {
#pragma unroll
    for (int p = 0; p < R; ++p) {
      if (Gm::first_layout(b + p) == g) {
        const Real cx = sm.ccx[b + p], cy = sm.ccy[b + p];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const C2 v = own[a ^ (1 << p)];
          const Real sy = ((a >> p) & 1) ? -cy : cy;
          acc[a].x += cx * v.x - sy * v.y;
          acc[a].y += cx * v.y + sy * v.x;
        }
      }
    }
  }

  // Couplings (b + p, j) with j above the group: one partner block per j,
  // serving the R couplings (b + p, j) at once.  The loop over j stays rolled
  // to keep the order loop inside the instruction cache.
#pragma unroll 1
  for (int j = b + R; j < (Gm::any_cross(g) ? L : 0); ++j) {
    const uint32_t m = 1u << j;
    const bool bj = (kb & m) != 0;
    Real c0[R], c1[R];
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const bool mine = Gm::cross_mine(g, p);
      const Real ff = mine ? sm.cff[(b + p) * LS + j] : Real(0);
      const Real fb = mine ? sm.cfb[(b + p) * LS + j] : Real(0);
      c0[p] = bj ? ff : fb;  // register bit clear: aligned iff bit j clear
      c1[p] = bj ? fb : ff;  // register bit set
    }
    // (kb | (x << b)) ^ m == (kb ^ m) | (x << b): bit j is not a group bit.
    cross_block<R, b>(acc, cur + pad<R>(kb ^ m), c0, c1, bj, has_fb);
  }

  // Couplings (i, L + jb) with a CTA bit: the partner block is this thread's
  // own block in the CTA across bit jb.  Layout 0 leaves its register bits'
  // couplings to layout 1, where those spins are lane bits: there the peer
  // block is read with consecutive lanes on consecutive amplitudes (layout
  // 0's pattern strides 2^R + 1 elements between lanes, a separate memory
  // sector per lane across the cluster network), and the partner of spin
  // q < b is the same slot in lane ^ 2^q, fetched with a warp shuffle.
  if constexpr (CB > 0 && (g > 0 || Gm::G == 1)) {
    constexpr int LB = (g == 1 && Gm::G > 1) ? b : 0;  // layout 0's bits, here lane bits
    static_assert(LB <= 5, "layout 0's bits must be lane bits of layout 1");
#pragma unroll 1
    for (int jb = 0; jb < CB; ++jb) {
      const int j = L + jb;
      const bool bj = ((part >> jb) & 1u) != 0;
      Real c0[R], c1[R];
#pragma unroll
      for (int p = 0; p < R; ++p) {
        const bool mine = Gm::first_layout(b + p) == g;
        const Real ff = mine ? sm.cff[(b + p) * LS + j] : Real(0);
        const Real fb = mine ? sm.cfb[(b + p) * LS + j] : Real(0);
        c0[p] = bj ? ff : fb;
        c1[p] = bj ? fb : ff;
      }
      Real cq[LB > 0 ? LB : 1];
#pragma unroll
      for (int q = 0; q < LB; ++q) {
        const bool anti = (((t >> q) & 1u) != 0) != bj;
        cq[q] = anti ? sm.cff[q * LS + j] : sm.cfb[q * LS + j];
      }
      const C2* partner = rcur[jb] + pad<R>(kb);
      if (!has_fb && bj) {
        cta_cross<R, b, 1, LB>(acc, partner, c0, c1, cq);
      } else if (!has_fb) {
        cta_cross<R, b, 2, LB>(acc, partner, c0, c1, cq);
      } else {
        cta_cross<R, b, 0, LB>(acc, partner, c0, c1, cq);
      }
    }
  }
}

template <int L, int R, typename Real, int g>
__device__ __forceinline__ void store_partial(const Smem<Real>& sm,
                                              const typename Cplx<Real>::T (&acc)[Geo<L, R>::NA],
                                              uint32_t t) {
  constexpr int b = Geo<L, R>::base(g);
  const uint32_t kb = ((t >> b) << (b + R)) | (t & ((1u << b) - 1u));
  typename Cplx<Real>::T* part = sm.buf[2] + pad<R>(kb);
#pragma unroll
  for (int a = 0; a < Geo<L, R>::NA; ++a) part[pad<R>(uint32_t(a) << b)] = acc[a];
}

// Layouts 0 .. G-2, each followed by a barrier.
template <int L, int R, typename Real, int g, int LS = L, int CB = 0>
__device__ __forceinline__ void front_layouts(const Smem<Real>& sm, const typename Cplx<Real>::T* cur,
                                              uint32_t t, bool has_trans, bool has_fb,
                                              const typename Cplx<Real>::T* const* rcur = nullptr,
                                              uint32_t part = 0) {
  if constexpr (g < Geo<L, R>::G - 1) {
    typename Cplx<Real>::T acc[Geo<L, R>::NA], own[Geo<L, R>::NA];
    layout_pass<L, R, Real, g, LS, CB>(sm, cur, acc, own, t, has_trans, has_fb, rcur, part);
    store_partial<L, R, Real, g>(sm, acc, t);
    __syncthreads();
    front_layouts<L, R, Real, g + 1, LS, CB>(sm, cur, t, has_trans, has_fb, rcur, part);
  }
}

}  // namespace batch
}  // namespace ss
