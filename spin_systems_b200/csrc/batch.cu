// The batched engine: many disorder realisations of one pulse program in one
// persistent fused launch per system size, captured with its set-up as a CUDA
// graph.  Host side: the program is linearised, every realisation is
// assembled bit for bit as the reference does (geometry, disorder, psi0), and
// each distinct Evolve step gets a per-realisation table (spectral bound,
// Chebyshev series weights, prescaled couplings).  Device side: see
// batch_kernel.cuh.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <fstream>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>
#include <numeric>
#include <thread>
#include <tuple>

#include <cooperative_groups.h>

#include "batch_kernel.cuh"
#include "hamiltonian.cuh"

namespace ss {

void rotation_matrix(const double axis[3], double angle, double u[8]);
void validate_config(const ss_run_config& c);

namespace batch {
namespace {

constexpr int kPrepThreads = 256;
constexpr int kClusterSize = 2;  // state and reference of one realisation
// Time of an FP64 amplitude-order relative to a mixed one (B200, L = 12).
constexpr double kFp64CostFactor = 1.45;
// Split clusters: device memory for the snapshots of one launch, and the
// fewest realisations a launch must hold for the split schedule to be used.
std::atomic<int64_t> g_snap_budget{int64_t{16} << 30};
constexpr size_t kSnapMinSlots = 64;

// ---------------------------------------------------------------- device
__device__ __forceinline__ double2 sigma_at(const double2* in, uint32_t k, int s, int axis) {
  const uint32_t m = 1u << s;
  if (axis == SS_AXIS_Z) {
    const double2 a = in[k];
    return (k & m) ? a : make_double2(-a.x, -a.y);
  }
  const double2 p = in[k ^ m];
  if (axis == SS_AXIS_X) return p;
  return (k & m) ? make_double2(p.y, -p.x) : make_double2(-p.y, p.x);
}

// psi0 -> state slot, reference = sum_s sigma_b(s) psi0 summed in spin order
// (bit-identical to src/ensemble/Ensemble.cpp:47-58).
__global__ void k_batch_prepare(const RealDev* reals, const double2* psi0, const long long* psi0_off,
                                double2* states, int ref_axis) {
  const RealDev rd = reals[blockIdx.x];
  const uint32_t n = 1u << rd.L;
  const double2* src = psi0 + psi0_off[blockIdx.x];
  double2* st = states + rd.state_off;
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
    st[k] = src[k];
    double re = 0.0, im = 0.0;
    for (int s = 0; s < rd.L; ++s) {
      const double2 v = sigma_at(src, k, s, ref_axis);
      re += v.x;
      im += v.y;
    }
    st[n + k] = make_double2(re, im);
  }
}

template <int L, int R, typename Real, int PSI>
__device__ void evolve_op(const Args& args, const Smem<Real>& sm, const RealDev& rd, double2* st,
                          const Op& op, const TypeDev& ty, int vec) {
  using Gm = Geo<L, R>;
  using C2 = typename Cplx<Real>::T;
  constexpr int NT = Gm::NT, NA = Gm::NA, G = Gm::G, N = Gm::N;
  constexpr int bl = Gm::base(G - 1);  // = L - R: thread t owns k = t | a << bl
  constexpr bool kMixed = std::is_same<Real, float>::value;
  const uint32_t t = threadIdx.x;
  const int P = rd.npairs;
  const double* cb = args.cpool + ty.c_off;
  const int2* pl = args.pairs + rd.pair_off;

  __syncthreads();  // earlier readers of the coefficient tables are done
  for (int i = t; i < L * L; i += NT) {
    sm.cff[i] = Real(0);
    sm.cfb[i] = Real(0);
  }
  __syncthreads();
  for (int p = t; p < P; p += NT) {
    const int2 q = pl[p];
    sm.cff[q.x * L + q.y] = Real(cb[p]);
    sm.cfb[q.x * L + q.y] = Real(cb[P + p]);
  }
  for (int s = t; s < L; s += NT) {
    sm.ccx[s] = Real(cb[3 * P + L + s]);
    sm.ccy[s] = Real(cb[3 * P + 2 * L + s]);
  }
  if (t == 0) {
    int nc = 0;
    if (kMixed) {
      const double* ct = cb + 3 * P + 3 * L;
      for (int c = 0; c < kCorr; ++c) {
        const int pi = static_cast<int>(ct[4 * c]);
        if (pi < 0) continue;
        const int2 q = pl[pi];
        sm.corr_mask[nc] = make_uint2(1u << q.x, 1u << q.y);
        sm.corr_coef[nc] = make_double2(ct[4 * c + 1], ct[4 * c + 2]);
        ++nc;
      }
    }
    *sm.corr_n = nc;
  }
  // Scaled diagonal of this thread's amplitudes in FP64, summed in the
  // reference's order (src/core/Hamiltonian.cpp:54-80).
  double dg[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    const uint32_t k = t | (uint32_t(a) << bl);
    double d = 0.0;
    for (int s = 0; s < L; ++s) {
      const double c = cb[3 * P + s];
      d += ((k >> s) & 1u) ? c : -c;
    }
    for (int p = 0; p < P; ++p) {
      const int2 q = pl[p];
      const double c = cb[2 * P + p];
      d += (((k >> q.x) ^ (k >> q.y)) & 1u) ? -c : c;
    }
    dg[a] = ty.scale * d;
  }
  __syncthreads();

  const bool has_trans = (ty.flags & 1) != 0, has_fb = (ty.flags & 2) != 0;
  const int ncorr = *sm.corr_n;
  const double2* wts = args.wpool + ty.w_off;
  const double a0 = wts[0].x;

  {
    double2* psig = st + vec * N;
    double2 preg[PSI == PSI_REG ? NA : 1] = {};
    // psi of amplitude slot a, wherever it lives
    auto psi_ld = [&](int a) -> double2 {
      const uint32_t k = t | (uint32_t(a) << bl);
      if constexpr (PSI == PSI_REG) return preg[a];
      else if constexpr (PSI == PSI_SMEM) return sm.psi[k];
      else return __ldcg(&psig[k]);
    };
    auto psi_st = [&](int a, double2 p) {
      const uint32_t k = t | (uint32_t(a) << bl);
      if constexpr (PSI == PSI_REG) preg[a] = p;
      else if constexpr (PSI == PSI_SMEM) sm.psi[k] = p;
      else __stcg(&psig[k], p);
    };
    if constexpr (PSI != PSI_GLOBAL) {
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const double2 p = psig[t | (uint32_t(a) << bl)];
        if constexpr (PSI == PSI_REG) preg[a] = p;
        else sm.psi[t | (uint32_t(a) << bl)] = p;
      }
    }
    for (int step = 0; step < op.b; ++step) {
      C2* cur = sm.buf[0];
      C2* prv = sm.buf[1];
      // T_0 = psi; psi *= a_0  (src/core/Propagator.cpp:53-55)
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const uint32_t k = t | (uint32_t(a) << bl);
        double2 p = psi_ld(a);
        C2 c;
        c.x = Real(p.x);
        c.y = Real(p.y);
        cur[pad<R>(k)] = c;
        p.x *= a0;
        p.y *= a0;
        psi_st(a, p);
      }
      __syncthreads();
      for (int n = 1; n <= ty.order; ++n) {
        const double2 cn = wts[n];
        front_layouts<L, R, Real, 0>(sm, cur, t, has_trans, has_fb);
        C2 acc[NA], own[NA];
        layout_pass<L, R, Real, G - 1>(sm, cur, acc, own, t, has_trans, has_fb);
        C2* prv_mine = prv + pad<R>(t);  // last layout: pad(t | a << bl) = pad(t) + pad(a << bl)
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const uint32_t k = t | (uint32_t(a) << bl);
          // T_n in FP64: the FP32 partial sum, the FP64 diagonal, the FP64
          // rounding residuals of the strongest couplings, the recurrence.
          double hx = double(acc[a].x) + dg[a] * double(own[a].x);
          double hy = double(acc[a].y) + dg[a] * double(own[a].y);
#pragma unroll
          for (int c = 0; c < kCorr; ++c) {
            if (c < ncorr) {
              const uint2 mk = sm.corr_mask[c];
              const double2 cc = sm.corr_coef[c];
              const C2 w = cur[pad<R>(k ^ mk.x ^ mk.y)];
              const double co = (((k & mk.x) != 0) == ((k & mk.y) != 0)) ? cc.y : cc.x;
              hx += co * double(w.x);
              hy += co * double(w.y);
            }
          }
          const uint32_t off = pad<R>(uint32_t(a) << bl);
          if (n == 1) {
            hx *= 0.5;
            hy *= 0.5;
          } else {
            const C2 q = prv_mine[off];
            hx -= double(q.x);
            hy -= double(q.y);
          }
          C2 tn;
          tn.x = Real(hx);
          tn.y = Real(hy);
          prv_mine[off] = tn;
          double2 p = psi_ld(a);
          p.x += cn.x * hx - cn.y * hy;
          p.y += cn.x * hy + cn.y * hx;
          psi_st(a, p);
        }
        __syncthreads();
        C2* tmp = cur;
        cur = prv;
        prv = tmp;
      }
      if (op.c) {  // autonormalise (src/core/Propagator.cpp:98)
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const double2 p = psi_ld(a);
          s += p.x * p.x + p.y * p.y;
        }
        const double nrm = sqrt(cta_sum2<NT>(make_double2(s, 0.0), sm.red).x);
        if (nrm == 0.0 || !isfinite(nrm)) {
          if (t == 0) atomicExch(args.flags, nrm == 0.0 ? SS_ERR_DOMAIN : SS_ERR_NUMERIC);
        } else {
          const double f = 1.0 / nrm;
#pragma unroll
          for (int a = 0; a < NA; ++a) {
            double2 p = psi_ld(a);
            p.x *= f;
            p.y *= f;
            psi_st(a, p);
          }
        }
        __syncthreads();
      }
    }
    if constexpr (PSI != PSI_GLOBAL) {
#pragma unroll
      for (int a = 0; a < NA; ++a) psig[t | (uint32_t(a) << bl)] = psi_ld(a);
    }
    __syncthreads();
  }
}

template <int NT>
__device__ void pulse_op(const Args& args, int L, double2* st, const Op& op, int vec,
                         long long rot_off) {
  const double* u = args.rots + rot_off + 8 * op.a;
  const double llr = u[0], lli = u[1], lhr = u[2], lhi = u[3];
  const double hlr = u[4], hli = u[5], hhr = u[6], hhi = u[7];
  const uint32_t n = 1u << L;
  const int s0 = op.b < 0 ? 0 : op.b, s1 = op.b < 0 ? L : op.b + 1;
  {
    double2* psi = st + vec * n;
    for (int s = s0; s < s1; ++s) {
      const uint32_t low = (1u << s) - 1u;
      for (uint32_t j = threadIdx.x; j < n / 2; j += NT) {
        const uint32_t lo = ((j & ~low) << 1) | (j & low);
        const uint32_t hi = lo | (1u << s);
        const double2 a = psi[lo], b = psi[hi];
        psi[lo] = make_double2((llr * a.x - lli * a.y) + (lhr * b.x - lhi * b.y),
                               (llr * a.y + lli * a.x) + (lhr * b.y + lhi * b.x));
        psi[hi] = make_double2((hlr * a.x - hli * a.y) + (hhr * b.x - hhi * b.y),
                               (hlr * a.y + hli * a.x) + (hhr * b.y + hhi * b.x));
      }
      __syncthreads();
    }
  }
}

// One thread's share of observable i of a realisation with state psi and
// reference ref: amplitudes k0 + threadIdx.x, k0 + threadIdx.x + NT, ... < k1.
// CORR (x, y) = <ref| sum_s sigma^axis_s |psi>, MAG = <psi|sigma^axis_spin|psi>,
// NORM = (<psi|psi>, <ref|ref>), ENERGY = <psi|H|psi> with the realisation's
// own fields, all in FP64.
template <int NT>
__device__ __forceinline__ double2 obs_thread(const Args& args, const RealDev& rd, int L,
                                              const double2* psi, const double2* ref, int i,
                                              uint32_t k0, uint32_t k1) {
  const int kind = args.obs[3 * i], axis = args.obs[3 * i + 1], spin = args.obs[3 * i + 2];
  double2 v = make_double2(0.0, 0.0);
  if (kind == SS_OBS_CORR) {
    for (uint32_t k = k0 + threadIdx.x; k < k1; k += NT) {
      double sr = 0.0, si = 0.0;
      for (int s = 0; s < L; ++s) {
        const double2 q = sigma_at(psi, k, s, axis);
        sr += q.x;
        si += q.y;
      }
      const double2 r = ref[k];
      v.x += r.x * sr + r.y * si;
      v.y += r.x * si - r.y * sr;
    }
  } else if (kind == SS_OBS_MAG) {
    for (uint32_t k = k0 + threadIdx.x; k < k1; k += NT) {
      const double2 q = sigma_at(psi, k, spin, axis);
      const double2 p = psi[k];
      v.x += p.x * q.x + p.y * q.y;
    }
  } else if (kind == SS_OBS_NORM) {
    for (uint32_t k = k0 + threadIdx.x; k < k1; k += NT) {
      const double2 p = psi[k], r = ref[k];
      v.x += p.x * p.x + p.y * p.y;
      v.y += r.x * r.x + r.y * r.y;
    }
  } else {
    const TypeDev ty = args.types[rd.type_off + args.measure_type];
    const double* cb = args.cpool + ty.c_off;
    const int2* pl = args.pairs + rd.pair_off;
    const int P = rd.npairs;
    for (uint32_t k = k0 + threadIdx.x; k < k1; k += NT) {
      const double2 p = psi[k];
      double d = 0.0;
      for (int s = 0; s < L; ++s) d += ((k >> s) & 1u) ? cb[3 * P + s] : -cb[3 * P + s];
      for (int q = 0; q < P; ++q) {
        const int2 pr = pl[q];
        d += (((k >> pr.x) ^ (k >> pr.y)) & 1u) ? -cb[2 * P + q] : cb[2 * P + q];
      }
      double hr = d * p.x, hi = d * p.y;
      for (int s = 0; s < L; ++s) {
        const double cx = cb[3 * P + L + s];
        const double cy = ((k >> s) & 1u) ? -cb[3 * P + 2 * L + s] : cb[3 * P + 2 * L + s];
        const double2 w = psi[k ^ (1u << s)];
        hr += cx * w.x - cy * w.y;
        hi += cx * w.y + cy * w.x;
      }
      for (int q = 0; q < P; ++q) {
        const int2 pr = pl[q];
        const bool anti = (((k >> pr.x) ^ (k >> pr.y)) & 1u) != 0;
        const double c = anti ? cb[q] : cb[P + q];
        const double2 w = psi[k ^ (1u << pr.x) ^ (1u << pr.y)];
        hr += c * w.x;
        hi += c * w.y;
      }
      v.x += hr * p.x + hi * p.y;
    }
  }
  return v;
}

// Writes observable i's total into the row at column col and returns the
// next column (CORR and NORM take two).
__device__ __forceinline__ int obs_store(const Args& args, double* row, int col, int i, double2 v) {
  const int kind = args.obs[3 * i];
  if (kind == SS_OBS_CORR) {
    row[col] = v.x;
    row[col + 1] = v.y;
  } else if (kind == SS_OBS_NORM) {
    row[col] = sqrt(v.x);
    row[col + 1] = sqrt(v.y);
  } else {
    row[col] = v.x;
  }
  return col + ((kind == SS_OBS_CORR || kind == SS_OBS_NORM) ? 2 : 1);
}

template <int L, int NT>
__device__ void measure_op(const Args& args, double2* stage, double2* red, const RealDev& rd,
                           const double2* st, const Op& op) {
  constexpr uint32_t N = 1u << L;
  const uint32_t t = threadIdx.x;
  __syncthreads();
  for (uint32_t k = t; k < N; k += NT) stage[k] = st[k];
  __syncthreads();
  const double2* ref = st + N;
  double* row = args.rows + rd.row_off + static_cast<long long>(op.a) * args.width;
  int col = 0;
  for (int i = 0; i < args.nobs; ++i) {
    const double2 v = cta_sum2<NT>(obs_thread<NT>(args, rd, L, stage, ref, i, 0u, N), red);
    if (t == 0) col = obs_store(args, row, col, i, v);
  }
  __syncthreads();
}

// Shared-memory carve-up: three recursion buffers, psi (when it lives here),
// the coupling tables, the correction terms and the reduction slots.
template <int L, int R, typename Real, int PSI>
struct SmemLayout {
  using C2 = typename Cplx<Real>::T;
  static constexpr size_t N = size_t{1} << L;
  static constexpr size_t NP = (size_t{1} << L) + (size_t{1} << (L - R));  // padded
  static constexpr size_t bufs = 3 * NP * sizeof(C2);
  static constexpr size_t psi = PSI == PSI_SMEM ? N * sizeof(double2) : 0;
  static constexpr size_t at_psi = bufs;
  static constexpr size_t at_coef = at_psi + psi;
  static constexpr size_t coef = (2 * L * L + 2 * L) * sizeof(Real);
  static constexpr size_t at_corr = (at_coef + coef + 15) & ~size_t{15};
  static constexpr size_t corr = kCorr * (sizeof(uint2) + sizeof(double2)) + 16;
  static constexpr size_t at_red = (at_corr + corr + 15) & ~size_t{15};
  static constexpr size_t total = at_red + 32 * sizeof(double2);
};

// One realisation per cluster of two CTAs: rank 0 carries the state, rank 1
// the reference, each through every evolve and pulse of the program.  The
// two meet only at measurements, where rank 0 reads both vectors from
// global memory between two cluster barriers.  Co-scheduling of a cluster's
// CTAs is guaranteed by the hardware, so the barriers always complete.
template <int L, int R, typename Real, int PSI>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Geo<L, R>::NT)
    k_batch(const __grid_constant__ Args args) {
  using Gm = Geo<L, R>;
  using C2 = typename Cplx<Real>::T;
  using SL = SmemLayout<L, R, Real, PSI>;
  constexpr int NT = Gm::NT, N = static_cast<int>(SL::NP);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<Real> sm;
  C2* base = reinterpret_cast<C2*>(smem_raw);
  sm.buf[0] = base;
  sm.buf[1] = base + N;
  sm.buf[2] = base + 2 * N;
  sm.psi = reinterpret_cast<double2*>(smem_raw + SL::at_psi);
  Real* coef = reinterpret_cast<Real*>(smem_raw + SL::at_coef);
  sm.cff = coef;
  sm.cfb = coef + L * L;
  sm.ccx = coef + 2 * L * L;
  sm.ccy = coef + 2 * L * L + L;
  sm.corr_coef = reinterpret_cast<double2*>(smem_raw + SL::at_corr);
  sm.corr_mask = reinterpret_cast<uint2*>(smem_raw + SL::at_corr + kCorr * sizeof(double2));
  sm.corr_n = reinterpret_cast<int*>(smem_raw + SL::at_corr + kCorr * (sizeof(double2) + sizeof(uint2)));
  sm.red = reinterpret_cast<double2*>(smem_raw + SL::at_red);
  __shared__ int s_work;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int vec = static_cast<int>(cluster.block_rank());
  int* lead_work = cluster.map_shared_rank(&s_work, 0);

  for (;;) {
    if (vec == 0 && threadIdx.x == 0) s_work = static_cast<int>(atomicAdd(args.counter, 1u));
    cluster.sync();
    const int w = *lead_work;
    cluster.sync();  // rank 1 has read the item before rank 0 may fetch again
    if (w >= args.nwork) break;
    const RealDev rd = args.reals[args.work[w]];
    double2* st = args.states + rd.state_off;
    for (int i = args.op_begin; i < args.op_end; ++i) {
      const Op op = args.ops[i];
      if (op.kind == OP_EVOLVE) {
        const TypeDev ty = args.types[rd.type_off + op.a];
        if (ty.order > 0 && op.b > 0) evolve_op<L, R, Real, PSI>(args, sm, rd, st, op, ty, vec);
      } else if (op.kind == OP_PULSE) {
        pulse_op<NT>(args, L, st, op, vec, rd.rot_off);
      } else {
        __threadfence();
        cluster.sync();  // both vectors are at this point of the program
        if (vec == 0) {
          measure_op<L, NT>(args, reinterpret_cast<double2*>(smem_raw), sm.red, rd, st, op);
        }
        cluster.sync();  // the reference stays put until it has been read
      }
    }
  }
}

// ------------------------------------------------- vectors over a cluster
// Sizes whose three recursion buffers exceed one CTA's shared memory spread
// each vector over C = 2^CB CTAs of the cluster: CTA `part` of a vector holds
// the amplitudes whose top CB bits equal `part`, with the same layout schedule
// over the L - CB local bits.  Couplings that reach a CTA bit read the partner
// block from the peer CTA's shared memory (distributed shared memory); one
// cluster barrier per Chebyshev order publishes T_n to the peers.  The
// cluster holds 2C CTAs: ranks 0 .. C-1 the state, C .. 2C-1 the reference;
// both run the same number of orders, so their barriers pair up.
//
// Split clusters hold C CTAs and carry one vector: a work item is a
// (realisation, vector) pair, so the state and the reference of a
// realisation run on different clusters and never wait for each other.  At
// each measurement point a vector copies itself to its snapshot slot, and
// k_batch_measure_snap computes the observables from the snapshot pairs once
// the bucket is done.  Half the cluster size lets more CTAs be resident (at
// L = 16 on B200: 15 clusters of 8, 120 SMs, instead of 7 of 16, 112 SMs),
// for one vector write and read per measurement point.
namespace cg = cooperative_groups;

template <typename T>
__device__ __forceinline__ T* peer_ptr(cg::cluster_group& cl, T* local, unsigned rank, unsigned mine) {
  return rank == mine ? local : cl.map_shared_rank(local, rank);
}

template <int L, int R, int CB, typename Real>
__device__ void evolve_dist(const Args& args, const Smem<Real>& sm, const RealDev& rd, double2* st,
                            const Op& op, const TypeDev& ty, int vec, uint32_t part,
                            cg::cluster_group& cl, double* s_norm) {
  constexpr int Ll = L - CB;
  constexpr int C = 1 << CB;
  using Gm = Geo<Ll, R>;
  using C2 = typename Cplx<Real>::T;
  constexpr int NT = Gm::NT, NA = Gm::NA, G = Gm::G;
  constexpr uint32_t N = 1u << L;
  constexpr int bl = Gm::base(G - 1);
  constexpr bool kMixed = std::is_same<Real, float>::value;
  const uint32_t t = threadIdx.x;
  const unsigned me = cl.block_rank();
  const unsigned group = me - part;  // cluster rank of this vector's part 0
  const uint32_t hi = part << Ll;
  const int P = rd.npairs;
  const double* cb = args.cpool + ty.c_off;
  const int2* pl = args.pairs + rd.pair_off;

  __syncthreads();
  for (int i = t; i < L * L; i += NT) {
    sm.cff[i] = Real(0);
    sm.cfb[i] = Real(0);
  }
  __syncthreads();
  for (int p = t; p < P; p += NT) {
    const int2 q = pl[p];
    sm.cff[q.x * L + q.y] = Real(cb[p]);
    sm.cfb[q.x * L + q.y] = Real(cb[P + p]);
  }
  for (int s = t; s < L; s += NT) {
    sm.ccx[s] = Real(cb[3 * P + L + s]);
    sm.ccy[s] = Real(cb[3 * P + 2 * L + s]);
  }
  if (t == 0) {
    int nc = 0;
    if (kMixed) {
      const double* ct = cb + 3 * P + 3 * L;
      for (int c = 0; c < kCorr; ++c) {
        const int pi = static_cast<int>(ct[4 * c]);
        if (pi < 0) continue;
        const int2 q = pl[pi];
        sm.corr_mask[nc] = make_uint2(1u << q.x, 1u << q.y);
        sm.corr_coef[nc] = make_double2(ct[4 * c + 1], ct[4 * c + 2]);
        ++nc;
      }
    }
    *sm.corr_n = nc;
  }
  double dg[NA];
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    const uint32_t k = hi | t | (uint32_t(a) << bl);
    double d = 0.0;
    for (int s = 0; s < L; ++s) {
      const double c = cb[3 * P + s];
      d += ((k >> s) & 1u) ? c : -c;
    }
    for (int p = 0; p < P; ++p) {
      const int2 q = pl[p];
      const double c = cb[2 * P + p];
      d += (((k >> q.x) ^ (k >> q.y)) & 1u) ? -c : c;
    }
    dg[a] = ty.scale * d;
  }
  __syncthreads();

  const bool has_trans = (ty.flags & 1) != 0, has_fb = (ty.flags & 2) != 0;
  const int ncorr = *sm.corr_n;
  const double2* wts = args.wpool + ty.w_off;
  const double a0 = wts[0].x;
  double2* psig = st + vec * N;
  // CTA-bit fields and CTA-CTA couplings, uniform over this CTA
  Real tcx[CB > 0 ? CB : 1], tcy[CB > 0 ? CB : 1];
#pragma unroll
  for (int jb = 0; jb < CB; ++jb) {
    tcx[jb] = has_trans ? sm.ccx[Ll + jb] : Real(0);
    tcy[jb] = has_trans ? (((part >> jb) & 1u) ? -sm.ccy[Ll + jb] : sm.ccy[Ll + jb]) : Real(0);
  }
  constexpr int NCC = CB * (CB - 1) / 2;
  Real ccc[NCC > 0 ? NCC : 1];
  uint32_t cmask[NCC > 0 ? NCC : 1];
  {
    int q = 0;
#pragma unroll
    for (int j1 = 0; j1 < CB; ++j1) {
#pragma unroll
      for (int j2 = j1 + 1; j2 < CB; ++j2) {
        const bool anti = (((part >> j1) ^ (part >> j2)) & 1u) != 0;
        ccc[q] = anti ? sm.cff[(Ll + j1) * L + Ll + j2] : (has_fb ? sm.cfb[(Ll + j1) * L + Ll + j2] : Real(0));
        cmask[q] = (1u << j1) | (1u << j2);
        ++q;
      }
    }
  }

  for (int step = 0; step < op.b; ++step) {
    int ic = 0;  // which of buf[0], buf[1] holds T_{n-1}
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      const uint32_t kl = t | (uint32_t(a) << bl);
      double2 p = __ldcg(&psig[hi | kl]);
      C2 c;
      c.x = Real(p.x);
      c.y = Real(p.y);
      sm.buf[0][pad<R>(kl)] = c;
      p.x *= a0;
      p.y *= a0;
      __stcg(&psig[hi | kl], p);
    }
    cl.sync();  // every slice of T_0 is in place
    for (int n = 1; n <= ty.order; ++n) {
      const double2 cn = wts[n];
      C2* cur = sm.buf[ic];
      C2* prv = sm.buf[ic ^ 1];
      const C2* rc[CB > 0 ? CB : 1];
#pragma unroll
      for (int jb = 0; jb < CB; ++jb) rc[jb] = cl.map_shared_rank(cur, group + (part ^ (1u << jb)));
      front_layouts<Ll, R, Real, 0, L, CB>(sm, cur, t, has_trans, has_fb, rc, part);
      C2 acc[NA], own[NA];
      layout_pass<Ll, R, Real, G - 1, L, CB>(sm, cur, acc, own, t, has_trans, has_fb, rc, part);
      C2* prv_mine = prv + pad<R>(t);
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const uint32_t kl = t | (uint32_t(a) << bl);
        const uint32_t off = pad<R>(kl);
#pragma unroll
        for (int jb = 0; jb < CB; ++jb) {
          if (has_trans) {
            const C2 w = rc[jb][off];
            acc[a].x += tcx[jb] * w.x - tcy[jb] * w.y;
            acc[a].y += tcx[jb] * w.y + tcy[jb] * w.x;
          }
        }
#pragma unroll
        for (int q = 0; q < NCC; ++q) {
          const C2 w = cl.map_shared_rank(cur, group + (part ^ cmask[q]))[off];
          acc[a].x += ccc[q] * w.x;
          acc[a].y += ccc[q] * w.y;
        }
        const uint32_t k = hi | kl;
        double hx = double(acc[a].x) + dg[a] * double(own[a].x);
        double hy = double(acc[a].y) + dg[a] * double(own[a].y);
#pragma unroll
        for (int c = 0; c < kCorr; ++c) {
          if (c < ncorr) {
            const uint2 mk = sm.corr_mask[c];
            const double2 cc = sm.corr_coef[c];
            const uint32_t kp = k ^ mk.x ^ mk.y;
            const C2 w = peer_ptr(cl, cur, group + (kp >> Ll), me)[pad<R>(kp & ((1u << Ll) - 1u))];
            const double co = (((k & mk.x) != 0) == ((k & mk.y) != 0)) ? cc.y : cc.x;
            hx += co * double(w.x);
            hy += co * double(w.y);
          }
        }
        const uint32_t offs = pad<R>(uint32_t(a) << bl);
        if (n == 1) {
          hx *= 0.5;
          hy *= 0.5;
        } else {
          const C2 q = prv_mine[offs];
          hx -= double(q.x);
          hy -= double(q.y);
        }
        C2 tn;
        tn.x = Real(hx);
        tn.y = Real(hy);
        prv_mine[offs] = tn;
        double2 p = __ldcg(&psig[k]);
        p.x += cn.x * hx - cn.y * hy;
        p.y += cn.x * hy + cn.y * hx;
        __stcg(&psig[k], p);
      }
      cl.sync();  // T_n published; every peer is done reading T_{n-1}
      ic ^= 1;
    }
    if (op.c) {  // autonormalise over the C CTAs of this vector, in part order
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        const double2 p = __ldcg(&psig[hi | t | (uint32_t(a) << bl)]);
        s += p.x * p.x + p.y * p.y;
      }
      s = cta_sum2<NT>(make_double2(s, 0.0), sm.red).x;
      if (t == 0) *s_norm = s;
      cl.sync();
      double tot = 0.0;
      for (int q = 0; q < C; ++q) tot += *peer_ptr(cl, s_norm, group + q, me);
      const double nrm = sqrt(tot);
      if (nrm == 0.0 || !isfinite(nrm)) {
        if (t == 0 && part == 0) atomicExch(args.flags, nrm == 0.0 ? SS_ERR_DOMAIN : SS_ERR_NUMERIC);
      } else {
        const double f = 1.0 / nrm;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
          const uint32_t k = hi | t | (uint32_t(a) << bl);
          double2 p = __ldcg(&psig[k]);
          p.x *= f;
          p.y *= f;
          __stcg(&psig[k], p);
        }
      }
      cl.sync();  // s_norm may be reused
    }
  }
}

// A pulse on a vector spread over C CTAs: each CTA rotates a slice of the
// amplitude pairs of every target spin, a cluster barrier between spins.
template <int NT, int C>
__device__ void pulse_dist(const Args& args, int L, double2* st, const Op& op, int vec,
                           uint32_t part, long long rot_off, cg::cluster_group& cl) {
  const double* u = args.rots + rot_off + 8 * op.a;
  const double llr = u[0], lli = u[1], lhr = u[2], lhi = u[3];
  const double hlr = u[4], hli = u[5], hhr = u[6], hhi = u[7];
  const uint32_t n = 1u << L;
  const uint32_t slice = (n / 2) / C;
  const int s0 = op.b < 0 ? 0 : op.b, s1 = op.b < 0 ? L : op.b + 1;
  double2* psi = st + vec * n;
  for (int s = s0; s < s1; ++s) {
    const uint32_t low = (1u << s) - 1u;
    for (uint32_t j = part * slice + threadIdx.x; j < (part + 1) * slice; j += NT) {
      const uint32_t lo = ((j & ~low) << 1) | (j & low);
      const uint32_t hi = lo | (1u << s);
      const double2 a = __ldcg(&psi[lo]), b = __ldcg(&psi[hi]);
      __stcg(&psi[lo], make_double2((llr * a.x - lli * a.y) + (lhr * b.x - lhi * b.y),
                                    (llr * a.y + lli * a.x) + (lhr * b.y + lhi * b.x)));
      __stcg(&psi[hi], make_double2((hlr * a.x - hli * a.y) + (hhr * b.x - hhi * b.y),
                                    (hlr * a.y + hli * a.x) + (hhr * b.y + hhi * b.x)));
    }
    __threadfence();
    cl.sync();
  }
}

// Observables of a realisation whose vectors live in global memory, the
// amplitude range split over the cluster's CTAs; rank 0 adds the per-CTA
// partial sums in rank order and writes the row.
template <int NT>
__device__ void measure_dist(const Args& args, double2* red, double2* s_part, const RealDev& rd,
                             const double2* st, const Op& op, cg::cluster_group& cl) {
  const int L = rd.L;
  const uint32_t N = 1u << L;
  const unsigned me = cl.block_rank(), nb = cl.num_blocks();
  const uint32_t chunk = N / nb;
  const uint32_t k0 = me * chunk, k1 = k0 + chunk;
  for (int i = 0; i < args.nobs; ++i) {
    const double2 v = cta_sum2<NT>(obs_thread<NT>(args, rd, L, st, st + N, i, k0, k1), red);
    if (threadIdx.x == 0) s_part[i] = v;
  }
  cl.sync();
  if (me == 0 && threadIdx.x == 0) {
    double* row = args.rows + rd.row_off + static_cast<long long>(op.a) * args.width;
    int col = 0;
    for (int i = 0; i < args.nobs; ++i) {
      double2 v = make_double2(0.0, 0.0);
      for (unsigned b = 0; b < nb; ++b) v += *peer_ptr(cl, &s_part[i], b, me);
      col = obs_store(args, row, col, i, v);
    }
  }
  cl.sync();  // partial slots may be reused
}

constexpr int kMaxDistObs = 8;

template <int L, int R, int CB, typename Real>
struct DistLayout {
  static constexpr int Ll = L - CB;
  using SL = SmemLayout<Ll, R, Real, PSI_GLOBAL>;
  // the coupling tables cover all L spins
  static constexpr size_t NP = SL::NP;
  using C2 = typename Cplx<Real>::T;
  static constexpr size_t bufs = 3 * NP * sizeof(C2);
  static constexpr size_t at_coef = bufs;
  static constexpr size_t coef = (2 * L * L + 2 * L) * sizeof(Real);
  static constexpr size_t at_corr = (at_coef + coef + 15) & ~size_t{15};
  static constexpr size_t corr = kCorr * (sizeof(uint2) + sizeof(double2)) + 16;
  static constexpr size_t at_red = (at_corr + corr + 15) & ~size_t{15};
  static constexpr size_t at_part = at_red + 32 * sizeof(double2);
  static constexpr size_t at_norm = at_part + kMaxDistObs * sizeof(double2);
  static constexpr size_t total = at_norm + 16;
};

// One realisation per cluster of 2 * 2^CB CTAs, or with SPLIT one vector per
// cluster of 2^CB CTAs (cluster size given at launch).
template <int L, int R, int CB, typename Real, bool SPLIT>
__global__ void __launch_bounds__(Geo<L - CB, R>::NT) k_batch_dist(const __grid_constant__ Args args) {
  constexpr int Ll = L - CB, C = 1 << CB;
  using Gm = Geo<Ll, R>;
  using C2 = typename Cplx<Real>::T;
  using DL = DistLayout<L, R, CB, Real>;
  constexpr int NT = Gm::NT, NP = static_cast<int>(DL::NP);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<Real> sm;
  C2* base = reinterpret_cast<C2*>(smem_raw);
  sm.buf[0] = base;
  sm.buf[1] = base + NP;
  sm.buf[2] = base + 2 * NP;
  sm.psi = nullptr;
  Real* coef = reinterpret_cast<Real*>(smem_raw + DL::at_coef);
  sm.cff = coef;
  sm.cfb = coef + L * L;
  sm.ccx = coef + 2 * L * L;
  sm.ccy = coef + 2 * L * L + L;
  sm.corr_coef = reinterpret_cast<double2*>(smem_raw + DL::at_corr);
  sm.corr_mask = reinterpret_cast<uint2*>(smem_raw + DL::at_corr + kCorr * sizeof(double2));
  sm.corr_n = reinterpret_cast<int*>(smem_raw + DL::at_corr + kCorr * (sizeof(double2) + sizeof(uint2)));
  sm.red = reinterpret_cast<double2*>(smem_raw + DL::at_red);
  double2* s_part = reinterpret_cast<double2*>(smem_raw + DL::at_part);
  double* s_norm = reinterpret_cast<double*>(smem_raw + DL::at_norm);
  __shared__ int s_work, s_item;
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  const uint32_t part = rank % C;
  // a split cluster's work item, re-read from shared memory where it is
  // needed rather than held in registers across the recursion
  const volatile int* item = &s_item;
  int* lead_work = cluster.map_shared_rank(&s_work, 0);
  const int nitems = SPLIT ? 2 * args.nwork : args.nwork;

  for (;;) {
    if (rank == 0 && threadIdx.x == 0) s_work = static_cast<int>(atomicAdd(args.counter, 1u));
    cluster.sync();
    const int w = *lead_work;
    if (SPLIT && threadIdx.x == 0) s_item = w;
    cluster.sync();
    if (w >= nitems) break;
    const RealDev rd = args.reals[args.work[SPLIT ? w >> 1 : w]];
    double2* st = args.states + rd.state_off;
    for (int i = args.op_begin; i < args.op_end; ++i) {
      const Op op = args.ops[i];
      if (op.kind == OP_EVOLVE) {
        const TypeDev ty = args.types[rd.type_off + op.a];
        if (ty.order > 0 && op.b > 0) {
          const int vec = SPLIT ? (*item & 1) : static_cast<int>(rank / C);
          evolve_dist<L, R, CB, Real>(args, sm, rd, st, op, ty, vec, part, cluster, s_norm);
          __threadfence();
          cluster.sync();  // psi complete in global memory
        }
      } else if (op.kind == OP_PULSE) {
        const int vec = SPLIT ? (*item & 1) : static_cast<int>(rank / C);
        pulse_dist<NT, C>(args, L, st, op, vec, part, rd.rot_off, cluster);
      } else if (SPLIT) {
        // evolve and pulse end on a fenced cluster barrier, so every part
        // of the vector is in global memory; each CTA copies its own part
        constexpr uint32_t N = 1u << L, chunk = N / C;
        const int slot = *item >> 1, vec = *item & 1;
        const double2* src = st + vec * N + part * chunk;
        double2* dst = args.snap + ((static_cast<long long>(slot) * args.nmeas + op.a) * 2 + vec) * N +
                       part * chunk;
        for (uint32_t k = threadIdx.x; k < chunk; k += NT) __stcg(&dst[k], __ldcg(&src[k]));
        cluster.sync();  // no part is overwritten before its copy is taken
      } else {
        __threadfence();
        cluster.sync();
        measure_dist<NT>(args, sm.red, s_part, rd, st, op, cluster);
      }
    }
  }
}

// Observables from the snapshots of split clusters: one CTA per (work slot,
// measurement point), the same per-thread sums as the one-CTA kernel.
constexpr int kSnapThreads = 256;

__global__ void __launch_bounds__(kSnapThreads) k_batch_measure_snap(const __grid_constant__ Args args) {
  __shared__ double2 red[32];
  const long long items = static_cast<long long>(args.nwork) * args.nmeas;
  for (long long it = blockIdx.x; it < items; it += gridDim.x) {
    const int slot = static_cast<int>(it / args.nmeas), m = static_cast<int>(it % args.nmeas);
    const RealDev rd = args.reals[args.work[slot]];
    const uint32_t N = 1u << rd.L;
    const double2* psi = args.snap + it * 2 * N;
    double* row = args.rows + rd.row_off + static_cast<long long>(m) * args.width;
    int col = 0;
    for (int i = 0; i < args.nobs; ++i) {
      const double2 v =
          cta_sum2<kSnapThreads>(obs_thread<kSnapThreads>(args, rd, rd.L, psi, psi + N, i, 0u, N), red);
      if (threadIdx.x == 0) col = obs_store(args, row, col, i, v);
    }
  }
}

// ------------------------------------------------------------ variants
struct Variant {
  int L, R;
  bool mixed;
  int psi;
  int threads;
  size_t smem;
  void (*kernel)(Args);
  int cb;  // each vector spread over 2^cb CTAs (k_batch_dist); 0 = one CTA
  bool split;  // one vector per cluster, observables from snapshots
  int cluster() const { return split ? 1 << cb : 2 << cb; }
};

template <int L, int R, typename Real, int PSI>
Variant make_variant() {
  return Variant{L, R, std::is_same<Real, float>::value, PSI, Geo<L, R>::NT,
                 SmemLayout<L, R, Real, PSI>::total, &k_batch<L, R, Real, PSI>, 0, false};
}

template <int L, int R, int CB, typename Real, bool SPLIT = false>
Variant make_dist_variant() {
  return Variant{L, R, std::is_same<Real, float>::value, PSI_GLOBAL, Geo<L - CB, R>::NT,
                 DistLayout<L, R, CB, Real>::total, &k_batch_dist<L, R, CB, Real, SPLIT>, CB, SPLIT};
}

// The per-size schedules: register bits R and where psi lives.  Chosen so a
// realisation fits one CTA (threads = 2^(L-R) >= 32), the three shared
// buffers fit 227 KB, and the registers fit the thread count.
const std::vector<Variant>& variants() {
  static const std::vector<Variant> v = {
      make_variant<6, 1, float, PSI_REG>(),     make_variant<7, 2, float, PSI_REG>(),
      make_variant<8, 3, float, PSI_REG>(),     make_variant<9, 4, float, PSI_SMEM>(),
      make_variant<10, 4, float, PSI_SMEM>(),   make_variant<11, 4, float, PSI_SMEM>(),
      make_variant<12, 4, float, PSI_SMEM>(),   make_variant<13, 4, float, PSI_GLOBAL>(),
      make_variant<6, 1, double, PSI_REG>(),    make_variant<7, 2, double, PSI_REG>(),
      make_variant<8, 3, double, PSI_REG>(),    make_variant<9, 3, double, PSI_SMEM>(),
      make_variant<10, 3, double, PSI_SMEM>(),  make_variant<11, 3, double, PSI_SMEM>(),
      make_variant<12, 3, double, PSI_GLOBAL>(),
      // vectors over clusters: 2 / 4 / 8 CTAs per vector
      make_dist_variant<14, 4, 1, float>(),     make_dist_variant<15, 4, 2, float>(),
      make_dist_variant<16, 4, 3, float>(),     make_dist_variant<13, 3, 1, double>(),
      make_dist_variant<14, 3, 2, double>(),    make_dist_variant<15, 3, 3, double>(),
      // alternative schedules the autotuner may pick (the first entry of a
      // size is its default): fewer register bits (more threads), or a
      // second CTA per vector
      make_variant<10, 3, float, PSI_SMEM>(),   make_variant<11, 3, float, PSI_SMEM>(),
      make_variant<12, 3, float, PSI_SMEM>(),   make_dist_variant<13, 4, 1, float>(),
      make_variant<11, 4, double, PSI_SMEM>(),  make_dist_variant<12, 3, 1, double>(),
      // cluster sizes with five register bits: 256 threads of 32 amplitudes,
      // three layouts instead of four and no 128-register cap
      make_dist_variant<14, 5, 1, float>(),     make_dist_variant<15, 5, 2, float>(),
      make_dist_variant<16, 5, 3, float>(),
      // L = 12 with four register bits in FP64 (256 threads of 16
      // amplitudes) and with the FP32 path's psi in registers; both keep one
      // CTA per SM, which the buckets' shares of the device assume
      make_variant<12, 4, double, PSI_GLOBAL>(), make_variant<12, 4, float, PSI_REG>(),
      // psi in registers for the FP64 routing target at L = 12 and the
      // mid-size FP32 schedules
      make_variant<12, 3, double, PSI_REG>(),   make_variant<12, 4, double, PSI_REG>(),
      make_variant<11, 4, float, PSI_REG>(),    make_variant<10, 4, float, PSI_REG>(),
      make_variant<10, 3, double, PSI_REG>(),   make_variant<11, 3, double, PSI_REG>(),
      // split clusters: the state and the reference of a realisation on
      // clusters of their own
      make_dist_variant<14, 4, 1, float, true>(), make_dist_variant<15, 4, 2, float, true>(),
      make_dist_variant<16, 4, 3, float, true>(),
      // FP64 at L = 16: 16 CTAs per vector (Ll = 12, the FP64 L = 13..15
      // layout), which only the split form fits in one cluster
      make_dist_variant<16, 3, 4, double, true>(),
  };
  return v;
}

// The default schedule of a size: its first entry.
const Variant* find_variant(int L, bool mixed) {
  for (const Variant& v : variants()) {
    if (v.L == L && v.mixed == mixed) return &v;
  }
  return nullptr;
}

std::string variant_name(const Variant& v) {
  static const char* homes[] = {"reg", "smem", "global"};
  return "L" + std::to_string(v.L) + ".R" + std::to_string(v.R) + (v.mixed ? ".f32." : ".f64.") +
         homes[v.psi] + ".c" + std::to_string(1 << v.cb) + (v.split ? ".split" : "");
}

}  // namespace

// ------------------------------------------------------------- schedules
// The schedule table: for (device name, L, precision) the variant the
// autotuner measured fastest and its cost in nanoseconds per amplitude-order.
// Batches use it for the kernel of each size bucket and, when every bucket
// has a measured cost, for the buckets' shares of the device.  A tuning run
// forces one candidate at a time through `g_force`.
struct Choice {
  std::string variant;
  double ns = 0.0;
};
std::mutex g_sched_mu;
std::map<std::tuple<std::string, int, int>, Choice> g_sched;
thread_local const Variant* g_force = nullptr;

std::string device_name(int dev) {
  cudaDeviceProp p{};
  SS_CUDA(cudaGetDeviceProperties(&p, dev));
  return p.name;
}

const Variant* scheduled_variant(const std::string& dev, int L, bool mixed, double* ns) {
  *ns = 0.0;
  if (g_force && g_force->L == L && g_force->mixed == mixed) return g_force;
  {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    auto it = g_sched.find({dev, L, mixed ? 1 : 0});
    if (it != g_sched.end()) {
      for (const Variant& v : variants()) {
        if (v.L == L && v.mixed == mixed && variant_name(v) == it->second.variant) {
          *ns = it->second.ns;
          return &v;
        }
      }
    }
  }
  return find_variant(L, mixed);
}

// ------------------------------------------------------------------ host
struct TypeKey {
  int table;
  int from_draw;
  int mode;
  double tau;
  bool operator<(const TypeKey& o) const {
    return std::tie(table, from_draw, mode, tau) < std::tie(o.table, o.from_draw, o.mode, o.tau);
  }
};

struct Bucket {
  int L = 0;
  const Variant* var = nullptr;
  std::vector<int> work;
  int grid = 0;
  unsigned int* counter = nullptr;
  int* dev_work = nullptr;
  cudaStream_t side = nullptr;
  // split clusters: realisations per launch and their snapshots
  int chunk = 0;
  double2* snap = nullptr;
};

}  // namespace batch
}  // namespace ss

using namespace ss;
using namespace ss::batch;

struct ss_batch {
  ss_engine* engine = nullptr;
  int precision = SS_PRECISION_MIXED;
  uint64_t first = 0;
  int64_t count = 0;
  int64_t points = 0, width = 0;
  int ntypes = 0;  // evolve step types; slot ntypes is the energy table
  std::vector<double> times;
  // host staging
  std::vector<Op> ops;
  std::vector<double> rots;
  std::vector<RealDev> reals;
  std::vector<TypeDev> types;
  std::vector<double> cpool;
  std::vector<double> wpool;  // (re, im) pairs
  std::vector<int2> pairs;
  std::vector<double> psi0;   // (re, im) pairs
  std::vector<long long> psi0_off;
  std::vector<int> obs;
  std::vector<Bucket> buckets;
  int ref_axis = 0;
  long long state_len = 0, rows_len = 0;
  int64_t orders_total = 0;
  double amp_orders = 0.0;
  int64_t launches_per_run = 0;
  std::vector<int32_t> real_precision;  // ss_precision per realisation, index order
  std::vector<double> real_amp_orders;  // amplitudes x orders per realisation
  std::vector<double> real_error_estimate;  // mixed precision: orders x uncorrected residual
  // device
  Op* d_ops = nullptr;
  double* d_rots = nullptr;
  RealDev* d_reals = nullptr;
  TypeDev* d_types = nullptr;
  double* d_cpool = nullptr;
  double2* d_wpool = nullptr;
  int2* d_pairs = nullptr;
  double2* d_psi0 = nullptr;
  long long* d_psi0_off = nullptr;
  double2* d_states = nullptr;
  double* d_rows = nullptr;
  int* d_obs = nullptr;
  int* d_flags = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool uploaded = false;
};

namespace ss {
namespace batch {
namespace {

template <typename T>
void dev_alloc(T** p, size_t n) {
  SS_CUDA(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(n, 1)));
}

template <typename T>
void upload_vec(T* dst, const std::vector<T>& src, cudaStream_t s) {
  if (!src.empty()) {
    SS_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, s));
  }
}

void linearise(const ss_run_config& c, int begin, int end, std::vector<Op>& ops,
               std::map<TypeKey, int>& types, std::vector<TypeKey>& keys,
               std::map<std::vector<double>, int>& rot_ids, std::vector<double>& rots,
               std::vector<std::array<double, 4>>& rot_src, int64_t& point) {
  for (int at = begin; at < end;) {
    const ss_step& s = c.steps[at];
    if (s.kind == SS_STEP_EVOLVE) {
      const TypeKey key{s.field_table, s.tau_from_draw ? 1 : 0, s.mode, s.tau};
      auto it = types.find(key);
      if (it == types.end()) {
        it = types.emplace(key, static_cast<int>(keys.size())).first;
        keys.push_back(key);
      }
      require(s.count >= 0 && s.count < (int64_t{1} << 30), SS_ERR_CONFIG, "step count out of range");
      ops.push_back(Op{OP_EVOLVE, it->second, static_cast<int>(s.count), s.autonormalize ? 1 : 0});
      ++at;
    } else if (s.kind == SS_STEP_PULSE) {
      double u[8];
      rotation_matrix(s.axis, s.angle, u);
      std::vector<double> key(u, u + 8);
      auto it = rot_ids.find(key);
      if (it == rot_ids.end()) {
        it = rot_ids.emplace(key, static_cast<int>(rots.size() / 8)).first;
        rots.insert(rots.end(), u, u + 8);
        rot_src.push_back({s.axis[0], s.axis[1], s.axis[2], s.angle});
      }
      ops.push_back(Op{OP_PULSE, it->second, s.target, 0});
      ++at;
    } else if (s.kind == SS_STEP_MEASURE) {
      ops.push_back(Op{OP_MEASURE, static_cast<int>(point++), 0, 0});
      ++at;
    } else {
      for (int64_t i = 0; i < s.count; ++i) {
        linearise(c, at + 1, at + 1 + s.body_len, ops, types, keys, rot_ids, rots, rot_src, point);
      }
      at += 1 + s.body_len;
    }
  }
}

// Coefficient block of one table (see TypeDev) with the reference's skip rule.
void coefficient_block(int L, const double* f, const std::vector<PairTerm>& pairs, double scale,
                       std::vector<double>& out, int* flags) {
  const size_t P = pairs.size();
  const size_t at = out.size();
  out.resize(at + 3 * P + 3 * L + 4 * kCorr, 0.0);
  double* cb = out.data() + at;
  for (size_t p = 0; p < P; ++p) {
    const double q = scale * 0.25;
    const double ff = q * (pairs[p].jx + pairs[p].jy);
    const double fb = q * (pairs[p].jx - pairs[p].jy);
    if (std::abs(ff) > kNegligible) cb[p] = ff;
    if (std::abs(fb) > kNegligible) {
      cb[P + p] = fb;
      *flags |= 2;
    }
    const double z = 0.25 * pairs[p].jz;
    if (std::abs(z) > kNegligible) cb[2 * P + p] = z;
  }
  for (int s = 0; s < L; ++s) {
    const double z = 0.5 * f[3 * s + 2];
    if (std::abs(z) > kNegligible) cb[3 * P + s] = z;
    const double cx = scale * 0.5 * f[3 * s], cy = scale * 0.5 * f[3 * s + 1];
    if (std::abs(cx) > kNegligible || std::abs(cy) > kNegligible) {
      cb[3 * P + L + s] = cx;
      cb[3 * P + 2 * L + s] = cy;
      *flags |= 1;
    }
  }
  // The kCorr strongest couplings and their FP32 rounding residuals.
  std::vector<size_t> idx(P);
  std::iota(idx.begin(), idx.end(), size_t{0});
  std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
    return std::abs(cb[x]) + std::abs(cb[P + x]) > std::abs(cb[y]) + std::abs(cb[P + y]);
  });
  double* ct = cb + 3 * P + 3 * L;
  for (int c = 0; c < kCorr; ++c) {
    ct[4 * c] = -1.0;
    if (static_cast<size_t>(c) >= P) continue;
    const size_t p = idx[static_cast<size_t>(c)];
    const double rff = cb[p] - static_cast<double>(static_cast<float>(cb[p]));
    const double rfb = cb[P + p] - static_cast<double>(static_cast<float>(cb[P + p]));
    if (rff == 0.0 && rfb == 0.0) continue;
    ct[4 * c] = static_cast<double>(p);
    ct[4 * c + 1] = rff;
    ct[4 * c + 2] = rfb;
  }
}

// Sum of the FP32 rounding residuals a mixed-precision table leaves
// uncorrected: every coupling channel except the kCorr strongest (whose
// residuals coefficient_block hands to the kernel) and the transverse
// fields, all in the table's scaled units.  The kernel applies this
// perturbation of H at every order, coherently, so orders x residual sum
// estimates the echo error a realisation accumulates in mixed precision.
double uncorrected_residual(int L, const double* f, const std::vector<PairTerm>& pairs,
                            double scale) {
  const size_t P = pairs.size();
  std::vector<double> ff(P), fb(P);
  auto rounding = [](double c) { return std::abs(c - static_cast<double>(static_cast<float>(c))); };
  for (size_t p = 0; p < P; ++p) {
    const double q = scale * 0.25;
    const double a = q * (pairs[p].jx + pairs[p].jy), b = q * (pairs[p].jx - pairs[p].jy);
    ff[p] = std::abs(a) > kNegligible ? a : 0.0;
    fb[p] = std::abs(b) > kNegligible ? b : 0.0;
  }
  std::vector<size_t> idx(P);
  std::iota(idx.begin(), idx.end(), size_t{0});
  std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) {
    return std::abs(ff[x]) + std::abs(fb[x]) > std::abs(ff[y]) + std::abs(fb[y]);
  });
  double sum = 0.0;
  for (size_t r = static_cast<size_t>(kCorr); r < P; ++r) {
    sum += rounding(ff[idx[r]]) + rounding(fb[idx[r]]);
  }
  for (int s = 0; s < L; ++s) {
    const double cx = scale * 0.5 * f[3 * s], cy = scale * 0.5 * f[3 * s + 1];
    if (std::abs(cx) > kNegligible || std::abs(cy) > kNegligible) {
      sum += rounding(cx) + rounding(cy);
    }
  }
  return sum;
}

struct PerReal {
  int L = 0;
  double error_estimate = 0.0;  // orders x uncorrected residual, both vectors
  double tau_draw = 1.0;
  std::vector<int2> pairs;
  std::vector<double> psi0;
  std::vector<TypeDev> types;
  std::vector<double> cpool, wpool;
  double cost = 0.0;
  int64_t orders = 0;
  double amp_orders = 0.0;
  bool mixed = false;
  int error = 0;
  std::string message;
};

// Mixed precision applies a pulse's transverse field as one FP32 number per
// spin; its rounding is a coherent flip-angle error repeated at every pulse.
// When the field is uniform (the same hx, or the same hy, on every spin) the
// expansion is rebuilt on a normalisation bound' within 1e-7 of the bound,
// chosen so that the scaled field is exactly an FP32 number.  Any bound' at
// least ||H|| gives the same propagator (the sum of term norms overestimates
// ||H|| by percents), and the truncation order is kept, so the FP64 result is
// unchanged to the level of the truncated tail.
void exact_transverse(int L, const double* f, int mode, double tau, Expansion& ex) {
  if (ex.order() == 0) return;
  const double hx = f[0], hy = f[1];
  if ((hx == 0.0) == (hy == 0.0)) return;  // none, or both components
  for (int s = 1; s < L; ++s) {
    if (f[3 * s] != hx || f[3 * s + 1] != hy) return;
  }
  const double h = hx != 0.0 ? hx : hy;
  const double scale = -2.0 / ex.bound;
  const double c32 = static_cast<double>(static_cast<float>(scale * 0.5 * h));
  const double scale2 = c32 / (0.5 * h);
  const double c2 = scale2 * 0.5 * h;
  if (!(scale2 < 0.0) || c2 != static_cast<double>(static_cast<float>(c2))) return;
  const double bound2 = -2.0 / scale2;
  if (std::abs(bound2 - ex.bound) > 1e-7 * ex.bound) return;
  const size_t order = ex.order();
  std::vector<double> a = bessel(mode == SS_TIME_IMAGINARY ? 1 : 0, bound2 * std::abs(tau),
                                 order + 1, nullptr);
  if (tau < 0.0) {
    for (size_t n = 1; n < a.size(); n += 2) a[n] = -a[n];
  }
  ex.a = a;
  ex.bound = bound2;
}

// Default routing of mixed batches: a realisation whose Chebyshev orders per
// state vector exceed its size's limit runs in FP64.  Measured on B200 with
// routing off (1024-2048 realisations per size of the CPMG and XY-8
// programs): the echo error of a mixed curve grows as orders^0.86 and falls
// with L (the FP32 rounding of 2^L amplitudes averages out in the overlap),
// so the order count at which the first curve passes 1e-6 grows by ~1.5x
// per spin: 9.3K / 14.5K / 48K / 121K orders at L = 8 / 10 / 12 / 14, none at
// L = 16 (max 2.7e-7 at 1.1e5 orders).  Up to L = 12 the limits are those
// counts times 0.8 (interpolated for odd L).  At L = 13..15 they stay at
// 40000, below what accuracy needs: the FP64 bucket's wider clusters finish
// the heavy tail sooner than the mixed bucket's split clusters, so routing
// it shortens the batch (L = 14 CPMG-32, 296 realisations: 39.0 curves/s at
// 40000, 24.7 at 97000).  L = 16 is not routed by default (its FP64 kernel
// needs 16-CTA clusters).  `mixed_order_limit` > 0 replaces the limits by one
// for every size; < 0 keeps every realisation mixed.
constexpr int64_t kDefaultMixedOrderLimit[17] = {
    2000, 2000, 2000, 2000, 2000, 2000,  // L < 6 has no batched kernel
    3500, 5000, 7400, 9500, 11600, 21000, 38600, 40000, 40000, 40000,
    std::numeric_limits<int64_t>::max()};

bool stays_mixed(const ss_run_config& c, int L, int64_t orders_per_state) {
  if (c.mixed_order_limit < 0) return true;
  const int64_t limit = c.mixed_order_limit > 0
                            ? c.mixed_order_limit
                            : kDefaultMixedOrderLimit[std::min(std::max(L, 0), 16)];
  if (orders_per_state <= limit) return true;
  return find_variant(L, false) == nullptr;
}

void build_realization(const ss_run_config& c, uint64_t index, const std::vector<TypeKey>& keys,
                       const std::vector<Op>& ops, bool mixed, PerReal& out,
                       double tau_override = 0.0) {
  try {
    Realization rz = assemble_realization(c, index);
    if (tau_override > 0.0) rz.tau_draw = tau_override;
    out.L = rz.nspins;
    out.tau_draw = rz.tau_draw;
    out.psi0 = rz.psi0;
    for (const PairTerm& p : rz.pairs) out.pairs.push_back(make_int2(p.lo, p.hi));
    const int L = rz.nspins;
    std::vector<int> orders(keys.size(), 0);
    std::vector<Expansion> exps;
    std::vector<const double*> tables;
    for (size_t t = 0; t < keys.size(); ++t) {
      const TypeKey& k = keys[t];
      const double* f = k.table >= 0 ? c.step_fields + static_cast<size_t>(3) * c.nspins * k.table
                                     : rz.fields.data();
      const double tau = k.from_draw ? k.tau * rz.tau_draw : k.tau;
      exps.push_back(chebyshev(k.mode, spectral_bound(L, f, rz.pairs), tau, c.epsilon));
      tables.push_back(f);
      orders[t] = static_cast<int>(exps.back().order());
    }
    int64_t per_state = 0;
    std::vector<double> residual(keys.size(), 0.0);
    for (size_t t = 0; t < keys.size(); ++t) {
      if (orders[t] > 0) {
        residual[t] = uncorrected_residual(L, tables[t], rz.pairs, -2.0 / exps[t].bound);
      }
    }
    double estimate = 0.0;
    for (const Op& op : ops) {
      if (op.kind == OP_EVOLVE) {
        per_state += static_cast<int64_t>(orders[op.a]) * op.b;
        estimate += 2.0 * static_cast<double>(orders[op.a]) * op.b * residual[op.a];
      }
    }
    out.error_estimate = estimate;
    out.mixed = mixed && stays_mixed(c, L, per_state);
    for (size_t t = 0; t < keys.size(); ++t) {
      const TypeKey& k = keys[t];
      const double* f = tables[t];
      const double tau = k.from_draw ? k.tau * rz.tau_draw : k.tau;
      Expansion& ex = exps[t];
      if (out.mixed) exact_transverse(L, f, k.mode, tau, ex);
      TypeDev ty{};
      ty.order = static_cast<int>(ex.order());
      orders[t] = ty.order;
      ty.c_off = static_cast<long long>(out.cpool.size());
      if (ty.order > 0) {
        ty.scale = -2.0 / ex.bound;
        ty.w_off = static_cast<long long>(out.wpool.size() / 2);
        const std::vector<double> w = series_weights(ex, k.mode);
        out.wpool.insert(out.wpool.end(), w.begin(), w.end());
        coefficient_block(L, f, rz.pairs, ty.scale, out.cpool, &ty.flags);
      }
      out.types.push_back(ty);
    }
    TypeDev energy{};
    energy.scale = 1.0;
    energy.c_off = static_cast<long long>(out.cpool.size());
    coefficient_block(L, rz.fields.data(), rz.pairs, 1.0, out.cpool, &energy.flags);
    out.types.push_back(energy);
    for (const Op& op : ops) {
      if (op.kind == OP_EVOLVE) {
        const double work = static_cast<double>(orders[op.a]) * op.b;
        out.orders += 2 * static_cast<int64_t>(orders[op.a]) * op.b;
        out.amp_orders += 2.0 * work * static_cast<double>(size_t{1} << L);
      }
    }
    out.cost = out.amp_orders + 64.0 * static_cast<double>(size_t{1} << L);
  } catch (const Error& e) {
    out.error = e.code;
    out.message = e.what();
  } catch (const std::exception& e) {
    out.error = SS_ERR_RUNTIME;
    out.message = e.what();
  }
}

void build_plan(ss_batch* b, const ss_run_config& c) {
  validate_config(c);
  std::map<TypeKey, int> type_ids;
  std::vector<TypeKey> keys;
  std::map<std::vector<double>, int> rot_ids;
  std::vector<std::array<double, 4>> rot_src;
  int64_t point = 0;
  linearise(c, 0, c.n_steps, b->ops, type_ids, keys, rot_ids, b->rots, rot_src, point);
  // A sweep: consecutive blocks of realisation slots share the geometry
  // indices first .. first + per_point - 1 and take their point's scales;
  // rotation table 1 + p holds the pulses of point p with scaled angles.
  const int64_t npoints = c.sweep_points;
  int64_t per_point = b->count;
  if (npoints > 0) {
    require(c.sweep_params != nullptr && b->count % npoints == 0, SS_ERR_INVALID_ARGUMENT,
            "a sweep needs sweep_params and a realisation count divisible by sweep_points");
    per_point = b->count / npoints;
    const size_t nrot = rot_src.size();
    for (int64_t q = 0; q < npoints; ++q) {
      const double* sp = c.sweep_params + 4 * q;
      require(sp[0] >= 0.0 && sp[1] >= 0.0 && sp[2] > 0.0 && std::isfinite(sp[3]),
              SS_ERR_INVALID_ARGUMENT, "sweep parameters out of range");
      for (size_t r = 0; r < nrot; ++r) {
        double u[8];
        const double axis[3] = {rot_src[r][0], rot_src[r][1], rot_src[r][2]};
        rotation_matrix(axis, rot_src[r][3] * sp[3], u);
        b->rots.insert(b->rots.end(), u, u + 8);
      }
    }
  }
  b->points = point;
  b->width = observable_width(c.observables, c.n_observables);
  b->ntypes = static_cast<int>(keys.size());
  b->ref_axis = c.reference_axis;
  for (int i = 0; i < c.n_observables; ++i) {
    const ss_observable& o = c.observables[i];
    require(o.kind >= 0 && o.kind <= 3, SS_ERR_CONFIG, "unknown observable");
    require(o.axis >= 0 && o.axis <= 2, SS_ERR_CONFIG, "unknown axis; expected x, y or z");
    b->obs.insert(b->obs.end(), {o.kind, o.axis, o.spin});
  }
  for (const Op& op : b->ops) {
    if (op.kind == OP_PULSE) {
      require(op.b < c.nspins, SS_ERR_OUT_OF_RANGE, "rotation names a spin outside the system");
    }
  }

  std::vector<PerReal> per(static_cast<size_t>(b->count));
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t workers = std::min<size_t>(hw, per.size());
  {
    std::vector<std::thread> pool;
    std::atomic<size_t> next{0};
    for (size_t w = 0; w < workers; ++w) {
      pool.emplace_back([&] {
        for (size_t i = next.fetch_add(1); i < per.size(); i = next.fetch_add(1)) {
          if (npoints > 0) {
            const double* sp = c.sweep_params + 4 * (static_cast<int64_t>(i) / per_point);
            ss_run_config ci = c;
            ci.dipolar_scale = sp[0];
            ci.field_disorder = sp[1];
            build_realization(ci, b->first + i % per_point, keys, b->ops,
                              b->precision == SS_PRECISION_MIXED, per[i], sp[2]);
          } else {
            build_realization(c, b->first + i, keys, b->ops, b->precision == SS_PRECISION_MIXED,
                              per[i]);
          }
        }
      });
    }
    for (auto& th : pool) th.join();
  }
  for (const PerReal& pr : per) {
    if (pr.error) fail(pr.error, pr.message);
  }

  long long state_off = 0, row_off = 0;
  std::map<std::pair<int, bool>, std::vector<int>> by_size;
  for (size_t i = 0; i < per.size(); ++i) {
    PerReal& pr = per[i];
    for (int o = 0; o < c.n_observables; ++o) {
      if (c.observables[o].kind == SS_OBS_MAG) {
        require(c.observables[o].spin >= 0 && c.observables[o].spin < pr.L, SS_ERR_OUT_OF_RANGE,
                "observable names a spin outside the system");
      }
    }
    RealDev rd{};
    rd.L = pr.L;
    rd.npairs = static_cast<int>(pr.pairs.size());
    rd.pair_off = static_cast<long long>(b->pairs.size());
    rd.state_off = state_off;
    rd.type_off = static_cast<long long>(b->types.size());
    rd.row_off = row_off;
    rd.rot_off = npoints > 0
                     ? static_cast<long long>(8 * rot_src.size()) *
                           (1 + static_cast<long long>(i) / per_point)
                     : 0;
    const long long c_base = static_cast<long long>(b->cpool.size());
    const long long w_base = static_cast<long long>(b->wpool.size() / 2);
    for (TypeDev ty : pr.types) {
      ty.c_off += c_base;
      ty.w_off += w_base;
      b->types.push_back(ty);
    }
    b->pairs.insert(b->pairs.end(), pr.pairs.begin(), pr.pairs.end());
    b->cpool.insert(b->cpool.end(), pr.cpool.begin(), pr.cpool.end());
    b->wpool.insert(b->wpool.end(), pr.wpool.begin(), pr.wpool.end());
    b->psi0_off.push_back(static_cast<long long>(b->psi0.size() / 2));
    b->psi0.insert(b->psi0.end(), pr.psi0.begin(), pr.psi0.end());
    b->reals.push_back(rd);
    state_off += 2LL << pr.L;
    row_off += b->points * b->width;
    b->orders_total += pr.orders;
    b->amp_orders += pr.amp_orders;
    by_size[{pr.L, pr.mixed}].push_back(static_cast<int>(i));
    b->real_precision.push_back(pr.mixed ? SS_PRECISION_MIXED : SS_PRECISION_FP64);
    b->real_amp_orders.push_back(pr.amp_orders);
    b->real_error_estimate.push_back(pr.error_estimate);
  }
  b->state_len = state_off;
  b->rows_len = row_off;

  // Times of the first realisation (the reference reports the first's,
  // src/ensemble/EnsembleRunner.cpp:72).
  {
    double time = 0.0;
    for (const Op& op : b->ops) {
      if (op.kind == OP_EVOLVE) {
        const TypeKey& k = keys[op.a];
        const double tau = k.from_draw ? k.tau * per.front().tau_draw : k.tau;
        time += tau * static_cast<double>(op.b);
      } else if (op.kind == OP_MEASURE) {
        b->times.push_back(time);
      }
    }
  }

  // Buckets (one per size and precision) run side by side.  Each gets a
  // share of the device in proportion to its cost, in clusters that can be
  // resident together, so that no bucket's persistent CTAs wait for another
  // bucket to drain; within a bucket the most expensive realisations go first.
  std::vector<double> weight, measured;
  double total_weight = 0.0;
  const std::string dev = device_name(b->engine->device);
  for (auto& [key, list] : by_size) {
    const auto [L, mixed] = key;
    Bucket bk;
    bk.L = L;
    double ns = 0.0;
    bk.var = scheduled_variant(dev, L, mixed, &ns);
    measured.push_back(ns);
    if (!bk.var) {
      fail(SS_ERR_INVALID_ARGUMENT,
           "the batched engine covers L = 6..16; got L = " + std::to_string(L));
    }
    // Split clusters keep both vectors of every realisation of a launch at
    // every measurement point; the bucket runs in launches of `chunk`
    // realisations within the snapshot budget, or with the paired schedule
    // when too few fit.
    if (bk.var->split) {
      const size_t per_slot = b->times.size() * 2 * (size_t{1} << L) * sizeof(double2);
      const size_t fit = per_slot > 0 ? static_cast<size_t>(g_snap_budget.load()) / per_slot : list.size();
      const Variant* paired = find_variant(L, mixed);
      if (fit < std::min(list.size(), kSnapMinSlots) && !paired->split) {
        bk.var = paired;
      } else {  // a size whose only schedule is split runs at least one per launch
        bk.chunk = static_cast<int>(std::max<size_t>(1, std::min(fit, list.size())));
      }
    }
    // The paired cluster kernel's measurement keeps one partial sum per
    // observable in a fixed shared slot array.
    require(bk.var->cb == 0 || bk.var->split || b->obs.size() / 3 <= static_cast<size_t>(kMaxDistObs),
            SS_ERR_CONFIG, "sizes above 13 spins (FP32) / 12 (FP64) measure at most 8 observables");
    std::stable_sort(list.begin(), list.end(),
                     [&](int x, int y) { return per[x].cost > per[y].cost; });
    bk.work = list;
    double w = 0.0;
    for (int x : list) w += per[x].cost;
    weight.push_back(w);
    b->buckets.push_back(std::move(bk));
  }
  // Cost of a bucket: amplitude-orders times the tuned nanoseconds per
  // amplitude-order when every bucket has been measured, else the
  // heuristic FP64 / mixed ratio.
  const bool all_measured =
      std::all_of(measured.begin(), measured.end(), [](double v) { return v > 0.0; });
  for (size_t i = 0; i < weight.size(); ++i) {
    if (all_measured) {
      weight[i] *= measured[i];
    } else if (!b->buckets[i].var->mixed) {
      weight[i] *= kFp64CostFactor;
    }
    total_weight += weight[i];
  }
  for (size_t i = 0; i < b->buckets.size(); ++i) {
    Bucket& bk = b->buckets[i];
    SS_CUDA(cudaFuncSetAttribute(bk.var->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(bk.var->smem)));
    cudaLaunchConfig_t lc{};
    cudaLaunchAttribute attr[1];
    lc.blockDim = dim3(bk.var->threads);
    lc.dynamicSmemBytes = bk.var->smem;
    if (bk.var->cb > 0) {
      if (bk.var->cluster() > 8) {
        SS_CUDA(cudaFuncSetAttribute(bk.var->kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      }
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = static_cast<unsigned>(bk.var->cluster());
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      lc.attrs = attr;
      lc.numAttrs = 1;
      lc.gridDim = dim3(bk.var->cluster());
    } else {
      lc.gridDim = dim3(2 * kClusterSize);
    }
    int resident = 0;
    SS_CUDA(cudaOccupancyMaxActiveClusters(&resident, bk.var->kernel, &lc));
    require(resident > 0, SS_ERR_RUNTIME, "batched kernel cluster does not fit the device");
    const double share = total_weight > 0.0 ? weight[i] / total_weight : 1.0;
    int clusters = static_cast<int>(share * resident);
    const int items = bk.var->split ? 2 * bk.chunk : static_cast<int>(bk.work.size());
    clusters = std::max(1, std::min(clusters, items));
    bk.grid = (bk.var->cb > 0 ? bk.var->cluster() : kClusterSize) * clusters;
  }
}

void capture(ss_batch* b) {
  ss_engine* e = b->engine;
  cudaStream_t s = e->stream;
  SS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    SS_CUDA(cudaMemsetAsync(b->d_flags, 0, sizeof(int), s));
    k_batch_prepare<<<static_cast<unsigned>(b->count), kPrepThreads, 0, s>>>(
        b->d_reals, b->d_psi0, b->d_psi0_off, b->d_states, b->ref_axis);
    SS_CUDA(cudaGetLastError());
    int64_t launches = 1;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork;
    SS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    SS_CUDA(cudaEventRecord(fork, s));
    for (size_t i = 0; i < b->buckets.size(); ++i) {
      Bucket& bk = b->buckets[i];
      cudaStream_t ks = s;
      if (i > 0) {
        ks = bk.side;
        SS_CUDA(cudaStreamWaitEvent(ks, fork, 0));
      }
      Args a{};
      a.ops = b->d_ops;
      a.op_begin = 0;
      a.op_end = static_cast<int>(b->ops.size());
      a.rots = b->d_rots;
      a.reals = b->d_reals;
      a.work = bk.dev_work;
      a.nwork = static_cast<int>(bk.work.size());
      a.counter = bk.counter;
      a.types = b->d_types;
      a.cpool = b->d_cpool;
      a.wpool = b->d_wpool;
      a.pairs = b->d_pairs;
      a.states = b->d_states;
      a.rows = b->d_rows;
      a.obs = b->d_obs;
      a.nobs = static_cast<int>(b->obs.size() / 3);
      a.width = static_cast<int>(b->width);
      a.measure_type = b->ntypes;
      a.flags = b->d_flags;
      a.snap = bk.snap;
      a.nmeas = static_cast<int>(b->times.size());
      // one launch for the bucket, or launches of `chunk` realisations
      // (split clusters), each followed by its snapshot measurement
      const int total = static_cast<int>(bk.work.size());
      const int step = bk.var->split ? bk.chunk : total;
      for (int c0 = 0; c0 < total; c0 += step) {
        a.work = bk.dev_work + c0;
        a.nwork = std::min(step, total - c0);
        SS_CUDA(cudaMemsetAsync(bk.counter, 0, sizeof(unsigned int), ks));
        if (bk.var->cb > 0) {
          // vectors over clusters: the cluster size is a launch attribute
          cudaLaunchConfig_t lc{};
          cudaLaunchAttribute attr[1];
          attr[0].id = cudaLaunchAttributeClusterDimension;
          attr[0].val.clusterDim.x = static_cast<unsigned>(bk.var->cluster());
          attr[0].val.clusterDim.y = 1;
          attr[0].val.clusterDim.z = 1;
          lc.gridDim = dim3(bk.grid);
          lc.blockDim = dim3(bk.var->threads);
          lc.dynamicSmemBytes = bk.var->smem;
          lc.stream = ks;
          lc.attrs = attr;
          lc.numAttrs = 1;
          SS_CUDA(cudaLaunchKernelEx(&lc, bk.var->kernel, a));
        } else {
          bk.var->kernel<<<bk.grid, bk.var->threads, bk.var->smem, ks>>>(a);
        }
        SS_CUDA(cudaGetLastError());
        ++launches;
        if (bk.var->split && a.nmeas > 0) {
          const long long items = static_cast<long long>(a.nwork) * a.nmeas;
          const unsigned grid = static_cast<unsigned>(std::min<long long>(items, 8LL * e->sm_count));
          k_batch_measure_snap<<<grid, kSnapThreads, 0, ks>>>(a);
          SS_CUDA(cudaGetLastError());
          ++launches;
        }
      }
      if (i > 0) {
        cudaEvent_t j;
        SS_CUDA(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        SS_CUDA(cudaEventRecord(j, ks));
        joins.push_back(j);
      }
    }
    for (cudaEvent_t j : joins) SS_CUDA(cudaStreamWaitEvent(s, j, 0));
    SS_CUDA(cudaStreamEndCapture(s, &b->graph));
    cudaEventDestroy(fork);
    for (cudaEvent_t j : joins) cudaEventDestroy(j);
    b->launches_per_run = launches;
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  SS_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
}

void upload(ss_batch* b) {
  cudaStream_t s = b->engine->stream;
  upload_vec(b->d_ops, b->ops, s);
  upload_vec(b->d_rots, b->rots, s);
  upload_vec(b->d_reals, b->reals, s);
  upload_vec(b->d_types, b->types, s);
  upload_vec(b->d_cpool, b->cpool, s);
  if (!b->wpool.empty()) {
    SS_CUDA(cudaMemcpyAsync(b->d_wpool, b->wpool.data(), sizeof(double) * b->wpool.size(),
                            cudaMemcpyHostToDevice, s));
  }
  upload_vec(b->d_pairs, b->pairs, s);
  SS_CUDA(cudaMemcpyAsync(b->d_psi0, b->psi0.data(), sizeof(double) * b->psi0.size(),
                          cudaMemcpyHostToDevice, s));
  upload_vec(b->d_psi0_off, b->psi0_off, s);
  upload_vec(b->d_obs, b->obs, s);
  for (Bucket& bk : b->buckets) upload_vec(bk.dev_work, bk.work, s);
  sync(b->engine);
  b->uploaded = true;
}

void execute(ss_batch* b) {
  require(b->uploaded, SS_ERR_RUNTIME, "batch inputs were not uploaded");
  if (!b->exec) capture(b);
  SS_CUDA(cudaGraphLaunch(b->exec, b->engine->stream));
  b->engine->launches.fetch_add(b->launches_per_run, std::memory_order_relaxed);
}

void download(ss_batch* b, double* rows, double* times) {
  ss_engine* e = b->engine;
  int flag = 0;
  SS_CUDA(cudaMemcpyAsync(&flag, b->d_flags, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  if (rows) {
    SS_CUDA(cudaMemcpyAsync(rows, b->d_rows, sizeof(double) * b->rows_len,
                            cudaMemcpyDeviceToHost, e->stream));
  }
  sync(e);
  if (flag == SS_ERR_DOMAIN) fail(flag, "cannot normalize a zero state");
  if (flag) fail(flag, "a norm reduction saw NaN or Inf");
  if (times) std::copy(b->times.begin(), b->times.end(), times);
}

void release(ss_batch* b) {
  if (b->engine && b->engine->stream) cudaStreamSynchronize(b->engine->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_ops);
  cudaFree(b->d_rots);
  cudaFree(b->d_reals);
  cudaFree(b->d_types);
  cudaFree(b->d_cpool);
  cudaFree(b->d_wpool);
  cudaFree(b->d_pairs);
  cudaFree(b->d_psi0);
  cudaFree(b->d_psi0_off);
  cudaFree(b->d_states);
  cudaFree(b->d_rows);
  cudaFree(b->d_obs);
  cudaFree(b->d_flags);
  for (Bucket& bk : b->buckets) {
    cudaFree(bk.counter);
    cudaFree(bk.dev_work);
    cudaFree(bk.snap);
    if (bk.side) cudaStreamDestroy(bk.side);
  }
}

}  // namespace
}  // namespace batch
}  // namespace ss

extern "C" {

int ss_batch_create(ss_engine* engine, const ss_run_config* config, uint64_t first, int64_t count,
                    int precision, ss_batch** out) {
  return guarded([&] {
    TraceRange trace("ss_batch_create");
    require(engine != nullptr && config != nullptr && out != nullptr, SS_ERR_INVALID_ARGUMENT,
            "null argument");
    require(count >= 1, SS_ERR_INVALID_ARGUMENT, "an ensemble needs at least one realisation");
    require(precision == SS_PRECISION_FP64 || precision == SS_PRECISION_MIXED,
            SS_ERR_INVALID_ARGUMENT, "unknown precision");
    auto* b = new ss_batch;
    b->engine = engine;
    b->precision = precision;
    b->first = first;
    b->count = count;
    try {
      SS_CUDA(cudaSetDevice(engine->device));
      build_plan(b, *config);
      dev_alloc(&b->d_ops, b->ops.size());
      dev_alloc(&b->d_rots, b->rots.size());
      dev_alloc(&b->d_reals, b->reals.size());
      dev_alloc(&b->d_types, b->types.size());
      dev_alloc(&b->d_cpool, b->cpool.size());
      dev_alloc(&b->d_wpool, b->wpool.size() / 2);
      dev_alloc(&b->d_pairs, b->pairs.size());
      dev_alloc(&b->d_psi0, b->psi0.size() / 2);
      dev_alloc(&b->d_psi0_off, b->psi0_off.size());
      dev_alloc(&b->d_states, static_cast<size_t>(b->state_len));
      dev_alloc(&b->d_rows, static_cast<size_t>(b->rows_len));
      dev_alloc(&b->d_obs, b->obs.size());
      dev_alloc(&b->d_flags, 1);
      for (Bucket& bk : b->buckets) {
        dev_alloc(&bk.counter, 1);
        dev_alloc(&bk.dev_work, bk.work.size());
        if (bk.var->split) {
          dev_alloc(&bk.snap, static_cast<size_t>(bk.chunk) * b->times.size() * 2 * (size_t{1} << bk.L));
        }
        SS_CUDA(cudaStreamCreateWithFlags(&bk.side, cudaStreamNonBlocking));
      }
    } catch (...) {
      release(b);
      delete b;
      throw;
    }
    *out = b;
  });
}

int ss_batch_destroy(ss_batch* b) {
  return guarded([&] {
    if (!b) return;
    release(b);
    delete b;
  });
}

int ss_batch_shape(const ss_batch* b, int64_t* points, int64_t* width) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    if (points) *points = b->points;
    if (width) *width = b->width;
  });
}

int ss_batch_upload(ss_batch* b) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    upload(b);
  });
}

int ss_batch_execute(ss_batch* b) {
  return guarded([&] {
    TraceRange trace("ss_batch_execute");
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    execute(b);
  });
}

int ss_batch_download(ss_batch* b, double* rows, double* times) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    download(b, rows, times);
  });
}

int ss_batch_run(ss_batch* b, double* rows, double* times) {
  return guarded([&] {
    TraceRange trace("ss_batch_run");
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    upload(b);
    execute(b);
    download(b, rows, times);
  });
}

int ss_batch_stats(const ss_batch* b, int64_t* orders, double* amplitude_orders,
                   int64_t* launches) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    if (orders) *orders = b->orders_total;
    if (amplitude_orders) *amplitude_orders = b->amp_orders;
    if (launches) *launches = b->launches_per_run > 0 ? b->launches_per_run
                                                      : 1 + static_cast<int64_t>(b->buckets.size());
  });
}

int ss_batch_io_bytes(const ss_batch* b, int64_t* h2d, int64_t* d2h) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    int64_t in = 0;
    in += static_cast<int64_t>(sizeof(Op) * b->ops.size() + sizeof(double) * b->rots.size());
    in += static_cast<int64_t>(sizeof(RealDev) * b->reals.size() + sizeof(TypeDev) * b->types.size());
    in += static_cast<int64_t>(sizeof(double) * (b->cpool.size() + b->wpool.size() + b->psi0.size()));
    in += static_cast<int64_t>(sizeof(int2) * b->pairs.size() + sizeof(long long) * b->psi0_off.size());
    in += static_cast<int64_t>(sizeof(int) * b->obs.size());
    for (const Bucket& bk : b->buckets) in += static_cast<int64_t>(sizeof(int) * bk.work.size());
    if (h2d) *h2d = in;
    if (d2h) *d2h = static_cast<int64_t>(sizeof(double) * b->rows_len + sizeof(int));
  });
}

int ss_batch_error_estimates(const ss_batch* b, double* estimate) {
  return guarded([&] {
    require(b != nullptr && estimate != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    std::copy(b->real_error_estimate.begin(), b->real_error_estimate.end(), estimate);
  });
}

int ss_batch_precisions(const ss_batch* b, int32_t* precision, double* amplitude_orders) {
  return guarded([&] {
    require(b != nullptr, SS_ERR_INVALID_ARGUMENT, "null batch");
    if (precision) std::copy(b->real_precision.begin(), b->real_precision.end(), precision);
    if (amplitude_orders) {
      std::copy(b->real_amp_orders.begin(), b->real_amp_orders.end(), amplitude_orders);
    }
  });
}

}  // extern "C"

// ---------------------------------------------------------------- autotuner
namespace ss {
namespace batch {
namespace {

void write_cache(const char* path) {
  std::ofstream f(path, std::ios::trunc);
  require(static_cast<bool>(f), SS_ERR_RUNTIME, "cannot write the schedule cache");
  f << "# device\tL\tprecision\tvariant\tns_per_amplitude_order\n";
  std::lock_guard<std::mutex> lk(g_sched_mu);
  for (const auto& [key, ch] : g_sched) {
    f << std::get<0>(key) << '\t' << std::get<1>(key) << '\t'
      << (std::get<2>(key) ? "mixed" : "fp64") << '\t' << ch.variant << '\t' << ch.ns << '\n';
  }
}

void load_cache(const char* path) {
  std::ifstream f(path);
  if (!f) return;  // nothing tuned yet
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream in(line);
    std::string dev, L, prec, var, ns;
    if (!std::getline(in, dev, '\t') || !std::getline(in, L, '\t') ||
        !std::getline(in, prec, '\t') || !std::getline(in, var, '\t') ||
        !std::getline(in, ns)) {
      fail(SS_ERR_CONFIG, "malformed schedule cache line: " + line);
    }
    require(prec == "mixed" || prec == "fp64", SS_ERR_CONFIG, "schedule cache: unknown precision");
    Choice c;
    c.variant = var;
    try {
      c.ns = std::stod(ns);
      const int l = std::stoi(L);
      std::lock_guard<std::mutex> lk(g_sched_mu);
      g_sched[{dev, l, prec == "mixed" ? 1 : 0}] = c;
    } catch (const std::logic_error&) {
      fail(SS_ERR_CONFIG, "malformed schedule cache line: " + line);
    }
  }
}

// Clusters of a schedule that fit the device at once.
int resident_clusters(const Variant& v) {
  SS_CUDA(cudaFuncSetAttribute(v.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(v.smem)));
  cudaLaunchConfig_t lc{};
  cudaLaunchAttribute attr[1];
  lc.blockDim = dim3(v.threads);
  lc.dynamicSmemBytes = v.smem;
  if (v.cb > 0) {
    if (v.cluster() > 8) {
      SS_CUDA(cudaFuncSetAttribute(v.kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(v.cluster());
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    lc.gridDim = dim3(v.cluster());
  } else {
    lc.gridDim = dim3(2 * kClusterSize);
  }
  int resident = 0;
  SS_CUDA(cudaOccupancyMaxActiveClusters(&resident, v.kernel, &lc));
  return resident;
}

// Times one candidate on realisations of `c` (every one of size L): at least
// `sample` and at least four waves of the candidate's resident clusters, so
// the figure is a throughput rather than the longest realisation's latency;
// a warm-up run, then one timed run of the captured program.
double time_candidate(ss_engine* e, const ss_run_config& c, uint64_t first, int64_t sample,
                      int precision, const Variant& v) {
  // a split cluster carries one of a realisation's two vectors
  const int64_t per_wave = resident_clusters(v) / (v.split ? 2 : 1);
  sample = std::max<int64_t>(sample, 4 * std::max<int64_t>(per_wave, 1));
  ss_batch* b = nullptr;
  g_force = &v;
  const int rc = ss_batch_create(e, &c, first, sample, precision, &b);
  g_force = nullptr;
  if (rc) fail(rc, ss_last_error());
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  double ns = 0.0;
  try {
    if (int r = ss_batch_upload(b)) fail(r, ss_last_error());
    if (int r = ss_batch_execute(b)) fail(r, ss_last_error());
    SS_CUDA(cudaEventCreate(&t0));
    SS_CUDA(cudaEventCreate(&t1));
    SS_CUDA(cudaEventRecord(t0, e->stream));
    if (int r = ss_batch_execute(b)) fail(r, ss_last_error());
    SS_CUDA(cudaEventRecord(t1, e->stream));
    SS_CUDA(cudaEventSynchronize(t1));
    float ms = 0.0f;
    SS_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    ns = double(ms) * 1e6 / std::max(1.0, b->amp_orders);
  } catch (...) {
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    ss_batch_destroy(b);
    throw;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  ss_batch_destroy(b);
  return ns;
}

}  // namespace
}  // namespace batch
}  // namespace ss

extern "C" {

int ss_batch_tune(ss_engine* e, const ss_run_config* config, uint64_t first, int64_t sample,
                  int precision, const char* cache_path) {
  return guarded([&] {
    TraceRange trace("ss_batch_tune");
    require(e != nullptr && config != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    require(sample >= 1, SS_ERR_INVALID_ARGUMENT, "the tuning sample needs a realisation");
    require(precision == SS_PRECISION_FP64 || precision == SS_PRECISION_MIXED,
            SS_ERR_INVALID_ARGUMENT, "unknown precision");
    if (cache_path) load_cache(cache_path);
    const std::string dev = device_name(e->device);
    std::vector<int> sizes;
    if (config->n_spin_choices > 0) {
      sizes.assign(config->spin_choices, config->spin_choices + config->n_spin_choices);
    } else {
      sizes.push_back(config->nspins);
    }
    std::sort(sizes.begin(), sizes.end());
    sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
    std::vector<int> precs = {precision};
    if (precision == SS_PRECISION_MIXED) precs.push_back(SS_PRECISION_FP64);  // routing target
    for (int L : sizes) {
      for (int prec : precs) {
        // FP64 as the routing target only where this config's mixed
        // realisations of size L can be routed at all
        if (prec != precision && stays_mixed(*config, L, std::numeric_limits<int64_t>::max())) {
          continue;
        }
        const bool mixed = prec == SS_PRECISION_MIXED;
        ss_run_config c = *config;
        c.n_spin_choices = 1;  // every sampled realisation has L spins (the
        c.spin_choices[0] = L; // per-spin tables keep the config's stride)
        c.mixed_order_limit = -1;
        c.sweep_points = 0;
        c.sweep_params = nullptr;
        Choice best;
        for (const Variant& v : variants()) {
          if (v.L != L || v.mixed != mixed) continue;
          const double ns = time_candidate(e, c, first, sample, prec, v);
          if (best.variant.empty() || ns < best.ns) {
            best.variant = variant_name(v);
            best.ns = ns;
          }
        }
        if (best.variant.empty()) continue;  // no kernel for this size and precision
        std::lock_guard<std::mutex> lk(g_sched_mu);
        g_sched[{dev, L, mixed ? 1 : 0}] = best;
      }
    }
    if (cache_path) write_cache(cache_path);
  });
}

int ss_schedule_load(const char* cache_path) {
  return guarded([&] {
    require(cache_path != nullptr, SS_ERR_INVALID_ARGUMENT, "null path");
    std::ifstream f(cache_path);
    require(static_cast<bool>(f), SS_ERR_INVALID_ARGUMENT, "schedule cache not found");
    load_cache(cache_path);
  });
}

int ss_schedule_clear(void) {
  return guarded([&] {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched.clear();
  });
}

int ss_set_snapshot_budget(int64_t bytes) {
  return guarded([&] {
    require(bytes >= 0, SS_ERR_INVALID_ARGUMENT, "the snapshot budget is a byte count");
    g_snap_budget.store(bytes);
  });
}

int ss_schedule_describe(char* buf, size_t cap, size_t* needed) {
  return guarded([&] {
    std::ostringstream out;
    {
      std::lock_guard<std::mutex> lk(g_sched_mu);
      for (const auto& [key, ch] : g_sched) {
        out << std::get<0>(key) << '\t' << std::get<1>(key) << '\t'
            << (std::get<2>(key) ? "mixed" : "fp64") << '\t' << ch.variant << '\t' << ch.ns << '\n';
      }
    }
    const std::string text = out.str();
    if (needed) *needed = text.size() + 1;
    if (buf && cap > 0) {
      const size_t n = std::min(cap - 1, text.size());
      std::memcpy(buf, text.data(), n);
      buf[n] = '\0';
    }
  });
}

int ss_batch_variants(char* buf, size_t cap, size_t* needed) {
  return guarded([&] {
    std::ostringstream out;
    for (const Variant& v : variants()) {
      out << variant_name(v) << '\t' << v.threads << '\t' << v.smem << '\n';
    }
    const std::string text = out.str();
    if (needed) *needed = text.size() + 1;
    if (buf && cap > 0) {
      const size_t n = std::min(cap - 1, text.size());
      std::memcpy(buf, text.data(), n);
      buf[n] = '\0';
    }
  });
}

}  // extern "C"
