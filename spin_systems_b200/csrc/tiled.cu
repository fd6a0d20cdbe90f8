// The plain propagator's order kernel for large vectors.
//
// The fused gather kernel (propagator.cu) reads all ~L^2/4 anti-aligned
// partners of every amplitude one double2 at a time through L1: at L = 24
// that is 138 partner loads per amplitude-order, and the kernel is bound by
// their delivery.  Here one Chebyshev order is a few passes instead.  Pass p
// owns a set S_p of B spins (a "tile" pattern, B = 12 in FP64, 13 in mixed
// precision); the vector splits into 2^(L-B) tiles, each holding the 2^B
// amplitudes that agree on every spin outside S_p.  A CTA copies its tile of
// T_{n-1} into shared memory (cp.async, contiguous runs along the tile's low
// bits), applies every coupling assigned to the pass with the batched
// engine's register-blocked layouts (each partner block read from shared
// memory serves up to R couplings, couplings inside a register group come
// from registers), and accumulates the partial H T_{n-1} in a vector `part`
// of the same layout as the state.  The patterns are a pair covering: every
// coupling (i, j) has a pass whose tile holds both spins, so every coupling
// is applied on chip, exactly once.  The last pass also adds the diagonal
// (streamed, FP64) and forms T_n = 2H^ T_{n-1} - T_{n-2} and psi += c_n T_n,
// the reference's recurrence (src/core/Propagator.cpp:58-72) and its
// Hamiltonian (src/core/Hamiltonian.cpp:95-127) in one sweep per pass.
//
// The last pass holds T_{n-1} (its tile) and forms T_n, so psi is read and
// written every second order only, taking c_{n-1} T_{n-1} + c_n T_n at once.
//
// DRAM traffic per amplitude-order with P passes: T_{n-1} once per pass,
// the partial written by the first pass, read and written by the middle
// ones, read by the last, and the last pass's diagonal, T_{n-2}, T_n and
// (every second order) psi:
//   FP64  (16 B amplitudes):  16 P + 32 (P - 1) + 8 + 32 + 16  = 48 P + 24 B
//   mixed ( 8 B amplitudes):   8 P + 16 (P - 1) + 8 + 16 + 16  = 24 P + 24 B
// against the single-sweep 80 / 56 B (+8 B of diagonal) that needs every
// partner on chip at once.  Every tile keeps the lowest spins, so each copy
// moves whole 128-byte lines (8 FP64 or 16 FP32 amplitudes): at L = 24 that
// takes P = 7.
//
// Mixed precision: T vectors and the partial sums are FP32 and the couplings
// are applied as FP32 numbers; the diagonal, T_n's formation, the series
// weights and psi are FP64 (the batched engine's scheme).
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "batch_kernel.cuh"
#include "hamiltonian.cuh"
#include "tiled.hpp"

namespace ss {
namespace tiled {

using batch::cross_block;
using batch::Cplx;
using batch::cz;
using batch::Geo;
using batch::pad;
using batch::Padded;

constexpr int kMaxTile = 13;
constexpr int kMaxLayouts = 8;

enum PassKind { PASS_FIRST = 0, PASS_MID = 1, PASS_LAST = 2, PASS_ONLY = 3 };

// One pass: where the tile's spins sit in the basis index, which couplings it
// applies (tile-local upper-triangular tables, zero where another pass owns
// the pair), and per layout the partner blocks worth reading.
struct PassDev {
  uint32_t tile_pos[kMaxTile];   // basis bit of tile-local bit b
  uint32_t outer_pos[kMaxSpins]; // basis bits of the tile index, low to high
  int nouter;
  int has_trans;                 // a transverse field is applied in this pass
  int has_fb;                    // a |dd><uu| coefficient is non-zero
  int pad_;
  uint32_t jmask[kMaxLayouts];   // layout g: tile-local spins j with a partner block
  uint32_t rmask[kMaxLayouts];   // layout g: register pairs (p * R + q) with a coefficient
  uint32_t active;               // bit g: layout g applies something (the last always runs)
  double cff[kMaxTile * kMaxTile];  // [i * B + j], i < j: scale (jx + jy) / 4
  double cfb[kMaxTile * kMaxTile];  // scale (jx - jy) / 4
  double ccx[kMaxTile];             // scale hx / 2
  double ccy[kMaxTile];             // scale hy / 2
};

struct OrderArgs {
  const void* cur;      // T_{n-1}
  void* prev;           // T_{n-2}; T_n in the last pass
  void* part;           // partial H T_{n-1}
  double2* psi;
  const double* diag;   // sigma_z diagonal, unscaled
  double dscale;        // scale of the diagonal
  double cr, ci;        // series weight c_n
  double pr, pi;        // series weight c_{n-1}
  uint32_t ntiles;
  int first;            // order 1: T_1 = H^ T_0
  int psi_terms;        // 0: psi untouched; 1: psi += c_n T_n; 2: also + c_{n-1} T_{n-1}
};

// ------------------------------------------------------------------ host: plan

namespace {

// Local search for a pair covering of spins u .. L-1 by P tiles of B - u
// spins (spins 0 .. u-1 are in every tile).  Deterministic for a seed.
bool search_cover(int L, int B, int u, int P, uint64_t seed, int iters,
                  std::vector<uint32_t>* out) {
  const int n = L - u, c = B - u;
  if (c <= 0 || c > n) return false;
  std::mt19937_64 rng(seed);
  auto rnd = [&](int m) { return static_cast<int>(rng() % static_cast<uint64_t>(m)); };
  std::vector<std::vector<int>> tiles(P);
  std::vector<std::vector<char>> in(P, std::vector<char>(n, 0));
  for (int t = 0; t < P; ++t) {
    std::vector<int> all(n);
    for (int x = 0; x < n; ++x) all[x] = x;
    for (int x = 0; x < c; ++x) std::swap(all[x], all[x + rnd(n - x)]);
    tiles[t].assign(all.begin(), all.begin() + c);
    for (int x : tiles[t]) in[t][x] = 1;
  }
  std::vector<int> cnt(static_cast<size_t>(n) * n, 0);
  for (int t = 0; t < P; ++t) {
    for (int a = 0; a < c; ++a) {
      for (int b = a + 1; b < c; ++b) {
        ++cnt[tiles[t][a] * n + tiles[t][b]];
        ++cnt[tiles[t][b] * n + tiles[t][a]];
      }
    }
  }
  int uncovered = 0;
  for (int a = 0; a < n; ++a) {
    for (int b = a + 1; b < n; ++b) uncovered += cnt[a * n + b] == 0;
  }
  for (int it = 0; it < iters && uncovered > 0; ++it) {
    const int t = rnd(P), slot = rnd(c);
    const int gone = tiles[t][slot];
    int come = rnd(n - c);
    for (int x = 0; x < n; ++x) {  // the come-th spin outside the tile
      if (!in[t][x] && come-- == 0) {
        come = x;
        break;
      }
    }
    int delta = 0;
    for (int y : tiles[t]) {
      if (y == gone) continue;
      delta += cnt[gone * n + y] == 1;
      delta -= cnt[come * n + y] == 0;
    }
    if (delta > 0 && rng() % 64 != 0) continue;
    for (int y : tiles[t]) {
      if (y == gone) continue;
      --cnt[gone * n + y];
      --cnt[y * n + gone];
      ++cnt[come * n + y];
      ++cnt[y * n + come];
    }
    tiles[t][slot] = come;
    in[t][gone] = 0;
    in[t][come] = 1;
    uncovered += delta;
  }
  if (uncovered != 0) return false;
  out->clear();
  for (int t = 0; t < P; ++t) {
    uint32_t m = (1u << u) - 1u;
    for (int x : tiles[t]) m |= 1u << (u + x);
    out->push_back(m);
  }
  return true;
}

// Always available: the free spins in m groups of at most (B - u) / 2, one
// tile per pair of groups.
std::vector<uint32_t> group_cover(int L, int B, int u) {
  const int n = L - u, c = B - u;
  const uint32_t low = (1u << u) - 1u;
  if (n <= c) return {low | (((1u << n) - 1u) << u)};
  int m = 2;
  while ((n + m - 1) / m * 2 > c) ++m;
  std::vector<uint32_t> groups(m, 0);
  for (int x = 0; x < n; ++x) groups[x * m / n] |= 1u << (u + x);
  std::vector<uint32_t> out;
  for (int a = 0; a < m; ++a) {
    for (int b = a + 1; b < m; ++b) out.push_back(low | groups[a] | groups[b]);
  }
  return out;
}

bool covers(int L, const std::vector<uint32_t>& tiles) {
  for (int i = 0; i < L; ++i) {
    for (int j = i + 1; j < L; ++j) {
      const uint32_t m = (1u << i) | (1u << j);
      if (std::none_of(tiles.begin(), tiles.end(), [m](uint32_t t) { return (t & m) == m; })) {
        return false;
      }
    }
  }
  return true;
}

int low_run(uint32_t m) {
  int r = 0;
  while (r < 32 && ((m >> r) & 1u)) ++r;
  return r;
}

// Tiles of B spins that all hold spins 0 .. u-1 (so every copy of a tile
// moves runs of 2^u consecutive amplitudes), as few as the search finds.
std::vector<uint32_t> make_plan(int L, int B, int u) {
  if (L <= B) return {L >= 32 ? ~0u : (1u << L) - 1u};
  u = std::max(0, std::min(u, B - 2));
  std::vector<uint32_t> best = group_cover(L, B, u);
  const int n = L - u, c = B - u;
  const int r = (n - 1 + c - 2) / (c - 1);  // tiles per spin, at least
  const int lb = std::max(2, (n * r + c - 1) / c);
  for (int P = lb; P < static_cast<int>(best.size()); ++P) {
    std::vector<uint32_t> found;
    bool ok = false;
    for (uint64_t seed = 1; seed <= 8 && !ok; ++seed) {
      ok = search_cover(L, B, u, P, seed * 0x9E3779B97F4A7C15ULL + uint64_t(L * 64 + B), 60000,
                        &found);
    }
    if (ok) {
      best = found;
      break;
    }
  }
  // The kernel's tiles hold exactly B spins: top up smaller ones with the
  // lowest spins they lack (longer contiguous runs).
  for (uint32_t& m : best) {
    for (int s = 0; s < L && __builtin_popcount(m) < B; ++s) m |= 1u << s;
  }
  // The pass that forms T_n streams psi, T_{n-2} and the diagonal: give it
  // the longest contiguous run.
  auto last = std::max_element(best.begin(), best.end(),
                               [](uint32_t a, uint32_t b) { return low_run(a) < low_run(b); });
  std::iter_swap(last, best.end() - 1);
  return best;
}

}  // namespace

// ------------------------------------------------------------- device side

__device__ __forceinline__ uint32_t deposit(uint32_t x, const uint32_t* pos, int n) {
  uint32_t r = 0;
  for (int b = 0; b < n; ++b) r |= ((x >> b) & 1u) << pos[b];
  return r;
}

// Length of the run of tile-local bits that sit on basis bits 0, 1, 2, ...
__device__ __forceinline__ int low_run_of(const PassDev* pd) {
  int r = 0;
  while (r < kMaxTile && pd->tile_pos[r] == static_cast<uint32_t>(r)) ++r;
  return r;
}

template <typename C2>
__device__ __forceinline__ void cp_async(C2* dst, const C2* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(C2) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
  }
}

// Brings the 128-byte line holding `p` into L2 (no register or shared-memory
// destination: a later load of the line hits L2 instead of DRAM).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Waits until at most the most recently committed group is in flight.
__device__ __forceinline__ void cp_async_wait_prior() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <typename Real, int B, int R>
struct Tile {
  using Gm = Geo<B, R>;
  using C2 = typename Cplx<Real>::T;
  static constexpr int NT = Gm::NT, NA = Gm::NA, G = Gm::G;
  static constexpr uint32_t NP = Padded<B, R>::N;
  // Two T_{n-1} tile buffers (the next tile's copy lands while this one is
  // worked on), the partial sums between layouts, the pass's coefficients.
  static constexpr size_t kSmem =
      3 * NP * sizeof(C2) + (2 * B * B + 2 * B) * sizeof(Real) + 2 * NA * sizeof(uint32_t);
  static_assert(G <= kMaxLayouts && B <= kMaxTile, "tile too wide");
};

// The pass's per-layout masks and tile-index bits, copied to shared memory
// once per launch (they are read in every tile's layouts).
struct PassMeta {
  uint32_t jmask[kMaxLayouts];
  uint32_t rmask[kMaxLayouts];
  uint32_t active;
  int nouter;
  uint32_t outer_pos[kMaxSpins];
};

// Shared-memory view of one CTA.
template <typename Real>
struct TileSmem {
  using C2 = typename Cplx<Real>::T;
  C2* buf;        // T_{n-1} tile
  C2* acc;        // partial sums between layouts
  const Real* cff;
  const Real* cfb;
  const Real* ccx;
  const Real* ccy;
};

// The couplings (b + p, j), p < R, from one partner block held in registers:
// slot x of the block (amplitude k ^ 2^j with register bits x) feeds the
// thread's slot x ^ 2^p with c1[p] when that slot's bit p is set, c0[p] when
// it is clear.  MODE 1 keeps only the clear targets, MODE 2 only the set ones
// (the other half multiplies a zero coefficient when there is no |dd><uu|
// channel and bit j is the same across the warp).
template <int R, int MODE, typename C2, typename Real, int NA>
__device__ __forceinline__ void block_apply(C2 (&acc)[NA], const C2 (&v)[NA], const Real (&c0)[R],
                                            const Real (&c1)[R]) {
#pragma unroll
  for (int x = 0; x < NA; ++x) {
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const int dst = x ^ (1 << p);
      const bool set = ((dst >> p) & 1) != 0;
      if ((MODE == 1 && set) || (MODE == 2 && !set)) continue;
      const Real c = set ? c1[p] : c0[p];
      acc[dst].x += c * v[x].x;
      acc[dst].y += c * v[x].y;
    }
  }
}

// One register-blocked layout over the tile (the batched engine's
// layout_pass, restricted to the pass's couplings): own[] receives the
// thread's T_{n-1} amplitudes, acc[] the partial sums (from shared memory when
// `acc_in`, else zero).
template <typename Real, int B, int R, int g>
__device__ __forceinline__ void tile_layout(const TileSmem<Real>& sm,
                                            typename Cplx<Real>::T (&acc)[Geo<B, R>::NA],
                                            typename Cplx<Real>::T (&own)[Geo<B, R>::NA],
                                            uint32_t t, uint32_t jmask, uint32_t rmask,
                                            bool acc_in, bool has_trans, bool has_fb) {
  using Gm = Geo<B, R>;
  using C2 = typename Cplx<Real>::T;
  constexpr int b = Gm::base(g);
  constexpr int NA = Gm::NA;
  const uint32_t kb = ((t >> b) << (b + R)) | (t & ((1u << b) - 1u));
  const C2* mine = sm.buf + pad<R>(kb);
#pragma unroll
  for (int a = 0; a < NA; ++a) own[a] = mine[pad<R>(uint32_t(a) << b)];
  if (acc_in) {
    const C2* pp = sm.acc + pad<R>(kb);
#pragma unroll
    for (int a = 0; a < NA; ++a) acc[a] = pp[pad<R>(uint32_t(a) << b)];
  } else {
#pragma unroll
    for (int a = 0; a < NA; ++a) acc[a] = cz<C2>();
  }

  // Couplings with both spins in this register group.
#pragma unroll
  for (int p = 0; p < R; ++p) {
#pragma unroll
    for (int q = p + 1; q < R; ++q) {
      if (Gm::pair_layout(b + p, b + q) == g && ((rmask >> (p * R + q)) & 1u)) {
        const Real ff = sm.cff[(b + p) * B + (b + q)];
        const Real fb = sm.cfb[(b + p) * B + (b + q)];
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

  // Transverse fields assigned to this pass, on this group's spins.
  if (has_trans) {
#pragma unroll
    for (int p = 0; p < R; ++p) {
      if (Gm::first_layout(b + p) == g) {
        const Real cx = sm.ccx[b + p], cy = sm.ccy[b + p];
        if (cx != Real(0) || cy != Real(0)) {
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
  }

  // Couplings (b + p, j) with j above the group, one partner block per j
  // that has a coupling in this pass.  The first half of the next block is
  // loaded before this block's products, so its latency overlaps them.
  constexpr int H = NA / 2;
  if (jmask == 0u) return;
  int j = __ffs(jmask) - 1;
  jmask &= jmask - 1u;
  C2 v[NA];
#pragma unroll
  for (int x = 0; x < NA; ++x) v[x] = sm.buf[pad<R>(kb ^ (1u << j)) + pad<R>(uint32_t(x) << b)];
#pragma unroll 1
  for (;;) {
    const bool bj = ((kb >> j) & 1u) != 0u;
    Real c0[R], c1[R];
#pragma unroll
    for (int p = 0; p < R; ++p) {
      const bool mine_p = Gm::cross_mine(g, p);
      const Real ff = mine_p ? sm.cff[(b + p) * B + j] : Real(0);
      const Real fb = mine_p ? sm.cfb[(b + p) * B + j] : Real(0);
      c0[p] = bj ? ff : fb;  // register bit clear: aligned iff bit j clear
      c1[p] = bj ? fb : ff;  // register bit set
    }
    const int jn = jmask != 0u ? __ffs(jmask) - 1 : -1;
    const C2* nb = sm.buf + pad<R>(kb ^ (1u << (jn >= 0 ? jn : j)));
    C2 w[H];
#pragma unroll
    for (int x = 0; x < H; ++x) w[x] = nb[pad<R>(uint32_t(x) << b)];
    if (!has_fb && __all_sync(0xffffffffu, bj)) {
      block_apply<R, 1>(acc, v, c0, c1);
    } else if (!has_fb && __all_sync(0xffffffffu, !bj)) {
      block_apply<R, 2>(acc, v, c0, c1);
    } else {
      block_apply<R, 0>(acc, v, c0, c1);
    }
    if (jn < 0) break;
    jmask &= jmask - 1u;
    j = jn;
#pragma unroll
    for (int x = 0; x < H; ++x) v[x] = w[x];
#pragma unroll
    for (int x = H; x < NA; ++x) v[x] = nb[pad<R>(uint32_t(x) << b)];
  }
}

// Layouts 0 .. G-2 that apply something in this pass, each handing its
// partial sums to the next through shared memory.  `acc_in`: the partial sums
// in shared memory already hold something (the previous passes' sums, or an
// earlier layout's).
template <typename Real, int B, int R, int g>
__device__ __forceinline__ void tile_front(const TileSmem<Real>& sm, const PassMeta* pd, uint32_t t,
                                           bool acc_in, bool has_trans, bool has_fb) {
  using Gm = Geo<B, R>;
  if constexpr (g < Gm::G - 1) {
    if ((pd->active >> g) & 1u) {
      using C2 = typename Cplx<Real>::T;
      C2 acc[Gm::NA], own[Gm::NA];
      tile_layout<Real, B, R, g>(sm, acc, own, t, pd->jmask[g], pd->rmask[g], acc_in, has_trans,
                                 has_fb);
      constexpr int b = Gm::base(g);
      const uint32_t kb = ((t >> b) << (b + R)) | (t & ((1u << b) - 1u));
      C2* pp = sm.acc + pad<R>(kb);
#pragma unroll
      for (int a = 0; a < Gm::NA; ++a) pp[pad<R>(uint32_t(a) << b)] = acc[a];
      __syncthreads();
      acc_in = true;
    }
    tile_front<Real, B, R, g + 1>(sm, pd, t, acc_in, has_trans, has_fb);
  }
}

// One pass of one Chebyshev order over every tile (persistent CTAs).  The
// CTA's tiles are taken in turn; the copy of the next tile's T_{n-1} is
// issued before this tile is worked on, and (middle and last passes) the
// next tile's partial sums are copied into the accumulator buffer as soon as
// the last layout has read this tile's.
template <typename Real, int B, int R, int KIND>
__global__ void __launch_bounds__(Geo<B, R>::NT, 1)
    k_tile(const PassDev* __restrict__ pd, OrderArgs a) {
  using T = Tile<Real, B, R>;
  using C2 = typename T::C2;
  constexpr int NT = T::NT, NA = T::NA, G = T::G;
  constexpr uint32_t NP = T::NP;
  constexpr int bl = Geo<B, R>::base(G - 1);
  constexpr bool kAccIn = KIND == PASS_MID || KIND == PASS_LAST;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2* bufs = reinterpret_cast<C2*>(smem_raw);  // [2][NP]
  C2* accb = bufs + 2 * NP;
  Real* cff = reinterpret_cast<Real*>(accb + NP);
  Real* cfb = cff + B * B;
  Real* ccx = cfb + B * B;
  Real* ccy = ccx + B;
  uint32_t* dep_ld = reinterpret_cast<uint32_t*>(ccy + B);
  uint32_t* dep_rg = dep_ld + NA;

  __shared__ PassMeta meta;
  const uint32_t t = threadIdx.x;
  for (int i = t; i < B * B; i += NT) {
    cff[i] = Real(pd->cff[i]);
    cfb[i] = Real(pd->cfb[i]);
  }
  if (t < kMaxLayouts) {
    meta.jmask[t] = pd->jmask[t];
    meta.rmask[t] = pd->rmask[t];
  }
  if (t < kMaxSpins) meta.outer_pos[t] = pd->outer_pos[t];
  if (t == 0) {
    meta.active = pd->active;
    meta.nouter = pd->nouter;
  }
  if (t < B) {
    ccx[t] = Real(pd->ccx[t]);
    ccy[t] = Real(pd->ccy[t]);
  }
  if (t < NA) {
    dep_ld[t] = deposit(t << (B - R), pd->tile_pos, B);
    dep_rg[t] = deposit(t << bl, pd->tile_pos, B);
  }
  // Copies: thread t moves tile elements t + m NT, m < NA (consecutive lanes
  // on consecutive tile-local indices, i.e. along the tile's low bits).
  const uint32_t dep_t = deposit(t, pd->tile_pos, B - R);
  const uint32_t kb_last = ((t >> bl) << (bl + R)) | (t & ((1u << bl) - 1u));
  const uint32_t dep_kb = deposit(kb_last, pd->tile_pos, B);
  // Runs of 2^U consecutive amplitudes (the tile's low spins), 128 bytes of
  // T_{n-1}: thread t looks after runs t + i NT; dep_run[i] is where run
  // starts relative to the tile's base.
  constexpr int U = sizeof(C2) == 16 ? 3 : 4;
  constexpr int kRuns = 1 << (B - U);
  constexpr int kRunsPerThread = (kRuns + NT - 1) / NT;
  const bool runs_ok = low_run_of(pd) >= U;
  uint32_t dep_run[kRunsPerThread];
#pragma unroll
  for (int i = 0; i < kRunsPerThread; ++i) {
    const uint32_t r = t + uint32_t(i) * NT;
    dep_run[i] = r < uint32_t(kRuns) ? deposit(r << U, pd->tile_pos, B) : 0u;
  }
  // L2 prefetch of a tile's runs of vector v (elements of type E).
  auto prefetch_tile = [&](const auto* v, uint32_t base) {
    if (!runs_ok) return;
#pragma unroll
    for (int i = 0; i < kRunsPerThread; ++i) {
      if (t + uint32_t(i) * NT < uint32_t(kRuns)) {
        const auto* q = v + (base | dep_run[i]);
        constexpr int kLines = (sizeof(*q) << U) / 128 > 0 ? (sizeof(*q) << U) / 128 : 1;
#pragma unroll
        for (int l = 0; l < kLines; ++l) {
          prefetch_l2(reinterpret_cast<const char*>(q) + 128 * l);
        }
      }
    }
  };
  const bool has_trans = pd->has_trans != 0, has_fb = pd->has_fb != 0;
  __syncthreads();

  const C2* cur = static_cast<const C2*>(a.cur);
  C2* part = static_cast<C2*>(a.part);
  C2* prev = static_cast<C2*>(a.prev);
  auto copy_tile = [&](C2* dst, const C2* src, uint32_t base) {
#pragma unroll
    for (int m = 0; m < NA; ++m) {
      const uint32_t s = t + uint32_t(m) * NT;
      cp_async(dst + pad<R>(s), src + (base | dep_t | dep_ld[m]));
    }
  };
  const PassMeta* pm = &meta;
  uint32_t tile = blockIdx.x;
  if (tile < a.ntiles) {
    const uint32_t base = deposit(tile, pm->outer_pos, pm->nouter);
    copy_tile(bufs, cur, base);
    if constexpr (kAccIn) copy_tile(accb, part, base);
  }
  cp_async_commit();
  for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
    const uint32_t base = deposit(tile, pm->outer_pos, pm->nouter);
    const uint32_t next = tile + gridDim.x;
    const uint32_t next_base = next < a.ntiles ? deposit(next, pm->outer_pos, pm->nouter) : 0u;
    if (next < a.ntiles) copy_tile(bufs + ((it + 1) & 1) * NP, cur, next_base);
    cp_async_commit();
    // Lines this tile's epilogue and the next tile's partial-sum copy will
    // touch go to L2 now, a tile's work ahead of their use.
    if constexpr (kAccIn) {
      if (next < a.ntiles) prefetch_tile(part, next_base);
    }
    if constexpr (KIND == PASS_LAST || KIND == PASS_ONLY) {
      prefetch_tile(a.diag, base);
      prefetch_tile(prev, base);
      if (a.psi_terms != 0) prefetch_tile(a.psi, base);
    }
    cp_async_wait_prior();  // every copy but the one just issued has landed
    __syncthreads();

    const TileSmem<Real> sm{bufs + (it & 1) * NP, accb, cff, cfb, ccx, ccy};
    tile_front<Real, B, R, 0>(sm, pm, t, kAccIn, has_trans, has_fb);
    C2 acc[NA], own[NA];
    const bool acc_in = kAccIn || (pm->active & ((1u << (G - 1)) - 1u)) != 0u;
    tile_layout<Real, B, R, G - 1>(sm, acc, own, t, pm->jmask[G - 1], pm->rmask[G - 1], acc_in,
                                   has_trans, has_fb);
    if constexpr (kAccIn) {
      __syncthreads();  // every thread has read its partial sums
      if (next < a.ntiles) copy_tile(accb, part, next_base);
      cp_async_commit();
    }
    const size_t g0 = base | dep_kb;
    if constexpr (KIND == PASS_FIRST || KIND == PASS_MID) {
#pragma unroll
      for (int x = 0; x < NA; ++x) part[g0 | dep_rg[x]] = acc[x];
    } else {
      const double ds = a.dscale, cr = a.cr, ci = a.ci;
#pragma unroll
      for (int x = 0; x < NA; ++x) {
        const size_t gi = g0 | dep_rg[x];
        const double d = ds * __ldg(&a.diag[gi]);
        double hx = double(acc[x].x) + d * double(own[x].x);
        double hy = double(acc[x].y) + d * double(own[x].y);
        if (a.first) {
          hx *= 0.5;
          hy *= 0.5;
        } else {
          const C2 q = prev[gi];
          hx -= double(q.x);
          hy -= double(q.y);
        }
        C2 tn;
        tn.x = Real(hx);
        tn.y = Real(hy);
        prev[gi] = tn;
        if (a.psi_terms != 0) {
          double2 p = a.psi[gi];
          p.x += cr * hx - ci * hy;
          p.y += cr * hy + ci * hx;
          if (a.psi_terms == 2) {
            const double ox = double(own[x].x), oy = double(own[x].y);
            p.x += a.pr * ox - a.pi * oy;
            p.y += a.pr * oy + a.pi * ox;
          }
          a.psi[gi] = p;
        }
      }
    }
    __syncthreads();  // this tile's buffer is free for the copy after next
  }
  cp_async_wait_all();
}

// -------------------------------------------------------------- host glue

using Kernel = void (*)(const PassDev*, OrderArgs);

struct Family {
  int B = 0, R = 0, nt = 0;
  int line_bits = 0;  // every tile holds spins 0 .. line_bits-1: 128-byte runs
  size_t smem = 0;
  Kernel k[4] = {nullptr, nullptr, nullptr, nullptr};
};

template <typename Real, int B, int R>
Family family() {
  using T = Tile<Real, B, R>;
  Family f;
  f.B = B;
  f.R = R;
  f.nt = T::NT;
  f.line_bits = sizeof(typename T::C2) == 16 ? 3 : 4;
  f.smem = T::kSmem;
  f.k[PASS_FIRST] = k_tile<Real, B, R, PASS_FIRST>;
  f.k[PASS_MID] = k_tile<Real, B, R, PASS_MID>;
  f.k[PASS_LAST] = k_tile<Real, B, R, PASS_LAST>;
  f.k[PASS_ONLY] = k_tile<Real, B, R, PASS_ONLY>;
  return f;
}

// Register bits per thread of the tiled kernel, per precision (a schedule
// choice: fewer bits, more threads per tile; ss_tiled_select changes it).
std::atomic<int> g_register_bits[2] = {3, 4};

const Family& family_for(int precision, int kernel) {
  static const Family f64r3 = family<double, 12, 3>();
  static const Family f64r4 = family<double, 12, 4>();
  static const Family f32r4 = family<float, 13, 4>();
  static const Family f32r5 = family<float, 13, 5>();
  static const Family s64 = family<double, 8, 3>();
  static const Family s32 = family<float, 8, 3>();
  const bool mixed = precision == SS_PRECISION_MIXED;
  if (kernel == SS_KERNEL_TILED_SMALL) return mixed ? s32 : s64;
  const int r = g_register_bits[mixed ? 1 : 0].load();
  if (mixed) return r == 5 ? f32r5 : f32r4;
  return r == 4 ? f64r4 : f64r3;
}

// Builds pass p's table for layouts of R register bits.
void fill_pass(PassDev* pd, int L, int B, int R, uint32_t tile, const std::vector<int>& owner,
               int pass, const std::vector<uint32_t>& field_owner, const ss_ham* h,
               double scale) {
  std::memset(pd, 0, sizeof(PassDev));
  int local[32];
  int nb = 0, no = 0;
  for (int s = 0; s < L; ++s) {
    if ((tile >> s) & 1u) {
      local[s] = nb;
      pd->tile_pos[nb++] = static_cast<uint32_t>(s);
    } else {
      local[s] = -1;
      pd->outer_pos[no++] = static_cast<uint32_t>(s);
    }
  }
  pd->nouter = no;
  for (size_t i = 0; i < h->pairs.size(); ++i) {
    if (owner[i] != pass) continue;
    const PairTerm& p = h->pairs[i];
    const double quarter = scale * 0.25;
    const double ff = quarter * (p.jx + p.jy), fb = quarter * (p.jx - p.jy);
    const int li = local[p.lo], lj = local[p.hi];  // li < lj: positions keep their order
    pd->cff[li * B + lj] = std::abs(ff) > kNegligible ? ff : 0.0;
    pd->cfb[li * B + lj] = std::abs(fb) > kNegligible ? fb : 0.0;
    if (pd->cfb[li * B + lj] != 0.0) pd->has_fb = 1;
  }
  for (int s = 0; s < L; ++s) {
    if (field_owner[s] != static_cast<uint32_t>(pass)) continue;
    const double cx = scale * 0.5 * h->fields[3 * s], cy = scale * 0.5 * h->fields[3 * s + 1];
    if (std::abs(cx) > kNegligible || std::abs(cy) > kNegligible) {
      pd->ccx[local[s]] = cx;
      pd->ccy[local[s]] = cy;
      pd->has_trans = 1;
    }
  }
  // Layout schedule of the tile (Geo<B, R>, written out for run-time B, R).
  const int G = (B + R - 1) / R;
  auto base = [&](int g) { return (g + 1) * R <= B ? g * R : B - R; };
  auto holds = [&](int g, int s) { return s >= base(g) && s < base(g) + R; };
  auto first_layout = [&](int s) {
    for (int g = 0; g < G; ++g) {
      if (holds(g, s)) return g;
    }
    return -1;
  };
  auto pair_layout = [&](int i, int j) {
    for (int g = 0; g < G; ++g) {
      if (holds(g, i) && holds(g, j)) return g;
    }
    return first_layout(i);
  };
  auto cross_mine = [&](int g, int p) {
    return first_layout(base(g) + p) == g && !(g < G - 1 && base(g) + p >= B - R);
  };
  for (int g = 0; g < G; ++g) {
    const int b = base(g);
    for (int p = 0; p < R; ++p) {
      for (int q = p + 1; q < R; ++q) {
        const int i = b + p, j = b + q;
        if (pair_layout(i, j) == g && (pd->cff[i * B + j] != 0.0 || pd->cfb[i * B + j] != 0.0)) {
          pd->rmask[g] |= 1u << (p * R + q);
        }
      }
      if (first_layout(b + p) == g && (pd->ccx[b + p] != 0.0 || pd->ccy[b + p] != 0.0)) {
        pd->active |= 1u << g;
      }
      if (!cross_mine(g, p)) continue;
      for (int j = b + R; j < B; ++j) {
        const int i = b + p;
        if (pd->cff[i * B + j] != 0.0 || pd->cfb[i * B + j] != 0.0) pd->jmask[g] |= 1u << j;
      }
    }
    if (pd->rmask[g] != 0u || pd->jmask[g] != 0u) pd->active |= 1u << g;
  }
  pd->active |= 1u << (G - 1);
}

}  // namespace tiled

// Per-Hamiltonian device tables of the tiled kernel.
struct TiledTables {
  int precision = -1, kernel = -1, nspins = 0, register_bits = 0;
  double scale = 0.0;
  bool valid = false;
  std::vector<uint32_t> plan;
  tiled::PassDev* dev = nullptr;
};

std::vector<uint32_t> tile_plan(int nspins, int tile_bits, int line_bits) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, std::vector<uint32_t>> cache;
  require(nspins >= 1 && nspins <= kMaxSpins, SS_ERR_OUT_OF_RANGE,
          "number of spins must be in [1, kMaxSpins]");
  require(tile_bits >= 2 && tile_bits <= tiled::kMaxTile, SS_ERR_INVALID_ARGUMENT,
          "tile width out of range");
  require(line_bits >= 0 && line_bits <= 8, SS_ERR_INVALID_ARGUMENT, "line bits out of range");
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({nspins, tile_bits, line_bits});
  if (it != cache.end()) return it->second;
  std::vector<uint32_t> p = tiled::make_plan(nspins, tile_bits, line_bits);
  require(tiled::covers(nspins, p), SS_ERR_RUNTIME, "tile plan does not cover every pair");
  for (uint32_t m : p) {
    require(__builtin_popcount(m) == std::min(nspins, tile_bits), SS_ERR_RUNTIME,
            "tile plan has a tile of the wrong width");
  }
  cache.emplace(std::make_tuple(nspins, tile_bits, line_bits), p);
  return p;
}

int tile_bits_for(int precision, int kernel) {
  return tiled::family_for(precision, kernel).B;
}

int tile_variant(int precision, int kernel) {
  return tiled::family_for(precision, kernel).R;
}

int tile_line_bits(int precision, int kernel) {
  return tiled::family_for(precision, kernel).line_bits;
}

void tiled_release(ss_ham* h) {
  if (h->tiled == nullptr) return;
  cudaFree(h->tiled->dev);
  delete h->tiled;
  h->tiled = nullptr;
}

const void* tiled_prepare(ss_ham* h, double scale, int precision, int kernel) {
  const tiled::Family& f = tiled::family_for(precision, kernel);
  const int L = h->nspins;
  require(L >= f.B, SS_ERR_INVALID_ARGUMENT, "the tiled kernel needs at least one full tile");
  {
    // Opt in to the tile's shared memory once per kernel, outside any capture.
    static std::mutex mu;
    static std::map<tiled::Kernel, bool> configured;
    std::lock_guard<std::mutex> lock(mu);
    for (tiled::Kernel k : f.k) {
      if (!configured[k]) {
        SS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(f.smem)));
        configured[k] = true;
      }
    }
  }
  if (h->tiled == nullptr) h->tiled = new TiledTables;
  TiledTables* tt = h->tiled;
  if (tt->precision != precision || tt->kernel != kernel || tt->nspins != L ||
      tt->register_bits != f.R) {
    std::vector<uint32_t> plan = tile_plan(L, f.B, f.line_bits);
    if (tt->dev == nullptr || plan.size() > tt->plan.size()) {
      sync(h->engine);
      cudaFree(tt->dev);
      tt->dev = nullptr;
      SS_CUDA(cudaMalloc(&tt->dev, sizeof(tiled::PassDev) * plan.size()));
    }
    tt->plan = std::move(plan);
    tt->precision = precision;
    tt->kernel = kernel;
    tt->nspins = L;
    tt->register_bits = f.R;
    tt->valid = false;
  }
  if (!tt->valid || tt->scale != scale || !h->tiled_terms_valid) {
    const int P = static_cast<int>(tt->plan.size());
    // Each coupling to the last pass holding both spins (a pass's cost grows
    // with the partner blocks it reads, so concentrating the couplings on
    // few passes leaves the others fewer blocks); each field to the first
    // pass holding its spin.
    std::vector<int> owner(h->pairs.size(), -1);
    for (size_t i = 0; i < h->pairs.size(); ++i) {
      const uint32_t m = (1u << h->pairs[i].lo) | (1u << h->pairs[i].hi);
      for (int p = 0; p < P; ++p) {
        if ((tt->plan[p] & m) == m) owner[i] = p;
      }
    }
    std::vector<uint32_t> field_owner(L, 0);
    for (int s = 0; s < L; ++s) {
      for (int p = 0; p < P; ++p) {
        if ((tt->plan[p] >> s) & 1u) {
          field_owner[s] = static_cast<uint32_t>(p);
          break;
        }
      }
    }
    std::vector<tiled::PassDev> host(P);
    for (int p = 0; p < P; ++p) {
      tiled::fill_pass(&host[p], L, f.B, f.R, tt->plan[p], owner, p, field_owner, h, scale);
    }
    // Pageable source: staged before the call returns.
    SS_CUDA(cudaMemcpyAsync(tt->dev, host.data(), sizeof(tiled::PassDev) * P,
                            cudaMemcpyHostToDevice, h->engine->stream));
    tt->scale = scale;
    tt->valid = true;
    h->tiled_terms_valid = true;
  }
  return tt->dev;
}

void tiled_order(ss_ham* h, int precision, int kernel, const void* cur, void* prev, void* part,
                 double2* psi, int first, double cr, double ci, int psi_terms, double pr,
                 double pi) {
  const tiled::Family& f = tiled::family_for(precision, kernel);
  TiledTables* tt = h->tiled;
  ss_engine* e = h->engine;
  const int P = static_cast<int>(tt->plan.size());
  tiled::OrderArgs a;
  a.cur = cur;
  a.prev = prev;
  a.part = part;
  a.psi = psi;
  a.diag = h->diag;
  a.dscale = tt->scale;
  a.cr = cr;
  a.ci = ci;
  a.pr = pr;
  a.pi = pi;
  a.first = first;
  a.psi_terms = psi_terms;
  a.ntiles = 1u << (h->nspins - f.B);
  const unsigned int grid = std::min<unsigned int>(a.ntiles, static_cast<unsigned int>(e->sm_count));
  for (int p = 0; p < P; ++p) {
    const int kind = P == 1 ? tiled::PASS_ONLY
                     : p == 0 ? tiled::PASS_FIRST
                     : p == P - 1 ? tiled::PASS_LAST
                                  : tiled::PASS_MID;
    launch(e, f.k[kind], grid, f.nt, f.smem, static_cast<const tiled::PassDev*>(tt->dev + p), a);
  }
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_tiled_select(int precision, int register_bits) {
  return guarded([&] {
    require(precision == SS_PRECISION_FP64 || precision == SS_PRECISION_MIXED,
            SS_ERR_INVALID_ARGUMENT, "unknown precision");
    const int def = precision == SS_PRECISION_MIXED ? 4 : 3;
    const int r = register_bits == 0 ? def : register_bits;
    const bool ok = precision == SS_PRECISION_MIXED ? (r == 4 || r == 5) : (r == 3 || r == 4);
    require(ok, SS_ERR_INVALID_ARGUMENT,
            "register bits: 3 or 4 for FP64 tiles, 4 or 5 for mixed-precision tiles");
    tiled::g_register_bits[precision == SS_PRECISION_MIXED ? 1 : 0].store(r);
  });
}

int ss_tile_plan(int nspins, int tile_bits, int line_bits, int32_t* npass, uint32_t* masks,
                 int32_t cap) {
  return guarded([&] {
    require(npass != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    const std::vector<uint32_t> p = tile_plan(nspins, tile_bits, line_bits);
    *npass = static_cast<int32_t>(p.size());
    if (masks != nullptr) {
      require(cap >= static_cast<int32_t>(p.size()), SS_ERR_INVALID_ARGUMENT,
              "mask buffer too small");
      std::copy(p.begin(), p.end(), masks);
    }
  });
}

}  // extern "C"
