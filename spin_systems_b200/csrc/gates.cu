// Ideal pulses: SpinRotation::apply (src/core/Gate.cpp:60-85), its 2x2 matrix
// (Gate.cpp:20-33), and the two-spin unitary of Gate.cpp:90-121.
#include <cmath>

#include "common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

struct Rot {
  double ll_r, ll_i, lh_r, lh_i, hl_r, hl_i, hh_r, hh_i;
};

// One target spin: every (lo, hi) pair differing in bit `spin` gets
// (lo, hi) <- U (lo, hi); thread j handles pair j of the 2^(L-1).
__global__ void k_rotate(double2* psi, size_t half, int spin, Rot u) {
  const size_t j = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (j >= half) return;
  const size_t low_mask = (size_t{1} << spin) - 1;
  const size_t lo = ((j & ~low_mask) << 1) | (j & low_mask);
  const size_t hi = lo | (size_t{1} << spin);
  const double2 a = psi[lo], b = psi[hi];
  const double lr = (u.ll_r * a.x - u.ll_i * a.y) + (u.lh_r * b.x - u.lh_i * b.y);
  const double li = (u.ll_r * a.y + u.ll_i * a.x) + (u.lh_r * b.y + u.lh_i * b.x);
  const double hr = (u.hl_r * a.x - u.hl_i * a.y) + (u.hh_r * b.x - u.hh_i * b.y);
  const double hi_ = (u.hl_r * a.y + u.hl_i * a.x) + (u.hh_r * b.y + u.hh_i * b.x);
  psi[lo] = make_double2(lr, li);
  psi[hi] = make_double2(hr, hi_);
}

struct Mat4 {
  double m[32];
};

// 4x4 unitary on (dd, low-up, high-up, uu) of the pair (lo, hi); thread j
// handles block j of the 2^(L-2).
__global__ void k_two_spin(double2* psi, size_t quarter, int lo, int hi, Mat4 g) {
  const size_t j = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (j >= quarter) return;
  // Insert zero bits at positions lo and hi (lo < hi).
  const size_t ml = (size_t{1} << lo) - 1;
  size_t dd = ((j & ~ml) << 1) | (j & ml);
  const size_t mh = (size_t{1} << hi) - 1;
  dd = ((dd & ~mh) << 1) | (dd & mh);
  const size_t idx[4] = {dd, dd | (size_t{1} << lo), dd | (size_t{1} << hi),
                         dd | (size_t{1} << lo) | (size_t{1} << hi)};
  double2 v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = psi[idx[q]];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double ar = 0.0, ai = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double mr = g.m[2 * (4 * r + c)], mi = g.m[2 * (4 * r + c) + 1];
      ar += mr * v[c].x - mi * v[c].y;
      ai += mr * v[c].y + mi * v[c].x;
    }
    psi[idx[r]] = make_double2(ar, ai);
  }
}

}  // namespace

void rotation_matrix(const double axis[3], double angle, double u[8]) {
  const double len = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
  require(len > 0.0, SS_ERR_INVALID_ARGUMENT, "rotation axis must have non-zero length");
  const double nx = axis[0] / len, ny = axis[1] / len, nz = axis[2] / len;
  const double c = std::cos(0.5 * angle), s = std::sin(0.5 * angle);
  // exp(-i theta/2 n.sigma) in the (down, up) basis, sigma_z = diag(-1, +1).
  u[0] = c;       u[1] = s * nz;
  u[2] = s * ny;  u[3] = -s * nx;
  u[4] = -s * ny; u[5] = -s * nx;
  u[6] = c;       u[7] = -s * nz;
}

void rotate(ss_state* psi, const double u[8], const int32_t* targets, int ntargets) {
  const Rot r{u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7]};
  const size_t half = psi->size() / 2;
  const unsigned int grid = static_cast<unsigned int>((half + kThreads - 1) / kThreads);
  for (int i = 0; i < ntargets; ++i) {
    require(targets[i] >= 0 && targets[i] < psi->nspins, SS_ERR_OUT_OF_RANGE,
            "rotation names a spin outside the system");
    launch(psi->engine, k_rotate, grid, kThreads, 0, psi->data, half, targets[i], r);
  }
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_rotation_matrix(const double axis[3], double angle, double u[8]) {
  return guarded([&] {
    require(axis != nullptr && u != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    rotation_matrix(axis, angle, u);
  });
}

int ss_rotate(ss_state* psi, const double u[8], const int32_t* targets, int32_t ntargets) {
  return guarded([&] {
    check_state(psi);
    require(u != nullptr, SS_ERR_INVALID_ARGUMENT, "null rotation matrix");
    require(ntargets >= 1 && targets != nullptr, SS_ERR_INVALID_ARGUMENT,
            "a rotation must name at least one spin");
    rotate(psi, u, targets, ntargets);
  });
}

int ss_two_spin_gate(ss_state* psi, const double m[32], int a, int b) {
  return guarded([&] {
    check_state(psi);
    require(m != nullptr, SS_ERR_INVALID_ARGUMENT, "null gate matrix");
    require(a != b, SS_ERR_INVALID_ARGUMENT, "a spin cannot couple to itself");
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    require(lo >= 0 && hi < psi->nspins, SS_ERR_OUT_OF_RANGE,
            "gate names a spin outside the system");
    require(psi->nspins >= 2, SS_ERR_OUT_OF_RANGE, "gate names a spin outside the system");
    Mat4 g;
    std::memcpy(g.m, m, sizeof g.m);
    const size_t quarter = psi->size() / 4;
    launch(psi->engine, k_two_spin,
           static_cast<unsigned int>((quarter + kThreads - 1) / kThreads), kThreads, 0, psi->data,
           quarter, lo, hi, g);
  });
}

}  // extern "C"
