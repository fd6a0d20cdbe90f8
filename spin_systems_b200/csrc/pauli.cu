// Pauli-operator kernels (core/SpinOperators.hpp:22-58): sigma acting on one
// spin, the three-axis coupling of one pair, and the total-spin operator used
// by reference-state preparation and the correlator.
//
// Each output amplitude is gathered from its partner(s), so there are no
// write conflicts and no atomics: out[k] depends on in[k] and in[k ^ mask].
#include "common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

// (sigma_axis(spin) in)[k], with sigma_y|down> = -i|up> (SpinOperators.cpp:105-119).
__device__ __forceinline__ double2 sigma_gather(const double2* __restrict__ in, size_t k,
                                                size_t mask, int axis) {
  if (axis == SS_AXIS_Z) {
    const double2 a = in[k];
    return (k & mask) ? a : make_double2(-a.x, -a.y);
  }
  const double2 p = in[k ^ mask];
  if (axis == SS_AXIS_X) return p;
  // up component receives -i * down; down component receives +i * up.
  return (k & mask) ? make_double2(p.y, -p.x) : make_double2(-p.y, p.x);
}

__global__ void k_axpy_sigma(double c, const double2* __restrict__ in, size_t mask, int axis,
                             double2* out, size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double2 t = sigma_gather(in, k, mask, axis);
  double2 o = out[k];
  o.x += c * t.x;
  o.y += c * t.y;
  out[k] = o;
}

__global__ void k_apply_sigma(const double2* __restrict__ in, size_t mask, int axis, double2* out,
                              size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k < n) out[k] = sigma_gather(in, k, mask, axis);
}

// out += (jx sx.sx + jy sy.sy + jz sz.sz) in  (SpinOperators.cpp:179-209)
__global__ void k_axpy_coupling(double flip_both, double flip_one, double jz,
                                const double2* __restrict__ in, size_t mlo, size_t mhi,
                                double2* out, size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const bool aligned = ((k & mlo) != 0) == ((k & mhi) != 0);
  const double2 self = in[k];
  const double2 p = in[k ^ (mlo | mhi)];
  const double c = aligned ? flip_both : flip_one;
  const double z = aligned ? jz : -jz;
  double2 o = out[k];
  o.x += c * p.x + z * self.x;
  o.y += c * p.y + z * self.y;
  out[k] = o;
}

// out = sum_s sigma_axis(s) in, summed in spin order from zero, which is
// exactly the sequence of additions of Ensemble.cpp:47-58.
__global__ void k_total_spin(const double2* __restrict__ in, int nspins, int axis, double2* out,
                             size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  double re = 0.0, im = 0.0;
  for (int s = 0; s < nspins; ++s) {
    const double2 t = sigma_gather(in, k, size_t{1} << s, axis);
    re += t.x;
    im += t.y;
  }
  out[k] = make_double2(re, im);
}

// out += c * d[k] * in[k]  (SpinOperators.cpp:211-226)
__global__ void k_axpy_diagonal(double c, const double* __restrict__ d,
                                const double2* __restrict__ in, double2* out, size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k >= n) return;
  const double f = c * d[k];
  const double2 a = in[k];
  double2 o = out[k];
  o.x += f * a.x;
  o.y += f * a.y;
  out[k] = o;
}

inline unsigned int blocks_for(size_t n) {
  return static_cast<unsigned int>((n + kThreads - 1) / kThreads);
}

void check_distinct(const ss_state* in, const ss_state* out) {
  check_same_space(in, out);
  require(in != out && in->data != out->data, SS_ERR_INVALID_ARGUMENT,
          "kernels require distinct input and output");
}

void check_spin(const ss_state* s, int spin) {
  require(spin >= 0 && spin < s->nspins, SS_ERR_OUT_OF_RANGE, "spin index out of range");
}

void check_axis(int axis) {
  require(axis >= 0 && axis <= 2, SS_ERR_INVALID_ARGUMENT, "unknown axis; expected x, y or z");
}

}  // namespace

void total_spin(int axis, const ss_state* in, ss_state* out) {
  launch(in->engine, k_total_spin, blocks_for(in->size()), kThreads, 0, in->data, in->nspins, axis,
         out->data, in->size());
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_axpy_sigma(double c, const ss_state* in, int spin, int axis, ss_state* out) {
  return guarded([&] {
    check_distinct(in, out);
    check_spin(in, spin);
    check_axis(axis);
    launch(in->engine, k_axpy_sigma, blocks_for(in->size()), kThreads, 0, c, in->data,
           size_t{1} << spin, axis, out->data, in->size());
  });
}

int ss_apply_sigma(const ss_state* in, int spin, int axis, ss_state* out) {
  return guarded([&] {
    check_distinct(in, out);
    check_spin(in, spin);
    check_axis(axis);
    launch(in->engine, k_apply_sigma, blocks_for(in->size()), kThreads, 0, in->data,
           size_t{1} << spin, axis, out->data, in->size());
  });
}

int ss_axpy_coupling(double jx, double jy, double jz, const ss_state* in, int a, int b,
                     ss_state* out) {
  return guarded([&] {
    check_distinct(in, out);
    check_spin(in, a);
    check_spin(in, b);
    require(a != b, SS_ERR_INVALID_ARGUMENT, "a spin cannot couple to itself");
    launch(in->engine, k_axpy_coupling, blocks_for(in->size()), kThreads, 0, jx - jy, jx + jy, jz,
           in->data, size_t{1} << (a < b ? a : b), size_t{1} << (a < b ? b : a), out->data,
           in->size());
  });
}

int ss_axpy_diagonal(double c, const double* diagonal, const ss_state* in, ss_state* out) {
  return guarded([&] {
    check_distinct(in, out);
    require(diagonal != nullptr, SS_ERR_INVALID_ARGUMENT, "null diagonal");
    ss_engine* e = in->engine;
    double* d = nullptr;
    SS_CUDA(cudaMallocAsync(&d, sizeof(double) * in->size(), e->stream));
    SS_CUDA(cudaMemcpyAsync(d, diagonal, sizeof(double) * in->size(), cudaMemcpyHostToDevice,
                            e->stream));
    launch(e, k_axpy_diagonal, blocks_for(in->size()), kThreads, 0, c, d, in->data, out->data,
           in->size());
    SS_CUDA(cudaFreeAsync(d, e->stream));
  });
}

int ss_apply_total_spin(int axis, const ss_state* in, ss_state* out) {
  return guarded([&] {
    check_distinct(in, out);
    check_axis(axis);
    total_spin(axis, in, out);
  });
}

}  // extern "C"
