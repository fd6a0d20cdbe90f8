// Engine lifetime and the StateVector operations of core/StateVector.hpp:82-140
// (src/core/StateVector.cpp:10-75) on device-resident amplitudes.
#include "common.cuh"

namespace ss {

thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

void check_state(const ss_state* s) {
  require(s != nullptr && s->data != nullptr, SS_ERR_INVALID_ARGUMENT, "null state vector");
}

void check_same_space(const ss_state* a, const ss_state* b) {
  check_state(a);
  check_state(b);
  require(a->nspins == b->nspins, SS_ERR_INVALID_ARGUMENT, "state vectors span different spaces");
  require(a->engine == b->engine, SS_ERR_INVALID_ARGUMENT, "state vectors live on different engines");
}

namespace {

constexpr int kThreads = 256;

inline unsigned int blocks_for(size_t n) {
  return static_cast<unsigned int>((n + kThreads - 1) / kThreads);
}

__global__ void k_scale(double2* v, size_t n, double f) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k < n) {
    const double2 a = v[k];
    v[k] = make_double2(a.x * f, a.y * f);
  }
}

__global__ void k_negate(double2* v, size_t n) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k < n) {
    const double2 a = v[k];
    v[k] = make_double2(-a.x, -a.y);
  }
}

// this += (cr + i ci) * other  (StateVector.cpp:20-31)
__global__ void k_add_scaled(double2* dst, const double2* __restrict__ src, size_t n, double cr,
                             double ci) {
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k < n) {
    const double2 o = src[k];
    double2 d = dst[k];
    d.x += cr * o.x - ci * o.y;
    d.y += cr * o.y + ci * o.x;
    dst[k] = d;
  }
}

__global__ void k_set_one(double2* v, size_t index) { v[index] = make_double2(1.0, 0.0); }

// sum |c_k|^2
__global__ void k_norm2(const double2* __restrict__ v, size_t n, double2* partials,
                        unsigned int* counter, double2* result) {
  double s = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    const double2 a = v[k];
    s += a.x * a.x + a.y * a.y;
  }
  grid_reduce2<kReduceThreads>(make_double2(s, 0.0), partials, counter, result);
}

// <b|a> = sum conj(b_k) a_k  (StateVector.cpp:58-70)
__global__ void k_inner(const double2* __restrict__ a, const double2* __restrict__ b, size_t n,
                        double2* partials, unsigned int* counter, double2* result) {
  double re = 0.0, im = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    const double2 x = a[k], y = b[k];
    re += y.x * x.x + y.y * x.y;
    im += y.x * x.y - y.y * x.x;
  }
  grid_reduce2<kReduceThreads>(make_double2(re, im), partials, counter, result);
}

// v *= 1/sqrt(result.x), flagging a zero norm instead of dividing by it.
__global__ void k_normalize_apply(double2* v, size_t n, const double2* result, int* flag) {
  const double nrm = sqrt(result->x);
  if (nrm == 0.0 || !isfinite(nrm)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *flag = nrm == 0.0 ? SS_ERR_DOMAIN : SS_ERR_NUMERIC;
    return;
  }
  const double f = 1.0 / nrm;
  const size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x;
  if (k < n) {
    const double2 a = v[k];
    v[k] = make_double2(a.x * f, a.y * f);
  }
}

}  // namespace

void state_scale(ss_state* s, double f) {
  launch(s->engine, k_scale, blocks_for(s->size()), kThreads, 0, s->data, s->size(), f);
}

void state_negate(ss_state* s) {
  launch(s->engine, k_negate, blocks_for(s->size()), kThreads, 0, s->data, s->size());
}

void state_add_scaled(ss_state* dst, double cr, double ci, const ss_state* src) {
  launch(dst->engine, k_add_scaled, blocks_for(dst->size()), kThreads, 0, dst->data, src->data,
         dst->size(), cr, ci);
}

// Queues ||s||^2 into result slot `slot` (no synchronisation).
void state_norm2_async(const ss_state* s, int slot) {
  ss_engine* e = s->engine;
  launch(e, k_norm2, reduce_blocks(s->size()), kReduceThreads, 0, s->data, s->size(),
         e->red_partials, e->red_counter, e->red_result + slot);
}

// Queues normalisation by the norm in `slot`, raising flag 0 on a zero norm.
void state_normalize_async(ss_state* s, int slot) {
  state_norm2_async(s, slot);
  ss_engine* e = s->engine;
  launch(e, k_normalize_apply, blocks_for(s->size()), kThreads, 0, s->data, s->size(),
         e->red_result + slot, e->dev_flags);
}

// Raises the first device status flag as an error (synchronises).
void check_flags(ss_engine* e) {
  SS_CUDA(cudaMemcpyAsync(e->host_flags, e->dev_flags, sizeof(int) * 16, cudaMemcpyDeviceToHost,
                          e->stream));
  sync(e);
  for (int i = 0; i < 16; ++i) {
    if (e->host_flags[i] != 0) {
      const int code = e->host_flags[i];
      SS_CUDA(cudaMemsetAsync(e->dev_flags, 0, sizeof(int) * 16, e->stream));
      sync(e);
      if (code == SS_ERR_DOMAIN) fail(code, "cannot normalize a zero state");
      if (code == SS_ERR_TIMEOUT) fail(code, "a bounded device wait gave up");
      fail(code, "a norm reduction saw NaN or Inf");
    }
  }
}

}  // namespace ss

using namespace ss;

extern "C" {

const char* ss_last_error(void) { return g_last_error.c_str(); }

int ss_version(void) { return 100; }

int ss_engine_create(int device, ss_engine** out) {
  return guarded([&] {
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output handle");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      fail(SS_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    require(device >= 0 && device < count, SS_ERR_NO_DEVICE, "device index out of range");
    cudaDeviceProp prop{};
    SS_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) fail(SS_ERR_NO_DEVICE, "this build targets sm_100a (B200) only");
    SS_CUDA(cudaSetDevice(device));
    auto* e = new ss_engine;
    e->device = device;
    e->sm_count = prop.multiProcessorCount;
    try {
      SS_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
      SS_CUDA(cudaMalloc(&e->red_partials, sizeof(double2) * kMaxReduceBlocks));
      SS_CUDA(cudaMalloc(&e->red_counter, sizeof(unsigned int)));
      SS_CUDA(cudaMalloc(&e->red_result, sizeof(double2) * 64));
      SS_CUDA(cudaMalloc(&e->dev_flags, sizeof(int) * 16));
      SS_CUDA(cudaMallocHost(&e->host_result, sizeof(double2) * 64));
      SS_CUDA(cudaMallocHost(&e->host_flags, sizeof(int) * 16));
      SS_CUDA(cudaMemsetAsync(e->red_counter, 0, sizeof(unsigned int), e->stream));
      SS_CUDA(cudaMemsetAsync(e->red_result, 0, sizeof(double2) * 64, e->stream));
      SS_CUDA(cudaMemsetAsync(e->dev_flags, 0, sizeof(int) * 16, e->stream));
      sync(e);
    } catch (...) {
      ss_engine_destroy(e);
      throw;
    }
    *out = e;
  });
}

int ss_engine_destroy(ss_engine* e) {
  return guarded([&] {
    if (e == nullptr) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    cudaFree(e->red_partials);
    cudaFree(e->red_counter);
    cudaFree(e->red_result);
    cudaFree(e->dev_flags);
    cudaFree(e->evolve_t[0]);
    cudaFree(e->evolve_t[1]);
    cudaFree(e->evolve_part);
    for (ss::StepGraph& g : e->step_graphs) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
    }
    cudaFreeHost(e->host_result);
    cudaFreeHost(e->host_flags);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
  });
}

int ss_engine_synchronize(ss_engine* e) {
  return guarded([&] {
    require(e != nullptr, SS_ERR_INVALID_ARGUMENT, "null engine");
    sync(e);
  });
}

void* ss_engine_stream(ss_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

int64_t ss_engine_launch_count(const ss_engine* e) { return e ? e->launches.load() : 0; }

int ss_state_create(ss_engine* e, int nspins, ss_state** out) {
  return guarded([&] {
    require(e != nullptr && out != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    require(nspins >= 1 && nspins <= kMaxSpins, SS_ERR_OUT_OF_RANGE,
            "number of spins must be in [1, kMaxSpins]");
    auto* s = new ss_state;
    s->engine = e;
    s->nspins = nspins;
    if (cudaMalloc(&s->data, sizeof(double2) * s->size()) != cudaSuccess) {
      cudaGetLastError();
      delete s;
      fail(SS_ERR_CUDA, "device allocation of a state vector failed");
    }
    SS_CUDA(cudaMemsetAsync(s->data, 0, sizeof(double2) * s->size(), e->stream));
    *out = s;
  });
}

int ss_state_destroy(ss_state* s) {
  return guarded([&] {
    if (s == nullptr) return;
    cudaStreamSynchronize(s->engine->stream);
    cudaFree(s->data);
    delete s;
  });
}

int ss_state_nspins(const ss_state* s) { return s ? s->nspins : -1; }

int ss_state_upload(ss_state* s, const double* host) {
  return guarded([&] {
    check_state(s);
    require(host != nullptr, SS_ERR_INVALID_ARGUMENT, "null host buffer");
    SS_CUDA(cudaMemcpyAsync(s->data, host, sizeof(double2) * s->size(), cudaMemcpyHostToDevice,
                            s->engine->stream));
    sync(s->engine);
  });
}

int ss_state_download(const ss_state* s, double* host) {
  return guarded([&] {
    check_state(s);
    require(host != nullptr, SS_ERR_INVALID_ARGUMENT, "null host buffer");
    SS_CUDA(cudaMemcpyAsync(host, s->data, sizeof(double2) * s->size(), cudaMemcpyDeviceToHost,
                            s->engine->stream));
    sync(s->engine);
  });
}

int ss_state_copy(ss_state* dst, const ss_state* src) {
  return guarded([&] {
    check_same_space(dst, src);
    if (dst == src) return;
    SS_CUDA(cudaMemcpyAsync(dst->data, src->data, sizeof(double2) * src->size(),
                            cudaMemcpyDeviceToDevice, dst->engine->stream));
  });
}

int ss_state_set_zero(ss_state* s) {
  return guarded([&] {
    check_state(s);
    SS_CUDA(cudaMemsetAsync(s->data, 0, sizeof(double2) * s->size(), s->engine->stream));
  });
}

int ss_state_scale(ss_state* s, double f) {
  return guarded([&] {
    check_state(s);
    state_scale(s, f);
  });
}

int ss_state_negate(ss_state* s) {
  return guarded([&] {
    check_state(s);
    state_negate(s);
  });
}

int ss_state_add_scaled(ss_state* dst, double cr, double ci, const ss_state* other) {
  return guarded([&] {
    check_same_space(dst, other);
    state_add_scaled(dst, cr, ci, other);
  });
}

int ss_state_set_basis(ss_state* s, uint64_t index) {
  return guarded([&] {
    check_state(s);
    require(index < s->size(), SS_ERR_OUT_OF_RANGE, "basis state index outside the 2^L state space");
    SS_CUDA(cudaMemsetAsync(s->data, 0, sizeof(double2) * s->size(), s->engine->stream));
    launch(s->engine, k_set_one, 1, 1, 0, s->data, static_cast<size_t>(index));
  });
}

int ss_state_norm(const ss_state* s, double* out) {
  return guarded([&] {
    check_state(s);
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    state_norm2_async(s, 0);
    read_results(s->engine, 1);
    *out = std::sqrt(s->engine->host_result[0].x);
  });
}

int ss_state_normalize(ss_state* s, double* norm_before) {
  return guarded([&] {
    check_state(s);
    state_norm2_async(s, 0);
    read_results(s->engine, 1);
    const double n = std::sqrt(s->engine->host_result[0].x);
    if (norm_before) *norm_before = n;
    require(n != 0.0, SS_ERR_DOMAIN, "cannot normalize a zero state");
    state_scale(s, 1.0 / n);
  });
}

int ss_state_inner_product(const ss_state* self, const ss_state* other, double out[2]) {
  return guarded([&] {
    check_same_space(self, other);
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    ss_engine* e = self->engine;
    launch(e, k_inner, reduce_blocks(self->size()), kReduceThreads, 0, self->data, other->data,
           self->size(), e->red_partials, e->red_counter, e->red_result);
    read_results(e, 1);
    out[0] = e->host_result[0].x;
    out[1] = e->host_result[0].y;
  });
}

int ss_state_swap(ss_state* a, ss_state* b) {
  return guarded([&] {
    check_same_space(a, b);
    std::swap(a->data, b->data);
  });
}

}  // extern "C"
