// Shared plumbing of the B200 echo engine: error model, engine and state
// objects, launch accounting and the deterministic FP64 reductions.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/spinsim_b200.h"
#include "common_host.hpp"

namespace ss {

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    fail(SS_ERR_CUDA, std::string(what) + " failed at " + file + ":" + std::to_string(line) +
                          ": " + cudaGetErrorString(e));
  }
}
#define SS_CUDA(call) ::ss::cuda_check((call), #call, __FILE__, __LINE__)

inline void require(bool ok, int code, const char* msg) {
  if (!ok) fail(code, msg);
}

constexpr int kMaxSpins = 30;               // core/Bits.hpp:13
constexpr int kMaxPairs = kMaxSpins * (kMaxSpins - 1) / 2;
constexpr double kNegligible = 1.0e-14;     // src/core/Hamiltonian.cpp:16
constexpr int kReduceThreads = 256;
constexpr int kMaxReduceBlocks = 1184;      // 8 x 148 SMs

}  // namespace ss

namespace ss {
// One captured Chebyshev step of the plain propagator (init + every order +
// the optional renormalisation) for fixed vectors, tables and weights.
struct StepGraph {
  const void* terms = nullptr;
  const void* diag = nullptr;
  const void* psi = nullptr;
  const void* t0 = nullptr;
  const void* t1 = nullptr;
  const void* part = nullptr;    // tiled kernel: the partial-sum vector
  const void* passes = nullptr;  // tiled kernel: the per-pass tables
  size_t n = 0;
  int autonormalize = 0;
  int precision = 0;
  int kernel = 0;
  std::vector<double> weights;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;  // kernel nodes per replay
  uint64_t used = 0;    // last use, for eviction
};
}  // namespace ss

// Device-side scratch of one engine: reduction partials, the completion
// counter of the last-block reduction and result slots read by the host.
struct ss_engine {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  double2* red_partials = nullptr;  // kMaxReduceBlocks entries
  unsigned int* red_counter = nullptr;
  double2* red_result = nullptr;    // 64 result slots
  int* dev_flags = nullptr;         // 16 status flags written by kernels
  double2* host_result = nullptr;   // pinned mirror of red_result
  int* host_flags = nullptr;
  double2* evolve_t[2] = {nullptr, nullptr};  // the propagator's two work vectors
  int evolve_nspins = 0;                      // their capacity, as L
  double2* evolve_part = nullptr;             // tiled kernel: partial sums of H T_{n-1}
  int evolve_part_nspins = 0;
  std::vector<ss::StepGraph> step_graphs;     // the plain propagator's captured steps
  uint64_t graph_clock = 0;
  std::atomic<int64_t> launches{0};
};

struct ss_state {
  ss_engine* engine = nullptr;
  int nspins = 0;
  double2* data = nullptr;  // 2^L complex amplitudes, interleaved re/im
  size_t size() const { return size_t{1} << nspins; }
};

namespace ss {

// Launches a kernel on the engine's stream, counting it and surfacing launch
// errors immediately.
template <typename... KArgs, typename... Args>
void launch(ss_engine* e, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
            Args&&... args) {
  kernel<<<grid, block, smem, e->stream>>>(std::forward<Args>(args)...);
  SS_CUDA(cudaGetLastError());
  e->launches.fetch_add(1, std::memory_order_relaxed);
}

inline void sync(ss_engine* e) { SS_CUDA(cudaStreamSynchronize(e->stream)); }

// Blocks for a grid-stride reduction over n items: a fixed function of n, so
// the summation order (and hence the result) is the same on every run.
inline int reduce_blocks(size_t n) {
  const size_t per_block = size_t{kReduceThreads} * 4;
  size_t b = (n + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > size_t{kMaxReduceBlocks}) b = kMaxReduceBlocks;
  return static_cast<int>(b);
}

// Reads `count` result slots back to the host (synchronises the stream).
inline void read_results(ss_engine* e, int count) {
  SS_CUDA(cudaMemcpyAsync(e->host_result, e->red_result, sizeof(double2) * count,
                          cudaMemcpyDeviceToHost, e->stream));
  sync(e);
}

void check_state(const ss_state* s);
void check_same_space(const ss_state* a, const ss_state* b);

}  // namespace ss

// ---------------------------------------------------------------- device side
__device__ __forceinline__ double2 operator+(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2& operator+=(double2& a, double2 b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}

namespace ss {

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, off);
    v.y += __shfl_down_sync(0xffffffffu, v.y, off);
  }
  return v;
}

// Block-wide sum of a double2; thread 0 receives the total.
template <int NT>
__device__ __forceinline__ double2 block_sum2(double2 v, double2* warp_buf) {
  v = warp_sum2(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_buf[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < NT / 32 ? warp_buf[lane] : make_double2(0.0, 0.0);
    v = warp_sum2(v);
  }
  __syncthreads();
  return v;
}

// Grid-wide deterministic reduction: every block stores its partial, and the
// last block to arrive adds the partials in block order into `*result`.
template <int NT>
__device__ void grid_reduce2(double2 v, double2* partials, unsigned int* counter,
                             double2* result) {
  __shared__ double2 warp_buf[NT / 32];
  __shared__ bool last;
  v = block_sum2<NT>(v, warp_buf);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v;
    __threadfence();
    const unsigned int prev = atomicAdd(counter, 1u);
    last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double2 acc = make_double2(0.0, 0.0);
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += NT) acc += __ldcg(&partials[i]);
  acc = block_sum2<NT>(acc, warp_buf);
  if (threadIdx.x == 0) {
    *result = acc;
    *counter = 0u;
  }
}

}  // namespace ss
