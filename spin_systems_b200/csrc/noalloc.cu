// The echo correlator <ref| sum_s sigma_axis(s) |psi> over device vectors the
// caller owns, computed without allocating anything.  It is the same fused
// gather reduction as ss_measure_corr (src/core/Observable.cpp:66-73), but
// its scratch (block partials, the last-block counter, the result slot) is a
// fixed array in this module's device memory instead of engine memory, and
// the answer is copied straight into the caller's host array.
//
// Scratch: kNoAllocPartials double2 partials + one counter + one result,
// about 19 KB per device.  The grid is reduce_blocks(2^L) blocks, at most
// kMaxReduceBlocks, so every L in [1, 30] fits; anything else is rejected.
// The counter must be zero when a launch starts: static device memory is
// zero at module load and the last block of every launch puts it back to
// zero.  Calls that overlap on one device (two streams, two host threads)
// share this scratch and race; the caller serialises them.
#include <mutex>

#include "common.cuh"

namespace ss {
namespace {

constexpr int kNoAllocPartials = kMaxReduceBlocks;
constexpr int kNoAllocMaxDevices = 64;
static_assert(kMaxReduceBlocks <= kNoAllocPartials, "the largest grid must fit the scratch");

struct NoAllocScratch {
  double2 partials[kNoAllocPartials];
  double2 result;
  unsigned int counter;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch per device, looked up once per device
// (the first call on a device does this, with that device current).
NoAllocScratch* g_scratch_addr[kNoAllocMaxDevices] = {};
std::once_flag g_scratch_once[kNoAllocMaxDevices];
cudaError_t g_scratch_rc[kNoAllocMaxDevices] = {};

NoAllocScratch* scratch_for_current_device() {
  int dev = -1;
  SS_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kNoAllocMaxDevices, SS_ERR_RUNTIME,
          "device ordinal beyond the no-allocation scratch table");
  std::call_once(g_scratch_once[dev], [dev] {
    void* p = nullptr;
    g_scratch_rc[dev] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (g_scratch_rc[dev] == cudaSuccess) g_scratch_addr[dev] = static_cast<NoAllocScratch*>(p);
  });
  if (g_scratch_rc[dev] != cudaSuccess) {
    fail(SS_ERR_CUDA, std::string("cudaGetSymbolAddress of the correlator scratch failed: ") +
                          cudaGetErrorString(g_scratch_rc[dev]));
  }
  return g_scratch_addr[dev];
}

// Same arithmetic, in the same order, as the engine's correlator kernel.
__global__ void k_corr_noalloc(const double2* __restrict__ psi, const double2* __restrict__ ref,
                               int nspins, int axis, size_t n, NoAllocScratch* scratch) {
  double re = 0.0, im = 0.0;
  for (size_t k = blockIdx.x * size_t{blockDim.x} + threadIdx.x; k < n;
       k += size_t{gridDim.x} * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < nspins; ++s) {
      const size_t mask = size_t{1} << s;
      double2 t;
      if (axis == SS_AXIS_Z) {
        const double2 a = psi[k];
        t = (k & mask) ? a : make_double2(-a.x, -a.y);
      } else {
        const double2 p = psi[k ^ mask];
        if (axis == SS_AXIS_X) {
          t = p;
        } else {
          t = (k & mask) ? make_double2(p.y, -p.x) : make_double2(-p.y, p.x);
        }
      }
      sr += t.x;
      si += t.y;
    }
    const double2 r = ref[k];
    re += r.x * sr + r.y * si;
    im += r.x * si - r.y * sr;
  }
  grid_reduce2<kReduceThreads>(make_double2(re, im), scratch->partials, &scratch->counter,
                               &scratch->result);
}

void check_vector(const double* p, int dev, const char* what) {
  require(p != nullptr, SS_ERR_INVALID_ARGUMENT, "null state pointer");
  require(reinterpret_cast<uintptr_t>(p) % 16 == 0, SS_ERR_INVALID_ARGUMENT,
          "state pointer is not 16-byte aligned");
  cudaPointerAttributes a{};
  SS_CUDA(cudaPointerGetAttributes(&a, p));
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) {
    fail(SS_ERR_INVALID_ARGUMENT, std::string(what) + " is not device memory");
  }
  require(a.device == dev, SS_ERR_INVALID_ARGUMENT,
          "state lives on another device than the current one");
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" int ss_measure_corr_noalloc(const double* psi, const double* ref, int nspins, int axis,
                                       void* stream, double out[2]) {
  return guarded([&] {
    require(nspins >= 1 && nspins <= kMaxSpins, SS_ERR_OUT_OF_RANGE,
            "nspins must be in [1, 30] for the no-allocation correlator");
    require(axis >= 0 && axis <= 2, SS_ERR_INVALID_ARGUMENT, "unknown axis; expected x, y or z");
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    const size_t n = size_t{1} << nspins;
    const int blocks = reduce_blocks(n);
    require(blocks <= kNoAllocPartials, SS_ERR_OUT_OF_RANGE,
            "state too large for the no-allocation correlator scratch");
    NoAllocScratch* scratch = scratch_for_current_device();
    int dev = -1;
    SS_CUDA(cudaGetDevice(&dev));
    check_vector(psi, dev, "psi");
    check_vector(ref, dev, "ref");
    auto s = static_cast<cudaStream_t>(stream);
    k_corr_noalloc<<<blocks, kReduceThreads, 0, s>>>(reinterpret_cast<const double2*>(psi),
                                                      reinterpret_cast<const double2*>(ref),
                                                      nspins, axis, n, scratch);
    SS_CUDA(cudaGetLastError());
    double2 r;
    SS_CUDA(cudaMemcpyAsync(&r, &scratch->result, sizeof(r), cudaMemcpyDeviceToHost, s));
    SS_CUDA(cudaStreamSynchronize(s));
    out[0] = r.x;
    out[1] = r.y;
  });
}
