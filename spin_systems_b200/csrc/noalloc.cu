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
// share this scratch and race; the caller serialises them.  Each vector is
// checked to lie in device memory of the current device, 16-byte aligned,
// with its 2 * 2^nspins doubles inside one allocation.
#include <cuda.h>

#include <mutex>

#include "observables.cuh"

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

// Device address of g_noalloc_scratch per device, looked up with that device
// current by the first call on it that succeeds (a failed lookup, e.g. one
// made during a stream capture, is not remembered: the next call retries).
// The address stays valid while the device's primary context lives; it is
// kept for the life of the process.
NoAllocScratch* g_scratch_addr[kNoAllocMaxDevices] = {};
std::mutex g_scratch_mu[kNoAllocMaxDevices];

NoAllocScratch* scratch_for_current_device() {
  int dev = -1;
  SS_CUDA(cudaGetDevice(&dev));
  require(dev >= 0 && dev < kNoAllocMaxDevices, SS_ERR_RUNTIME,
          "device ordinal beyond the no-allocation scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mu[dev]);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (rc != cudaSuccess) {
      cudaGetLastError();
      fail(SS_ERR_CUDA, std::string("cudaGetSymbolAddress of the correlator scratch failed: ") +
                            cudaGetErrorString(rc));
    }
    g_scratch_addr[dev] = static_cast<NoAllocScratch*>(p);
  }
  return g_scratch_addr[dev];
}

// Same per-thread sums, in the same order, as the engine's correlator kernel
// (observables.cuh), reduced into the static scratch.
__global__ void k_corr_noalloc(const double2* __restrict__ psi, const double2* __restrict__ ref,
                               int nspins, int axis, size_t n, NoAllocScratch* scratch) {
  grid_reduce2<kReduceThreads>(corr_thread_sum(psi, ref, nspins, axis, n), scratch->partials,
                               &scratch->counter, &scratch->result);
}

// The driver's cuMemGetAddressRange, fetched through the runtime (the
// library links no driver library): the allocation holding a pointer.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

AddressRangeFn address_range_fn() {
  static std::once_flag once;
  static AddressRangeFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = reinterpret_cast<AddressRangeFn>(p);
    } else {
      cudaGetLastError();
    }
  });
  require(fn != nullptr, SS_ERR_RUNTIME, "cuMemGetAddressRange is not available");
  return fn;
}

// A state vector the kernel may read: device (or managed) memory of the
// current device, 16-byte aligned, and `bytes` long inside one allocation.
void check_vector(const double* p, int dev, size_t bytes, const char* what) {
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
  CUdeviceptr base = 0;
  size_t size = 0;
  const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p);
  if (address_range_fn()(&base, &size, at) != CUDA_SUCCESS) {
    fail(SS_ERR_INVALID_ARGUMENT, std::string(what) + " is not inside a device allocation");
  }
  if (at - base > size || size - (at - base) < bytes) {
    fail(SS_ERR_INVALID_ARGUMENT,
         std::string(what) + " is shorter than 2 * 2^nspins doubles (its allocation ends first)");
  }
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
    check_vector(psi, dev, n * sizeof(double2), "psi");
    check_vector(ref, dev, n * sizeof(double2), "ref");
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
