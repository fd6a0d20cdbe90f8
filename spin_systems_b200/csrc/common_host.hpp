// Error model shared by host-only and CUDA translation units: every failure
// is an ss::Error carrying the C ABI status it maps to.
#pragma once

#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/spinsim_b200.h"

namespace ss {

// A named NVTX range over one host call of the C ABI (batch execution, a
// propagation, a training run): a marker on a profiler's timeline and a
// filter for `ncu --nvtx --nvtx-include`.  NVTX is header-only and the push
// and pop cost a pointer check unless a tool is attached.
class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void host_fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void host_require(bool ok, int code, const char* msg) {
  if (!ok) host_fail(code, msg);
}

void set_last_error(const std::string& msg);

// Runs `body`, mapping exceptions to a status and the thread-local message.
template <typename F>
int guarded(F&& body) noexcept {
  try {
    body();
    return SS_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("out of host memory");
    return SS_ERR_RUNTIME;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SS_ERR_RUNTIME;
  } catch (...) {
    set_last_error("unknown failure");
    return SS_ERR_RUNTIME;
  }
}

}  // namespace ss
