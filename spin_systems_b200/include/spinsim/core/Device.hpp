// The device behind the spinsim C++ API: one ss_engine (device + stream) per
// host thread, created on first use, and the mapping of C ABI statuses back
// onto the exception types the reference throws.
#pragma once

#include "spinsim_b200.h"

namespace spinsim {

/// The calling thread's engine on device 0 (or $SPINSIM_DEVICE).
ss_engine* threadEngine();

/// Throws the exception the reference would for a non-zero status.
void checkStatus(int status);

}  // namespace spinsim
