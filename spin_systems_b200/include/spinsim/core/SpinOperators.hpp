// Pauli-operator kernels (reference: include/spinsim/core/SpinOperators.hpp:22-82),
// all running on the device.  `in` and `out` must be distinct.
#pragma once

#include <span>

#include "spinsim/core/Bits.hpp"
#include "spinsim/core/StateVector.hpp"

namespace spinsim {

void axpySigmaX(double c, const StateVector& in, SpinIndex spin, StateVector& out);
void axpySigmaY(double c, const StateVector& in, SpinIndex spin, StateVector& out);
void axpySigmaZ(double c, const StateVector& in, SpinIndex spin, StateVector& out);
void applySigmaX(const StateVector& in, SpinIndex spin, StateVector& out);
void applySigmaY(const StateVector& in, SpinIndex spin, StateVector& out);
void applySigmaZ(const StateVector& in, SpinIndex spin, StateVector& out);
void axpyCoupling(double jx, double jy, double jz, const StateVector& in, SpinPair pair,
                  StateVector& out);
void axpyDiagonal(double c, std::span<const double> diagonal, const StateVector& in,
                  StateVector& out);
void axpyTransverse(double cx, double cy, const StateVector& in, SpinIndex spin, StateVector& out);
void axpyFlipFlop(double c, const StateVector& in, SpinPair pair, StateVector& out);
void axpyFlipBoth(double c, const StateVector& in, SpinPair pair, StateVector& out);

}  // namespace spinsim
