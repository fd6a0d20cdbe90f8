// Host interface of the tiled order kernel (tiled.cu) for the plain
// propagator (propagator.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

struct ss_ham;

namespace ss {

// Tile sets of an L-spin vector for tiles of `tile_bits` spins that all hold
// spins 0 .. line_bits-1: every pair of spins shares at least one tile, and
// the last tile is the one with the longest run of low bits (it forms T_n,
// streaming psi, T_{n-2} and the diagonal).  A tile is a bit mask over the
// spins.
std::vector<uint32_t> tile_plan(int nspins, int tile_bits, int line_bits);

// Tile width of a kernel family in a precision (SS_KERNEL_TILED: 12 spins in
// FP64, 13 in mixed; SS_KERNEL_TILED_SMALL: 8 in both).
int tile_bits_for(int precision, int kernel);

// Register bits per thread of the family's current schedule (part of a
// captured step's identity).
int tile_variant(int precision, int kernel);

// Low spins every tile of the family holds (2^line_bits amplitudes = 128 B).
int tile_line_bits(int precision, int kernel);

// Frees the Hamiltonian's per-pass tables.
void tiled_release(ss_ham* h);

// Makes the Hamiltonian's per-pass coefficient tables current for `scale`
// (the -2/bound of the expansion), the precision and the kernel family, and
// returns their device address (part of a captured step's identity).
const void* tiled_prepare(ss_ham* h, double scale, int precision, int kernel);

// Queues one Chebyshev order: every pass of the plan over T_{n-1} = cur, the
// partial sums in `part`, and in the last pass T_n = 2H^ T_{n-1} - T_{n-2}
// written over `prev` (T_1 = H^ T_0 when `first`) and, as `psi_terms` says
// (0, 1 or 2), psi += (cr + i ci) T_n + (pr + i pi) T_{n-1}.
void tiled_order(ss_ham* h, int precision, int kernel, const void* cur, void* prev, void* part,
                 double2* psi, int first, double cr, double ci, int psi_terms, double pr,
                 double pi);

}  // namespace ss
