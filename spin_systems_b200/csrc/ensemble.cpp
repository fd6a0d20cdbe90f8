// C ABI of the host-side realisation assembly (io/Experiment.cpp:10-35).
#include <cstring>

#include "common_host.hpp"
#include "host_numerics.hpp"

using namespace ss;

extern "C" int ss_realization_setup(const ss_run_config* config, uint64_t index, int32_t* nspins,
                                    double* fields, int32_t* pairs, double* couplings,
                                    int32_t* npairs, double* psi0) {
  return guarded([&] {
    host_require(config != nullptr, SS_ERR_INVALID_ARGUMENT, "null config");
    const Realization r = assemble_realization(*config, index);
    if (nspins) *nspins = r.nspins;
    if (fields) std::memcpy(fields, r.fields.data(), sizeof(double) * r.fields.size());
    if (pairs || couplings) {
      for (size_t p = 0; p < r.pairs.size(); ++p) {
        if (pairs) {
          pairs[2 * p] = r.pairs[p].lo;
          pairs[2 * p + 1] = r.pairs[p].hi;
        }
        if (couplings) {
          couplings[3 * p] = r.pairs[p].jx;
          couplings[3 * p + 1] = r.pairs[p].jy;
          couplings[3 * p + 2] = r.pairs[p].jz;
        }
      }
    }
    if (npairs) *npairs = static_cast<int32_t>(r.pairs.size());
    if (psi0) std::memcpy(psi0, r.psi0.data(), sizeof(double) * r.psi0.size());
  });
}
