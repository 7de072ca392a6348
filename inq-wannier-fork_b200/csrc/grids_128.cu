// Compiled grids: 128^3 (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_128(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(128)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
