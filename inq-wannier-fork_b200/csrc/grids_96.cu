// Compiled grids: 96^3 (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_96(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(96)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
