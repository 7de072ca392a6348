// Compiled grids: 72^3 and 80^3 (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_72(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(72) INQB_CUBIC(80)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
