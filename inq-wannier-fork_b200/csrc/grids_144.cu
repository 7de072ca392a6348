// Compiled grids: 144^3 (the large-cell configuration) (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_144(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(144)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
