// Compiled grids: 64^3 and tetragonal 64 x 64 x 96 (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_64(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(64)
      INQB_GRID(64, 64, 96)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
