// Compiled grids: cubic grids 12 to 30 and the orthorhombic 18 x 24 x 20 of the reference's laplacian test (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_small(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(12) INQB_CUBIC(16) INQB_CUBIC(18) INQB_CUBIC(20) INQB_CUBIC(24) INQB_CUBIC(30)
      INQB_GRID(18, 24, 20)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
