// Compiled grids: cubic grids 32 to 60 and orthorhombic 36 x 48 x 60 (one translation unit per group, built in parallel).
#include "launch_h.cuh"

namespace inqb {

void register_grids_mid(GridRegistry& reg) {
  const GridRegistry plans = {
      INQB_CUBIC(32) INQB_CUBIC(36) INQB_CUBIC(40) INQB_CUBIC(48) INQB_CUBIC(60)
      INQB_GRID(36, 48, 60) INQB_GRID(24, 24, 48) INQB_GRID(32, 32, 48)
  };
  reg.insert(plans.begin(), plans.end());
}

}  // namespace inqb
