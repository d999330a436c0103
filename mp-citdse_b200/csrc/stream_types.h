// stream_types.h -- launch arguments of the dipole-streaming kernel.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "plan.h"

namespace mpc {

// One 2-D tensor map per dipole block (row-major, padded pitch).
struct TmapSet {
  CUtensorMap m[kMaxBlocks];
};

struct StreamArgs {
  const double2* y;       // stage input, ntot complex (+ kVecPad zeroed tail)
  double2* RP;            // row partials
  double2* CP;            // column partial slots, kStripW complex each
  const int* cta_slot0;   // first CP slot of each CTA
  unsigned* status;
  // the first keep_frac of every CTA's tiles are loaded with an L2 evict-last
  // hint (they stay in L2 from pass to pass), the rest evict-first
  float keep_frac;
  Geometry g;
};

}  // namespace mpc
