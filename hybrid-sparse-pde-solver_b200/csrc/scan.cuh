// scan.cuh -- device prefix sums used by the setup phases (ILU levels, AMG).
#pragma once

#include "engine.cuh"

namespace hamlss {

// In-place exclusive scan of `count` int32 values on the context stream; returns the
// total (synchronises).  Deterministic: three passes (block sums, scan of the block
// sums, add offsets).
long long exclusive_scan(Ctx& ctx, int* data, int count);

}  // namespace hamlss
