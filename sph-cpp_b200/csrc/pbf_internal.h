// Internal declarations shared by the host (.cpp) and CUDA (.cu) halves of
// libpbf_b200.  Not part of the public C ABI.
#pragma once
#include <cstdint>

namespace pbf {
// ceil(extent/s) + 2 grid cells per axis, in float (neighbors.h:69-71).
int64_t grid_dim(float extent, float s);
// floor((c + s)/s) in float (neighbors.h:109-114), as a signed integer.
int64_t axis_bin(float c, float s);
}  // namespace pbf
