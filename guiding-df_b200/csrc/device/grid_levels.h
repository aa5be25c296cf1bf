// grid_levels.h -- plain-data per-level tables of a multiresolution grid
// encoding, shared by host and device code.
#pragma once

#include <cstdint>

namespace gdf {

// Per-level tables of one grid encoding (tcnn encodings/grid.h:967-1012),
// computed on the host once per context.
struct GridLevels {
  float scale[24];
  uint32_t offset[24];   // first entry of the level (entries of F features)
  uint32_t hsize[24];    // entries in the level
  uint32_t res[24];      // vertices per axis
  uint32_t ndims[24];    // axes folded into the dense index (grid_index loop)
  uint32_t hashed[24];   // 1 = CoherentPrime hash replaces the dense index
  uint32_t pow2[24];     // 1 = hsize is a power of two (modulo by mask)
  int32_t n_levels;
  int32_t interp;        // 0 linear, 1 smoothstep, 2 nearest
};

}  // namespace gdf
