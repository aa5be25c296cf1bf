// grid_features.cu -- multiresolution grid encoding of both DF networks for
// a batch of queries, written in the tensor-core tile layout.
//
// The grid gathers (tcnn kernel_grid, encodings/grid.h:220-330: 8 corner
// reads per level) dominate inference. Inside the fused kernel they ran at
// one 128-thread warpgroup per tile between the MMA and epilogue phases,
// which left L2 mostly idle. Here every thread computes one 16-byte chunk of
// one row's features -- 8/F levels of one network, 8x that many independent
// 4- or 8-byte gathers -- at full occupancy, and stores it where the fused
// kernel's bulk copy expects it: tiles of 128 rows x L*F fp16 columns in the
// canonical no-swizzle K-major layout (8x8 core matrices), tile t at
// feat + t * 128 * L*F. A warp covers 32 consecutive rows of one chunk, so
// each group of 8 rows writes one contiguous 128-byte line.
#include <cuda_fp16.h>

#include "../device/df_tile.cuh"
#include "../device/records.cuh"
#include "../device/sm100.cuh"
#include "df_kernels.h"

namespace gdf {
namespace {

template <int L, int F>
__global__ void __launch_bounds__(256, 4) grid_features_kernel(const __grid_constant__ GridFeatParams p) {
  constexpr int LPC = 8 / F;  // levels per 16-byte chunk
  constexpr int NCH = L / LPC;
  constexpr uint32_t LF = L * F;
  const int64_t rows = p.n_tiles * 128;
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= rows * NCH * 2) return;
  const int64_t row = gid % rows;
  const int64_t rest = gid / rows;
  const int chunk = static_cast<int>(rest % NCH);
  const int net = static_cast<int>(rest / NCH);
  float pos[3] = {0.5f, 0.5f, 0.5f};
  if (row < p.n) {
    if (p.shading_pos != nullptr) {
      float raw[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) raw[k] = __ldg(p.shading_pos + row * 3 + k);
      rec::normalize_spatial(raw, rec::scene_frame(p.aabb), pos);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) pos[k] = __ldg(p.queries + row * 9 + k);
    }
  }
  const GridLevels& gl = net ? p.gl_phi : p.gl_theta;
  const __half* tab = net ? p.grid_phi : p.grid_theta;
  uint32_t packed[4];
#pragma unroll
  for (int j = 0; j < LPC; ++j) {
    float f[F];
    tile::grid_level<F>(gl, chunk * LPC + j, gl.interp, tab, pos[0], pos[1], pos[2], f);
#pragma unroll
    for (int k = 0; k < F; k += 2) {
      const __half2 h = __floats2half2_rn(f[k], f[k + 1]);
      packed[(j * F + k) / 2] = *reinterpret_cast<const uint32_t*>(&h);
    }
  }
  __half* out = (net ? p.feat_phi : p.feat_theta) + (row >> 7) * (128 * LF) +
                sm100::canon_offset(static_cast<uint32_t>(row & 127), static_cast<uint32_t>(chunk * 8), LF);
  *reinterpret_cast<uint4*>(out) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
}

template <int L, int F>
cudaError_t launch_l(const GridFeatParams& p, cudaStream_t st) {
  constexpr int NCH = L * F / 8;
  const int64_t threads = p.n_tiles * 128 * NCH * 2;
  grid_features_kernel<L, F><<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_grid_features(const DfShape& s, const GridFeatParams& p, cudaStream_t st) {
  if (p.n_tiles <= 0) return cudaSuccess;
  if (s.levels == 8 && s.features == 2) return launch_l<8, 2>(p, st);
  if (s.levels == 16 && s.features == 2) return launch_l<16, 2>(p, st);
  if (s.levels == 8 && s.features == 4) return launch_l<8, 4>(p, st);
  return cudaErrorNotSupported;
}

}  // namespace gdf
