// grid_features.cu -- multiresolution grid encoding of both DF networks for
// a batch of queries, written in the tensor-core tile layout.
//
// The grid gathers (tcnn kernel_grid, encodings/grid.h:220-330: 8 corner
// reads per level and network) dominate inference, and with random query
// positions their cost is the number of L1 misses sent to L2 (about 4
// random sectors per level). Both networks use the same grid configuration
// at the same position, so their corner indices coincide: inference reads
// an interleaved copy of the two EMA tables (entry e = [theta F halves |
// phi F halves]) and one 4F-byte gather serves both networks, halving the
// requests. Every thread computes one 16-byte chunk (8/F levels) of one
// row for both networks at full occupancy and stores the two chunks where
// the fused kernel's bulk copies expect them: tiles of 128 rows x L*F fp16
// columns in the canonical no-swizzle K-major layout (8x8 core matrices),
// tile t at feat + t * 128 * L*F. A warp covers 32 consecutive rows of one
// chunk, so each group of 8 rows writes one contiguous 128-byte line.
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
  if (gid >= rows * NCH) return;
  const int64_t row = gid % rows;
  const int chunk = static_cast<int>(gid / rows);
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
  const GridLevels& gl = p.gl;
  uint32_t pt[4], pp[4];
#pragma unroll
  for (int j = 0; j < LPC; ++j) {
    float ft[F], fp[F];
    tile::grid_level_pair<F>(gl, chunk * LPC + j, gl.interp, p.grid_il, pos[0], pos[1], pos[2], ft, fp);
#pragma unroll
    for (int k = 0; k < F; k += 2) {
      pt[(j * F + k) / 2] = tile::pack2(ft[k], ft[k + 1], p.bf16 != 0);
      pp[(j * F + k) / 2] = tile::pack2(fp[k], fp[k + 1], p.bf16 != 0);
    }
  }
  const int64_t off = (row >> 7) * (128 * LF) +
                      sm100::canon_offset(static_cast<uint32_t>(row & 127), static_cast<uint32_t>(chunk * 8), LF);
  *reinterpret_cast<uint4*>(p.feat_theta + off) = make_uint4(pt[0], pt[1], pt[2], pt[3]);
  *reinterpret_cast<uint4*>(p.feat_phi + off) = make_uint4(pp[0], pp[1], pp[2], pp[3]);
}

// Both networks' grid features of a training batch from the fp16 training
// tables (one table per network, each network at its own record's
// position), in the tile layout the training forward and backward read;
// same arithmetic as the training forward's own gathers
// (tile::grids_to_tiles). Rows the forward's validity filter rejects (a NaN
// in any field of the three records, or wi_pdf = 0; train.cu:77-81) and
// padding rows use position 0.5, as the forward does.
template <int L, int F>
__global__ void __launch_bounds__(256, 4) train_features_kernel(const __grid_constant__ TrainFeatParams p) {
  constexpr int LPC = 8 / F;
  constexpr int NCH = L / LPC;
  constexpr uint32_t LF = L * F;
  const int64_t rows = p.n_tiles * 128;
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= rows * NCH) return;
  const int64_t row = gid % rows;
  const int chunk = static_cast<int>(gid / rows);
  const int64_t n = p.n_dev ? min(*p.n_dev, p.n) : p.n;
  if (row >= (n + 127) / 128 * 128) return;  // tiles beyond this batch's records
  float pt[3] = {0.5f, 0.5f, 0.5f}, pp[3] = {0.5f, 0.5f, 0.5f};
  if (row < n) {
    bool ok = true;
    float a[3], b[3];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float x = __ldg(p.in_theta + row * 9 + i), y = __ldg(p.target + row * 9 + i);
      ok &= !isnan(x) && !isnan(y);
      if (i < 3) a[i] = x;
      if (i == 5) ok &= y != 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      const float x = __ldg(p.in_phi + row * 10 + i);
      ok &= !isnan(x);
      if (i < 3) b[i] = x;
    }
    if (ok) {
#pragma unroll
      for (int k = 0; k < 3; ++k) { pt[k] = a[k]; pp[k] = b[k]; }
    }
  }
  uint32_t ot[4], op[4];
#pragma unroll
  for (int j = 0; j < LPC; ++j) {
    float ft[F], fp[F];
    const int l = chunk * LPC + j;
    tile::grid_level<F>(p.gl_theta, l, p.gl_theta.interp, p.grid_theta, pt[0], pt[1], pt[2], ft);
    tile::grid_level<F>(p.gl_phi, l, p.gl_phi.interp, p.grid_phi, pp[0], pp[1], pp[2], fp);
#pragma unroll
    for (int k = 0; k < F; k += 2) {
      ot[(j * F + k) / 2] = tile::pack2(ft[k], ft[k + 1], p.bf16 != 0);
      op[(j * F + k) / 2] = tile::pack2(fp[k], fp[k + 1], p.bf16 != 0);
    }
  }
  const int64_t off = (row >> 7) * (128 * LF) +
                      sm100::canon_offset(static_cast<uint32_t>(row & 127), static_cast<uint32_t>(chunk * 8), LF);
  *reinterpret_cast<uint4*>(p.feat_theta + off) = make_uint4(ot[0], ot[1], ot[2], ot[3]);
  *reinterpret_cast<uint4*>(p.feat_phi + off) = make_uint4(op[0], op[1], op[2], op[3]);
}

// il[e][0..F) = theta[e][..], il[e][F..2F) = phi[e][..]
__global__ void interleave_grids_kernel(const __half* __restrict__ t, const __half* __restrict__ ph,
                                        __half* __restrict__ il, int64_t n_entries, int F) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n_entries * F) return;
  const int64_t e = i / F;
  const int f = static_cast<int>(i % F);
  il[e * 2 * F + f] = t[i];
  il[e * 2 * F + F + f] = ph[i];
}

template <int L, int F>
cudaError_t launch_l(const GridFeatParams& p, cudaStream_t st) {
  constexpr int NCH = L * F / 8;
  const int64_t threads = p.n_tiles * 128 * NCH;
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

cudaError_t launch_train_features(const DfShape& s, const TrainFeatParams& p, cudaStream_t st) {
  if (p.n_tiles <= 0) return cudaSuccess;
  const int nch = s.levels * s.features / 8;
  const unsigned blocks = static_cast<unsigned>((p.n_tiles * 128 * nch + 255) / 256);
  if (s.levels == 8 && s.features == 2) train_features_kernel<8, 2><<<blocks, 256, 0, st>>>(p);
  else if (s.levels == 16 && s.features == 2) train_features_kernel<16, 2><<<blocks, 256, 0, st>>>(p);
  else if (s.levels == 8 && s.features == 4) train_features_kernel<8, 4><<<blocks, 256, 0, st>>>(p);
  else return cudaErrorNotSupported;
  return cudaGetLastError();
}

cudaError_t launch_interleave_grids(const __half* theta, const __half* phi, __half* il,
                                    int64_t n_entries, int features, cudaStream_t st) {
  const int64_t n = n_entries * features;
  if (n == 0) return cudaSuccess;
  interleave_grids_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(theta, phi, il, n_entries,
                                                                                  features);
  return cudaGetLastError();
}

}  // namespace gdf
