// nrc.cu -- Neural Radiance Cache query and training backward on sm_100a.
//
// The NRC is an RGB MLP (common/configs/nn/base_hashgrid_nrc_df.json): input
// [pos 3 | dir 3 | n_theta', n_phi', r' | diffuse 3 | specular 3]
// (GuidedInputNRC, src/render/guided/guideditem.h:89-93) encoded as
// Frequency(pos, 12) | OneBlob(dims 3..8, 4 bins) | Identity(dims 9..14),
// padded with ones to 112 columns; 64-wide ReLU layers; 3 outputs padded to 16.
//
// nrc_query_kernel: NRC::inferenceStep (src/render/guided/nrc.cpp:172-181) —
//   persistent tile kernel like the DF inference kernel, EMA weights.
// nrc_train_bwd_kernel: one NRC::trainStep iteration (nrc.cpp:132-167) —
//   forward with tile-resident activations, RelativeL2Luminance loss and
//   gradient (tcnn losses/relative_l2_luminance.h:40-86) on the fp16
//   outputs, tcgen05 data- and weight-gradient MMAs, per-CTA weight-gradient
//   partials (the optimizer kernel of df_train.cu reduces them).
#include <cuda_fp16.h>

#include "../device/df_math.cuh"
#include "../device/df_tile.cuh"
#include "../device/sm100.cuh"
#include "../device/train_tile.cuh"
#include "nrc_kernels.h"
#include "launch_util.h"

namespace gdf {
namespace {

using namespace sm100;
using namespace train_tile;

constexpr int kNrcK0 = 112;  // 72 frequency + 24 OneBlob + 6 identity + 10 ones
constexpr int kNrcOut = 16;
constexpr int kNrcWgs = 4;

// GuidedInputNRC row -> fp16 network input in columns [0, 112) of `tile`.
__device__ __forceinline__ void nrc_encode_to_tile(const float* x, uint8_t* tile, uint32_t row) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float f[24];
    frequency_encode<12>(x[d], f);
    tile::store_run(tile, row, d * 24, kNrcK0, f, 24);
  }
  float ob[24];
#pragma unroll
  for (int d = 0; d < 6; ++d) oneblob_encode<4>(x[3 + d], ob + 4 * d);
  tile::store_run(tile, row, 72, kNrcK0, ob, 24);
  tile::store_run(tile, row, 96, kNrcK0, x + 9, 6);
  tile::ones_to_tile(tile, row, 102, kNrcK0, kNrcK0);
}

__global__ void __launch_bounds__(128 * kNrcWgs, 1) nrc_query_kernel(const __grid_constant__ NrcParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, wg = tid >> 7, warp = tid >> 5;
  const uint32_t off_tiles = (p.blob_bytes + 127u) & ~127u;
  constexpr uint32_t kTile = 128u * kNrcK0 * 2u;
  const uint32_t off_bars = off_tiles + kNrcWgs * kTile;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bars);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bars + 8 * (kNrcWgs + 1));
  if (warp == 0) {
    tmem_alloc(tmem_slot, 64 * kNrcWgs);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i <= kNrcWgs; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], p.blob_bytes);
    for (uint32_t o = 0; o < p.blob_bytes; o += 32768u)
      bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(p.blob) + o, min(32768u, p.blob_bytes - o), &bars[0]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  mbar_wait(&bars[0], 0, p.err, kErrWeightLoad);

  tile::Wg c;
  c.tile_a = smem + off_tiles + wg * kTile;
  c.tile_a_s = smem_addr(c.tile_a);
  c.tile_p = nullptr;
  c.tile_p_s = 0;
  c.tmem = tmem_base + wg * 64u;
  c.lane_base = ((warp & 3u) * 32u) << 16;
  c.bar = &bars[1 + wg];
  c.phase = 0;
  c.bar_id = 1 + wg;
  c.row = tid & 127u;
  c.leader = c.row == 0;
  c.err = p.err;
  c.bf16 = false;  // the NRC runs in fp16 (tile::issue and mlp_tail read it)
  const uint32_t w0 = smem_addr(smem);

  const int64_t n_tiles = (p.n + 127) / 128;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kNrcWgs + wg; t < n_tiles;
       t += static_cast<int64_t>(gridDim.x) * kNrcWgs) {
    const int64_t row = t * 128 + c.row;
    const bool valid = row < p.n;
    float x[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) x[i] = valid ? __ldg(p.in + row * 15 + i) : 0.5f;
    nrc_encode_to_tile(x, c.tile_a, c.row);
    tile::publish(c);
    {
      const tile::ASeg a{c.tile_a_s, kNrcK0, kNrcK0 / 16};
      tile::issue(c, &a, 1, w0, kNrcK0, 64);
    }
    tile::mlp_tail(c, w0 + 64u * kNrcK0 * 2u, p.hidden, kNrcOut);
    uint32_t r[16];
    tmem_ld16(c.tmem + c.lane_base, r);
    tmem_ld_wait();
    tc_fence_before();
    if (valid) {
      p.out[row * 3 + 0] = __uint_as_float(r[0]);
      p.out[row * 3 + 1] = __uint_as_float(r[1]);
      p.out[row * 3 + 2] = __uint_as_float(r[2]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, 64 * kNrcWgs);
}

// RelativeL2Luminance (relative_l2_luminance.h:40-86) of one record on the
// fp16 network outputs: gradient rows (fp16) into the D tile, loss value of
// the record returned.
__device__ __forceinline__ float nrc_loss_to_tile(uint32_t taddr, const float* target, bool ok, float scale,
                                                  float n_total, uint8_t* d_tile, uint32_t row) {
  uint32_t r[16];
  tmem_ld16(taddr, r);
  tmem_ld_wait();
  tc_fence_before();
  float y[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) y[k] = __half2float(__float2half_rn(__uint_as_float(r[k])));
  const float lum = 0.299f * y[0] + 0.587f * y[1] + 0.114f * y[2];
  const float denom = lum * lum + 0.01f;
  float g[16];
  float loss = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) g[k] = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float diff = y[k] - target[k];
    loss += diff * diff / denom / 1.0f / n_total;
    g[k] = ok ? scale * (2 * diff / denom / 1.0f) / n_total : 0.f;
  }
#pragma unroll
  for (int kc = 0; kc < 2; ++kc) {
    __half2 h[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) h[j] = __floats2half2_rn(g[kc * 8 + 2 * j], g[kc * 8 + 2 * j + 1]);
    *reinterpret_cast<uint4*>(d_tile + tile::chunk_off(row, kc, 64)) = *reinterpret_cast<uint4*>(h);
  }
  return ok ? loss : 0.f;
}

__global__ void __launch_bounds__(128, 1) nrc_train_bwd_kernel(const __grid_constant__ NrcTrainParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const int H = p.hidden;
  const uint32_t off_x = (p.blob_bytes + 127u) & ~127u;
  constexpr uint32_t kX = 128u * kNrcK0 * 2u, kT = 128u * 64u * 2u;
  const uint32_t off_h = off_x + kX;
  const uint32_t off_d = off_h + static_cast<uint32_t>(H) * kT;
  const uint32_t off_bar = off_d + kT;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bar);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bar + 16);
  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], p.blob_bytes);
    for (uint32_t o = 0; o < p.blob_bytes; o += 32768u)
      bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(p.blob) + o, min(32768u, p.blob_bytes - o), &bars[0]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  mbar_wait(&bars[0], 0, p.err, kErrWeightLoad);

  tile::Wg c;
  c.tile_a = smem + off_x;
  c.tile_a_s = smem_addr(c.tile_a);
  c.tile_p = nullptr;
  c.tile_p_s = 0;
  c.tmem = tmem;
  c.lane_base = (warp * 32u) << 16;
  c.bar = &bars[1];
  c.phase = 0;
  c.bar_id = 1;
  c.row = tid;
  c.leader = tid == 0;
  c.err = p.err;
  uint8_t* const x_tile = smem + off_x;
  uint8_t* const d_tile = smem + off_d;
  const uint32_t x_s = smem_addr(x_tile), d_s = smem_addr(d_tile), h_s0 = smem_addr(smem + off_h);
  auto h_tile = [&](int l) { return smem + off_h + static_cast<uint32_t>(l - 1) * kT; };
  auto h_addr = [&](int l) { return h_s0 + static_cast<uint32_t>(l - 1) * kT; };
  const uint32_t w0 = smem_addr(smem);
  auto w_addr = [&](int l) {
    return l == 0 ? w0 : w0 + 64u * kNrcK0 * 2u + static_cast<uint32_t>(l - 1) * 64u * 64u * 2u;
  };
  // TMEM: work [0,64) | G_0 [64,176) | G_l at 192+64(l-1) | G_H^T at 192+64(H-1)
  auto t_g = [&](int l) { return tmem + (l == 0 ? 64u : 192u + 64u * static_cast<uint32_t>(l - 1)); };
  const uint32_t lane = c.lane_base;
  constexpr uint32_t kIdFwd64 = idesc_f16(128, 64, 0, 0, 0);
  constexpr uint32_t kIdFwdOut = idesc_f16(128, kNrcOut, 0, 0, 0);
  constexpr uint32_t kIdDgrad = idesc_f16(128, 64, 0, 0, 1);
  constexpr uint32_t kIdWg64 = idesc_f16(64, 64, 0, 1, 1);
  constexpr uint32_t kIdWgK0 = idesc_f16(64, kNrcK0, 0, 1, 1);
  constexpr uint32_t kIdWgOut = idesc_f16(64, kNrcOut, 0, 1, 1);

  const int64_t n_tiles = (p.n + 127) / 128;
  bool first = true;
  for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int64_t row = t * 128 + c.row;
    const bool valid = row < p.n;
    float x[15], y[3];
    bool ok = valid;
#pragma unroll
    for (int i = 0; i < 15; ++i) {
      x[i] = valid ? __ldg(p.in + row * 15 + i) : 0.5f;
      ok &= !isnan(x[i]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      y[k] = valid ? __ldg(p.target + row * 3 + k) : 0.f;
      ok &= !isnan(y[k]);
    }
    if (!ok) {
#pragma unroll
      for (int i = 0; i < 15; ++i) x[i] = 0.5f;
#pragma unroll
      for (int k = 0; k < 3; ++k) y[k] = 0.f;
    }
    if (valid && !ok) atomicAdd(p.n_dropped, 1ull);
    nrc_encode_to_tile(x, x_tile, c.row);
    for (int l = 0; l <= H; ++l) {
      tile::publish(c);
      if (c.leader) {
        tc_fence_after();
        const uint32_t a_s = l == 0 ? x_s : h_addr(l);
        const uint32_t ka = l == 0 ? kNrcK0 : 64u;
        mma_steps(tmem, a_s, 128, ka * 16u, 256, w_addr(l), 128, ka * 16u, 256, l == H ? kIdFwdOut : kIdFwd64,
                  static_cast<int>(ka / 16), false);
        mma_commit(c.bar);
      }
      tile::wait_mma(c);
      if (l < H) relu_to(c, tmem + lane, h_tile(l + 1));
    }
    const float loss = nrc_loss_to_tile(tmem + lane, y, ok, p.loss_scale, p.n_total, d_tile, c.row);
    if (valid) p.loss_out[row * 4 + 3] = loss;
    for (int l = H; l >= 0; --l) {
      tile::publish(c);
      if (c.leader) {
        tc_fence_after();
        const bool acc = !first;
        if (l == H) {
          mma_steps(t_g(H), h_addr(H), 64u * 16u, 128, 2u * 64u * 16u, d_s, 64u * 16u, 128, 2u * 64u * 16u,
                    kIdWgOut, 8, acc);
          mma_steps(tmem, d_s, 128, 64u * 16u, 256, w_addr(H), 64u * 16u, 128, 2u * 64u * 16u, kIdDgrad,
                    kNrcOut / 16, false);
        } else if (l > 0) {
          mma_steps(t_g(l), d_s, 64u * 16u, 128, 2u * 64u * 16u, h_addr(l), 64u * 16u, 128, 2u * 64u * 16u,
                    kIdWg64, 8, acc);
          mma_steps(tmem, d_s, 128, 64u * 16u, 256, w_addr(l), 64u * 16u, 128, 2u * 64u * 16u, kIdDgrad, 4,
                    false);
        } else {
          mma_steps(t_g(0), d_s, 64u * 16u, 128, 2u * 64u * 16u, x_s, kNrcK0 * 16u, 128, 2u * kNrcK0 * 16u,
                    kIdWgK0, 8, acc);
        }
        mma_commit(c.bar);
      }
      tile::wait_mma(c);
      if (l > 0) dgrad_relu_to_tile(c, tmem + lane, h_tile(l), d_tile);
    }
    first = false;
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  float* part = p.wgrad_partial + static_cast<size_t>(blockIdx.x) * p.n_mlp;
  const uint32_t mrow = warp * 16u + (tid & 31u);
  const bool mvalid = (tid & 31u) < 16u;
  for (int l = 0; l <= H; ++l) {
    const int ncols = l == 0 ? kNrcK0 : (l == H ? kNrcOut : 64);
    const size_t base = l == 0 ? 0 : static_cast<size_t>(64) * kNrcK0 + static_cast<size_t>(l - 1) * 64 * 64;
    for (int c0 = 0; c0 < ncols; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(t_g(l) + lane + c0, r);
      tmem_ld_wait();
      if (mvalid) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float v = first ? 0.f : __uint_as_float(r[j]);
          if (l == H) part[base + static_cast<size_t>(c0 + j) * 64 + mrow] = v;
          else part[base + static_cast<size_t>(mrow) * ncols + c0 + j] = v;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

}  // namespace

cudaError_t launch_nrc_query(const NrcParams& p, int num_sms, cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  const size_t smem = ((p.blob_bytes + 127u) & ~127u) + kNrcWgs * 128u * kNrcK0 * 2u + 8u * (kNrcWgs + 1) + 16u;
  cudaError_t e = allow_dynamic_smem(nrc_query_kernel);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (p.n + 127) / 128;
  int64_t ctas = (tiles + kNrcWgs - 1) / kNrcWgs;
  if (ctas > num_sms) ctas = num_sms;
  nrc_query_kernel<<<static_cast<unsigned>(ctas), 128 * kNrcWgs, smem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_nrc_train_bwd(const NrcTrainParams& p, int ctas, cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  const size_t smem = ((p.blob_bytes + 127u) & ~127u) + 128u * kNrcK0 * 2u +
                      static_cast<size_t>(p.hidden + 1) * 128u * 64u * 2u + 64u;
  cudaError_t e = allow_dynamic_smem(nrc_train_bwd_kernel);
  if (e != cudaSuccess) return e;
  nrc_train_bwd_kernel<<<ctas, 128, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace gdf
