// df_train.cu -- backward pass and optimizer of the DF training step.
//
// df_train_bwd_kernel: one network per launch. Each CTA (one warpgroup, 128
// records per tile, persistent over tiles):
//   1. recomputes the forward of its network with every activation kept in
//      shared memory (tcgen05, fp32 accumulators in TMEM, fp16 activations);
//      the grid features are the training forward's, bulk-copied per tile
//      (the next tile's while this one finishes), not gathered again;
//   2. builds the fp16 pdf table and dL/dlogits of combine_AR_pdf_and_dl_doutput
//      (src/render/guided/train.h:932-965, AR.h:51-104) from the per-record
//      pdf of the other network and the loss prefix computed by the forward
//      kernel;
//   3. back-propagates (tcnn/src/fully_fused_mlp.cu:755-850): per layer one
//      tcgen05 MMA for the data gradient (M=128) and one for the weight
//      gradient (M=64, operands read MN-major from the same tiles), the
//      weight gradients accumulating across all of the CTA's tiles in TMEM;
//   4. writes dL/dgrid-features (level-major) for grid_scatter_kernel, which
//      scatters them times the corner weights into the fp32 grid gradient
//      with vector atomics at full occupancy (grid.h:395-520; tcnn uses fp16
//      atomics).
// At the end each CTA writes its weight-gradient partial sums; the optimizer
// kernel reduces them in fixed CTA order (deterministic).
//
// adam_ema_kernel: Adam (tcnn optimizers/adam.h:48-117) + EMA (ema.h:63-130)
// over one network, fused with the gradient reduction, the re-zeroing of the
// grid gradient and the re-layout of the MLP weights for the tensor cores.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../device/df_math.cuh"
#include "../device/df_tile.cuh"
#include "../device/sm100.cuh"
#include "../device/train_tile.cuh"
#include "df_kernels.h"
#include "train_kernels.h"
#include "launch_util.h"

namespace gdf {
namespace {

using namespace sm100;
using namespace train_tile;

__host__ __device__ constexpr int pad16t(int v) { return (v + 15) / 16 * 16; }

// dL/dlogits of one row into the D tile (fp16, 64 columns; first NB used).
// compute_gradients_specialized_linear_interpolation / _nearest (AR.h:51-104).
template <int NB, bool LINEAR, bool BF16>
__device__ __noinline__ void dlogits_to_tile(uint32_t taddr, float u, float pdf_other, float prefix,
                                            bool ok, uint8_t* d_tile, uint32_t row) {
  float v[NB];
  if constexpr (NB == 16) {
    uint32_t r[16];
    tmem_ld16(taddr, r);
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
  } else {
    uint32_t r[NB];
#pragma unroll
    for (int c = 0; c < NB / 32; ++c) tmem_ld32(taddr + c * 32, *reinterpret_cast<uint32_t(*)[32]>(r + c * 32));
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < NB; ++i) v[i] = __uint_as_float(r[i]);
  }
  tc_fence_before();
  softmax_table_fp16<NB>(v);
  const float inv_res = 1.0f / static_cast<float>(NB);
  const float multiplier = prefix * pdf_other * static_cast<float>(NB);
  int f, cidx;
  float w;
  if constexpr (LINEAR) {
    const float idx = u * static_cast<float>(NB) - 0.5f;
    f = safe_floor<NB>(idx);
    cidx = f + 1;
    w = idx - static_cast<float>(f);
    if (f < 0) { f = NB - 1; w = 1.0f; }
    if (cidx > NB - 1) { cidx = 0; w = 0.0f; }
  } else {
    f = min(static_cast<int>(u * static_cast<float>(NB)), NB - 1);
    cidx = f;
    w = 0.f;
  }
  const float p0 = select_bin<NB>(v, f) * inv_res;
  const float p1 = select_bin<NB>(v, cidx) * inv_res;
#pragma unroll
  for (int kc = 0; kc < NB / 8; ++kc) {
    uint32_t out[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float g[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = kc * 8 + 2 * j + e;
        const float pi = v[i] * inv_res;
        const float j0 = f == i ? p0 * (1.0f - p0) : -p0 * pi;
        float jj;
        if constexpr (LINEAR) {
          const float j1 = cidx == i ? p1 * (1.0f - p1) : -p1 * pi;
          jj = (1.0f - w) * j0 + w * j1;
        } else {
          jj = j0;
        }
        g[e] = ok ? multiplier * jj : 0.f;
      }
      out[j] = tile::pack2(g[0], g[1], BF16);
    }
    *reinterpret_cast<uint4*>(d_tile + tile::chunk_off(row, kc, 64)) = make_uint4(out[0], out[1], out[2], out[3]);
  }
}

// Grid backward of one level of one row: dL/dfeatures (F fp32 values)
// times each corner's weight scattered into the fp32 gradient table
// (kernel_grid_backward, grid.h:395-520).
template <int F>
__device__ __forceinline__ void grid_backward_level(const GridLevels& g, int l, const float* pos,
                                                    const float* dl, float* __restrict__ grad) {
  const float scale = g.scale[l];
  float fr[3];
  uint32_t pg[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float pp = fmaf(pos[d], scale, 0.5f);
    const float t = floorf(pp);
    pg[d] = static_cast<uint32_t>(static_cast<int>(t));
    pp -= t;
    if (g.interp == 1) pp = pp * pp * (3.0f - 2.0f * pp);
    fr[d] = pp;
  }
  float* gl = grad + static_cast<size_t>(g.offset[l]) * F;
  if (g.interp == 2) {
    const uint32_t e = grid_entry(g, l, pg[0], pg[1], pg[2]);
#pragma unroll
    for (int f = 0; f < F; ++f) atomicAdd(gl + static_cast<size_t>(e) * F + f, dl[f]);
    return;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    float w = 1.f;
    w *= (c & 1) ? fr[0] : 1.f - fr[0];
    w *= (c & 2) ? fr[1] : 1.f - fr[1];
    w *= (c & 4) ? fr[2] : 1.f - fr[2];
    const uint32_t e = grid_entry(g, l, pg[0] + (c & 1), pg[1] + ((c >> 1) & 1), pg[2] + ((c >> 2) & 1));
    if constexpr (F == 2) {
      atomicAdd(reinterpret_cast<float2*>(gl) + e, make_float2(w * dl[0], w * dl[1]));
    } else {
      atomicAdd(reinterpret_cast<float4*>(gl) + e, make_float4(w * dl[0], w * dl[1], w * dl[2], w * dl[3]));
    }
  }
}

// The grid backward of a batch at full occupancy: one thread per (level,
// record), level-major so a warp reads 32 records' dL/dfeatures of one
// level in one 256-byte line. Records the forward rejected (prefix 0, as
// the backward's `ok`) are skipped.
template <int L, int F>
__global__ void __launch_bounds__(256) grid_scatter_kernel(const __grid_constant__ GridScatterParams p) {
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= p.n * L) return;
  const int l = static_cast<int>(gid / p.n);
  const int64_t row = gid - static_cast<int64_t>(l) * p.n;
  if (p.n_dev && row >= *p.n_dev) return;  // beyond this batch's records
  if (__ldg(p.fwd + row * 4 + 2) == 0.f) return;
  float pos[3], dl[F];
#pragma unroll
  for (int d = 0; d < 3; ++d) pos[d] = __ldg(p.in + row * p.in_stride + d);
  const float* src = p.dx + (static_cast<int64_t>(l) * p.dx_rows + row) * F;
  if constexpr (F == 2) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(src));
    dl[0] = v.x;
    dl[1] = v.y;
  } else {
    const float4 v = __ldg(reinterpret_cast<const float4*>(src));
    dl[0] = v.x; dl[1] = v.y; dl[2] = v.z; dl[3] = v.w;
  }
  grid_backward_level<F>(p.gl, l, pos, dl, p.grid_grad);
}

// BF16: the bf16 training form (weights, grid features, encodings,
// activations and gradients in bf16; fp32 accumulation).
template <int L, int F, int NB, bool LINEAR, bool PHI, bool BF16>
__global__ void __launch_bounds__(128, 1) df_train_bwd_kernel(const __grid_constant__ DfBwdParams p) {
  constexpr int LF = L * F;
  constexpr int K0 = PHI ? pad16t(LF + 40) : pad16t(LF + 28);
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x;
  const uint32_t warp = tid >> 5;
  const int H = p.hidden;

  // shared memory: weights | XF (grid features) | XR (rest of the input) |
  // H_1..H_H tiles | D tile | barriers
  constexpr int KR0 = K0 - LF;
  const uint32_t off_xf = (p.blob_bytes + 127u) & ~127u;
  constexpr uint32_t kXF = 128u * LF * 2u, kXR = 128u * KR0 * 2u, kT = 128u * 64u * 2u;
  const uint32_t off_x = off_xf + kXF;
  const uint32_t off_h = off_x + kXR;
  const uint32_t off_d = off_h + static_cast<uint32_t>(H) * kT;
  const uint32_t off_bar = off_d + kT;
  // [0] weights, [1] MMA completion, [2] feature tile
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bar);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bar + 32);
  const int64_t n_rows = p.n_dev ? min(*p.n_dev, p.n) : p.n;
  const int64_t n_tiles = (n_rows + 127) / 128;
  auto fetch_features = [&](int64_t t) {
    mbar_arrive_expect_tx(&bars[2], kXF);
    bulk_g2s(smem + off_xf, p.feat + t * (128 * LF), kXF, &bars[2]);
  };

  if (warp == 0) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], p.blob_bytes);
    for (uint32_t o = 0; o < p.blob_bytes; o += 32768u)
      bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(p.blob) + o, min(32768u, p.blob_bytes - o), &bars[0]);
    if (blockIdx.x < n_tiles) fetch_features(blockIdx.x);
  }
  uint32_t fphase = 0;
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
  uint8_t* const x_tile = smem + off_x;  // XR: columns LF..K0 of the input
  uint8_t* const d_tile = smem + off_d;
  const uint32_t xf_s = smem_addr(smem + off_xf);
  const uint32_t x_s = smem_addr(x_tile), d_s = smem_addr(d_tile), h_s0 = smem_addr(smem + off_h);
  auto h_tile = [&](int l) { return smem + off_h + static_cast<uint32_t>(l - 1) * kT; };  // H_l, l >= 1
  auto h_addr = [&](int l) { return h_s0 + static_cast<uint32_t>(l - 1) * kT; };
  const uint32_t w0 = smem_addr(smem);
  auto w_addr = [&](int l) {  // W_l, l in [0, H]; W_H is the output layer
    return l == 0 ? w0 : w0 + 64u * K0 * 2u + static_cast<uint32_t>(l - 1) * 64u * 64u * 2u;
  };
  // TMEM columns: work [0,64) | dX [64,96) | G_0 [96, 96+K0) | G_l at 192+64(l-1) | G_H^T after
  const uint32_t t_work = tmem, t_dx = tmem + 64;
  auto t_g = [&](int l) { return tmem + (l == 0 ? 96u : 192u + 64u * static_cast<uint32_t>(l - 1)); };
  const uint32_t lane = c.lane_base;

  constexpr uint32_t kFmt = BF16 ? 1u : 0u;  // A and B share one type
  constexpr uint32_t kIdFwd64 = idesc_f16(128, 64, kFmt, 0, 0);
  constexpr uint32_t kIdFwdNB = idesc_f16(128, NB, kFmt, 0, 0);
  constexpr uint32_t kIdDgrad = idesc_f16(128, 64, kFmt, 0, 1);    // B = W^T read MN-major
  constexpr uint32_t kIdDx = idesc_f16(128, LF, kFmt, 0, 1);
  constexpr uint32_t kIdWg64 = idesc_f16(64, 64, kFmt, 1, 1);      // A, B MN-major
  constexpr uint32_t kIdWgF = idesc_f16(64, LF, kFmt, 1, 1);
  constexpr uint32_t kIdWgR = idesc_f16(64, KR0, kFmt, 1, 1);
  constexpr uint32_t kIdWgOut = idesc_f16(64, NB, kFmt, 1, 1);

  bool first = true;
  for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int64_t row = t * 128 + c.row;
    const bool valid = row < n_rows;
    float q[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) q[i] = 0.5f;
    const int ninp = PHI ? 10 : 9;
    for (int i = 0; i < ninp; ++i) q[i] = valid ? __ldg(p.in + row * p.in_stride + i) : 0.5f;
    const float4 fw = valid ? *reinterpret_cast<const float4*>(p.fwd + row * 4) : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool ok = valid && fw.z != 0.f;
    float u_own = valid ? __ldg(p.target + row * 9 + (PHI ? 1 : 0)) : 0.5f;
    if (!ok) {
#pragma unroll
      for (int i = 0; i < 10; ++i) q[i] = 0.5f;
      u_own = 0.5f;
    }

    // ---- forward: X = [XF | XR] | H_1 .. H_H | logits
    if constexpr (PHI) {
      tile::sh_ob_to_tile(q, x_tile, c.row, 0, KR0, BF16);
      float tw[12];
      triangle_wave_encode<12>(q[9], tw);
      tile::store_run(x_tile, c.row, 28, KR0, tw, 12, BF16);
      tile::ones_to_tile(x_tile, c.row, 40, KR0, KR0, BF16);
    } else {
      tile::theta_rest_to_tile(q, x_tile, c.row, 0, KR0, BF16);
    }
    mbar_wait(&bars[2], fphase, p.err, kErrMbarTimeout);
    fphase ^= 1u;
    for (int l = 0; l <= H; ++l) {
      tile::publish(c);
      if (c.leader) {
        tc_fence_after();
        if (l == 0) {
          mma_steps(t_work, xf_s, 128, LF * 16u, 256, w_addr(0), 128, K0 * 16u, 256, kIdFwd64, LF / 16, false);
          mma_steps(t_work, x_s, 128, KR0 * 16u, 256, w_addr(0) + (LF / 16) * 256u, 128, K0 * 16u, 256,
                    kIdFwd64, KR0 / 16, true);
        } else {
          mma_steps(t_work, h_addr(l), 128, 64u * 16u, 256, w_addr(l), 128, 64u * 16u, 256,
                    l == H ? kIdFwdNB : kIdFwd64, 4, false);
        }
        mma_commit(c.bar);
      }
      tile::wait_mma(c);
      if (l < H) relu_to<BF16>(c, t_work + lane, h_tile(l + 1));
    }
    // ---- dL/dlogits -> D tile
    dlogits_to_tile<NB, LINEAR, BF16>(t_work + lane, u_own, fabsf(PHI ? fw.x : fw.y), fw.z, ok, d_tile, c.row);

    // ---- backward: output layer, hidden layers, first layer
    for (int l = H; l >= 0; --l) {
      tile::publish(c);
      if (c.leader) {
        tc_fence_after();
        const bool acc = !first;
        if (l == H) {
          // G_H^T (i x o) += H_H^T D: A = H_H, B = D, both MN-major, K = 128 rows
          mma_steps(t_g(H), h_addr(H), 64u * 16u, 128, 2u * 64u * 16u, d_s, 64u * 16u, 128,
                    2u * 64u * 16u, kIdWgOut, 8, acc);
          // work = D W_H: A = D K-major (K = NB), B = W_H MN-major
          mma_steps(t_work, d_s, 128, 64u * 16u, 256, w_addr(H), 64u * 16u, 128, 2u * 64u * 16u,
                    kIdDgrad, NB / 16, false);
        } else if (l > 0) {
          // G_l (o x i) += D^T H_l
          mma_steps(t_g(l), d_s, 64u * 16u, 128, 2u * 64u * 16u, h_addr(l), 64u * 16u, 128,
                    2u * 64u * 16u, kIdWg64, 8, acc);
          mma_steps(t_work, d_s, 128, 64u * 16u, 256, w_addr(l), 64u * 16u, 128, 2u * 64u * 16u,
                    kIdDgrad, 4, false);
        } else {
          // G_0 (o x K0) += D^T X, as its XF and XR column blocks ; dX = D W_0[:, :LF]
          mma_steps(t_g(0), d_s, 64u * 16u, 128, 2u * 64u * 16u, xf_s, LF * 16u, 128, 2u * LF * 16u,
                    kIdWgF, 8, acc);
          mma_steps(t_g(0) + LF, d_s, 64u * 16u, 128, 2u * 64u * 16u, x_s, KR0 * 16u, 128, 2u * KR0 * 16u,
                    kIdWgR, 8, acc);
          mma_steps(t_dx, d_s, 128, 64u * 16u, 256, w_addr(0), K0 * 16u, 128, 2u * K0 * 16u, kIdDx, 4,
                    false);
        }
        mma_commit(c.bar);
      }
      tile::wait_mma(c);
      if (l > 0) dgrad_relu_to_tile<BF16>(c, t_work + lane, h_tile(l), d_tile);
    }
    // every MMA reading XF has completed: the next tile's features
    if (c.leader && t + gridDim.x < n_tiles) fetch_features(t + gridDim.x);
    // ---- dL/dfeatures, level-major, for grid_scatter_kernel
    {
      float dx[LF];
      if constexpr (LF == 16) {
        uint32_t r[16];
        tmem_ld16(t_dx + lane, r);
        tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) dx[i] = __uint_as_float(r[i]);
      } else {
        uint32_t r[32];
        tmem_ld32(t_dx + lane, r);
        tmem_ld_wait();
#pragma unroll
        for (int i = 0; i < 32; ++i) dx[i] = __uint_as_float(r[i]);
      }
      tc_fence_before();
      if (valid) {
#pragma unroll
        for (int l = 0; l < L; ++l) {
          float* dst = p.dx + (static_cast<int64_t>(l) * p.dx_rows + row) * F;
          if constexpr (F == 2) *reinterpret_cast<float2*>(dst) = make_float2(dx[l * F], dx[l * F + 1]);
          else *reinterpret_cast<float4*>(dst) = make_float4(dx[l * F], dx[l * F + 1], dx[l * F + 2], dx[l * F + 3]);
        }
      }
    }
    first = false;
  }

  // ---- weight-gradient partials of this CTA (zeros if it had no tile)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  float* part = p.wgrad_partial + static_cast<size_t>(blockIdx.x) * p.n_mlp;
  // M=64 accumulators: warp q holds rows 16q + t in its lanes t < 16
  const uint32_t mrow = warp * 16u + (tid & 31u);
  const bool mvalid = (tid & 31u) < 16u;
  for (int l = 0; l <= H; ++l) {
    const int ncols = l == 0 ? K0 : (l == H ? NB : 64);
    const size_t base = l == 0 ? 0 : static_cast<size_t>(64) * K0 + static_cast<size_t>(l - 1) * 64 * 64;
    for (int c0 = 0; c0 < ncols; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(t_g(l) + lane + c0, r);
      tmem_ld_wait();
      if (mvalid) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float v = first ? 0.f : __uint_as_float(r[j]);
          if (l == H) part[base + static_cast<size_t>(c0 + j) * 64 + mrow] = v;  // G_H stored transposed
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

template <int L, int F, int NB, bool LIN, bool PHI, bool BF16>
cudaError_t launch_bwd_f(const DfBwdParams& p, int ctas, cudaStream_t st) {
  constexpr int LF = L * F;
  constexpr int K0 = PHI ? pad16t(LF + 40) : pad16t(LF + 28);
  if (p.feat == nullptr) return cudaErrorInvalidValue;
  const size_t smem = ((p.blob_bytes + 127u) & ~127u) + 128u * K0 * 2u +
                      static_cast<size_t>(p.hidden + 1) * 128u * 64u * 2u + 64u;
  auto k = df_train_bwd_kernel<L, F, NB, LIN, PHI, BF16>;
  cudaError_t e = allow_dynamic_smem(k);
  if (e != cudaSuccess) return e;
  k<<<ctas, 128, smem, st>>>(p);
  return cudaGetLastError();
}

template <int L, int F, int NB, bool LIN, bool PHI>
cudaError_t launch_bwd_t(const DfBwdParams& p, int ctas, cudaStream_t st) {
  if (p.bf16) return launch_bwd_f<L, F, NB, LIN, PHI, true>(p, ctas, st);
  return launch_bwd_f<L, F, NB, LIN, PHI, false>(p, ctas, st);
}

// ----------------------------------------------------------------- Adam
// One parameter of AdamOptimizer::step (tcnn optimizers/adam.h:48-117)
// followed by EmaOptimizer's update (ema.h:102-130). The step size for a
// parameter whose own step counter is k, lr sqrt(1 - beta2^k) / (1 - beta1^k),
// comes from a table filled by adam_lr_table_kernel with the same float
// expression; past the table's end the value is lr exactly.
__device__ __forceinline__ void adam_param(const AdamParams& p, const float2 debias, bool matrix, float graw, float& wf,
                                           float& m1, float& m2, uint32_t& step, __half& w16h,
                                           __half& emah, double& sq) {
  float g = graw / p.loss_scale;
  sq += static_cast<double>(g) * g;
  float w16;
  if (matrix || g != 0.0f) {  // non-matrix parameters with a zero gradient are skipped
    if (matrix) g += p.l2_reg * wf;
    m1 = p.beta1 * m1 + (1 - p.beta1) * g;
    m2 = p.beta2 * m2 + (1 - p.beta2) * (g * g);
    const uint32_t cs = ++step;
    const float lr = p.lr_table[cs < static_cast<uint32_t>(p.lr_table_n) ? cs : p.lr_table_n - 1];
    const float eff = fminf(fmaxf(lr / (sqrtf(m2) + p.eps), 0.0f), 3.402823466e38f);
    wf = wf - eff * m1;
    w16h = __float2half_rn(wf);
    w16 = __half2float(w16h);
  } else {
    w16 = __half2float(w16h);
  }
  emah = __float2half_rn((__half2float(emah) * p.ema_decay * debias.x + w16 * (1 - p.ema_decay)) *
                         debias.y);
}

__global__ void adam_lr_table_kernel(float lr, float beta1, float beta2, float* table, int32_t n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float cs = static_cast<float>(k);
  table[k] = lr * sqrtf(1 - powf(beta2, cs)) / (1 - powf(beta1, cs));
}

constexpr int kAdamTile = 1024;                     // grid parameters per staged tile
constexpr uint32_t kAdamStage = 24u * kAdamTile;    // grad, master, m, v, step (4 B) + w16, ema (2 B)
constexpr size_t kAdamSmem = 2u * kAdamStage + 16u;

// Four EMA halves of grid parameters j..j+3 into the interleaved inference
// table: entry e = [theta F | phi F].
__device__ __forceinline__ void write_il(const AdamParams& p, int64_t j, uint2 e4) {
  if (p.il_features == 2) {
    const int64_t e = j >> 1;
    *reinterpret_cast<uint32_t*>(p.grid_il + e * 4 + p.il_net * 2) = e4.x;
    *reinterpret_cast<uint32_t*>(p.grid_il + (e + 1) * 4 + p.il_net * 2) = e4.y;
  } else {
    const int64_t e = j >> 2;
    *reinterpret_cast<uint2*>(p.grid_il + e * 8 + p.il_net * 4) = e4;
  }
}

__global__ void __launch_bounds__(256) adam_ema_kernel(const __grid_constant__ AdamParams p) {
  if (p.n_dev && *p.n_dev <= 0) return;  // empty batch: no optimizer step
  // AdamOptimizer::step increments its counter before use (adam.h:150-152);
  // EmaOptimizer::step debiases with it (ema.h:102-110). Every block reads
  // the counter here; the last block to finish stores the new value.
  __shared__ float2 debias_s;
  __shared__ uint32_t opt_step_s;
  if (threadIdx.x == 0) {
    const uint32_t opt_step = p.opt->step + 1;
    const double d = static_cast<double>(p.ema_decay);
    debias_s = make_float2(1.0f - static_cast<float>(pow(d, static_cast<double>(opt_step - 1))),
                           1.0f / (1.0f - static_cast<float>(pow(d, static_cast<double>(opt_step)))));
    opt_step_s = opt_step;
  }
  __syncthreads();
  const float2 debias = debias_s;
  double local_sq = 0.0;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t nth = static_cast<int64_t>(gridDim.x) * blockDim.x;
  // MLP matrices: gradient = the per-CTA partials reduced in CTA order
  for (int64_t i = tid; i < p.n_mlp; i += nth) {
    float graw = 0.f;
#pragma unroll 8
    for (int cta = 0; cta < p.n_partials; ++cta) graw += p.partials[static_cast<size_t>(cta) * p.n_mlp + i];
    float wf = p.master[i], m1 = p.m[i], m2 = p.v[i];
    uint32_t step = p.step[i];
    __half w16h = p.w16[i], emah = p.ema16[i];
    adam_param(p, debias, true, graw, wf, m1, m2, step, w16h, emah, local_sq);
    p.master[i] = wf;
    p.m[i] = m1;
    p.v[i] = m2;
    p.step[i] = step;
    p.w16[i] = w16h;
    p.ema16[i] = emah;
    // re-layout for the tensor cores (canonical K-major per matrix)
    int l = 0;
    while (l + 1 < p.n_layers && i >= p.layer_off[l + 1]) ++l;
    const uint32_t k = static_cast<uint32_t>(i - p.layer_off[l]);
    const uint32_t cols = static_cast<uint32_t>(p.layer_cols[l]);
    const uint32_t off = static_cast<uint32_t>(p.layer_off[l]) + canon_offset(k / cols, k % cols, cols);
    if (p.blob_w16_bf16) {
      const __nv_bfloat16 b = __float2bfloat16_rn(__half2float(w16h));
      p.blob_w16[off] = *reinterpret_cast<const __half*>(&b);
    } else {
      p.blob_w16[off] = w16h;
    }
    if (p.blob_ema_bf16) {
      const __nv_bfloat16 b = __float2bfloat16_rn(__half2float(emah));
      p.blob_ema[off] = *reinterpret_cast<const __half*>(&b);
    } else {
      p.blob_ema[off] = emah;
    }
  }
  // grid tables, staged: tiles of kAdamTile parameters move global ->
  // shared by bulk copies (two stages: the next tile loads while this one
  // is updated), 4 parameters per thread, and back by bulk stores; the
  // gradient is re-zeroed by the threads. Needs n_mlp % 8 == 0 (16-byte
  // aligned grid parts); the rest goes through the register path below.
  extern __shared__ __align__(128) uint8_t stage_mem[];
  uint64_t* sbar = reinterpret_cast<uint64_t*>(stage_mem + 2 * kAdamStage);
  const int64_t ng = p.n - p.n_mlp;
  const int64_t n_tiles = (p.n_mlp % 8 == 0) ? ng / kAdamTile : 0;
  if (threadIdx.x == 0) {
    mbar_init(&sbar[0], 1);
    mbar_init(&sbar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t inflight = 0u;  // thread 0: bit k = a load of stage k not yet waited for
  auto issue_load = [&](int64_t tile, int st) {
    uint8_t* b = stage_mem + st * kAdamStage;
    const int64_t j = tile * kAdamTile, i = p.n_mlp + j;
    mbar_arrive_expect_tx(&sbar[st], kAdamStage);
    bulk_g2s(b, p.grid_grad + j, 4 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 4 * kAdamTile, p.master + i, 4 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 8 * kAdamTile, p.m + i, 4 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 12 * kAdamTile, p.v + i, 4 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 16 * kAdamTile, p.step + i, 4 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 20 * kAdamTile, p.w16 + i, 2 * kAdamTile, &sbar[st]);
    bulk_g2s(b + 22 * kAdamTile, p.ema16 + i, 2 * kAdamTile, &sbar[st]);
    inflight |= 1u << st;
  };
  uint32_t phase = 0u;  // bit k: parity of stage k's barrier
  int st = 0;
  if (threadIdx.x == 0 && blockIdx.x < n_tiles) issue_load(blockIdx.x, 0);
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, st ^= 1) {
    const int64_t next = tile + gridDim.x;
    if (threadIdx.x == 0 && next < n_tiles) {
      bulk_wait_read();  // the other stage's stores have read it
      issue_load(next, st ^ 1);
    }
    const bool ok = mbar_wait(&sbar[st], (phase >> st) & 1u, p.err, kErrMbarTimeout);
    phase ^= 1u << st;
    if (threadIdx.x == 0 && ok) inflight &= ~(1u << st);
    if (__syncthreads_or(!ok)) break;
    uint8_t* b = stage_mem + st * kAdamStage;
    const int t = threadIdx.x;
    const int64_t j = tile * kAdamTile + 4 * t;
    const float4 g4 = reinterpret_cast<const float4*>(b)[t];
    float4 w4 = reinterpret_cast<const float4*>(b + 4 * kAdamTile)[t];
    float4 m4 = reinterpret_cast<const float4*>(b + 8 * kAdamTile)[t];
    float4 v4 = reinterpret_cast<const float4*>(b + 12 * kAdamTile)[t];
    uint4 s4 = reinterpret_cast<const uint4*>(b + 16 * kAdamTile)[t];
    uint2 h4 = reinterpret_cast<const uint2*>(b + 20 * kAdamTile)[t];
    uint2 e4 = reinterpret_cast<const uint2*>(b + 22 * kAdamTile)[t];
    __half* hh = reinterpret_cast<__half*>(&h4);
    __half* ee = reinterpret_cast<__half*>(&e4);
    const float gg[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) adam_param(p, debias, false, gg[k], (&w4.x)[k], (&m4.x)[k], (&v4.x)[k], (&s4.x)[k], hh[k], ee[k], local_sq);
    reinterpret_cast<float4*>(b + 4 * kAdamTile)[t] = w4;
    reinterpret_cast<float4*>(b + 8 * kAdamTile)[t] = m4;
    reinterpret_cast<float4*>(b + 12 * kAdamTile)[t] = v4;
    reinterpret_cast<uint4*>(b + 16 * kAdamTile)[t] = s4;
    reinterpret_cast<uint2*>(b + 20 * kAdamTile)[t] = h4;
    reinterpret_cast<uint2*>(b + 22 * kAdamTile)[t] = e4;
    *reinterpret_cast<float4*>(p.grid_grad + j) = make_float4(0.f, 0.f, 0.f, 0.f);
    if (p.grid_il != nullptr) write_il(p, j, e4);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t i = p.n_mlp + tile * kAdamTile;
      bulk_s2g(p.master + i, b + 4 * kAdamTile, 4 * kAdamTile);
      bulk_s2g(p.m + i, b + 8 * kAdamTile, 4 * kAdamTile);
      bulk_s2g(p.v + i, b + 12 * kAdamTile, 4 * kAdamTile);
      bulk_s2g(p.step + i, b + 16 * kAdamTile, 4 * kAdamTile);
      bulk_s2g(p.w16 + i, b + 20 * kAdamTile, 2 * kAdamTile);
      bulk_s2g(p.ema16 + i, b + 22 * kAdamTile, 2 * kAdamTile);
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) {
    // loads abandoned after a timed-out wait land before the block exits
    for (int k = 0; k < 2; ++k)
      if ((inflight >> k) & 1u) mbar_wait(&sbar[k], (phase >> k) & 1u, p.err, kErrMbarTimeout);
    bulk_wait();
  }
  // the rest of the grid part: 4 parameters per thread and step
  const int64_t g0 = n_tiles * kAdamTile;
  const int64_t ng4 = ng >> 2;
  for (int64_t q = (g0 >> 2) + tid; q < ng4; q += nth) {
    const int64_t j = q * 4, i = p.n_mlp + j;
    const float4 g4 = *reinterpret_cast<const float4*>(p.grid_grad + j);
    *reinterpret_cast<float4*>(p.grid_grad + j) = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 w4 = *reinterpret_cast<const float4*>(p.master + i);
    float4 m4 = *reinterpret_cast<const float4*>(p.m + i);
    float4 v4 = *reinterpret_cast<const float4*>(p.v + i);
    uint4 s4 = *reinterpret_cast<const uint4*>(p.step + i);
    uint2 h4 = *reinterpret_cast<const uint2*>(p.w16 + i);
    uint2 e4 = *reinterpret_cast<const uint2*>(p.ema16 + i);
    __half* hh = reinterpret_cast<__half*>(&h4);
    __half* ee = reinterpret_cast<__half*>(&e4);
    const float gg[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) adam_param(p, debias, false, gg[k], (&w4.x)[k], (&m4.x)[k], (&v4.x)[k], (&s4.x)[k], hh[k], ee[k], local_sq);
    *reinterpret_cast<float4*>(p.master + i) = w4;
    *reinterpret_cast<float4*>(p.m + i) = m4;
    *reinterpret_cast<float4*>(p.v + i) = v4;
    *reinterpret_cast<uint4*>(p.step + i) = s4;
    *reinterpret_cast<uint2*>(p.w16 + i) = h4;
    *reinterpret_cast<uint2*>(p.ema16 + i) = e4;
    if (p.grid_il != nullptr) write_il(p, j, e4);
  }
  for (int64_t j = ng4 * 4 + tid; j < ng; j += nth) {  // remainder (none for tcnn grid sizes)
    const int64_t i = p.n_mlp + j;
    const float graw = p.grid_grad[j];
    p.grid_grad[j] = 0.f;
    float wf = p.master[i], m1 = p.m[i], m2 = p.v[i];
    uint32_t step = p.step[i];
    __half w16h = p.w16[i], emah = p.ema16[i];
    adam_param(p, debias, false, graw, wf, m1, m2, step, w16h, emah, local_sq);
    p.master[i] = wf;
    p.m[i] = m1;
    p.v[i] = m2;
    p.step[i] = step;
    p.w16[i] = w16h;
    p.ema16[i] = emah;
    if (p.grid_il != nullptr) {
      const int64_t F = p.il_features;
      p.grid_il[(j / F) * 2 * F + p.il_net * F + j % F] = emah;
    }
  }
  // per-block sum of squared gradients (FP64), reduced by the host-side kernel
  __shared__ double red[256];
  red[threadIdx.x] = local_sq;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    p.sq_partial[blockIdx.x] = red[0];
    // this block read the step counter at its start; the last block done
    // stores the advanced counter and resets the count for the next launch
    __threadfence();
    if (atomicAdd(&p.opt->blocks_done, 1u) == gridDim.x - 1) {
      p.opt->step = opt_step_s;
      p.opt->blocks_done = 0u;
    }
  }
}

// Deterministic FP64 reductions: loss = sum(likelihood) (column 3 of the
// forward output), grad_norm^2 = sum of the optimizer's block partials.
__global__ void train_stats_kernel(const float* __restrict__ fwd, int64_t n, const double* __restrict__ sq,
                                   int n_sq, double* out) {
  __shared__ double red[1024];
  double a = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) a += fwd[i * 4 + 3];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
  __syncthreads();
  double b = 0.0;
  for (int i = threadIdx.x; i < n_sq; i += blockDim.x) b += sq[i];
  red[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[1] = red[0];
}

// The same two FP64 sums over many blocks: each block sums the likelihood
// column over one contiguous range of records (fixed order) ...
__global__ void __launch_bounds__(512) loss_partials_kernel(const float* __restrict__ fwd, int64_t n,
                                                            const int64_t* n_dev, double* __restrict__ part) {
  __shared__ double red[512];
  if (n_dev) n = min(*n_dev, n);
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = min(n, b + per);
  double a = 0.0;
  for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) a += fwd[i * 4 + 3];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ... and one block adds the block sums and the optimizer's partials.
__global__ void __launch_bounds__(256) stats_final_kernel(const double* __restrict__ part, int n_part,
                                                          const double* __restrict__ sq, int n_sq,
                                                          double* out, int64_t n, const int64_t* n_dev,
                                                          double* loss_acc) {
  __shared__ double red[256];
  for (int k = 0; k < 2; ++k) {
    const double* v = k == 0 ? part : sq;
    const int m = k == 0 ? n_part : n_sq;
    double a = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) a += v[i];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = red[0];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss_acc) {
    const int64_t rows = n_dev ? min(*n_dev, n) : n;
    if (rows > 0) *loss_acc += out[0] / static_cast<double>(rows);
  }
}

}  // namespace

cudaError_t launch_df_train_bwd(const DfShape& s, bool phi, const DfBwdParams& p, int ctas,
                                cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
#define GDF_BWD(L, F, NBT, NBP)                                                                 \
  if (s.levels == L && s.features == F && s.bins_theta == NBT && s.bins_phi == NBP) {           \
    if (phi) return s.linear ? launch_bwd_t<L, F, NBP, true, true>(p, ctas, st)                 \
                             : launch_bwd_t<L, F, NBP, false, true>(p, ctas, st);               \
    return s.linear ? launch_bwd_t<L, F, NBT, true, false>(p, ctas, st)                         \
                    : launch_bwd_t<L, F, NBT, false, false>(p, ctas, st);                       \
  }
  GDF_BWD(8, 2, 32, 32)
  GDF_BWD(16, 2, 64, 64)
  GDF_BWD(16, 2, 32, 32)
  GDF_BWD(8, 4, 16, 32)
#undef GDF_BWD
  return cudaErrorNotSupported;
}

cudaError_t launch_grid_scatter(int levels, int features, const GridScatterParams& p, cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>((p.n * levels + 255) / 256);
  if (levels == 8 && features == 2) grid_scatter_kernel<8, 2><<<blocks, 256, 0, st>>>(p);
  else if (levels == 16 && features == 2) grid_scatter_kernel<16, 2><<<blocks, 256, 0, st>>>(p);
  else if (levels == 8 && features == 4) grid_scatter_kernel<8, 4><<<blocks, 256, 0, st>>>(p);
  else return cudaErrorNotSupported;
  return cudaGetLastError();
}

size_t df_train_bwd_smem_bytes(int levels, int features, bool phi, uint32_t blob_bytes, int hidden) {
  const int lf = levels * features;
  const int k0 = phi ? pad16t(lf + 40) : pad16t(lf + 28);
  return ((blob_bytes + 127u) & ~127u) + 128u * k0 * 2u + static_cast<size_t>(hidden + 1) * 128u * 64u * 2u + 64u;
}

cudaError_t launch_adam_lr_table(float lr, float beta1, float beta2, float* table, int32_t n,
                                 cudaStream_t st) {
  adam_lr_table_kernel<<<(n + 255) / 256, 256, 0, st>>>(lr, beta1, beta2, table, n);
  return cudaGetLastError();
}

cudaError_t launch_adam_ema(const AdamParams& p, cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  cudaError_t e = allow_dynamic_smem(adam_ema_kernel);
  if (e != cudaSuccess) return e;
  adam_ema_kernel<<<p.n_blocks, 256, kAdamSmem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_train_stats(const float* fwd, int64_t n, const double* sq, int n_sq, double* out,
                               cudaStream_t st) {
  train_stats_kernel<<<1, 1024, 0, st>>>(fwd, n, sq, n_sq, out);
  return cudaGetLastError();
}

cudaError_t launch_train_stats_mb(const float* fwd, int64_t n, const int64_t* n_dev, const double* sq, int n_sq,
                                  double* part, double* out, double* loss_acc, cudaStream_t st) {
  loss_partials_kernel<<<kStatBlocks, 512, 0, st>>>(fwd, n, n_dev, part);
  stats_final_kernel<<<1, 256, 0, st>>>(part, kStatBlocks, sq, n_sq, out, n, n_dev, loss_acc);
  return cudaGetLastError();
}

}  // namespace gdf
