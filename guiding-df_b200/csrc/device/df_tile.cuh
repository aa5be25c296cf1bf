// df_tile.cuh -- building blocks of the tile-based DF kernels: one warpgroup
// owns a 128-row tile, thread t of the warpgroup owns row t.
//
//   * operand tiles live in shared memory in the no-swizzle K-major
//     canonical layout (8x8 core matrices, 128 B each);
//   * layer accumulators live in tensor memory (lane = row);
//   * the softmax / CDF / sampling epilogue streams a row's logits out of
//     tensor memory in 32-column chunks instead of holding them in registers.
//
// Files including this header are compiled with -fmad=false (see df_math.cuh).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "df_math.cuh"
#include "sm100.cuh"

namespace gdf {
namespace tile {

using namespace sm100;

// Byte offset of the 16-byte chunk `kc` (8 fp16 columns) of row `row` in a
// canonical tile of K columns.
__device__ __forceinline__ uint32_t chunk_off(uint32_t row, uint32_t kc, uint32_t K) {
  return (((row >> 3) * (K >> 3) + kc) << 7) + ((row & 7u) << 4);
}

// Byte offset of column `col` of row `row`.
__device__ __forceinline__ uint32_t elem_off(uint32_t row, uint32_t col, uint32_t K) {
  return chunk_off(row, col >> 3, K) + ((col & 7u) << 1);
}

// Two values rounded to the MLP operand format (fp16, or bf16 for the
// bf16 inference form), packed low-first.
__device__ __forceinline__ uint32_t pack2(float a, float b, bool bf16) {
  if (bf16) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ void store_h2(uint8_t* t, uint32_t row, uint32_t col, uint32_t K, float a,
                                         float b, bool bf16 = false) {
  *reinterpret_cast<uint32_t*>(t + elem_off(row, col, K)) = pack2(a, b, bf16);
}

// Stores n (even) consecutive values starting at column col (even).
__device__ __forceinline__ void store_run(uint8_t* t, uint32_t row, uint32_t col, uint32_t K,
                                          const float* v, int n, bool bf16 = false) {
  for (int i = 0; i < n; i += 2) store_h2(t, row, col + i, K, v[i], v[i + 1], bf16);
}

// ------------------------------------------------------------------ grid
// One level of kernel_grid (tcnn encodings/grid.h:220-349) for F = 2 or 4,
// fp32 accumulation. interp: 0 linear, 1 smoothstep, 2 nearest.
// The level tables are read from the kernel's __grid_constant__ parameters
// with a warp-uniform dynamic level index (indexed constant-bank loads).
// Corner entries and per-axis weights of one level at one position
// (tcnn kernel_grid, encodings/grid.h:220-330; grid_index :165-188 with the
// CoherentPrime hash of :112-129 for hashed levels).
struct LevelCorners {
  uint32_t e[8];   // entry of corner c (bit 0: x, bit 1: y, bit 2: z), within the level
  float w[3][2];   // per-axis weight of the lower (0) and upper (1) corner
};

__device__ __forceinline__ LevelCorners level_corners(const GridLevels& s, int l, int interp, float px,
                                                      float py, float pz) {
  const float scale = s.scale[l];
  const float pin[3] = {px, py, pz};
  float fr[3];
  uint32_t pg[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float p = fmaf(pin[d], scale, 0.5f);
    const float t = floorf(p);
    pg[d] = static_cast<uint32_t>(static_cast<int>(t));
    p -= t;
    if (interp == 1) p = p * p * (3.0f - 2.0f * p);
    fr[d] = p;
  }
  const uint32_t hsize = s.hsize[l], r = s.res[l];
  const uint32_t mode = s.hashed[l] ? 0u : s.ndims[l];
  const uint32_t hmask = s.pow2[l] ? hsize - 1u : 0u;
  // Per-axis index terms for the lower (0) and upper (1) corner.
  uint32_t tx[2], ty[2], tz[2];
  if (mode == 0) {
    tx[0] = pg[0]; tx[1] = pg[0] + 1u;
    ty[0] = pg[1] * 2654435761u; ty[1] = ty[0] + 2654435761u;
    tz[0] = pg[2] * 805459861u; tz[1] = tz[0] + 805459861u;
  } else {
    tx[0] = pg[0]; tx[1] = pg[0] + 1u;
    ty[0] = mode > 1 ? pg[1] * r : 0u; ty[1] = mode > 1 ? ty[0] + r : 0u;
    tz[0] = mode > 2 ? pg[2] * r * r : 0u; tz[1] = mode > 2 ? tz[0] + r * r : 0u;
  }
  LevelCorners c;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t x = tx[k & 1], y = ty[(k >> 1) & 1], z = tz[(k >> 2) & 1];
    const uint32_t idx = mode == 0 ? (x ^ y ^ z) : (x + y + z);
    c.e[k] = hmask ? (idx & hmask) : (idx % hsize);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c.w[d][0] = 1.f - fr[d];
    c.w[d][1] = fr[d];
  }
  return c;
}

// weight of corner k = (x-term * y-term) * z-term, as kernel_grid's dim loop
__device__ __forceinline__ float corner_weight(const LevelCorners& c, int k) {
  return (1.f * c.w[0][k & 1]) * c.w[1][(k >> 1) & 1] * c.w[2][(k >> 2) & 1];
}

template <int F>
__device__ __forceinline__ void grid_level(const GridLevels& s, int l, int interp,
                                           const __half* __restrict__ table, float px, float py,
                                           float pz, float* out) {
  const LevelCorners c = level_corners(s, l, interp, px, py, pz);
  const __half* tab = table + static_cast<size_t>(s.offset[l]) * F;
  float acc[F];
#pragma unroll
  for (int f = 0; f < F; ++f) acc[f] = 0.f;
  if (interp == 2) {
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] = __half2float(tab[static_cast<size_t>(c.e[0]) * F + f]);
  } else if constexpr (F == 2) {
    uint32_t raw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) raw[k] = __ldg(reinterpret_cast<const unsigned int*>(tab) + c.e[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float w = corner_weight(c, k);
      const float2 v = __half22float2(*reinterpret_cast<const __half2*>(&raw[k]));
      acc[0] += w * v.x;
      acc[1] += w * v.y;
    }
  } else {
    uint2 raw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) raw[k] = __ldg(reinterpret_cast<const uint2*>(tab) + c.e[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float w = corner_weight(c, k);
      const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw[k].x));
      const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw[k].y));
      acc[0] += w * a.x;
      acc[1] += w * a.y;
      acc[2] += w * b.x;
      acc[3] += w * b.y;
    }
  }
#pragma unroll
  for (int f = 0; f < F; ++f) out[f] = acc[f];
}

// One level of both DF grids at the same position, from the interleaved
// table il: entry e holds [theta features (F) | phi features (F)], so each
// corner is one 2F-half gather for both networks. Same arithmetic as
// grid_level (shared corners and weights, accumulation in corner order).
template <int F>
__device__ __forceinline__ void grid_level_pair(const GridLevels& s, int l, int interp,
                                                const __half* __restrict__ il, float px, float py,
                                                float pz, float* out_t, float* out_p) {
  const LevelCorners c = level_corners(s, l, interp, px, py, pz);
  const __half* tab = il + static_cast<size_t>(s.offset[l]) * (2 * F);
  float at[F], ap[F];
#pragma unroll
  for (int f = 0; f < F; ++f) { at[f] = 0.f; ap[f] = 0.f; }
  if (interp == 2) {
#pragma unroll
    for (int f = 0; f < F; ++f) {
      at[f] = __half2float(tab[static_cast<size_t>(c.e[0]) * 2 * F + f]);
      ap[f] = __half2float(tab[static_cast<size_t>(c.e[0]) * 2 * F + F + f]);
    }
  } else if constexpr (F == 2) {
    uint2 raw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) raw[k] = __ldg(reinterpret_cast<const uint2*>(tab) + c.e[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float w = corner_weight(c, k);
      const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw[k].x));
      const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw[k].y));
      at[0] += w * a.x;
      at[1] += w * a.y;
      ap[0] += w * b.x;
      ap[1] += w * b.y;
    }
  } else {
    uint4 raw[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) raw[k] = __ldg(reinterpret_cast<const uint4*>(tab) + c.e[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float w = corner_weight(c, k);
      const uint32_t h[4] = {raw[k].x, raw[k].y, raw[k].z, raw[k].w};
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&h[j]));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&h[2 + j]));
        at[2 * j] += w * a.x;
        at[2 * j + 1] += w * a.y;
        ap[2 * j] += w * b.x;
        ap[2 * j + 1] += w * b.y;
      }
    }
  }
#pragma unroll
  for (int f = 0; f < F; ++f) { out_t[f] = at[f]; out_p[f] = ap[f]; }
}

// All levels of one grid, written as fp16 into columns [0, L*F) of a tile
// with K columns.
template <int F>
__device__ __forceinline__ void grid_to_tile(const GridLevels& s, int n_levels, int interp,
                                             const __half* __restrict__ table, const float* q,
                                             uint8_t* tile, uint32_t row, uint32_t K) {
#pragma unroll 2
  for (int l = 0; l < n_levels; ++l) {
    float f[F];
    grid_level<F>(s, l, interp, table, q[0], q[1], q[2], f);
#pragma unroll
    for (int j = 0; j < F; j += 2) store_h2(tile, row, l * F + j, K, f[j], f[j + 1]);
  }
}

// Both networks' grids in one fully unrolled level loop: per level the
// theta and phi gathers (16 independent loads) are in flight together.
// Features go out as 16-byte chunks: tile A (theta input, K = KA columns)
// and tile P (phi grid features, K = L*F columns).
template <int L, int F>
__device__ __forceinline__ void grids_to_tiles(const GridLevels& gt, const __half* __restrict__ tab_t,
                                               const GridLevels& gp, const __half* __restrict__ tab_p,
                                               const float* q, const float* qp, uint8_t* tile_a,
                                               uint32_t ka, uint8_t* tile_p, uint32_t row) {
  constexpr int kLevelsPerChunk = 8 / F;  // 8 fp16 features per 16-byte chunk
  __half2 ct[4], cp[4];
#pragma unroll
  for (int l = 0; l < L; ++l) {
    float ft[F], fp[F];
    grid_level<F>(gt, l, gt.interp, tab_t, q[0], q[1], q[2], ft);
    grid_level<F>(gp, l, gp.interp, tab_p, qp[0], qp[1], qp[2], fp);
#pragma unroll
    for (int j = 0; j < F; j += 2) {
      const int slot = ((l % kLevelsPerChunk) * F + j) / 2;
      ct[slot] = __floats2half2_rn(ft[j], ft[j + 1]);
      cp[slot] = __floats2half2_rn(fp[j], fp[j + 1]);
    }
    if (l % kLevelsPerChunk == kLevelsPerChunk - 1) {
      const uint32_t kc = static_cast<uint32_t>(l / kLevelsPerChunk);
      *reinterpret_cast<uint4*>(tile_a + chunk_off(row, kc, ka)) = *reinterpret_cast<uint4*>(ct);
      *reinterpret_cast<uint4*>(tile_p + chunk_off(row, kc, L * F)) = *reinterpret_cast<uint4*>(cp);
    }
  }
}

// SH(16) of q[3..5] and OneBlob(4 bins) of q[6..8] at columns [col, col+28).
__device__ __forceinline__ void sh_ob_to_tile(const float* q, uint8_t* tile, uint32_t row,
                                              uint32_t col, uint32_t K, bool bf16 = false) {
  float v[28];
  sh4_encode(q[3], q[4], q[5], v);
  oneblob_encode<4>(q[6], v + 16);
  oneblob_encode<4>(q[7], v + 20);
  oneblob_encode<4>(q[8], v + 24);
  store_run(tile, row, col, K, v, 28, bf16);
}

__device__ __forceinline__ void ones_to_tile(uint8_t* tile, uint32_t row, uint32_t col0,
                                             uint32_t col1, uint32_t K, bool bf16 = false) {
  for (uint32_t c = col0; c < col1; c += 2) store_h2(tile, row, c, K, 1.f, 1.f, bf16);
}

// The theta network's input after its grid features, at columns [col, K):
// SH(16) of q[3..5], OneBlob(4 bins) of q[6..8], then K - col - 28 alignment
// columns -- as the reference computes them. In the theta composite OneBlob
// is the last encoding, so it takes the alignment padding, and tiny-cuda-nn
// v1.6 writes that padding (encodings/oneblob.h:223-226, SoA layout) starting
// n_dims_to_encode = 3 rows into OneBlob's own outputs instead of after its
// 12: OneBlob outputs [3, 3 + pad) read 1, and the pad columns keep what the
// fresh buffer holds, 0. (The phi composite ends with TriangleWave, whose
// kernel pads correctly: ones_to_tile.)
__device__ __forceinline__ void theta_rest_from_values(const float (&v)[28], uint8_t* tile, uint32_t row,
                                                       uint32_t col, uint32_t K, bool bf16 = false) {
  constexpr uint32_t kObFirst = 16, kObDims = 3;
  const uint32_t pad = K - col - 28;
#pragma unroll
  for (uint32_t i = 0; i < 28; i += 2) {
    const bool one0 = i >= kObFirst + kObDims && i < kObFirst + kObDims + pad;
    const bool one1 = i + 1 >= kObFirst + kObDims && i + 1 < kObFirst + kObDims + pad;
    store_h2(tile, row, col + i, K, one0 ? 1.f : v[i], one1 ? 1.f : v[i + 1], bf16);
  }
  for (uint32_t c = col + 28; c < K; c += 2) {
    const uint32_t j = c - col - kObFirst;  // row within OneBlob's padded output
    store_h2(tile, row, c, K, j < kObDims + pad ? 1.f : 0.f, j + 1 < kObDims + pad ? 1.f : 0.f, bf16);
  }
}

// SH(16) of q[3..5] and OneBlob(4 bins) of q[6..8]: the 28 values both
// networks' inputs carry after their grid features.
__device__ __forceinline__ void sh_ob_values(const float* q, float (&v)[28]) {
  sh4_encode(q[3], q[4], q[5], v);
  oneblob_encode<4>(q[6], v + 16);
  oneblob_encode<4>(q[7], v + 20);
  oneblob_encode<4>(q[8], v + 24);
}

__device__ __forceinline__ void theta_rest_to_tile(const float* q, uint8_t* tile, uint32_t row,
                                                   uint32_t col, uint32_t K, bool bf16 = false) {
  float v[28];
  sh_ob_values(q, v);
  theta_rest_from_values(v, tile, row, col, K, bf16);
}

// n (even) values rounded to the operand format and packed in pairs, for a
// later store_packed_run.
template <int N>
__device__ __forceinline__ void pack_run(const float (&v)[N], bool bf16, uint32_t (&w)[N / 2]) {
#pragma unroll
  for (int i = 0; i < N / 2; ++i) w[i] = pack2(v[2 * i], v[2 * i + 1], bf16);
}

template <int W>
__device__ __forceinline__ void store_packed_run(uint8_t* t, uint32_t row, uint32_t col, uint32_t K,
                                                 const uint32_t (&w)[W]) {
#pragma unroll
  for (int i = 0; i < W; ++i) *reinterpret_cast<uint32_t*>(t + elem_off(row, col + 2 * i, K)) = w[i];
}

// ------------------------------------------------------------- warpgroup
struct Wg {
  uint8_t* tile_a;     // activations / first-layer input (generic pointer)
  uint32_t tile_a_s;   // shared-space address
  uint8_t* tile_p;     // side tile (phi grid features)
  uint32_t tile_p_s;
  uint32_t tmem;       // accumulator column base, lane 0
  uint32_t lane_base;  // this warp's TMEM lane offset (address units)
  uint64_t* bar;       // MMA-completion mbarrier
  uint32_t phase;
  uint32_t bar_id;     // named barrier id of the warpgroup
  uint32_t row;
  bool leader;
  uint32_t* err;
  bool bf16 = false;   // MLP operands in bf16 (inference form); fp16 otherwise
};

// One K segment of an MMA's A operand: `ksteps` K=16 steps read from a
// canonical tile at `saddr` with `K` columns.
struct ASeg {
  uint32_t saddr;
  uint32_t K;
  int ksteps;
};

// Makes this warpgroup's shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void publish(Wg& c) {
  fence_proxy_async_smem();
  __syncwarp();
  named_bar_sync(c.bar_id, 128);
}

// D[tmem] = concat(A segments) * W^T. W is the canonical [N x Kw] matrix at
// w_s. Issued by the leader after publish(); completion arrives on c.bar.
__device__ __forceinline__ void issue(Wg& c, const ASeg* segs, int nseg, uint32_t w_s, uint32_t Kw,
                                      uint32_t N) {
  if (!c.leader) return;
  tc_fence_after();
  const uint32_t idesc = idesc_f16(128, N, c.bf16 ? 1u : 0u, 0, 0);  // A and B share one type
  const uint32_t bsbo = Kw * 16u;
  int s = 0;
  for (int g = 0; g < nseg; ++g) {
    for (int j = 0; j < segs[g].ksteps; ++j, ++s) {
      const uint64_t ad = smem_desc(segs[g].saddr + j * 256, 128, segs[g].K * 16u);
      const uint64_t bd = smem_desc(w_s + s * 256, 128, bsbo);
      mma_f16_ss(c.tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
  }
  mma_commit(c.bar);
}

__device__ __forceinline__ void wait_mma(Wg& c) {
  mbar_wait(c.bar, c.phase, c.err, kErrMbarTimeout);
  c.phase ^= 1u;
  __syncwarp();
  tc_fence_after();
}

// ReLU of the 64 accumulator columns -> fp16 -> tile_a (K = 64). SCALED:
// the accumulators are first multiplied by d (a power of two: the FP8
// form's descale of its last e4m3 layer).
template <bool SCALED = false>
__device__ __forceinline__ void relu_to_tile(Wg& c, float d = 1.f) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t r[32];
    tmem_ld32(c.tmem + c.lane_base + h * 32, r);
    tmem_ld_wait();
    if constexpr (SCALED) {
#pragma unroll
      for (int j = 0; j < 32; ++j) r[j] = __float_as_uint(__uint_as_float(r[j]) * d);
    }
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t v[4];
      // ReLU after rounding: max(round(x), 0) = round(max(x, 0)), and
      // __hmax2 maps NaN to 0 like tcnn's relu (x > 0 ? x : 0)
      if (c.bf16) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const __nv_bfloat162 b = __hmax2(__floats2bfloat162_rn(__uint_as_float(r[kc * 8 + 2 * j]),
                                                                 __uint_as_float(r[kc * 8 + 2 * j + 1])),
                                           __float2bfloat162_rn(0.f));
          v[j] = *reinterpret_cast<const uint32_t*>(&b);
        }
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const __half2 b = __hmax2(__floats2half2_rn(__uint_as_float(r[kc * 8 + 2 * j]),
                                                      __uint_as_float(r[kc * 8 + 2 * j + 1])),
                                    __float2half2_rn(0.f));
          v[j] = *reinterpret_cast<const uint32_t*>(&b);
        }
      }
      *reinterpret_cast<uint4*>(c.tile_a + chunk_off(c.row, h * 4 + kc, 64)) =
          make_uint4(v[0], v[1], v[2], v[3]);
    }
  }
  tc_fence_before();
}

// Hidden layers 1..n_hidden-1 and the output layer, starting after the first
// layer's MMA was issued. w_s points at the first hidden matrix. Leaves the
// n_out logits in TMEM.
__device__ __forceinline__ void mlp_tail(Wg& c, uint32_t w_s, int n_hidden, uint32_t n_out) {
  const ASeg a{c.tile_a_s, 64, 4};
  for (int l = 1; l <= n_hidden; ++l) {
    wait_mma(c);
    relu_to_tile(c);
    publish(c);
    const bool last = l == n_hidden;
    issue(c, &a, 1, w_s, 64, last ? n_out : 64u);
    w_s += (last ? n_out : 64u) * 64u * 2u;
  }
  wait_mma(c);
}

// ------------------------------------------------------------ FP8 form
// The 64x64 hidden matrices run as e4m3 x e4m3 MMAs with fp32 accumulation;
// the first matrix (encoded inputs) and the output matrix stay fp16. A
// hidden matrix W is stored as e4m3(W * 2^kw) with one exponent per matrix,
// an activation row h as e4m3(h * 2^kr) with one exponent per row (query),
// both chosen from the absolute maximum, so the accumulator of row r is
// descaled exactly by 2^-(kw + kr).

// Exponent k of the largest power of two with amax * 2^k <= 448 (e4m3's
// largest finite value), clamped to [-100, 100]; 0 for a zero or
// non-finite amax.
__device__ __forceinline__ int e4m3_scale_exp(float amax) {
  const uint32_t b = __float_as_uint(amax);
  const uint32_t ef = (b >> 23) & 0xffu;
  if (amax == 0.f || ef == 0xffu) return 0;
  // amax = m * 2^e with m in [1, 2): m * 2^(e+k) <= 1.75 * 2^8
  const int k = ((b & 0x7fffffu) <= 0x600000u ? 8 : 7) - (static_cast<int>(ef) - 127);
  return k < -100 ? -100 : (k > 100 ? 100 : k);
}

__device__ __forceinline__ float exp2i(int k) { return __uint_as_float(static_cast<uint32_t>(k + 127) << 23); }

// Two values -> e4m3 (round to nearest even, saturating), low byte first.
__device__ __forceinline__ uint32_t pack_e4m3x2(float a, float b) {
  return static_cast<uint32_t>(__nv_cvt_float2_to_fp8x2(make_float2(a, b), __NV_SATFINITE, __NV_E4M3));
}

// ReLU(acc * d) of the 64 accumulator columns -> e4m3 with the row's
// exponent -> tile_a as a 64-byte row (canonical layout of 32 two-byte
// columns). Returns the row's descale 2^-k.
__device__ __forceinline__ float relu_to_tile_f8(Wg& c, float d) {
  uint32_t r0[32], r1[32];
  tmem_ld32(c.tmem + c.lane_base, r0);
  tmem_ld32(c.tmem + c.lane_base + 32, r1);
  tmem_ld_wait();
  float amax = 0.f;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    // fmaxf(NaN, 0) = 0, tcnn relu's NaN behaviour
    const float a = fmaxf(__uint_as_float(r0[j]) * d, 0.f), b = fmaxf(__uint_as_float(r1[j]) * d, 0.f);
    r0[j] = __float_as_uint(a);
    r1[j] = __float_as_uint(b);
    amax = fmaxf(amax, fmaxf(a, b));
  }
  const int k = e4m3_scale_exp(amax);
  const float s = exp2i(k);
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    const uint32_t* r = kc < 2 ? r0 + kc * 16 : r1 + (kc - 2) * 16;
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      v[j] = pack_e4m3x2(__uint_as_float(r[4 * j]) * s, __uint_as_float(r[4 * j + 1]) * s) |
             (pack_e4m3x2(__uint_as_float(r[4 * j + 2]) * s, __uint_as_float(r[4 * j + 3]) * s) << 16);
    *reinterpret_cast<uint4*>(c.tile_a + chunk_off(c.row, kc, 32)) = make_uint4(v[0], v[1], v[2], v[3]);
  }
  tc_fence_before();
  return exp2i(-k);
}

// D[tmem] = A8 * W8^T for a 64-byte-row e4m3 A tile at a_s and the e4m3
// [N x 64] matrix at w_s: two K = 32 steps.
__device__ __forceinline__ void issue_f8(Wg& c, uint32_t a_s, uint32_t w_s, uint32_t N) {
  if (!c.leader) return;
  tc_fence_after();
  const uint32_t idesc = idesc_f16(128, N, 0, 0, 0);  // format fields 0: E4M3 x E4M3
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const uint64_t ad = smem_desc(a_s + j * 256, 128, 32u * 16u);
    const uint64_t bd = smem_desc(w_s + j * 256, 128, 32u * 16u);
    mma_f8_ss(c.tmem, ad, bd, idesc, j > 0 ? 1u : 0u);
  }
  mma_commit(c.bar);
}

// mlp_tail of the FP8 form: matrices 1..n_hidden-1 e4m3 (4096 bytes each
// from w_s), then the fp16 output matrix; descale[l-1] = 2^-kw of matrix l.
__device__ __forceinline__ void mlp_tail_f8(Wg& c, uint32_t w_s, int n_hidden, uint32_t n_out,
                                            const float* descale) {
  const ASeg a{c.tile_a_s, 64, 4};
  float d = 1.f;
  for (int l = 1; l <= n_hidden; ++l) {
    wait_mma(c);
    if (l < n_hidden) {
      const float inv_s = relu_to_tile_f8(c, d);
      publish(c);
      issue_f8(c, c.tile_a_s, w_s, 64);
      w_s += 64u * 64u;
      d = descale[l - 1] * inv_s;
    } else {
      relu_to_tile<true>(c, d);
      publish(c);
      issue(c, &a, 1, w_s, 64, n_out);
    }
  }
  wait_mma(c);
}

// ------------------------------------------------------------ epilogue
// Streams the row's logits out of TMEM in chunks of 32 (or 16) columns.
template <int NB, typename Fn>
__device__ __forceinline__ void for_each_logit(const Wg& c, Fn&& fn) {
  constexpr int CH = NB >= 32 ? 32 : 16;
#pragma unroll 1
  for (int base = 0; base < NB; base += CH) {
    uint32_t r[CH];
    if constexpr (CH == 32) tmem_ld32(c.tmem + c.lane_base + base, r);
    else tmem_ld16(c.tmem + c.lane_base + base, r);
    tmem_ld_wait();
#pragma unroll
    for (int j = 0; j < CH; ++j) fn(base + j, __uint_as_float(r[j]));
  }
}

// softmax2 statistics (train.h:845-862): m = max(0, max z), ls = log(sum exp(z - m)).
struct SoftmaxStats {
  float m, ls;
  __device__ __forceinline__ float pdf(float z, float n) const { return __expf(z - m - ls) * n; }
};

template <int NB>
__device__ __forceinline__ SoftmaxStats softmax_stats(const Wg& c) {
  float m = 0.f;
  for_each_logit<NB>(c, [&](int, float z) { m = fmaxf(m, z); });
  float s = 0.f;
  for_each_logit<NB>(c, [&](int, float z) { s += __expf(z - m); });
  return SoftmaxStats{m, __logf(s)};
}

// Inversion sampling (sample_dir_guided_inputs_F, train.h:416-520) with the
// CDF walk streamed over the logits; identical float sequence to
// df_math.cuh sample_dir.
template <int NB, bool LINEAR>
__device__ __forceinline__ float sample_streamed(const Wg& c, const SoftmaxStats& st, float u, float u2) {
  const float n = static_cast<float>(NB);
  const float inv_n = 1.f / n;
  float cm1 = 0.f, ci = 0.f, prev_c = 0.f, prev_p = 0.f, lo = 0.f, hi = 0.f, p_last = 0.f;
  int seg = NB;
  bool found = false;
  for_each_logit<NB>(c, [&](int i, float z) {
    const float p = st.pdf(z, n);
    if constexpr (LINEAR) {
      const float cc = i == 0 ? p * 0.5f / n : prev_c + (prev_p + p) / static_cast<float>(2 * NB);
      if (!found && u < cc) {
        found = true; seg = i; cm1 = i == 0 ? 0.f : prev_c; ci = cc;
        lo = i == 0 ? p : prev_p; hi = p;
      }
      prev_c = cc;
    } else {
      const float cc = prev_c + p / n;
      if (!found && u < cc) { found = true; seg = i; cm1 = prev_c; ci = cc; }
      prev_c = cc;
    }
    prev_p = p;
    p_last = p;
  });
  if constexpr (LINEAR) {
    if (!found) { cm1 = prev_c; ci = prev_c + p_last * 0.5f / n; lo = hi = p_last; }
    int idx_m1 = seg - 1;
    float v = static_cast<float>(idx_m1) + 0.5f;
    float ecm = 1.f, v_off = 0.f;
    if (idx_m1 < 0) { v_off = 0.5f; ecm = 0.5f; }
    else if (seg > NB - 1) { ecm = 0.5f; }
    const float m = (hi - lo) * n;
    const float B = lo * (1 + v) - hi * v;
    v += v_off;
    const float A = m * 0.5f;
    float d;
    if (fabsf(A) < kEps) {
      const float w = (ci - cm1) > kEps ? (u - cm1) / (ci - cm1) : u2;
      d = (v + w * ecm) * inv_n;
    } else {
      const float C = -(m * 0.5f) * (v * v * inv_n * inv_n) - (B * v * inv_n) + cm1 - u;
      const float delta = B * B - 4 * A * C;
      if (delta < kEps) {
        d = (v + u2 * ecm) * inv_n;
      } else {
        const float sq = sqrtf(delta);
        const float s0 = (-B + sq) / (2 * A);
        const float s1 = (-B - sq) / (2 * A);
        d = A >= 0 ? fmaxf(s0, s1) : fminf(s0, s1);
      }
    }
    return fminf(d, 1.f - kEps);
  } else {
    if (!found) { cm1 = prev_c; ci = prev_c; }
    const float w = (ci - cm1) > kEps ? (u - cm1) / (ci - cm1) : u2;
    return fminf((static_cast<float>(seg) + w) / n, 1.f - kEps);
  }
}

// sample_pdf (train.h:655-681) with the two looked-up bins fetched by one
// streamed pass.
template <int NB, bool LINEAR>
__device__ __forceinline__ float pdf_streamed(const Wg& c, const SoftmaxStats& st, float u) {
  const float n = static_cast<float>(NB);
  float idx = u * n;
  int f, cidx;
  float w = 0.f;
  if constexpr (LINEAR) {
    idx -= 0.5f;
    f = safe_floor<NB>(idx);
    cidx = f + 1;
    w = idx - static_cast<float>(f);
    if (f < 0) { f = NB - 1; w = 1.0f; }
    if (cidx > NB - 1) { cidx = 0; w = 0.0f; }
  } else {
    f = safe_floor<NB>(idx);
    cidx = f;
  }
  float zf = 0.f, zc = 0.f;
  for_each_logit<NB>(c, [&](int i, float z) {
    zf = i == f ? z : zf;
    zc = i == cidx ? z : zc;
  });
  if constexpr (LINEAR) return (1.0f - w) * st.pdf(zf, n) + w * st.pdf(zc, n);
  else return st.pdf(zf, n);
}

// Result of the per-row DF epilogue of one network.
struct RowResult {
  float u;    // sampled (or given) square coordinate
  float pdf;  // interpolated pdf at u
};

// The whole thetaPostInference / phiPostInference row epilogue
// (train.h:896-929) for one network, logits read once from TMEM into
// registers: softmax2 x N, inversion sampling when `guided` (else u is the
// given coordinate), pdf interpolation at u. Out of line so the theta and
// phi networks share one copy of the code.
// COMP (the BF16 / FP8 inference forms): the softmax sum and the CDF use
// Neumaier's compensated summation.
template <int NB, bool LINEAR, bool COMP = false>
__device__ __noinline__ RowResult row_epilogue(uint32_t taddr, bool guided, float u_given, float u_main,
                                               float u_fallback) {
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
  // softmax2 (train.h:845-862): p_i = N exp(z_i - m - log sum_j exp(z_j - m))
  // with m = max(0, max z), evaluated as e_i = 2^(z_i log2 e - m log2 e),
  // p_i = e_i * (N / sum e): one exponential per bin instead of two.
  float m = 0.0f;
#pragma unroll
  for (int i = 0; i < NB; ++i) m = fmaxf(m, v[i]);
  constexpr float kLog2e = 1.4426950408889634074f;
  const float ml = m * kLog2e;
  float s = 0.0f, sc = 0.0f;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    v[i] = ex2_approx(fmaf(v[i], kLog2e, -ml));
    if constexpr (COMP) neumaier_add(s, sc, v[i]);
    else s += v[i];
  }
  const float k = static_cast<float>(NB) / (COMP ? s + sc : s);
#pragma unroll
  for (int i = 0; i < NB; ++i) v[i] *= k;
  const SampleResult sr = sample_and_pdf<NB, LINEAR, COMP>(v, guided, u_given, u_main, u_fallback);
  RowResult r;
  r.u = sr.u;
  r.pdf = sr.pdf;
  return r;
}

// The CDF normalisation check in FP64: recomputes the row's pdfs exactly as
// row_epilogue does (same operations, same order) from the logits still in
// TMEM, sums them in double and max-merges |1 - sum p_i / N| per warp into
// *norm_err as the bits of a non-negative double (NaN sorts above all).
// Called by every lane of the warp, right after row_epilogue.
template <int NB, bool COMP = false>
__device__ __noinline__ void row_norm_check(uint32_t taddr, unsigned long long* norm_err) {
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
  float m = 0.0f;
#pragma unroll
  for (int i = 0; i < NB; ++i) m = fmaxf(m, v[i]);
  constexpr float kLog2e = 1.4426950408889634074f;
  const float ml = m * kLog2e;
  float s = 0.0f, sc = 0.0f;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    v[i] = ex2_approx(fmaf(v[i], kLog2e, -ml));
    if constexpr (COMP) neumaier_add(s, sc, v[i]);
    else s += v[i];
  }
  const float k = static_cast<float>(NB) / (COMP ? s + sc : s);
  double sum = 0.0;
#pragma unroll
  for (int i = 0; i < NB; ++i) sum += static_cast<double>(v[i] * k);
  unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(fabs(1.0 - sum / NB)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
    b = x > b ? x : b;
  }
  if ((threadIdx.x & 31u) == 0) atomicMax(norm_err, b);
}

// Training flavour of the epilogue (forward of LearnedDistribution::trainStep,
// learnedDistribution.cpp:252-262): the logits are the network's fp16
// outputs, softmax2 is stored as fp16 and multiplied by N in fp16
// (softmaxMultFactor), and the pdf at the record's direction interpolates
// those fp16 values (combine_AR_pdf_and_dl_doutput, train.h:946-948).
template <int NB, bool LINEAR>
__device__ __noinline__ float row_pdf_train(uint32_t taddr, float u) {
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
  return sample_pdf<NB, LINEAR>(v, u);
}

}  // namespace tile
}  // namespace gdf
