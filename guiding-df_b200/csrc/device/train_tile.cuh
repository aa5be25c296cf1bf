// train_tile.cuh -- backward-pass helpers shared by the DF and NRC training
// kernels (one warpgroup per 128-row tile, see df_tile.cuh).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "df_tile.cuh"
#include "sm100.cuh"

namespace gdf {
namespace train_tile {

using namespace sm100;

// MMA with arbitrary majors: D (+)= A * B over `ksteps` K=16 steps. a/b
// descriptors advance by a_step / b_step bytes per step.
__device__ __forceinline__ void mma_steps(uint32_t d, uint32_t a_s, uint32_t a_lbo, uint32_t a_sbo,
                                          uint32_t a_step, uint32_t b_s, uint32_t b_lbo,
                                          uint32_t b_sbo, uint32_t b_step, uint32_t idesc,
                                          int ksteps, bool accumulate) {
  for (int s = 0; s < ksteps; ++s) {
    const uint64_t ad = smem_desc(a_s + s * a_step, a_lbo, a_sbo);
    const uint64_t bd = smem_desc(b_s + s * b_step, b_lbo, b_sbo);
    mma_f16_ss(d, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
  }
}

// Two floats from a packed pair of the operand format (fp16, or bf16).
template <bool BF16>
__device__ __forceinline__ float2 unpack2(uint32_t w) {
  if constexpr (BF16) return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
  else return __half22float2(*reinterpret_cast<const __half2*>(&w));
}

// ReLU'(forward activation) * accumulator -> operand format -> D tile (64
// columns); BF16: the bf16 training form.
template <bool BF16 = false>
__device__ __forceinline__ void dgrad_relu_to_tile(const tile::Wg& c, uint32_t taddr,
                                                   const uint8_t* h_tile, uint8_t* d_tile) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t r[32];
    tmem_ld32(taddr + h * 32, r);
    tmem_ld_wait();
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      const uint4 hv = *reinterpret_cast<const uint4*>(h_tile + tile::chunk_off(c.row, h * 4 + kc, 64));
      const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
      uint32_t out[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 f = unpack2<BF16>(hw[j]);
        const float a = f.x > 0.f ? __uint_as_float(r[kc * 8 + 2 * j]) : 0.f;
        const float b = f.y > 0.f ? __uint_as_float(r[kc * 8 + 2 * j + 1]) : 0.f;
        out[j] = tile::pack2(a, b, BF16);
      }
      *reinterpret_cast<uint4*>(d_tile + tile::chunk_off(c.row, h * 4 + kc, 64)) =
          *reinterpret_cast<uint4*>(out);
    }
  }
  tc_fence_before();
}

template <bool BF16 = false>
__device__ __forceinline__ void relu_to(const tile::Wg& c, uint32_t taddr, uint8_t* dst) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t r[32];
    tmem_ld32(taddr + h * 32, r);
    tmem_ld_wait();
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t v[4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
        v[j] = tile::pack2(fmaxf(__uint_as_float(r[kc * 8 + 2 * j]), 0.f),
                           fmaxf(__uint_as_float(r[kc * 8 + 2 * j + 1]), 0.f), BF16);
      *reinterpret_cast<uint4*>(dst + tile::chunk_off(c.row, h * 4 + kc, 64)) = *reinterpret_cast<uint4*>(v);
    }
  }
  tc_fence_before();
}

}  // namespace train_tile
}  // namespace gdf
