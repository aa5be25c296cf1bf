// df_fused.cu -- the fused DF inference kernel for sm_100a.
//
// One launch computes, for every query row, what the reference does in
// LearnedDistribution::inferenceStep (src/render/guided/learnedDistribution.cpp:
// 167-206): generate inputs, theta network (tcnn composite encoding +
// FullyFusedMLP), thetaPostInference (train.h:896-911), phi network
// conditioned on the sampled theta, phiPostInference (train.h:914-929).
//
// Layout of the work
//   * persistent CTAs, one per SM, 4 warpgroups each; a warpgroup owns a
//     128-query tile, thread t of the warpgroup owns query row t;
//   * both networks' MLP weights are bulk-copied (TMA engine) once per CTA
//     into shared memory in the tensor-core canonical layout;
//   * each layer is M=128 x N=64 (or n_bins) x K tcgen05.mma issued by one
//     thread of the warpgroup, A = activations in shared memory, B = weights,
//     fp32 accumulator in tensor memory (64 columns per warpgroup);
//   * the epilogue reads its row back with tcgen05.ld (lane = row), applies
//     ReLU, rounds to fp16 and writes the next layer's A operand; after the
//     last layer the row's logits stay in registers for the softmax / CDF /
//     sampling epilogue.
#include <cuda_fp16.h>

#include "../device/df_math.cuh"
#include "../device/sm100.cuh"
#include "df_kernels.h"

namespace gdf {
namespace {

using namespace sm100;

constexpr int pad16c(int v) { return (v + 15) / 16 * 16; }

// Composite widths of the built configurations: SH degree 4 (16),
// OneBlob 4 bins x 3 dims (12), TriangleWave 12 frequencies (phi only).
template <int L, int F>
struct DfWidths {
  static constexpr int kGrid = L * F;
  static constexpr int kTheta = pad16c(kGrid + 16 + 12);
  static constexpr int kPhi = pad16c(kGrid + 16 + 12 + 12);
  static constexpr int kMax = kPhi > 64 ? kPhi : 64;
};

// Store one row of K fp16 values (given as fp32) into the canonical K-major
// A tile (128 rows x K).
template <int K>
__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t row, const float* v) {
#pragma unroll
  for (int kc = 0; kc < K / 8; ++kc) {
    __half2 h[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) h[j] = __floats2half2_rn(v[kc * 8 + 2 * j], v[kc * 8 + 2 * j + 1]);
    const uint32_t off = (((row >> 3) * (K / 8) + kc) << 7) + ((row & 7u) << 4);
    *reinterpret_cast<uint4*>(tile + off) = *reinterpret_cast<uint4*>(h);
  }
}

// Reads N fp32 columns of this thread's TMEM lane.
template <int N>
__device__ __forceinline__ void tmem_load_row(uint32_t taddr, float (&v)[N]) {
  if constexpr (N == 16) {
    uint32_t r[16];
    tmem_ld16(taddr, r);
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
  } else {
#pragma unroll
    for (int c = 0; c < N / 32; ++c) {
      uint32_t r[32];
      tmem_ld32(taddr + c * 32, r);
      tmem_ld_wait();
#pragma unroll
      for (int i = 0; i < 32; ++i) v[c * 32 + i] = __uint_as_float(r[i]);
    }
  }
}

struct WgCtx {
  uint8_t* tile;       // this warpgroup's A tile (generic pointer)
  uint32_t tile_s;     // same, shared-space address
  uint32_t tmem;       // accumulator column base (lane 0)
  uint32_t lane_base;  // this warp's TMEM lane offset, in address units
  uint64_t* bar;       // MMA-completion mbarrier
  uint32_t phase;
  uint32_t bar_id;     // named barrier of the warpgroup
  uint32_t row;        // thread's row in the tile
  bool leader;
  uint32_t* err;
};

// Issue one layer: D = A[128 x K] * W[N x K]^T, then wait for completion.
__device__ __forceinline__ void mma_layer(WgCtx& c, uint32_t w_s, int K, int N) {
  fence_proxy_async_smem();
  __syncwarp();
  named_bar_sync(c.bar_id, 128);
  if (c.leader) {
    tc_fence_after();
    const uint32_t idesc = idesc_f16(128, N, 0, 0, 0);
    const uint32_t sbo = static_cast<uint32_t>(K) * 16u;
    for (int s = 0; s < K / 16; ++s) {
      const uint64_t ad = smem_desc(c.tile_s + s * 256, 128, sbo);
      const uint64_t bd = smem_desc(w_s + s * 256, 128, sbo);
      mma_f16_ss(c.tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
    mma_commit(c.bar);
  }
  mbar_wait(c.bar, c.phase, c.err, kErrMbarTimeout);
  c.phase ^= 1u;
  __syncwarp();
  tc_fence_after();
}

// Runs hidden layers + output layer of one network whose encoded input is
// already in the tile. Returns the NOUT logits of this thread's row.
template <int K0, int NOUT>
__device__ __forceinline__ void run_mlp(WgCtx& c, uint32_t w_s, int n_hidden, float (&logits)[NOUT]) {
  // First layer: K0 -> 64.
  mma_layer(c, w_s, K0, 64);
  w_s += 64u * K0 * 2u;
  for (int l = 1; l <= n_hidden; ++l) {
    float h[64];
    tmem_load_row<64>(c.tmem + c.lane_base, h);
    tc_fence_before();
#pragma unroll
    for (int i = 0; i < 64; ++i) h[i] = fmaxf(h[i], 0.0f);
    store_row<64>(c.tile, c.row, h);
    const bool last = (l == n_hidden);
    mma_layer(c, w_s, 64, last ? NOUT : 64);
    w_s += (last ? NOUT : 64) * 64u * 2u;
  }
  tmem_load_row<NOUT>(c.tmem + c.lane_base, logits);
  tc_fence_before();
}

template <int L, int F>
__device__ __forceinline__ void encode_common(const GridLevels& gl, const __half* grid,
                                              const float* q, float* x) {
  grid_encode<L, F>(gl, grid, q[0], q[1], q[2], x);
  sh4_encode(q[3], q[4], q[5], x + L * F);
  oneblob_encode<4>(q[6], x + L * F + 16);
  oneblob_encode<4>(q[7], x + L * F + 20);
  oneblob_encode<4>(q[8], x + L * F + 24);
}

template <int L, int F, int NBT, int NBP, bool LINEAR, int MODE>
__global__ void __launch_bounds__(kDfThreads, 1) df_fused_kernel(const __grid_constant__ DfKernelParams p) {
  using W = DfWidths<L, F>;
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x;
  const uint32_t wg = tid >> 7;
  const uint32_t warp = tid >> 5;

  // Shared-memory carve-up: weights | A tiles | barriers | tmem slot.
  const uint32_t off_phi = (p.blob_theta_bytes + 127u) & ~127u;
  const uint32_t off_tiles = (off_phi + p.blob_phi_bytes + 1023u) & ~1023u;
  constexpr uint32_t kTileBytes = 128u * W::kMax * 2u;
  const uint32_t off_bars = off_tiles + kDfWarpgroups * kTileBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bars);  // [0] weights, [1+g] MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bars + 8 * (kDfWarpgroups + 1));

  if (warp == 0) {
    tmem_alloc(tmem_slot, 64 * kDfWarpgroups);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i <= kDfWarpgroups; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], p.blob_theta_bytes + p.blob_phi_bytes);
    for (uint32_t o = 0; o < p.blob_theta_bytes; o += 32768u) {
      const uint32_t b = min(32768u, p.blob_theta_bytes - o);
      bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(p.blob_theta) + o, b, &bars[0]);
    }
    for (uint32_t o = 0; o < p.blob_phi_bytes; o += 32768u) {
      const uint32_t b = min(32768u, p.blob_phi_bytes - o);
      bulk_g2s(smem + off_phi + o, reinterpret_cast<const uint8_t*>(p.blob_phi) + o, b, &bars[0]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  mbar_wait(&bars[0], 0, p.err, kErrWeightLoad);

  WgCtx c;
  c.tile = smem + off_tiles + wg * kTileBytes;
  c.tile_s = smem_addr(c.tile);
  c.tmem = tmem_base + wg * 64u;
  c.lane_base = ((warp & 3u) * 32u) << 16;
  c.bar = &bars[1 + wg];
  c.phase = 0;
  c.bar_id = 1 + wg;
  c.row = tid & 127u;
  c.leader = (tid & 127u) == 0;
  c.err = p.err;
  const uint32_t w_theta = smem_addr(smem);
  const uint32_t w_phi = smem_addr(smem + off_phi);

  const int64_t n_tiles = (p.n + 127) / 128;
  for (int64_t tile = static_cast<int64_t>(blockIdx.x) * kDfWarpgroups + wg; tile < n_tiles;
       tile += static_cast<int64_t>(gridDim.x) * kDfWarpgroups) {
    const int64_t row = tile * 128 + c.row;
    const bool valid = row < p.n;
    float q[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) q[i] = valid ? __ldg(p.queries + row * 9 + i) : 0.5f;

    // ---- theta network
    {
      float x[W::kTheta];
      encode_common<L, F>(p.gl_theta, p.grid_theta, q, x);
#pragma unroll
      for (int i = W::kGrid + 28; i < W::kTheta; ++i) x[i] = 1.0f;
      store_row<W::kTheta>(c.tile, c.row, x);
    }
    float lt[NBT];
    run_mlp<W::kTheta, NBT>(c, w_theta, p.hidden_theta, lt);
    softmax2_times_n<NBT>(lt);

    float4 wi = make_float4(0.f, 0.f, 1.f, 1.f);
    float u[4] = {0.f, 0.f, 0.f, 0.f};
    bool guided = true;
    float u_theta;
    if constexpr (MODE == kModeInfer) {
      if (valid) {
        wi = *reinterpret_cast<const float4*>(p.wi + row * 4);
        guided = p.guided ? (p.guided[row] != 0) : true;
        if (p.uniforms) {
          const float4 uu = *reinterpret_cast<const float4*>(p.uniforms + row * 4);
          u[0] = uu.x; u[1] = uu.y; u[2] = uu.z; u[3] = uu.w;
        } else {
          uint32_t r[4];
          philox4x32_10(static_cast<uint32_t>(row), static_cast<uint32_t>(static_cast<uint64_t>(row) >> 32),
                        static_cast<uint32_t>(p.philox_offset),
                        static_cast<uint32_t>(p.philox_offset >> 32),
                        static_cast<uint32_t>(p.philox_seed),
                        static_cast<uint32_t>(p.philox_seed >> 32), r);
#pragma unroll
          for (int k = 0; k < 4; ++k) u[k] = u32_to_uniform(r[k]);
        }
      }
      u_theta = guided ? sample_dir<NBT, LINEAR>(lt, u[0], u[1]) : wi.x;
    } else {
      u_theta = valid ? __ldg(p.u_eval + row * 2) : 0.5f;
    }
    const float pdf_theta = sample_pdf<NBT, LINEAR>(lt, u_theta);
    const float cond = theta_condition<NBT, LINEAR>(u_theta);

    // ---- phi network (own grid; same SH / OneBlob inputs; TriangleWave of theta)
    {
      float x[W::kPhi];
      encode_common<L, F>(p.gl_phi, p.grid_phi, q, x);
      triangle_wave_encode<12>(cond, x + W::kGrid + 28);
#pragma unroll
      for (int i = W::kGrid + 40; i < W::kPhi; ++i) x[i] = 1.0f;
      store_row<W::kPhi>(c.tile, c.row, x);
    }
    float lp[NBP];
    run_mlp<W::kPhi, NBP>(c, w_phi, p.hidden_phi, lp);
    softmax2_times_n<NBP>(lp);

    if constexpr (MODE == kModeInfer) {
      const float u_phi = guided ? sample_dir<NBP, LINEAR>(lp, u[2], u[3]) : wi.y;
      const float pdf_phi = sample_pdf<NBP, LINEAR>(lp, u_phi);
      if (valid) {
        *reinterpret_cast<float4*>(p.wi + row * 4) =
            make_float4(u_theta, u_phi, wi.z * pdf_theta, wi.w * pdf_phi);
      }
    } else {
      const float u_phi = valid ? __ldg(p.u_eval + row * 2 + 1) : 0.5f;
      const float pdf_phi = sample_pdf<NBP, LINEAR>(lp, u_phi);
      if (valid) *reinterpret_cast<float2*>(p.pdf_out + row * 2) = make_float2(pdf_theta, pdf_phi);
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, 64 * kDfWarpgroups);
}

template <int NBT, int NBP, bool LINEAR>
__global__ void df_post_kernel(const float* __restrict__ lt_in, const float* __restrict__ lp_in,
                               const uint8_t* __restrict__ guided, const float* __restrict__ uni,
                               float* __restrict__ wi, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lt[NBT], lp[NBP];
#pragma unroll
  for (int k = 0; k < NBT; ++k) lt[k] = lt_in[i * NBT + k];
#pragma unroll
  for (int k = 0; k < NBP; ++k) lp[k] = lp_in[i * NBP + k];
  float4 w = *reinterpret_cast<const float4*>(wi + i * 4);
  const float4 u = *reinterpret_cast<const float4*>(uni + i * 4);
  const bool g = guided ? guided[i] != 0 : true;
  softmax2_times_n<NBT>(lt);
  if (g) w.x = sample_dir<NBT, LINEAR>(lt, u.x, u.y);
  softmax2_times_n<NBP>(lp);
  if (g) w.y = sample_dir<NBP, LINEAR>(lp, u.z, u.w);
  w.z *= sample_pdf<NBT, LINEAR>(lt, w.x);
  w.w *= sample_pdf<NBP, LINEAR>(lp, w.y);
  *reinterpret_cast<float4*>(wi + i * 4) = w;
}

__global__ void pack_mlp_kernel(const __half* __restrict__ src, __half* __restrict__ dst, int32_t rows,
                                int32_t cols, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = static_cast<uint32_t>(i / cols), cc = static_cast<uint32_t>(i % cols);
  dst[canon_offset(r, cc, static_cast<uint32_t>(cols))] = src[i];
}

template <int L, int F, int NBT, int NBP, bool LIN>
cudaError_t launch_t(int mode, const DfKernelParams& p, size_t smem, int num_sms, cudaStream_t st) {
  const int64_t n_tiles = (p.n + 127) / 128;
  int64_t ctas = (n_tiles + kDfWarpgroups - 1) / kDfWarpgroups;
  if (ctas > num_sms) ctas = num_sms;
  if (ctas < 1) ctas = 1;
  auto kern = mode == kModeInfer ? df_fused_kernel<L, F, NBT, NBP, LIN, kModeInfer>
                                 : df_fused_kernel<L, F, NBT, NBP, LIN, kModeEval>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  kern<<<static_cast<unsigned>(ctas), kDfThreads, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

bool df_shape_supported(const DfShape& s) {
  const bool a = s.levels == 8 && s.features == 2 && s.bins_theta == 32 && s.bins_phi == 32;
  const bool b = s.levels == 16 && s.features == 2 && s.bins_theta == 64 && s.bins_phi == 64;
  const bool c = s.levels == 8 && s.features == 4 && s.bins_theta == 16 && s.bins_phi == 32;
  return a || b || c;
}

size_t df_fused_smem_bytes(const DfShape& s, uint32_t bt, uint32_t bp) {
  const int grid = s.levels * s.features;
  const int kphi = pad16c(grid + 40);
  const int kmax = kphi > 64 ? kphi : 64;
  const size_t off_phi = (bt + 127u) & ~127u;
  const size_t off_tiles = (off_phi + bp + 1023u) & ~size_t(1023);
  return off_tiles + static_cast<size_t>(kDfWarpgroups) * 128u * kmax * 2u +
         8u * (kDfWarpgroups + 1) + 16u;
}

cudaError_t launch_df_fused(const DfShape& s, int mode, const DfKernelParams& p, int num_sms,
                            cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  const size_t smem = df_fused_smem_bytes(s, p.blob_theta_bytes, p.blob_phi_bytes);
#define GDF_DISPATCH(L, F, NBT, NBP)                                                  \
  if (s.levels == L && s.features == F && s.bins_theta == NBT && s.bins_phi == NBP) { \
    return s.linear ? launch_t<L, F, NBT, NBP, true>(mode, p, smem, num_sms, st)      \
                    : launch_t<L, F, NBT, NBP, false>(mode, p, smem, num_sms, st);    \
  }
  GDF_DISPATCH(8, 2, 32, 32)
  GDF_DISPATCH(16, 2, 64, 64)
  GDF_DISPATCH(8, 4, 16, 32)
#undef GDF_DISPATCH
  return cudaErrorNotSupported;
}

cudaError_t launch_df_post(int nbt, int nbp, bool linear, const float* lt, const float* lp,
                           const uint8_t* guided, const float* uni, float* wi, int64_t n,
                           cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
#define GDF_POST(NBT, NBP)                                                                   \
  if (nbt == NBT && nbp == NBP) {                                                            \
    if (linear) df_post_kernel<NBT, NBP, true><<<blocks, 128, 0, st>>>(lt, lp, guided, uni, wi, n); \
    else df_post_kernel<NBT, NBP, false><<<blocks, 128, 0, st>>>(lt, lp, guided, uni, wi, n);      \
    return cudaGetLastError();                                                               \
  }
  GDF_POST(32, 32)
  GDF_POST(64, 64)
  GDF_POST(16, 32)
#undef GDF_POST
  return cudaErrorNotSupported;
}

cudaError_t launch_pack_mlp(const __half* src, __half* dst, const int32_t* rows, const int32_t* cols,
                            int n_layers, cudaStream_t st) {
  for (int l = 0; l < n_layers; ++l) {
    const int64_t n = static_cast<int64_t>(rows[l]) * cols[l];
    pack_mlp_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(src, dst, rows[l], cols[l], n);
    src += n;
    dst += n;
  }
  return cudaGetLastError();
}

}  // namespace gdf
