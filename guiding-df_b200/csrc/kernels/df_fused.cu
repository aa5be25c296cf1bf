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
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "../device/df_math.cuh"
#include "../device/df_tile.cuh"
#include "../device/records.cuh"
#include "../device/sm100.cuh"
#include "df_kernels.h"
#include "launch_util.h"

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
  // columns of the per-warpgroup A tile: first-layer segment(s) and the
  // 64-wide hidden activations
  __host__ __device__ static constexpr uint32_t tile_a(uint32_t a, uint32_t b) {
    return a > 64u ? (a > b ? a : b) : (64u > b ? 64u : b);
  }
};

// ---------------------------------------------------------------------------
// Fused kernel, one warpgroup per 128-query tile:
//   1. theta input (grid | SH | OneBlob | 1-pad) -> tile A; theta layer 0 issued;
//   2. while it runs, the phi grid's gathers -> tile P (its own K=L*F tile);
//   3. theta hidden/output layers (tcgen05, TMEM accumulators);
//   4. softmax/CDF/sampling streamed from TMEM -> u_theta, pdf_theta;
//   5. phi input rest (SH | OneBlob | TriangleWave(u_theta) | 1-pad) -> tile A;
//      phi layer 0 reads K steps from tile P then tile A;
//   6. phi layers, epilogue -> u_phi, pdf_phi -> guiding data.
// FMT: MLP operand format of the inference forms, 0 fp16, 1 bf16, 2 FP8
// (e4m3 hidden matrices, mlp_tail_f8).
template <int L, int F, int NBT, int NBP, bool LINEAR, int MODE, int WGS, int FMT>
__global__ void __launch_bounds__(128 * WGS, 1) df_fused_kernel(const __grid_constant__ DfKernelParams p) {
  using Wd = DfWidths<L, F>;
  constexpr uint32_t LF = L * F;
  constexpr uint32_t KT = Wd::kTheta;            // theta input width
  constexpr uint32_t KR = Wd::kPhi - LF;         // phi input minus its grid part
  constexpr uint32_t KTR = KT - LF;              // theta input minus its grid part
  // Inference, pdf evaluation and the training step read both grids'
  // features precomputed (launch_grid_features, launch_train_features);
  // kModeTrainFwd gathers them itself.
  constexpr bool kFeat = MODE != kModeTrainFwd;
  constexpr bool kTrain = MODE == kModeTrainFwd || MODE == kModeTrainFeat;
  constexpr uint32_t KA = kFeat ? DfWidths<L, F>::tile_a(KTR, KR) : DfWidths<L, F>::tile_a(KT, KR);
  static_assert(LF % 16 == 0 && KT % 16 == 0 && KR % 16 == 0 && KTR % 16 == 0,
                "K segments must be multiples of 16");
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x;
  const uint32_t wg = tid >> 7;
  const uint32_t warp = tid >> 5;

  const uint32_t off_phi = (p.blob_theta_bytes + 127u) & ~127u;
  const uint32_t off_tiles = (off_phi + p.blob_phi_bytes + 127u) & ~127u;
  constexpr uint32_t kTileA = 128u * KA * 2u, kTileP = 128u * LF * 2u;
  constexpr uint32_t kWgBytes = kTileA + (kFeat ? 2u : 1u) * kTileP;
  const uint32_t off_bars = off_tiles + WGS * kWgBytes;
  // [0] weights, [1+g] MMA of warpgroup g, [1+WGS+g] its feature tiles
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bars);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bars + 8 * (2 * WGS + 1));
  constexpr uint32_t kTmemCols = 64 * WGS <= 128 ? 128 : (64 * WGS <= 256 ? 256 : 512);

  if (warp == 0) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i <= 2 * WGS; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bars[0], p.blob_theta_bytes + p.blob_phi_bytes);
    for (uint32_t o = 0; o < p.blob_theta_bytes; o += 32768u)
      bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(p.blob_theta) + o,
               min(32768u, p.blob_theta_bytes - o), &bars[0]);
    for (uint32_t o = 0; o < p.blob_phi_bytes; o += 32768u)
      bulk_g2s(smem + off_phi + o, reinterpret_cast<const uint8_t*>(p.blob_phi) + o,
               min(32768u, p.blob_phi_bytes - o), &bars[0]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  mbar_wait(&bars[0], 0, p.err, kErrWeightLoad);

  tile::Wg c;
  c.tile_a = smem + off_tiles + wg * kWgBytes;
  c.tile_a_s = smem_addr(c.tile_a);
  c.tile_p = c.tile_a + kTileA;
  c.tile_p_s = c.tile_a_s + kTileA;
  uint8_t* const tile_gt = c.tile_p + kTileP;  // theta grid features (kFeat)
  const uint32_t tile_gt_s = c.tile_p_s + kTileP;
  uint64_t* const fbar = &bars[1 + WGS + wg];
  uint32_t fphase = 0;
  c.tmem = tmem_base + wg * 64u;
  c.lane_base = ((warp & 3u) * 32u) << 16;
  c.bar = &bars[1 + wg];
  c.phase = 0;
  c.bar_id = 1 + wg;
  c.row = tid & 127u;
  c.leader = c.row == 0;
  c.err = p.err;
  c.bf16 = kFeat && FMT == 1;  // operand format of the inference forms
  constexpr bool kF8 = kFeat && FMT == 2;
  const uint32_t w_theta = smem_addr(smem);
  const uint32_t w_phi = smem_addr(smem + off_phi);
  const uint32_t w_theta_hidden = w_theta + 64u * KT * 2u;
  const uint32_t w_phi_hidden = w_phi + 64u * (LF + KR) * 2u;
  // FP8 form: descale factors after each blob's output matrix
  const float* ds_theta = reinterpret_cast<const float*>(
      smem + 64u * KT * 2u + static_cast<uint32_t>(p.hidden_theta - 1) * 4096u + NBT * 128u);
  const float* ds_phi = reinterpret_cast<const float*>(
      smem + off_phi + 64u * (LF + KR) * 2u + static_cast<uint32_t>(p.hidden_phi - 1) * 4096u + NBP * 128u);

  // training modes with a device-side record count: min(*n_dev, n) rows
  const int64_t n_rows = (kTrain && p.n_dev) ? min(*p.n_dev, p.n) : p.n;
  const float loss_scale_per_record = (kTrain && p.n_dev)
                                          ? (n_rows > 0 ? p.loss_scale / static_cast<float>(n_rows) : 0.f)
                                          : p.loss_scale_per_record;
  const int64_t n_tiles = (n_rows + 127) / 128;
  // Both feature tiles of tile t, one bulk copy each, completing on fbar.
  auto fetch_features = [&](int64_t t) {
    if (!c.leader) return;
    mbar_arrive_expect_tx(fbar, 2u * kTileP);
    bulk_g2s(tile_gt, p.feat_theta + t * (128 * LF), kTileP, fbar);
    bulk_g2s(c.tile_p, p.feat_phi + t * (128 * LF), kTileP, fbar);
  };
  if constexpr (kFeat) {
    const int64_t t0 = static_cast<int64_t>(blockIdx.x) * WGS + wg;
    if (t0 < n_tiles) fetch_features(t0);
  }
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * WGS + wg; t < n_tiles;
       t += static_cast<int64_t>(gridDim.x) * WGS) {
    const int64_t row = t * 128 + c.row;
    const bool valid = row < n_rows;
    float q[9], qp[10];
    if (MODE == kModeInfer && p.shading.pos != nullptr) {
      // generate_inference_data_AR (train.cu:344-361) in registers
#pragma unroll
      for (int i = 0; i < 9; ++i) q[i] = 0.5f;
      if (valid) {
        float pos[3], wo[3], nrm[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          pos[k] = __ldg(p.shading.pos + row * 3 + k);
          wo[k] = __ldg(p.shading.wo + row * 3 + k);
          nrm[k] = __ldg(p.shading.normal + row * 3 + k);
        }
        rec::shading_to_query(pos, wo, nrm, __ldg(p.shading.roughness + row), rec::scene_frame(p.aabb), q);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) q[i] = valid ? __ldg(p.queries + row * 9 + i) : 0.5f;
    }
    bool record_ok = true;
    float tg[9];
    if constexpr (kTrain) {
      // the phi network reads its own record (GuidedInputPhi, slot 9 = theta)
#pragma unroll
      for (int i = 0; i < 10; ++i) qp[i] = valid ? __ldg(p.in_phi + row * 10 + i) : 0.5f;
#pragma unroll
      for (int i = 0; i < 9; ++i) tg[i] = valid ? __ldg(p.target + row * 9 + i) : 0.5f;
      // generate_training_data_AR validity filter (train.cu:77-81)
#pragma unroll
      for (int i = 0; i < 9; ++i) record_ok &= !isnan(q[i]) && !isnan(tg[i]);
#pragma unroll
      for (int i = 0; i < 10; ++i) record_ok &= !isnan(qp[i]);
      record_ok &= tg[5] != 0.0f;
      if (!record_ok) {
#pragma unroll
        for (int i = 0; i < 9; ++i) { q[i] = 0.5f; qp[i] = 0.5f; }
        qp[9] = 0.5f;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) qp[i] = q[i];
    }

    // ---- 1. theta input (grid features | SH | OneBlob | padding), layer 0
    // Inference and pdf evaluation feed the phi network the same first nine
    // inputs, so its SH / OneBlob values are computed here once and kept,
    // packed, until its input tile is written (step 5).
    uint32_t phi_shob[14];
    if constexpr (kFeat) {
      float shob[28];
      tile::sh_ob_values(q, shob);
      if constexpr (!kTrain) tile::pack_run<28>(shob, c.bf16, phi_shob);
      tile::theta_rest_from_values(shob, c.tile_a, c.row, 0, KTR, c.bf16);
      mbar_wait(fbar, fphase, p.err, kErrMbarTimeout);
      fphase ^= 1u;
      tile::publish(c);
      const tile::ASeg a[2] = {{tile_gt_s, LF, static_cast<int>(LF / 16)},
                               {c.tile_a_s, KTR, static_cast<int>(KTR / 16)}};
      tile::issue(c, a, 2, w_theta, KT, 64);
    } else {
      tile::grids_to_tiles<L, F>(p.gl_theta, p.grid_theta, p.gl_phi, p.grid_phi, q, qp, c.tile_a, KT,
                                 c.tile_p, c.row);
      tile::theta_rest_to_tile(q, c.tile_a, c.row, LF, KT);
      tile::publish(c);
      const tile::ASeg a{c.tile_a_s, KT, static_cast<int>(KT / 16)};
      tile::issue(c, &a, 1, w_theta, KT, 64);
    }
    // ---- 2./3. theta layers
    if constexpr (kF8) tile::mlp_tail_f8(c, w_theta_hidden, p.hidden_theta, NBT, ds_theta);
    else tile::mlp_tail(c, w_theta_hidden, p.hidden_theta, NBT);
    // ---- 4. theta epilogue
    float4 wi = make_float4(0.f, 0.f, 1.f, 1.f);
    float u[4] = {0.f, 0.f, 0.f, 0.f};
    bool guided = true;
    if constexpr (MODE == kModeInfer) {
      if (valid) {
        wi = *reinterpret_cast<const float4*>(p.wi + row * 4);
        guided = p.guided ? (p.guided[row] != 0) : true;
        if (p.uniforms) {
          const float4 uu = *reinterpret_cast<const float4*>(p.uniforms + row * 4);
          u[0] = uu.x; u[1] = uu.y; u[2] = uu.z; u[3] = uu.w;
        } else {
          uint32_t r[4];
          const uint64_t ctr = static_cast<uint64_t>(row + p.philox_row_base);
          philox4x32_10(static_cast<uint32_t>(ctr), static_cast<uint32_t>(ctr >> 32),
                        static_cast<uint32_t>(p.philox_offset), static_cast<uint32_t>(p.philox_offset >> 32),
                        static_cast<uint32_t>(p.philox_seed), static_cast<uint32_t>(p.philox_seed >> 32), r);
#pragma unroll
          for (int k = 0; k < 4; ++k) u[k] = u32_to_uniform(r[k]);
        }
      }
    }
    float u_theta, pdf_theta, cond;
    if constexpr (kTrain) {
      u_theta = tg[0];
      pdf_theta = tile::row_pdf_train<NBT, LINEAR>(c.tmem + c.lane_base, tg[0]);
      cond = qp[9];
    } else {
      const float u_theta_given = MODE == kModeInfer ? wi.x : (valid ? __ldg(p.u_eval + row * 2) : 0.5f);
      const tile::RowResult rt = tile::row_epilogue<NBT, LINEAR, (FMT != 0)>(
          c.tmem + c.lane_base, MODE == kModeInfer && guided, u_theta_given, u[0], u[1]);
      if (p.norm_err != nullptr) tile::row_norm_check<NBT, (FMT != 0)>(c.tmem + c.lane_base, p.norm_err);
      u_theta = rt.u;
      pdf_theta = rt.pdf;
      cond = theta_condition<NBT, LINEAR>(u_theta);
    }

    // ---- 5. phi input rest, layer 0 over tile P (grid) + tile A (rest)
    if constexpr (kFeat && !kTrain) tile::store_packed_run<14>(c.tile_a, c.row, 0, KR, phi_shob);
    else tile::sh_ob_to_tile(qp, c.tile_a, c.row, 0, KR, c.bf16);
    {
      float tw[12];
      triangle_wave_encode<12>(cond, tw);
      tile::store_run(c.tile_a, c.row, 28, KR, tw, 12, c.bf16);
    }
    tile::ones_to_tile(c.tile_a, c.row, 40, KR, KR, c.bf16);
    tile::publish(c);
    {
      const tile::ASeg a[2] = {{c.tile_p_s, LF, static_cast<int>(LF / 16)},
                               {c.tile_a_s, KR, static_cast<int>(KR / 16)}};
      tile::issue(c, a, 2, w_phi, LF + KR, 64);
    }
    // ---- 6. phi layers and epilogue
    if constexpr (kF8) tile::mlp_tail_f8(c, w_phi_hidden, p.hidden_phi, NBP, ds_phi);
    else tile::mlp_tail(c, w_phi_hidden, p.hidden_phi, NBP);
    if constexpr (kFeat) {
      // every MMA that read this tile's feature tiles has completed
      const int64_t next = t + static_cast<int64_t>(gridDim.x) * WGS;
      if (next < n_tiles) fetch_features(next);
    }
    if constexpr (kTrain) {
      const float pdf_phi = tile::row_pdf_train<NBP, LINEAR>(c.tmem + c.lane_base, tg[1]);
      // combine_AR_pdf_and_dl_doutput (train.h:956-963): AutoRegressive takes
      // |pdf|, pdf() = pt * pp * (1/4pi), times its inverse, + M_EPSILON
      constexpr float kInv4Pi = 0.0795774715459476678844f;
      const float li = (tg[2] + tg[3] + tg[4]) / 3.0f;
      const float wi_pdf = tg[5] + kEps;
      const float gpdf = fabsf(pdf_theta) * fabsf(pdf_phi) * kInv4Pi * (1.f / kInv4Pi) + kEps;
      const float prefix = -li / wi_pdf / gpdf * loss_scale_per_record;
      const float lik = -li / wi_pdf * logf(gpdf);
      if (valid) {
        const float4 o = record_ok ? make_float4(pdf_theta, pdf_phi, prefix, lik)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
        *reinterpret_cast<float4*>(p.train_out + row * 4) = o;
        if (!record_ok) atomicAdd(p.n_dropped, 1ull);
      }
      continue;
    }
    const float u_phi_given = MODE == kModeInfer ? wi.y : (valid ? __ldg(p.u_eval + row * 2 + 1) : 0.5f);
    const tile::RowResult rp = tile::row_epilogue<NBP, LINEAR, (FMT != 0)>(
        c.tmem + c.lane_base, MODE == kModeInfer && guided, u_phi_given, u[2], u[3]);
    if (p.norm_err != nullptr) tile::row_norm_check<NBP, (FMT != 0)>(c.tmem + c.lane_base, p.norm_err);
    if constexpr (MODE == kModeInfer) {
      const float4 o = make_float4(u_theta, rp.u, wi.z * pdf_theta, wi.w * rp.pdf);
      if (valid) *reinterpret_cast<float4*>(p.wi + row * 4) = o;
      if (valid && p.dir_pdf != nullptr) {
        // AutoRegressive over the guiding data (AR.h:25-48)
        float d[3];
        rec::square_to_uniform_sphere(o.x, o.y, d);
        const float pdf = fabsf(o.z) * fabsf(o.w) * rec::kInv4Pi;
        *reinterpret_cast<float4*>(p.dir_pdf + row * 4) = make_float4(d[0], d[1], d[2], pdf);
      }
    } else {
      if (valid) *reinterpret_cast<float2*>(p.pdf_out + row * 2) = make_float2(pdf_theta, rp.pdf);
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
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
                                int32_t cols, int64_t n, bool to_bf16) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = static_cast<uint32_t>(i / cols), cc = static_cast<uint32_t>(i % cols);
  __half v = src[i];
  if (to_bf16) {  // bf16 inference form: the fp16 value rounded to bf16, stored bit for bit
    const __nv_bfloat16 b = __float2bfloat16_rn(__half2float(v));
    v = *reinterpret_cast<const __half*>(&b);
  }
  dst[canon_offset(r, cc, static_cast<uint32_t>(cols))] = v;
}

// One block per matrix (Fp8PackParams): fp16 copies for the first and last
// matrices, e4m3(W * 2^k) for the hidden ones with k from the matrix's
// absolute maximum (tile::e4m3_scale_exp) and descale 2^-k.
__global__ void __launch_bounds__(256) pack_fp8_kernel(const __grid_constant__ Fp8PackParams p) {
  const int l = blockIdx.x;
  const int rows = p.rows[l], cols = p.cols[l];
  const int n = rows * cols;
  const __half* src = p.src + p.src_off[l];
  if (l == 0 || l == p.n_layers - 1) {
    __half* dst = reinterpret_cast<__half*>(p.dst + p.dst_off[l]);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      dst[canon_offset(static_cast<uint32_t>(i / cols), static_cast<uint32_t>(i % cols),
                       static_cast<uint32_t>(cols))] = src[i];
    return;
  }
  __shared__ float red[8];
  float amax = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) amax = fmaxf(amax, fabsf(__half2float(src[i])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  amax = red[0];
  for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) amax = fmaxf(amax, red[w]);
  const int k = tile::e4m3_scale_exp(amax);
  const float s = tile::exp2i(k);
  if (threadIdx.x == 0) reinterpret_cast<float*>(p.dst + p.descale_off)[l - 1] = tile::exp2i(-k);
  uint8_t* dst = p.dst + p.dst_off[l];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t r = static_cast<uint32_t>(i / cols), cc = static_cast<uint32_t>(i % cols);
    // byte cc of a 64-byte row: two-byte column cc / 2 of the canonical layout
    const uint32_t off = 2u * canon_offset(r, cc >> 1, static_cast<uint32_t>(cols) >> 1) + (cc & 1u);
    dst[off] = static_cast<uint8_t>(__nv_cvt_float_to_fp8(__half2float(src[i]) * s, __NV_SATFINITE, __NV_E4M3));
  }
}

template <int L, int F, int NBT, int NBP, bool LIN>
cudaError_t launch_t(int mode, const DfKernelParams& p, size_t smem, int num_sms, cudaStream_t st) {
  const int64_t n_tiles = (p.n + 127) / 128;
  int64_t ctas = (n_tiles + kDfWarpgroups - 1) / kDfWarpgroups;
  if (ctas > num_sms) ctas = num_sms;
  if (ctas < 1) ctas = 1;
  // the training forward with feature tiles has an fp16 and a bf16 form;
  // the one with in-kernel gathers (static-workspace loss) fp16 only
  const int fmt = mode == kModeTrainFwd ? 0
                  : mode == kModeTrainFeat ? (p.bf16 ? 1 : 0)
                                           : (p.fp8 ? 2 : (p.bf16 ? 1 : 0));
  auto pick = [&](auto k16, auto kb16, auto k8) { return fmt == 2 ? k8 : (fmt == 1 ? kb16 : k16); };
  auto kern = mode == kModeInfer
                  ? pick(df_fused_kernel<L, F, NBT, NBP, LIN, kModeInfer, kDfWarpgroups, 0>,
                         df_fused_kernel<L, F, NBT, NBP, LIN, kModeInfer, kDfWarpgroups, 1>,
                         df_fused_kernel<L, F, NBT, NBP, LIN, kModeInfer, kDfWarpgroups, 2>)
              : mode == kModeEval
                  ? pick(df_fused_kernel<L, F, NBT, NBP, LIN, kModeEval, kDfWarpgroups, 0>,
                         df_fused_kernel<L, F, NBT, NBP, LIN, kModeEval, kDfWarpgroups, 1>,
                         df_fused_kernel<L, F, NBT, NBP, LIN, kModeEval, kDfWarpgroups, 2>)
              : mode == kModeTrainFeat
                  ? (fmt == 1 ? df_fused_kernel<L, F, NBT, NBP, LIN, kModeTrainFeat, kDfWarpgroups, 1>
                              : df_fused_kernel<L, F, NBT, NBP, LIN, kModeTrainFeat, kDfWarpgroups, 0>)
                  : df_fused_kernel<L, F, NBT, NBP, LIN, kModeTrainFwd, kDfWarpgroups, 0>;
  cudaError_t e = allow_dynamic_smem(kern);
  if (e != cudaSuccess) return e;
  kern<<<static_cast<unsigned>(ctas), kDfThreads, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

bool df_shape_supported(const DfShape& s) {
  const bool a = s.levels == 8 && s.features == 2 && s.bins_theta == 32 && s.bins_phi == 32;
  const bool b = s.levels == 16 && s.features == 2 && (s.bins_theta == 64 || s.bins_theta == 32) &&
                 s.bins_phi == s.bins_theta;
  const bool c = s.levels == 8 && s.features == 4 && s.bins_theta == 16 && s.bins_phi == 32;
  return a || b || c;
}

size_t df_fused_smem_bytes(const DfShape& s, int mode, uint32_t bt, uint32_t bp) {
  const uint32_t lf = static_cast<uint32_t>(s.levels * s.features);
  const uint32_t kt = static_cast<uint32_t>(pad16c(static_cast<int>(lf) + 28));
  const uint32_t kr = static_cast<uint32_t>(pad16c(static_cast<int>(lf) + 40)) - lf;
  const bool feat = mode != kModeTrainFwd;
  const uint32_t ka = feat ? DfWidths<8, 2>::tile_a(kt - lf, kr) : DfWidths<8, 2>::tile_a(kt, kr);
  const size_t off_phi = (bt + 127u) & ~127u;
  const size_t off_tiles = (off_phi + bp + 127u) & ~size_t(127);
  return off_tiles + static_cast<size_t>(kDfWarpgroups) * 128u * (ka + (feat ? 2u : 1u) * lf) * 2u +
         8u * (2 * kDfWarpgroups + 1) + 16u;
}

cudaError_t launch_df_fused(const DfShape& s, int mode, const DfKernelParams& p, int num_sms,
                            cudaStream_t st) {
  if (p.n <= 0) return cudaSuccess;
  const size_t smem = df_fused_smem_bytes(s, mode, p.blob_theta_bytes, p.blob_phi_bytes);
  if (mode != kModeTrainFwd && (p.feat_theta == nullptr || p.feat_phi == nullptr))
    return cudaErrorInvalidValue;
#define GDF_DISPATCH(L, F, NBT, NBP)                                                  \
  if (s.levels == L && s.features == F && s.bins_theta == NBT && s.bins_phi == NBP) { \
    return s.linear ? launch_t<L, F, NBT, NBP, true>(mode, p, smem, num_sms, st)      \
                    : launch_t<L, F, NBT, NBP, false>(mode, p, smem, num_sms, st);    \
  }
  GDF_DISPATCH(8, 2, 32, 32)
  GDF_DISPATCH(16, 2, 64, 64)
  GDF_DISPATCH(16, 2, 32, 32)
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

uint32_t fp8_blob_bytes(const int32_t* rows, const int32_t* cols, int n_layers, Fp8PackParams* lay) {
  uint32_t off = 0;
  int64_t src = 0;
  for (int l = 0; l < n_layers; ++l) {
    const bool f16 = l == 0 || l == n_layers - 1;
    if (lay) {
      lay->rows[l] = rows[l];
      lay->cols[l] = cols[l];
      lay->src_off[l] = src;
      lay->dst_off[l] = off;
    }
    off += static_cast<uint32_t>(rows[l] * cols[l] * (f16 ? 2 : 1));
    src += static_cast<int64_t>(rows[l]) * cols[l];
  }
  if (lay) {
    lay->n_layers = n_layers;
    lay->descale_off = off;
  }
  off += static_cast<uint32_t>(n_layers > 2 ? n_layers - 2 : 0) * 4u;
  return (off + 15u) & ~15u;
}

cudaError_t launch_pack_fp8(const Fp8PackParams& p, cudaStream_t st) {
  if (p.n_layers < 2 || p.n_layers > kMaxMlpLayers) return cudaErrorInvalidValue;
  for (int l = 1; l + 1 < p.n_layers; ++l)
    if (p.rows[l] != 64 || p.cols[l] != 64) return cudaErrorInvalidValue;
  pack_fp8_kernel<<<p.n_layers, 256, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_pack_mlp(const __half* src, __half* dst, const int32_t* rows, const int32_t* cols,
                            int n_layers, cudaStream_t st, bool to_bf16) {
  for (int l = 0; l < n_layers; ++l) {
    const int64_t n = static_cast<int64_t>(rows[l]) * cols[l];
    pack_mlp_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(src, dst, rows[l], cols[l], n,
                                                                            to_bf16);
    src += n;
    dst += n;
  }
  return cudaGetLastError();
}

}  // namespace gdf
