// grouped.cu -- DF inference for many jobs, each with its own networks, in
// one grid-feature launch and one persistent fused launch.
//
// The work is the inference of LearnedDistribution::inferenceStep
// (src/render/guided/learnedDistribution.cpp:167-206) for every job, with
// the same arithmetic as gdf_infer (df_fused.cu): a job's result does not
// depend on the other jobs in the launch. The jobs come from a table in
// device memory, so a CUDA graph of the two launches stays valid while the
// job set changes from call to call.
//
// Scheduling: each job's tiles (128 queries) are grouped into super-tiles of
// WGS consecutive tiles, one per warpgroup of a CTA, so every warpgroup of a
// CTA works for the same job at a time. A persistent CTA walks the
// super-tiles of all jobs; when it reaches another job it waits for its
// warpgroups to finish and bulk-copies that job's MLP weights into shared
// memory (one reload per CTA and job). Bin counts (16/32/64) are read per
// job, so jobs with different bin counts share the launch.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../device/df_math.cuh"
#include "../device/df_tile.cuh"
#include "../device/sm100.cuh"
#include "group_kernels.h"
#include "launch_util.h"

namespace gdf {
namespace {

using namespace sm100;

__host__ __device__ constexpr uint32_t pad16g(uint32_t v) { return (v + 15u) / 16u * 16u; }

__host__ __device__ constexpr uint32_t tile_a_cols(uint32_t a, uint32_t b) {
  return a > 64u ? (a > b ? a : b) : (64u > b ? 64u : b);
}

// last job whose first super-tile (or tile) is <= s; the table is ordered
__device__ __forceinline__ int find_job(const GroupJobDev* jobs, int n, int64_t s, bool by_super) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t b = by_super ? jobs[mid].super_begin : jobs[mid].tile_begin;
    if (b <= s) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <bool LINEAR, bool COMP>
__device__ __forceinline__ tile::RowResult epilogue_bins(int nb, uint32_t taddr, bool guided, float u_given,
                                                         float u0, float u1) {
  if (nb == 16) return tile::row_epilogue<16, LINEAR, COMP>(taddr, guided, u_given, u0, u1);
  if (nb == 32) return tile::row_epilogue<32, LINEAR, COMP>(taddr, guided, u_given, u0, u1);
  return tile::row_epilogue<64, LINEAR, COMP>(taddr, guided, u_given, u0, u1);
}

template <bool LINEAR>
__device__ __forceinline__ float condition_bins(int nb, float u) {
  if (nb == 16) return theta_condition<16, LINEAR>(u);
  if (nb == 32) return theta_condition<32, LINEAR>(u);
  return theta_condition<64, LINEAR>(u);
}

// One 16-byte chunk of one row per thread, as grid_features_kernel; the
// host sizes the grid to the call's rows (the graph's launch node is
// updated per call), so every thread has exactly one item.
template <int L, int F, bool BF16>
__global__ void __launch_bounds__(256, 4) group_features_kernel(const __grid_constant__ GroupParams g) {
  constexpr int LPC = 8 / F;
  constexpr int NCH = L / LPC;
  constexpr uint32_t LF = L * F;
  const int64_t rows = g.hdr->total_tiles * 128;
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (gid >= rows * NCH) return;  // whole warps: rows * NCH is a multiple of 256
  const int64_t row = gid % rows;
  const int chunk = static_cast<int>(gid / rows);
  const int64_t t = row >> 7;
  // a warp's 32 rows lie in one 128-row tile, hence in one job
  int jb = 0;
  if ((threadIdx.x & 31) == 0) jb = find_job(g.jobs, g.hdr->n_jobs, t, false);
  jb = __shfl_sync(0xffffffffu, jb, 0);
  const GroupJobDev& J = g.jobs[jb];
  const int64_t lr = row - J.tile_begin * 128;
  float pos[3] = {0.5f, 0.5f, 0.5f};
  if (lr < J.n) {
#pragma unroll
    for (int k = 0; k < 3; ++k) pos[k] = __ldg(J.queries + lr * 9 + k);
  }
  uint32_t pt[4], pp[4];
#pragma unroll
  for (int j = 0; j < LPC; ++j) {
    float ft[F], fp[F];
    tile::grid_level_pair<F>(g.gl, chunk * LPC + j, g.gl.interp, J.grid_il, pos[0], pos[1], pos[2], ft, fp);
#pragma unroll
    for (int k = 0; k < F; k += 2) {
      pt[(j * F + k) / 2] = tile::pack2(ft[k], ft[k + 1], BF16);
      pp[(j * F + k) / 2] = tile::pack2(fp[k], fp[k + 1], BF16);
    }
  }
  const int64_t off = t * (128 * LF) +
                      canon_offset(static_cast<uint32_t>(row & 127), static_cast<uint32_t>(chunk * 8), LF);
  *reinterpret_cast<uint4*>(g.feat_theta + off) = make_uint4(pt[0], pt[1], pt[2], pt[3]);
  *reinterpret_cast<uint4*>(g.feat_phi + off) = make_uint4(pp[0], pp[1], pp[2], pp[3]);
}

template <int L, int F, bool LINEAR, int WGS, bool BF16>
__global__ void __launch_bounds__(128 * WGS, 1) group_fused_kernel(const __grid_constant__ GroupParams g) {
  constexpr uint32_t LF = L * F;
  constexpr uint32_t KT = pad16g(LF + 28);
  constexpr uint32_t KR = pad16g(LF + 40) - LF;
  constexpr uint32_t KTR = KT - LF;
  constexpr uint32_t KA = tile_a_cols(KTR, KR);
  static_assert(LF % 16 == 0 && KT % 16 == 0 && KR % 16 == 0 && KTR % 16 == 0,
                "K segments must be multiples of 16");
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x;
  const uint32_t wg = tid >> 7;
  const uint32_t warp = tid >> 5;

  const uint32_t off_phi = (g.max_blob_theta + 127u) & ~127u;
  const uint32_t off_tiles = (off_phi + g.max_blob_phi + 127u) & ~127u;
  constexpr uint32_t kTileA = 128u * KA * 2u, kTileP = 128u * LF * 2u;
  constexpr uint32_t kWgBytes = kTileA + 2u * kTileP;
  const uint32_t off_bars = off_tiles + WGS * kWgBytes;
  // [0] weights, [1+g] MMA of warpgroup g, [1+WGS+g] its feature tiles
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + off_bars);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + off_bars + 8 * (2 * WGS + 1));
  constexpr uint32_t kTmemCols = 64 * WGS <= 128 ? 128 : 256;

  if (warp == 0) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i <= 2 * WGS; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  tile::Wg c;
  c.tile_a = smem + off_tiles + wg * kWgBytes;
  c.tile_a_s = smem_addr(c.tile_a);
  c.tile_p = c.tile_a + kTileA;
  c.tile_p_s = c.tile_a_s + kTileA;
  uint8_t* const tile_gt = c.tile_p + kTileP;
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
  c.err = g.err;
  c.bf16 = BF16;
  const uint32_t w_theta = smem_addr(smem);
  const uint32_t w_phi = smem_addr(smem + off_phi);
  const uint32_t w_theta_hidden = w_theta + 64u * KT * 2u;
  const uint32_t w_phi_hidden = w_phi + 64u * (LF + KR) * 2u;

  const int n_jobs = g.hdr->n_jobs;
  const int64_t n_super = g.hdr->n_super;
  // this warpgroup's tile of super-tile s (index into the feature buffer), or -1
  auto tile_of = [&](int64_t s, int& job) -> int64_t {
    job = find_job(g.jobs, n_jobs, s, true);
    const GroupJobDev& J = g.jobs[job];
    const int64_t lt = (s - J.super_begin) * WGS + wg;
    return lt < (J.n + 127) / 128 ? J.tile_begin + lt : -1;
  };
  auto fetch_features = [&](int64_t s) {
    if (s >= n_super) return;
    int j;
    const int64_t t = tile_of(s, j);
    if (t < 0 || !c.leader) return;
    mbar_arrive_expect_tx(fbar, 2u * kTileP);
    bulk_g2s(tile_gt, g.feat_theta + t * (128 * LF), kTileP, fbar);
    bulk_g2s(c.tile_p, g.feat_phi + t * (128 * LF), kTileP, fbar);
  };
  fetch_features(blockIdx.x);

  int loaded = -1;
  uint32_t wphase = 0;
  for (int64_t s = blockIdx.x; s < n_super; s += gridDim.x) {
    int j;
    const int64_t t = tile_of(s, j);
    const GroupJobDev& J = g.jobs[j];
    if (j != loaded) {
      // every warpgroup is between tiles: its MMAs have completed
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (tid == 0) {
        mbar_arrive_expect_tx(&bars[0], J.blob_theta_bytes + J.blob_phi_bytes);
        for (uint32_t o = 0; o < J.blob_theta_bytes; o += 32768u)
          bulk_g2s(smem + o, reinterpret_cast<const uint8_t*>(J.blob_theta) + o,
                   min(32768u, J.blob_theta_bytes - o), &bars[0]);
        for (uint32_t o = 0; o < J.blob_phi_bytes; o += 32768u)
          bulk_g2s(smem + off_phi + o, reinterpret_cast<const uint8_t*>(J.blob_phi) + o,
                   min(32768u, J.blob_phi_bytes - o), &bars[0]);
      }
      mbar_wait(&bars[0], wphase, g.err, kErrWeightLoad);
      wphase ^= 1u;
      loaded = j;
    }
    if (t < 0) {  // no tile for this warpgroup in this super-tile
      fetch_features(s + gridDim.x);
      continue;
    }
    const int64_t row = (t - J.tile_begin) * 128 + c.row;
    const bool valid = row < J.n;
    float q[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) q[i] = valid ? __ldg(J.queries + row * 9 + i) : 0.5f;
    // theta input (grid features | SH | OneBlob | padding), layer 0; the phi
    // network's SH / OneBlob values are the same, kept packed until its input
    uint32_t phi_shob[14];
    {
      float shob[28];
      tile::sh_ob_values(q, shob);
      tile::pack_run<28>(shob, BF16, phi_shob);
      tile::theta_rest_from_values(shob, c.tile_a, c.row, 0, KTR, BF16);
    }
    mbar_wait(fbar, fphase, g.err, kErrMbarTimeout);
    fphase ^= 1u;
    tile::publish(c);
    {
      const tile::ASeg a[2] = {{tile_gt_s, LF, static_cast<int>(LF / 16)},
                               {c.tile_a_s, KTR, static_cast<int>(KTR / 16)}};
      tile::issue(c, a, 2, w_theta, KT, 64);
    }
    tile::mlp_tail(c, w_theta_hidden, J.hidden_theta, static_cast<uint32_t>(J.bins_theta));
    float4 wi = make_float4(0.f, 0.f, 1.f, 1.f);
    float u[4] = {0.f, 0.f, 0.f, 0.f};
    bool guided = true;
    if (valid) {
      wi = *reinterpret_cast<const float4*>(J.wi + row * 4);
      guided = J.guided ? (J.guided[row] != 0) : true;
      if (J.uniforms) {
        const float4 uu = *reinterpret_cast<const float4*>(J.uniforms + row * 4);
        u[0] = uu.x; u[1] = uu.y; u[2] = uu.z; u[3] = uu.w;
      } else {
        uint32_t r[4];
        const uint64_t ctr = static_cast<uint64_t>(row);
        philox4x32_10(static_cast<uint32_t>(ctr), static_cast<uint32_t>(ctr >> 32),
                      static_cast<uint32_t>(J.offset), static_cast<uint32_t>(J.offset >> 32),
                      static_cast<uint32_t>(J.seed), static_cast<uint32_t>(J.seed >> 32), r);
#pragma unroll
        for (int k = 0; k < 4; ++k) u[k] = u32_to_uniform(r[k]);
      }
    }
    const tile::RowResult rt = epilogue_bins<LINEAR, BF16>(J.bins_theta, c.tmem + c.lane_base, guided, wi.x, u[0], u[1]);
    const float cond = condition_bins<LINEAR>(J.bins_theta, rt.u);
    // phi input rest (SH | OneBlob | TriangleWave(u_theta) | 1-pad), layer 0
    tile::store_packed_run<14>(c.tile_a, c.row, 0, KR, phi_shob);
    {
      float tw[12];
      triangle_wave_encode<12>(cond, tw);
      tile::store_run(c.tile_a, c.row, 28, KR, tw, 12, BF16);
    }
    tile::ones_to_tile(c.tile_a, c.row, 40, KR, KR, BF16);
    tile::publish(c);
    {
      const tile::ASeg a[2] = {{c.tile_p_s, LF, static_cast<int>(LF / 16)},
                               {c.tile_a_s, KR, static_cast<int>(KR / 16)}};
      tile::issue(c, a, 2, w_phi, LF + KR, 64);
    }
    tile::mlp_tail(c, w_phi_hidden, J.hidden_phi, static_cast<uint32_t>(J.bins_phi));
    fetch_features(s + gridDim.x);  // both feature tiles have been read
    const tile::RowResult rp = epilogue_bins<LINEAR, BF16>(J.bins_phi, c.tmem + c.lane_base, guided, wi.y, u[2], u[3]);
    if (valid)
      *reinterpret_cast<float4*>(J.wi + row * 4) = make_float4(rt.u, rp.u, wi.z * rt.pdf, wi.w * rp.pdf);
    // each warp counts its 32 rows; the job's last warp makes them visible
    // to the host through the flag (unless a bounded wait has failed)
    if (g.hdr->track == 0u) continue;
    __syncwarp();
    if ((tid & 31u) == 0u) {
      __threadfence();
      const uint32_t warps = 4u * static_cast<uint32_t>((J.n + 127) / 128);
      if (atomicAdd(g.job_tiles_done + j, 1u) + 1u == warps &&
          *reinterpret_cast<volatile uint32_t*>(g.err) == 0u) {
        __threadfence_system();
        *reinterpret_cast<volatile uint32_t*>(g.job_flag + j) = g.hdr->seq;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, kTmemCols);
}

template <int L, int F>
cudaError_t features_l(const GroupShape& s, const GroupParams& p, int blocks, int threads, cudaStream_t st) {
  if (s.bf16) group_features_kernel<L, F, true><<<blocks, threads, 0, st>>>(p);
  else group_features_kernel<L, F, false><<<blocks, threads, 0, st>>>(p);
  return cudaGetLastError();
}

template <int L, int F, bool LIN, int WGS>
cudaError_t fused_l(bool bf16, const GroupParams& p, size_t smem, int ctas, cudaStream_t st) {
  auto kern = bf16 ? group_fused_kernel<L, F, LIN, WGS, true> : group_fused_kernel<L, F, LIN, WGS, false>;
  cudaError_t e = allow_dynamic_smem(kern);
  if (e != cudaSuccess) return e;
  kern<<<ctas, 128 * WGS, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

bool group_shape_supported(const GroupShape& s) {
  return (s.levels == 8 && s.features == 2) || (s.levels == 16 && s.features == 2) ||
         (s.levels == 8 && s.features == 4);
}

size_t group_fused_smem_bytes(const GroupShape& s, int wgs, uint32_t bt, uint32_t bp) {
  const uint32_t lf = static_cast<uint32_t>(s.levels * s.features);
  const uint32_t kt = pad16g(lf + 28), kr = pad16g(lf + 40) - lf;
  const uint32_t ka = tile_a_cols(kt - lf, kr);
  const size_t off_phi = (bt + 127u) & ~127u;
  const size_t off_tiles = (off_phi + bp + 127u) & ~size_t(127);
  return off_tiles + static_cast<size_t>(wgs) * 128u * (ka + 2u * lf) * 2u + 8u * (2 * wgs + 1) + 16u;
}

cudaError_t launch_group_features(const GroupShape& s, const GroupParams& p, int blocks, int threads,
                                  cudaStream_t st) {
  if (s.levels == 8 && s.features == 2) return features_l<8, 2>(s, p, blocks, threads, st);
  if (s.levels == 16 && s.features == 2) return features_l<16, 2>(s, p, blocks, threads, st);
  if (s.levels == 8 && s.features == 4) return features_l<8, 4>(s, p, blocks, threads, st);
  return cudaErrorNotSupported;
}

cudaError_t launch_group_fused(const GroupShape& s, int wgs, const GroupParams& p, int num_sms, cudaStream_t st) {
  const size_t smem = group_fused_smem_bytes(s, wgs, p.max_blob_theta, p.max_blob_phi);
#define GDF_GROUP(L, F)                                                                     \
  if (s.levels == L && s.features == F) {                                                   \
    if (wgs == 4)                                                                           \
      return s.linear ? fused_l<L, F, true, 4>(s.bf16, p, smem, num_sms, st)               \
                      : fused_l<L, F, false, 4>(s.bf16, p, smem, num_sms, st);             \
    return s.linear ? fused_l<L, F, true, 2>(s.bf16, p, smem, num_sms, st)                 \
                    : fused_l<L, F, false, 2>(s.bf16, p, smem, num_sms, st);               \
  }
  GDF_GROUP(8, 2)
  GDF_GROUP(16, 2)
  GDF_GROUP(8, 4)
#undef GDF_GROUP
  return cudaErrorNotSupported;
}

}  // namespace gdf
