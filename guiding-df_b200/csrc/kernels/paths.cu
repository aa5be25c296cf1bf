// paths.cu -- training records from the path tracer's per-pixel vertex
// records, and the NRC target substitution.
//
// The reference appends records with an atomic counter
// (TrainBuffer::push, train.h:20-70), so their order changes from run to
// run. Here a pass counts each training pixel's records (a 16-bit mask of
// the depths it emits), a single-block scan turns the per-block counts into
// offsets, and a second pass writes every record at its place: records come
// out ordered by training pixel, then depth, and the producers are
// deterministic. All passes read the per-depth record arrays with unit
// stride across threads (stride 1 pixels) and are bandwidth bound.
#include <cuda_runtime.h>

#include "../device/records.cuh"
#include "paths_kernels.h"

namespace gdf {
namespace {

using rec::kEpsilon;
constexpr int kScanThreads = 1024;

__device__ __forceinline__ void load3(const float* a, uint32_t p, float v[3]) {
  v[0] = a[3ull * p];
  v[1] = a[3ull * p + 1];
  v[2] = a[3ull * p + 2];
}

// L / thp per channel where thp > M_EPSILON, times misWeight
// (train.cu:61-67, 188-194).
__device__ __forceinline__ void local_radiance(const gdf_record_fields& r, uint32_t p, float L[3]) {
  float l[3], t[3];
  load3(r.L, p, l);
  load3(r.thp, p, t);
  const float mis = r.mis_weight[p];
#pragma unroll
  for (int c = 0; c < 3; ++c) L[c] = (t[c] > kEpsilon ? l[c] / t[c] : 0.0f) * mis;
}

// GuidedInput / GuidedInputPhi / GuidedOutput of one vertex
// (generate_training_data_AR, train.cu:22-81). Returns the validity test of
// train.cu:77-81.
__device__ __forceinline__ bool df_record(const gdf_record_fields& r, uint32_t p,
                                          const rec::SceneFrame& f, int bins, bool linear,
                                          float in[9], float& phi_theta, float out[9]) {
  float v[3];
  load3(r.pos, p, v);
  rec::normalize_spatial(v, f, in);
  rec::spherical_to_cartesian(r.wo[2ull * p], r.wo[2ull * p + 1], v);
  rec::warp_direction_for_sh(v, in + 3);
  in[6] = r.normal[2ull * p] * rec::kInvPi;
  in[7] = r.normal[2ull * p + 1] * rec::kInv2Pi;
  in[8] = rec::warp_roughness_for_ob(r.roughness[p]);
  float wi[2];
  rec::spherical_to_cartesian(r.dir[2ull * p], r.dir[2ull * p + 1], v);
  rec::uniform_sphere_to_square(v, wi);
  const float nb = static_cast<float>(bins);
  int fl = static_cast<int>(floorf(wi[0] * nb));
  fl = fl < bins - 1 ? fl : bins - 1;  // safe_floor (train.h:650-652)
  if (linear) {
    const float w = wi[0] * nb - static_cast<float>(fl);
    phi_theta = (static_cast<float>(fl) + w) / nb;
  } else {
    phi_theta = static_cast<float>(fl) / nb;
  }
  float L[3];
  local_radiance(r, p, L);
  float bv[3];
  load3(r.bsdf_val, p, bv);
  const float wi_pdf = r.wi_pdf[p];
  out[0] = wi[0];
  out[1] = wi[1];
#pragma unroll
  for (int c = 0; c < 3; ++c) out[2 + c] = L[c] * bv[c];
  out[5] = wi_pdf;
#pragma unroll
  for (int c = 0; c < 3; ++c) out[6 + c] = bv[c];
  return !(rec::any_nan(in, 3) || rec::any_nan(wi, 2) || rec::any_nan(in + 3, 3) ||
           isnan(wi_pdf) || wi_pdf == 0.0f || rec::any_nan(L, 3));
}

// GuidedInputNRC of one vertex (train.cu:173-186); target = the local
// radiance times bsdfVal over (wiPdf + M_EPSILON) (train.cu:188-197).
__device__ __forceinline__ void nrc_input(const gdf_record_fields& r, uint32_t p,
                                          const rec::SceneFrame& f, float in[15]) {
  float v[3];
  load3(r.pos, p, v);
  rec::normalize_spatial(v, f, in);
  rec::spherical_to_cartesian(r.wo[2ull * p], r.wo[2ull * p + 1], v);
  rec::warp_direction_for_sh(v, in + 3);
  in[6] = r.normal[2ull * p] * rec::kInvPi;
  in[7] = r.normal[2ull * p + 1] * rec::kInv2Pi;
  in[8] = rec::warp_roughness_for_ob(r.roughness[p]);
  load3(r.diffuse, p, in + 9);
  load3(r.specular, p, in + 12);
}

__device__ __forceinline__ void nrc_target(const gdf_record_fields& r, uint32_t p, float L[3]) {
  local_radiance(r, p, L);
  float bv[3];
  load3(r.bsdf_val, p, bv);
  const float den = r.wi_pdf[p] + kEpsilon;
#pragma unroll
  for (int c = 0; c < 3; ++c) L[c] = L[c] * bv[c] / den;
}

template <int KIND>
__device__ __forceinline__ uint32_t pixel_mask(const ProduceParams& P, uint32_t p, int depth,
                                               const rec::SceneFrame& f) {
  uint32_t mask = 0;
  const int dmax = depth < GDF_MAX_TRAIN_DEPTH ? depth : GDF_MAX_TRAIN_DEPTH;
  for (int d = 0; d < dmax; ++d) {
    const gdf_record_fields& r = P.st.depth[d];
    if (r.delta[p]) continue;
    if constexpr (KIND == kRecordsDf) {
      float in[9], pt, out[9];
      if (df_record(r, p, f, P.bins_theta, P.linear != 0, in, pt, out)) mask |= 1u << d;
    } else {
      if (r.miss[p]) continue;
      float in[15];
      nrc_input(r, p, f, in);
      bool ok = !(rec::any_nan(in, 3) || rec::any_nan(in + 3, 3));
      if constexpr (KIND == kRecordsNrcTrain) {
        float L[3];
        nrc_target(r, p, L);
        ok &= !rec::any_nan(L, 3);
        if (ok && d < depth - 1) mask |= 1u << (8 + d);
      }
      if (ok) mask |= 1u << d;
    }
  }
  return mask;
}

// Block-wide inclusive sum of two counters (blockDim.x == kProduceBlock).
__device__ __forceinline__ int2 block_inclusive(int2 v, int2* warp_sums, int2* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ax = __shfl_up_sync(0xffffffffu, v.x, o);
    const int ay = __shfl_up_sync(0xffffffffu, v.y, o);
    if (lane >= o) { v.x += ax; v.y += ay; }
  }
  if (lane == 31) warp_sums[warp] = v;
  __syncthreads();
  int2 base = make_int2(0, 0);
  for (int w = 0; w < warp; ++w) { base.x += warp_sums[w].x; base.y += warp_sums[w].y; }
  if (total) {
    int2 t = make_int2(0, 0);
    for (int w = 0; w < kProduceBlock / 32; ++w) { t.x += warp_sums[w].x; t.y += warp_sums[w].y; }
    *total = t;
  }
  return make_int2(base.x + v.x, base.y + v.y);
}

template <int KIND>
__global__ void __launch_bounds__(kProduceBlock) produce_mask_kernel(const __grid_constant__ ProduceParams P) {
  __shared__ int2 warp_sums[kProduceBlock / 32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kProduceBlock + threadIdx.x;
  uint32_t mask = 0;
  if (i < P.n_train) {
    const uint32_t p = P.offset + static_cast<uint32_t>(i) * P.stride;
    const rec::SceneFrame f = rec::scene_frame(P.aabb);
    mask = pixel_mask<KIND>(P, p, static_cast<int>(P.st.cur_depth[p]), f);
    P.mask[i] = static_cast<uint16_t>(mask);
  }
  int2 total;
  block_inclusive(make_int2(__popc(mask & 0xffu), __popc(mask >> 8)), warp_sums, &total);
  if (threadIdx.x == 0) {
    P.block_counts[2 * blockIdx.x] = total.x;
    P.block_counts[2 * blockIdx.x + 1] = total.y;
  }
}

// Exclusive scan of the per-block counts by one block of kScanThreads.
__global__ void __launch_bounds__(kScanThreads) scan_blocks_kernel(const int32_t* __restrict__ counts,
                                                                  int64_t* __restrict__ offsets,
                                                                  int64_t* __restrict__ totals,
                                                                  int64_t n_blocks) {
  __shared__ long long sa[kScanThreads], sb[kScanThreads];
  const int t = threadIdx.x;
  const int64_t chunk = (n_blocks + kScanThreads - 1) / kScanThreads;
  const int64_t b0 = t * chunk, b1 = b0 + chunk < n_blocks ? b0 + chunk : n_blocks;
  long long a = 0, b = 0;
  for (int64_t k = b0; k < b1; ++k) { a += counts[2 * k]; b += counts[2 * k + 1]; }
  sa[t] = a;
  sb[t] = b;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {  // Hillis-Steele inclusive scan
    long long xa = 0, xb = 0;
    if (t >= o) { xa = sa[t - o]; xb = sb[t - o]; }
    __syncthreads();
    sa[t] += xa;
    sb[t] += xb;
    __syncthreads();
  }
  long long ea = sa[t] - a, eb = sb[t] - b;
  for (int64_t k = b0; k < b1; ++k) {
    offsets[2 * k] = ea;
    offsets[2 * k + 1] = eb;
    ea += counts[2 * k];
    eb += counts[2 * k + 1];
  }
  if (t == kScanThreads - 1) {
    totals[0] = sa[t];
    totals[1] = sb[t];
  }
}

template <int KIND>
__global__ void __launch_bounds__(kProduceBlock) produce_emit_kernel(const __grid_constant__ ProduceParams P) {
  __shared__ int2 warp_sums[kProduceBlock / 32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kProduceBlock + threadIdx.x;
  const uint32_t mask = i < P.n_train ? P.mask[i] : 0u;
  const int2 ca = make_int2(__popc(mask & 0xffu), __popc(mask >> 8));
  const int2 inc = block_inclusive(ca, warp_sums, nullptr);
  if (i >= P.n_train) return;
  int64_t ia = P.block_offsets[2 * blockIdx.x] + inc.x - ca.x;
  int64_t ib = P.block_offsets[2 * blockIdx.x + 1] + inc.y - ca.y;
  const uint32_t p = P.offset + static_cast<uint32_t>(i) * P.stride;
  const rec::SceneFrame f = rec::scene_frame(P.aabb);
  for (int d = 0; d < GDF_MAX_TRAIN_DEPTH; ++d) {
    const bool in_a = (mask >> d) & 1u, in_b = (mask >> (8 + d)) & 1u;
    if (!in_a && !in_b) continue;
    const gdf_record_fields& r = P.st.depth[d];
    if constexpr (KIND == kRecordsDf) {
      float in[9], pt, out[9];
      df_record(r, p, f, P.bins_theta, P.linear != 0, in, pt, out);
      if (ia < P.cap_a) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          P.out_a0[ia * 9 + k] = in[k];
          P.out_a1[ia * 10 + k] = in[k];
          P.out_a2[ia * 9 + k] = out[k];
        }
        P.out_a1[ia * 10 + 9] = pt;
      }
      ++ia;
    } else {
      float in[15];
      nrc_input(r, p, f, in);
      if (in_a) {
        if (ia < P.cap_a) {
#pragma unroll
          for (int k = 0; k < 15; ++k) P.out_a0[ia * 15 + k] = in[k];
          P.a_depth[ia] = d;
          P.a_pixel[ia] = static_cast<int32_t>(p);
        }
        ++ia;
      }
      if (KIND == kRecordsNrcTrain && in_b) {
        float L[3];
        nrc_target(r, p, L);
        if (ib < P.cap_b) {
#pragma unroll
          for (int k = 0; k < 15; ++k) P.out_b0[ib * 15 + k] = in[k];
#pragma unroll
          for (int k = 0; k < 3; ++k) P.out_b1[ib * 3 + k] = L[k];
        }
        ++ib;
      }
    }
  }
  // generate_training_data_nrc_with_inference / generate_NRCinput_from_
  // training_data end with curDepth-- (train.cu:213, 261), unsigned.
  if constexpr (KIND != kRecordsDf) P.st.cur_depth[p] = P.st.cur_depth[p] - 1u;
}

__global__ void prepare_queries_kernel(const gdf_shading s, const gdf_aabb aabb,
                                       float* __restrict__ q, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rec::SceneFrame f = rec::scene_frame(aabb);
  float pos[3], wo[3], nrm[3], row[9];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pos[k] = s.pos[i * 3 + k];
    wo[k] = s.wo[i * 3 + k];
    nrm[k] = s.normal[i * 3 + k];
  }
  rec::shading_to_query(pos, wo, nrm, s.roughness[i], f, row);
#pragma unroll
  for (int k = 0; k < 9; ++k) q[i * 9 + k] = row[k];
}

__device__ __forceinline__ bool valid_record(const gdf_path_state& st, int p, int depth) {
  return depth >= 0 && depth < GDF_MAX_TRAIN_DEPTH &&
         static_cast<uint32_t>(depth) < st.cur_depth[p];  // isValidRecord (workqueue.h:100-102)
}

// replaceIndirectRadianceSkipDelta (workqueue.h:122-129) at depth-1.
__global__ void apply_nrc_kernel(const gdf_path_state st, const float* __restrict__ out,
                                 const int32_t* __restrict__ depth, const int32_t* __restrict__ pixel,
                                 int64_t m) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int p = pixel[i];
  const int initial = depth[i] - 1;
  if (initial >= GDF_MAX_TRAIN_DEPTH) return;  // outside the record arrays
  int d = initial;
  while (d >= 0 && st.depth[d].delta[p]) --d;
  if (!valid_record(st, p, d)) return;
  const gdf_record_fields& ri = st.depth[initial];
  float* L = st.depth[d].L + 3ll * p;
#pragma unroll
  for (int c = 0; c < 3; ++c) L[c] = ri.thp[3ll * p + c] * (out[3 * i + c] + ri.Le[3ll * p + c]);
}

// divideRadiance (workqueue.h:104-111) at depth.
__global__ void divide_nrc_kernel(const gdf_path_state st, const float* __restrict__ out,
                                  const int32_t* __restrict__ depth, const int32_t* __restrict__ pixel,
                                  int64_t m) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int p = pixel[i];
  const int d = depth[i];
  if (!valid_record(st, p, d)) return;
  float* L = st.depth[d].L + 3ll * p;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float o = out[3 * i + c];
    if (o > kEpsilon) L[c] = L[c] / o;
  }
}

template <int KIND>
cudaError_t produce(const ProduceParams& p, cudaStream_t st) {
  const int64_t nb = produce_blocks(p.n_train);
  if (nb == 0) return cudaMemsetAsync(p.totals, 0, 2 * sizeof(int64_t), st);
  produce_mask_kernel<KIND><<<static_cast<unsigned>(nb), kProduceBlock, 0, st>>>(p);
  scan_blocks_kernel<<<1, kScanThreads, 0, st>>>(p.block_counts, p.block_offsets, p.totals, nb);
  produce_emit_kernel<KIND><<<static_cast<unsigned>(nb), kProduceBlock, 0, st>>>(p);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_produce(const ProduceParams& p, int kind, cudaStream_t st) {
  switch (kind) {
    case kRecordsDf: return produce<kRecordsDf>(p, st);
    case kRecordsNrcTrain: return produce<kRecordsNrcTrain>(p, st);
    case kRecordsNrcQuery: return produce<kRecordsNrcQuery>(p, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_prepare_queries(const gdf_shading& s, const gdf_aabb& aabb, float* queries,
                                   int64_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  prepare_queries_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(s, aabb, queries, n);
  return cudaGetLastError();
}

cudaError_t launch_apply_nrc(const gdf_path_state& st, const float* nrc_out, const int32_t* depth,
                             const int32_t* pixel, int64_t m, cudaStream_t s) {
  if (m == 0) return cudaSuccess;
  const unsigned g = static_cast<unsigned>((m + 255) / 256);
  apply_nrc_kernel<<<g, 256, 0, s>>>(st, nrc_out, depth, pixel, m);
  divide_nrc_kernel<<<g, 256, 0, s>>>(st, nrc_out, depth, pixel, m);
  return cudaGetLastError();
}

}  // namespace gdf
