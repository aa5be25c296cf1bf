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
#include "launch_util.h"

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
  // GuidedOutput::bsdfVal stays as value-initialised (train.cu:21 never
  // assigns it; bsdfVal enters only through L above)
#pragma unroll
  for (int c = 0; c < 3; ++c) out[6 + c] = 0.0f;
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

// A direction stored as (theta, phi) turns into a NaN through
// sphericalToCartesian exactly when an angle is NaN or infinite (sin and cos
// of finite floats are finite, and the unit-sphere maps that follow keep
// finite vectors finite), so the validity tests of the producers need no
// trigonometry: they test the stored angles.
__device__ __forceinline__ bool angles_ok(const float* a, uint32_t p) {
  return isfinite(a[2ull * p]) & isfinite(a[2ull * p + 1]);
}

__device__ __forceinline__ bool position_ok(const gdf_record_fields& r, uint32_t p, const rec::SceneFrame& f) {
  float v[3], o[3];
  load3(r.pos, p, v);
  rec::normalize_spatial(v, f, o);
  return !rec::any_nan(o, 3);
}

// The depths of one pixel that emit a record (bits 0-4: list A, 8-12: list
// B); the same decisions as df_record / nrc_input / nrc_target make. Every
// visited depth's fields are read whatever its delta / miss flags, so the
// loads of all depths go out together instead of one flag round trip
// before each depth's fields.
template <int KIND>
__device__ __forceinline__ uint32_t pixel_mask(const ProduceParams& P, uint32_t p, int depth,
                                               const rec::SceneFrame& f) {
  uint32_t mask = 0;
  const int dmax = depth < GDF_MAX_TRAIN_DEPTH ? depth : GDF_MAX_TRAIN_DEPTH;
#pragma unroll
  for (int d = 0; d < GDF_MAX_TRAIN_DEPTH; ++d) {
    if (d >= dmax) break;
    const gdf_record_fields& r = P.st.depth[d];
    const bool skip = r.delta[p] != 0;
    if constexpr (KIND == kRecordsDf) {
      // train.cu:77-81: pos, wi, wo direction, wiPdf, L / thp * misWeight
      float L[3];
      local_radiance(r, p, L);
      const float wi_pdf = r.wi_pdf[p];
      // & rather than &&: every term is evaluated, so no load waits on another
      const bool ok = position_ok(r, p, f) & angles_ok(r.dir, p) & angles_ok(r.wo, p) &
                      !isnan(wi_pdf) & (wi_pdf != 0.0f) & !rec::any_nan(L, 3);
      if (ok && !skip) mask |= 1u << d;
    } else {
      bool ok = !skip & (r.miss[p] == 0);
      ok &= position_ok(r, p, f) & angles_ok(r.wo, p);
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

// Words staged per record: DF [GuidedInput 9 | theta 1 | GuidedOutput 9]
// (GuidedInputPhi is the first 10); NRC list A [GuidedInputNRC 15 | depth | pixel], list B
// [GuidedInputNRC 15 | RGB 3].
template <int KIND> struct Stage;
// DF: [in (9) | theta of the phi record (1) | out (9)]; the phi record is
// words 0..9, the theta input's 9 words plus its theta
template <> struct Stage<kRecordsDf> { static constexpr int A = 19, B = 0; };
template <> struct Stage<kRecordsNrcTrain> { static constexpr int A = 17, B = 18; };
template <> struct Stage<kRecordsNrcQuery> { static constexpr int A = 17, B = 0; };
// Staged records per warp: 32 pixels average about 2.3 records each with a
// 0.7 survival per bounce, so 80 slots hold most warps' records; records
// past slot 80 are written straight to memory. Fewer slots than that would
// not raise occupancy (registers then allow 9 blocks per SM, as the staging
// does at 80); 96 slots allowed 7 (a 1080p frame: 0.71 ms, 0.64 ms at 80).
constexpr int kWarpRecords = 80;

template <int KIND>
constexpr size_t emit_smem_bytes() {
  return static_cast<size_t>(kProduceBlock / 32) * kWarpRecords * (Stage<KIND>::A + Stage<KIND>::B) * 4u;
}

// Warp-cooperative copy of `words` staged words per record (stride `stride`
// words, starting at word `first`) of records [0, n) to out + (base + r) * words:
// the destination range is contiguous, so lane l writes words l, l + 32, ...
template <typename T>
__device__ __forceinline__ void warp_copy(const uint32_t* stage, int stride, int first, int words, int n,
                                          int64_t base, int64_t cap, T* out, int lane) {
  if (out == nullptr) return;
  for (int w = lane; w < n * words; w += 32) {
    const int r = w / words, k = w - r * words;
    if (base + r < cap) out[(base + r) * words + k] = __uint_as_float(stage[r * stride + first + k]);
  }
}
__device__ __forceinline__ void warp_copy_i(const uint32_t* stage, int stride, int first, int n, int64_t base,
                                            int64_t cap, int32_t* out, int lane) {
  if (out == nullptr) return;
  for (int r = lane; r < n; r += 32)
    if (base + r < cap) out[base + r] = static_cast<int32_t>(stage[r * stride + first]);
}

// Writes each record of this block's pixels. A warp's records are
// contiguous in every output (pixel, then depth order), so they are staged
// in shared memory and copied out with consecutive lanes on consecutive
// words instead of scattered per-thread 36- to 60-byte rows.
template <int KIND>
__global__ void __launch_bounds__(kProduceBlock) produce_emit_kernel(const __grid_constant__ ProduceParams P) {
  constexpr int SA = Stage<KIND>::A, SB = Stage<KIND>::B;
  extern __shared__ uint32_t stage[];
  __shared__ int2 warp_sums[kProduceBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kProduceBlock + threadIdx.x;
  const uint32_t mask = i < P.n_train ? P.mask[i] : 0u;
  const int2 ca = make_int2(__popc(mask & 0xffu), __popc(mask >> 8));
  // warp-inclusive scan, then the warp's base within the block
  int2 inc = ca;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ax = __shfl_up_sync(0xffffffffu, inc.x, o);
    const int ay = __shfl_up_sync(0xffffffffu, inc.y, o);
    if (lane >= o) { inc.x += ax; inc.y += ay; }
  }
  const int2 wtot = make_int2(__shfl_sync(0xffffffffu, inc.x, 31), __shfl_sync(0xffffffffu, inc.y, 31));
  if (lane == 31) warp_sums[warp] = wtot;
  __syncthreads();
  int64_t base_a = P.block_offsets[2 * blockIdx.x], base_b = P.block_offsets[2 * blockIdx.x + 1];
  for (int w = 0; w < warp; ++w) { base_a += warp_sums[w].x; base_b += warp_sums[w].y; }
  uint32_t* sa = stage + static_cast<size_t>(warp) * kWarpRecords * (SA + SB);
  uint32_t* sb = sa + kWarpRecords * SA;
  int ra = inc.x - ca.x, rb = inc.y - ca.y;  // this thread's first slot in the warp
  if (i < P.n_train) {
    const uint32_t p = P.offset + static_cast<uint32_t>(i) * P.stride;
    const rec::SceneFrame f = rec::scene_frame(P.aabb);
    for (int d = 0; d < GDF_MAX_TRAIN_DEPTH; ++d) {
      const bool in_a = (mask >> d) & 1u, in_b = (mask >> (8 + d)) & 1u;
      if (!in_a && !in_b) continue;
      const gdf_record_fields& r = P.st.depth[d];
      if constexpr (KIND == kRecordsDf) {
        float in[9], pt, out[9];
        df_record(r, p, f, P.bins_theta, P.linear != 0, in, pt, out);
        if (ra < kWarpRecords) {
          uint32_t* o = sa + ra * SA;
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            o[k] = __float_as_uint(in[k]);
            o[10 + k] = __float_as_uint(out[k]);
          }
          o[9] = __float_as_uint(pt);
        } else if (base_a + ra < P.cap_a) {
          const int64_t g = base_a + ra;
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            P.out_a0[g * 9 + k] = in[k];
            P.out_a1[g * 10 + k] = in[k];
            P.out_a2[g * 9 + k] = out[k];
          }
          P.out_a1[g * 10 + 9] = pt;
        }
        ++ra;
      } else {
        float in[15];
        nrc_input(r, p, f, in);
        if (in_a) {
          if (ra < kWarpRecords) {
            uint32_t* o = sa + ra * SA;
#pragma unroll
            for (int k = 0; k < 15; ++k) o[k] = __float_as_uint(in[k]);
            o[15] = static_cast<uint32_t>(d);
            o[16] = p;
          } else if (base_a + ra < P.cap_a) {
            const int64_t g = base_a + ra;
#pragma unroll
            for (int k = 0; k < 15; ++k) P.out_a0[g * 15 + k] = in[k];
            P.a_depth[g] = d;
            P.a_pixel[g] = static_cast<int32_t>(p);
          }
          ++ra;
        }
        if (KIND == kRecordsNrcTrain && in_b) {
          float L[3];
          nrc_target(r, p, L);
          if (rb < kWarpRecords) {
            uint32_t* o = sb + rb * SB;
#pragma unroll
            for (int k = 0; k < 15; ++k) o[k] = __float_as_uint(in[k]);
#pragma unroll
            for (int k = 0; k < 3; ++k) o[15 + k] = __float_as_uint(L[k]);
          } else if (base_b + rb < P.cap_b) {
            const int64_t g = base_b + rb;
#pragma unroll
            for (int k = 0; k < 15; ++k) P.out_b0[g * 15 + k] = in[k];
#pragma unroll
            for (int k = 0; k < 3; ++k) P.out_b1[g * 3 + k] = L[k];
          }
          ++rb;
        }
      }
    }
    // generate_training_data_nrc_with_inference / generate_NRCinput_from_
    // training_data end with curDepth-- (train.cu:213, 261), unsigned.
    if constexpr (KIND != kRecordsDf) P.st.cur_depth[p] = P.st.cur_depth[p] - 1u;
  }
  __syncwarp();
  const int na = wtot.x < kWarpRecords ? wtot.x : kWarpRecords;
  const int nb = wtot.y < kWarpRecords ? wtot.y : kWarpRecords;
  if constexpr (KIND == kRecordsDf) {
    warp_copy(sa, SA, 0, 9, na, base_a, P.cap_a, P.out_a0, lane);
    warp_copy(sa, SA, 0, 10, na, base_a, P.cap_a, P.out_a1, lane);
    warp_copy(sa, SA, 10, 9, na, base_a, P.cap_a, P.out_a2, lane);
  } else {
    warp_copy(sa, SA, 0, 15, na, base_a, P.cap_a, P.out_a0, lane);
    warp_copy_i(sa, SA, 15, na, base_a, P.cap_a, P.a_depth, lane);
    warp_copy_i(sa, SA, 16, na, base_a, P.cap_a, P.a_pixel, lane);
    if constexpr (KIND == kRecordsNrcTrain) {
      warp_copy(sb, SB, 0, 15, nb, base_b, P.cap_b, P.out_b0, lane);
      warp_copy(sb, SB, 15, 3, nb, base_b, P.cap_b, P.out_b1, lane);
    }
  }
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
  constexpr size_t smem = emit_smem_bytes<KIND>();
  cudaError_t e = allow_dynamic_smem(produce_emit_kernel<KIND>);
  if (e != cudaSuccess) return e;
  produce_emit_kernel<KIND><<<static_cast<unsigned>(nb), kProduceBlock, smem, st>>>(p);
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

namespace {

__global__ void df_batch_plan_kernel(const int64_t* count, int64_t bs, int32_t per_frame, int64_t min_batch,
                                     int64_t* plan, double* loss_acc) {
  const int64_t n = *count;
  const int64_t batches = min(n / bs + 1, static_cast<int64_t>(per_frame));
  plan[0] = batches;
  bool stop = false;
  for (int32_t i = 0; i < per_frame; ++i) {
    int64_t local = i < batches ? min(n - i * bs, bs) : 0;
    local -= local % 128;
    if (stop || local < min_batch) {
      stop = true;
      local = 0;
    }
    plan[1 + i] = local;
  }
  *loss_acc = 0.0;
}

__global__ void df_frame_finish_kernel(const int64_t* plan, const double* loss_acc, const int64_t* count,
                                       float* loss_out, int64_t* n_out) {
  const int64_t batches = plan[0];
  if (loss_out) *loss_out = batches > 0 ? static_cast<float>(*loss_acc / static_cast<double>(batches)) : 0.f;
  if (n_out) *n_out = *count;
}

}  // namespace

cudaError_t launch_df_batch_plan(const int64_t* count, int64_t bs, int32_t per_frame, int64_t min_batch,
                                 int64_t* plan, double* loss_acc, cudaStream_t st) {
  df_batch_plan_kernel<<<1, 1, 0, st>>>(count, bs, per_frame, min_batch, plan, loss_acc);
  return cudaGetLastError();
}

cudaError_t launch_df_frame_finish(const int64_t* plan, const double* loss_acc, const int64_t* count,
                                   float* loss_out, int64_t* n_out, cudaStream_t st) {
  df_frame_finish_kernel<<<1, 1, 0, st>>>(plan, loss_acc, count, loss_out, n_out);
  return cudaGetLastError();
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
