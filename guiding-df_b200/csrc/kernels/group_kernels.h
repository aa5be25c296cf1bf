// group_kernels.h -- host-side declarations of the grouped (multi-job) DF inference.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../device/grid_levels.h"
#include "df_kernels.h"

namespace gdf {

// One job of a grouped launch, in device memory: its networks (the
// inference weight blobs and interleaved grid of its context), its inputs
// and outputs, and where its tiles sit in the launch.
struct GroupJobDev {
  const __half* blob_theta;
  const __half* blob_phi;
  uint32_t blob_theta_bytes, blob_phi_bytes;
  int32_t hidden_theta, hidden_phi;
  int32_t bins_theta, bins_phi;      // 16, 32 or 64 each
  const __half* grid_il;             // [entries][theta F | phi F]
  const float* queries;              // n x 9
  const uint8_t* guided;             // nullable
  const float* uniforms;             // nullable -> Philox(seed) at (row, offset)
  float* wi;                         // n x 4 in/out
  int64_t n;
  uint64_t seed, offset;
  int64_t tile_begin;                // first tile in the launch's feature buffer
  int64_t super_begin;               // first super-tile (WGS consecutive tiles)
};

struct GroupHeader {
  int32_t n_jobs;
  uint32_t seq;              // this call's sequence number (job completion flags)
  int64_t total_tiles;
  int64_t n_super;
  uint32_t track;            // report each job's completion (job_flag)
  uint32_t pad;
};

// Kernel parameters: fixed for a captured graph; the job set is read from
// device memory (hdr, jobs), so one graph serves any job set that fits.
struct GroupParams {
  const GroupHeader* hdr;
  const GroupJobDev* jobs;
  __half* feat_theta;                // [tile capacity][128 x L*F]
  __half* feat_phi;
  GridLevels gl;                     // the grid configuration all jobs share
  uint32_t max_blob_theta, max_blob_phi;
  uint32_t* err;
  // per-job completion: warps of 32 rows done (device, zeroed before each
  // launch) and the call's sequence number stored when a job's last one is
  // written
  // (host-mapped, so the host sees a job finish before the launch ends)
  uint32_t* job_tiles_done;
  uint32_t* job_flag;
};

struct GroupShape {
  int levels, features;
  bool linear, bf16;
};

bool group_shape_supported(const GroupShape& s);
// Grid features of every job's rows: one thread per 16-byte chunk (8 / F
// levels) of a row, so blocks * block_threads must equal the header's
// total_tiles * 128 * (levels * features / 8).
cudaError_t launch_group_features(const GroupShape& s, const GroupParams& p, int blocks, int block_threads,
                                  cudaStream_t st);
// The grouped fused kernel: wgs warpgroups per CTA (2 or 4), one CTA per SM.
cudaError_t launch_group_fused(const GroupShape& s, int wgs, const GroupParams& p, int num_sms,
                               cudaStream_t st);
size_t group_fused_smem_bytes(const GroupShape& s, int wgs, uint32_t max_blob_theta, uint32_t max_blob_phi);

}  // namespace gdf
