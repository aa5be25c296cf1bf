// paths_kernels.h -- host-side declarations of the record producers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../../include/gdf.h"

namespace gdf {

enum RecordKind : int {
  kRecordsDf = 0,          // generate_training_data_AR (train.cu:6-96)
  kRecordsNrcTrain = 1,    // generate_training_data_nrc_with_inference (train.cu:156-214)
  kRecordsNrcQuery = 2,    // generate_NRCinput_from_training_data (train.cu:216-262)
};

constexpr int kProduceBlock = 128;

// One record-production pass over the training pixels of a frame. List A
// holds DF records (in_a0/in_a1/in_a2 = GuidedInput, GuidedInputPhi,
// GuidedOutput) or NRC query rows (in_a0 = GuidedInputNRC, depth/pixel);
// list B holds NRC training rows (in_b0 = GuidedInputNRC, in_b1 = RGB).
struct ProduceParams {
  gdf_path_state st;
  gdf_aabb aabb;
  int64_t n_train;          // training pixels
  uint32_t offset, stride;  // pixel = offset + i * stride
  int32_t bins_theta;       // N_DIM_OUTPUT (phi-input theta quantisation)
  int32_t linear;           // AR_LINEAR_INTERPOLATION
  // scratch, n_blocks = ceil(n_train / kProduceBlock)
  uint16_t* mask;           // [n_train] bits 0-4 list A, 8-12 list B
  int32_t* block_counts;    // [n_blocks x 2]
  int64_t* block_offsets;   // [n_blocks x 2]
  int64_t* totals;          // [2]
  // outputs
  float* out_a0;
  float* out_a1;
  float* out_a2;
  int32_t* a_depth;
  int32_t* a_pixel;
  int64_t cap_a;
  float* out_b0;
  float* out_b1;
  int64_t cap_b;
};

inline int64_t produce_blocks(int64_t n_train) {
  return (n_train + kProduceBlock - 1) / kProduceBlock;
}

// mask -> block scan -> emit; totals[] hold the full counts afterwards.
cudaError_t launch_produce(const ProduceParams& p, int kind, cudaStream_t st);

// The frame-level batch plan of LearnedDistribution::trainStep
// (learnedDistribution.cpp:226-236) from the record count on the device:
// plan[0] = batches = min(count / bs + 1, per_frame); plan[1 + i] = the
// records of batch i (min(count - i bs, bs) rounded down to 128), or 0 from
// the first batch below min_batch on (the loop's break). Zeroes loss_acc.
cudaError_t launch_df_batch_plan(const int64_t* count, int64_t bs, int32_t per_frame, int64_t min_batch,
                                 int64_t* plan, double* loss_acc, cudaStream_t st);
// loss_out = loss_acc / batches (0 without batches), n_out = count.
cudaError_t launch_df_frame_finish(const int64_t* plan, const double* loss_acc, const int64_t* count,
                                   float* loss_out, int64_t* n_out, cudaStream_t st);

// generate_inference_data_AR (train.cu:334-362) alone.
cudaError_t launch_prepare_queries(const gdf_shading& s, const gdf_aabb& aabb, float* queries,
                                   int64_t n, cudaStream_t st);

// apply_NRCoutput_to_training_data then divide_training_data_by_NRCoutput
// (train.cu:265-308), one launch each.
cudaError_t launch_apply_nrc(const gdf_path_state& st, const float* nrc_out, const int32_t* depth,
                             const int32_t* pixel, int64_t m, cudaStream_t s);

}  // namespace gdf
