// nrc_kernels.h -- host-side declarations of the NRC kernels.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace gdf {

struct NrcParams {
  const float* in;       // m x 15 GuidedInputNRC
  float* out;            // m x 3 RGB
  int64_t n;
  const __half* blob;    // fp16 weights (EMA copy), canonical layout
  uint32_t blob_bytes;
  int32_t hidden;        // tcnn n_hidden_layers
  uint32_t* err;
};

struct NrcTrainParams {
  const float* in;       // m x 15
  const float* target;   // m x 3
  int64_t n;
  const __half* blob;    // fp16 training weights, canonical layout
  uint32_t blob_bytes;
  int32_t hidden;
  float* wgrad_partial;  // [gridDim.x][n_mlp]
  int64_t n_mlp;
  float loss_scale;      // TRAIN_LOSS_SCALE_NRC
  float n_total;         // 3 m (RelativeL2Luminance normalisation)
  float* loss_out;       // m x 4, column 3 = per-record loss value
  unsigned long long* n_dropped;
  uint32_t* err;
};

cudaError_t launch_nrc_query(const NrcParams& p, int num_sms, cudaStream_t st);
cudaError_t launch_nrc_train_bwd(const NrcTrainParams& p, int ctas, cudaStream_t st);

}  // namespace gdf
