// df_kernels.h -- host-side declarations of the DF / NRC kernel launchers.
// Parameter structs are plain data shared by host and device code.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../../include/gdf.h"
#include "../device/grid_levels.h"

namespace gdf {

// Warpgroups (128-row tiles in flight) per CTA of the fused DF kernel.
constexpr int kDfWarpgroups = 4;
constexpr int kDfThreads = 128 * kDfWarpgroups;

// kModeTrainFwd gathers the grid features in the kernel (gdf_train_loss_static);
// kModeTrainFeat reads them from launch_train_features' tiles (the training step).
enum DfMode : int { kModeInfer = 0, kModeEval = 1, kModeTrainFwd = 2, kModeTrainFeat = 3 };

struct DfKernelParams {
  const float* queries;      // n x 9
  const uint8_t* guided;     // n, nullable
  const float* uniforms;     // n x 4, nullable -> in-kernel Philox
  float* wi;                 // n x 4 in/out (infer)
  const float* u_eval;       // n x 2 (eval)
  float* pdf_out;            // n x 2 (eval)
  int64_t n;
  uint64_t philox_seed, philox_offset;
  int64_t philox_row_base;   // Philox counter of row r is row_base + r (chunked calls)
  const __half* grid_theta;  // grid tables (entries x F halfs), inference copy
  const __half* grid_phi;
  const __half* blob_theta;  // MLP weights in the canonical tensor-core layout
  const __half* blob_phi;
  uint32_t blob_theta_bytes, blob_phi_bytes;
  int32_t hidden_theta, hidden_phi;  // tcnn n_hidden_layers
  uint32_t* err;                     // device error word
  // training forward (kModeTrainFwd)
  const float* in_phi;               // n x 10 GuidedInputPhi
  const float* target;               // n x 9 GuidedOutput
  float* train_out;                  // n x 4: pdf_theta, pdf_phi, prefix, likelihood
  unsigned long long* n_dropped;     // records rejected by the validity filter
  float loss_scale_per_record;       // TRAIN_LOSS_SCALE / n
  // training modes: when set, the batch has min(*n_dev, n) records (n is
  // then the launch's bound) and the per-record scale is loss_scale / that
  const int64_t* n_dev;
  float loss_scale;
  GridLevels gl_theta, gl_phi;
  // grid features of both networks, precomputed by launch_grid_features
  // (inference and pdf evaluation): 128-row tiles, canonical layout
  const __half* feat_theta;
  const __half* feat_phi;
  // inference options (gdf_infer_ex)
  gdf_shading shading;               // raw shading points when shading.pos != nullptr
  gdf_aabb aabb;
  float* dir_pdf;                    // n x 4 world direction + solid-angle pdf, nullable
  int32_t bf16;                      // inference form with bf16 MLP operands
  int32_t fp8;                       // FP8 inference form: blobs from launch_pack_fp8
  unsigned long long* norm_err;      // FP64 CDF normalisation check (double bits, max-merged), nullable
};

// Both networks' grid features of a training batch (launch_train_features).
struct TrainFeatParams {
  const float* in_theta;     // n x 9 GuidedInput
  const float* in_phi;       // n x 10 GuidedInputPhi
  const float* target;       // n x 9 GuidedOutput (the validity filter reads it)
  int64_t n, n_tiles;
  const int64_t* n_dev;      // nullable: min(*n_dev, n) records (n, n_tiles: the launch's bound)
  const __half* grid_theta;  // fp16 training tables
  const __half* grid_phi;
  GridLevels gl_theta, gl_phi;
  __half* feat_theta;        // [n_tiles][128 x L*F] canonical
  __half* feat_phi;
  int32_t bf16;              // features rounded to bf16 (the bf16 training form)
};

struct GridFeatParams {
  const float* queries;      // n x 9 query rows (positions in columns 0-2), or
  const float* shading_pos;  // n x 3 world positions normalised against aabb
  gdf_aabb aabb;
  int64_t n, n_tiles;        // rows, 128-row tiles written (padding rows use 0.5)
  const __half* grid_il;     // interleaved EMA tables: [entries][theta F | phi F]
  GridLevels gl;             // the grid configuration both networks share
  __half* feat_theta;        // [n_tiles][128 x L*F] canonical
  __half* feat_phi;
  int32_t bf16;              // features rounded to bf16 (bit patterns in __half storage)
};

struct DfShape {
  int levels, features, bins_theta, bins_phi;
  bool linear;
};

// Returns cudaErrorNotSupported when no kernel is built for the shape.
cudaError_t launch_df_fused(const DfShape& s, int mode, const DfKernelParams& p, int num_sms,
                            cudaStream_t stream);
size_t df_fused_smem_bytes(const DfShape& s, int mode, uint32_t blob_theta_bytes, uint32_t blob_phi_bytes);
bool df_shape_supported(const DfShape& s);

// Both grids' features for inference / pdf evaluation.
cudaError_t launch_grid_features(const DfShape& s, const GridFeatParams& p, cudaStream_t st);
cudaError_t launch_train_features(const DfShape& s, const TrainFeatParams& p, cudaStream_t st);
// (Re)builds the interleaved inference table from the two EMA grids.
cudaError_t launch_interleave_grids(const __half* theta, const __half* phi, __half* il,
                                    int64_t n_entries, int features, cudaStream_t st);

// Epilogue-only kernel (gdf_post_inference).
cudaError_t launch_df_post(int bins_theta, int bins_phi, bool linear, const float* logits_theta,
                           const float* logits_phi, const uint8_t* guided, const float* uniforms,
                           float* wi, int64_t n, cudaStream_t stream);

// Packs fp16 row-major [rows x cols] matrices into the canonical layout,
// optionally rounded to bf16 (bf16 inference form).
cudaError_t launch_pack_mlp(const __half* src, __half* dst, const int32_t* rows,
                            const int32_t* cols, int n_layers, cudaStream_t stream,
                            bool to_bf16 = false);

// FP8 inference blob of one DF network from its fp16 EMA matrices (row-major,
// back to back): matrix 0 and the last matrix fp16 in the canonical layout,
// the 64x64 hidden matrices e4m3 scaled by a power of two per matrix
// (canonical layout of 64-byte rows, 4096 bytes each), then one float
// descale per hidden matrix. fp8_blob_bytes gives the size.
constexpr int kMaxMlpLayers = 10;
struct Fp8PackParams {
  const __half* src;
  uint8_t* dst;
  int32_t n_layers;
  int32_t rows[kMaxMlpLayers], cols[kMaxMlpLayers];
  int64_t src_off[kMaxMlpLayers];
  uint32_t dst_off[kMaxMlpLayers];
  uint32_t descale_off;
};
uint32_t fp8_blob_bytes(const int32_t* rows, const int32_t* cols, int n_layers, Fp8PackParams* layout);
cudaError_t launch_pack_fp8(const Fp8PackParams& p, cudaStream_t stream);

}  // namespace gdf
