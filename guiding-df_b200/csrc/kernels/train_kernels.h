// train_kernels.h -- host-side declarations of the training kernels.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../device/grid_levels.h"
#include "df_kernels.h"

namespace gdf {

// Backward of one DF network over a batch.
struct DfBwdParams {
  const float* in;          // records of this network (stride in_stride)
  int32_t in_stride;        // 9 (theta) or 10 (phi)
  const float* target;      // n x 9 GuidedOutput
  const float* fwd;         // n x 4 from the training forward: pdf_theta, pdf_phi, prefix, likelihood
  int64_t n;
  const int64_t* n_dev;     // nullable: min(*n_dev, n) records (n: the launch's bound)
  const __half* blob;       // fp16 training weights, canonical layout
  uint32_t blob_bytes;
  const __half* grid;       // fp16 training grid tables
  const __half* feat;       // [tiles][128 x L*F] canonical grid features of the training forward
  float* dx;                // [L][dx_rows][F] dL/dgrid-features out, level-major
  int64_t dx_rows;
  float* grid_grad;         // fp32 gradient of the grid tables (zeroed by the optimizer)
  float* wgrad_partial;     // [gridDim.x][n_mlp] per-CTA weight-gradient sums
  int64_t n_mlp;
  int32_t hidden;           // tcnn n_hidden_layers
  uint32_t* err;
  GridLevels gl;
  int32_t bf16;             // bf16 training form: bf16 weight blob, features and activations
};

// Grid backward of a batch (grid_scatter_kernel): dx from the backward.
struct GridScatterParams {
  const float* in;          // records (positions in columns 0-2), stride in_stride
  int32_t in_stride;
  const float* fwd;         // n x 4 from the training forward (prefix 0: rejected record)
  int64_t n;
  const int64_t* n_dev;     // nullable: min(*n_dev, n) records (n: the launch's bound)
  const float* dx;          // [L][dx_rows][F]
  int64_t dx_rows;
  float* grid_grad;
  GridLevels gl;
};

// A network's optimizer step counter (Adam m_current_step, adam.h:150-152),
// in device memory so that a step can be skipped on the device (an empty
// batch). The optimizer kernel's blocks all read it; the last block to
// finish advances it (blocks_done counts them and is reset to 0).
struct OptState {
  uint32_t step;
  uint32_t blocks_done;
};

// Adam + EMA over one network (tcnn optimizers/adam.h, ema.h).
struct AdamParams {
  int64_t n, n_mlp;
  const float* partials;    // [n_partials][n_mlp]
  int32_t n_partials;
  float* grid_grad;         // [n - n_mlp], read then zeroed
  float* master;
  __half* w16;
  __half* ema16;
  float* m;
  float* v;
  uint32_t* step;
  __half* blob_w16;
  __half* blob_ema;
  int64_t layer_off[12];
  int32_t layer_cols[12];
  int32_t n_layers;
  float loss_scale, lr, beta1, beta2, eps, l2_reg, ema_decay;
  OptState* opt;            // the step counter, advanced by this launch
  const int64_t* n_dev;     // nullable: the step is skipped when *n_dev == 0
  double* sq_partial;       // [n_blocks]
  int32_t n_blocks;
  // interleaved inference copy of the EMA grid ([entries][theta F | phi F]),
  // nullable; this network's half is at il_net * F
  __half* grid_il;
  int32_t il_net, il_features;
  // lr sqrt(1 - beta2^k) / (1 - beta1^k) for step counters k < lr_table_n;
  // the last entry equals lr (both powers below float resolution)
  const float* lr_table;
  int32_t lr_table_n;
  bool blob_ema_bf16;       // the inference blob holds bf16 (bf16 inference form)
  bool blob_w16_bf16;       // the training blob holds bf16 (bf16 training form)
  uint32_t* err;            // device error word (bounded waits of the staged grid part)
};

cudaError_t launch_grid_scatter(int levels, int features, const GridScatterParams& p, cudaStream_t st);
cudaError_t launch_df_train_bwd(const DfShape& s, bool phi, const DfBwdParams& p, int ctas,
                                cudaStream_t st);
size_t df_train_bwd_smem_bytes(int levels, int features, bool phi, uint32_t blob_bytes, int hidden);
cudaError_t launch_adam_ema(const AdamParams& p, cudaStream_t st);
cudaError_t launch_adam_lr_table(float lr, float beta1, float beta2, float* table, int32_t n,
                                 cudaStream_t st);
// The same two sums with the loss over kStatBlocks blocks; part holds
// kStatBlocks doubles of scratch.
constexpr int kStatBlocks = 148;
// n_dev (nullable): min(*n_dev, n) records; loss_acc (nullable): += out[0] / records, if any.
cudaError_t launch_train_stats_mb(const float* fwd, int64_t n, const int64_t* n_dev, const double* sq, int n_sq,
                                  double* part, double* out, double* loss_acc, cudaStream_t stream);
cudaError_t launch_train_stats(const float* fwd, int64_t n, const double* sq, int n_sq, double* out,
                               cudaStream_t st);

}  // namespace gdf
