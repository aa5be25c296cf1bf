// context.h -- internal state behind the gdf C ABI (not installed).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../../include/gdf.h"
#include "../device/grid_levels.h"
#include "../kernels/df_kernels.h"
#include "../kernels/train_kernels.h"

namespace gdf {

// One network with its encoding, in tcnn parameter order
// (network_with_input_encoding.h set_params): MLP matrices, then grid.
struct Net {
  bool present = false;
  int32_t k0 = 0, width = 64, hidden = 0, n_out = 0, n_out_pad = 0;
  int64_t n_mlp = 0, n_grid = 0, n_params = 0;
  int32_t levels = 0, features = 0;
  GridLevels gl{};
  std::vector<int32_t> rows, cols;  // per weight matrix

  // Device state (all n_params long unless noted).
  float* master = nullptr;   // fp32 master weights (Trainer params_full_precision)
  __half* w16 = nullptr;     // fp16 copy used by the training forward
  __half* ema16 = nullptr;   // fp16 EMA copy used by inference
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  uint32_t* adam_step = nullptr;
  float* grad = nullptr;     // fp32 gradient accumulator
  __half* blob_ema = nullptr;  // n_mlp, canonical tensor-core layout of ema16
  __half* blob_w16 = nullptr;  // n_mlp, canonical layout of w16
  uint32_t blob_bytes = 0;
  bool infer_bf16 = false;     // blob_ema holds bf16 (bf16 inference form, DF networks)
  bool train_bf16 = false;     // blob_w16 holds bf16 (bf16 training form, DF networks)
  // FP8 inference form (DF networks): e4m3 hidden matrices, rebuilt from
  // ema16 after every optimizer step (launch_pack_fp8)
  bool infer_f8 = false;
  uint8_t* blob_f8 = nullptr;
  uint32_t f8_bytes = 0;
  Fp8PackParams f8_pack{};
  OptState* opt = nullptr;     // optimizer step counter (device; the optimizer kernel advances it)
};

// Device workspace of the training step, sized by max_train_batch.
struct TrainWorkspace {
  int64_t capacity = 0;
  float* fwd = nullptr;                   // [capacity x 4]
  float* partial[3] = {nullptr, nullptr, nullptr};  // [num_sms x n_mlp] per net
  double* sq = nullptr;                   // [3 x kAdamBlocks] optimizer partials
  double* stats = nullptr;                // [2]: loss sum, squared gradient norm
  unsigned long long* dropped = nullptr;  // [1]
  __half* feat[2] = {nullptr, nullptr};   // [capacity rounded to 128 x L*F] per DF network
  float* dx[2] = {nullptr, nullptr};      // [L][capacity][F] dL/dgrid-features per DF network
  double* stat_part = nullptr;            // [kStatBlocks] per-block loss sums
};

constexpr int kAdamBlocks = 1184;  // 8 x 148 SMs

// Buffers of the frame-level record producers, grown on demand.
struct PathWorkspace {
  int64_t pixels = 0;               // training-pixel capacity of the scratch
  uint16_t* mask = nullptr;         // [pixels]
  int32_t* block_counts = nullptr;  // [blocks x 2]
  int64_t* block_offsets = nullptr; // [blocks x 2]
  int64_t* totals = nullptr;        // [2] device
  int64_t* totals_host = nullptr;   // [2] pinned
  int64_t df_cap = 0;               // DF records
  float* df_in = nullptr;           // [df_cap x 9]
  float* df_in_phi = nullptr;       // [df_cap x 10]
  float* df_target = nullptr;       // [df_cap x 9]
  int64_t nrc_cap = 0;              // NRC query / training rows
  float* nrc_query = nullptr;       // [nrc_cap x 15]
  int32_t* nrc_depth = nullptr;     // [nrc_cap]
  int32_t* nrc_pixel = nullptr;     // [nrc_cap]
  float* nrc_out = nullptr;         // [nrc_cap x 3]
  float* nrc_train_in = nullptr;    // [nrc_cap x 15]
  float* nrc_train_target = nullptr;// [nrc_cap x 3]
  int64_t nrc_rows = 0;             // query rows of the last NRC build
  // frame-level DF training with the record count on the device
  int32_t plan_len = 0;             // batches the plan holds
  int64_t* plan = nullptr;          // [1 + plan_len]: batches, records per batch
  double* loss_acc = nullptr;       // [1] sum of the batches' mean losses
  float* frame_loss = nullptr;      // [1] device results of gdf_train_paths
  int64_t* frame_n = nullptr;       // [1]
};

struct Context {
  gdf_config cfg{};
  int device = 0;
  int num_sms = 148;
  // CTAs of the training step's persistent kernels (0: one per SM). A server
  // that keeps SMs free for inference while training runs lowers it.
  int train_ctas = 0;
  // the training step's second half on the caller's stream alone, not
  // forked over train_aux (a server, whose other slots fill the device)
  bool train_one_stream = false;
  Net net[3];  // theta, phi, nrc
  uint32_t* d_err = nullptr;  // device error word of bounded waits
  TrainWorkspace ws;
  PathWorkspace pw;
  // the two DF networks' EMA grids interleaved per entry for inference:
  // [grid entries][theta F halves | phi F halves]
  __half* grid_il = nullptr;
  // grid features of both networks for inference: [2][feat_tiles][128 x L*F]
  __half* feat = nullptr;
  int64_t feat_tiles = 0;
  // device copies of host inputs for gdf_infer_host, two pipeline streams
  int64_t host_cap = 0;
  float* host_q = nullptr;       // [host_cap x 9]
  uint8_t* host_g = nullptr;     // [host_cap]
  float* host_u = nullptr;       // [host_cap x 4]
  float* host_wi = nullptr;      // [host_cap x 4]
  // the training step's second half: [0] the phi backward, grid backward and
  // optimizer, [1] the theta grid backward and optimizer;
  // events [0] fork, [1], [2] joins
  cudaStream_t train_aux[2] = {nullptr, nullptr};
  cudaEvent_t train_ev[3] = {nullptr, nullptr, nullptr};
  // gdf_infer_host's streams: [0] input copies, [1] kernels, [2] output copies
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};
  // Adam step sizes by per-parameter step counter: [0] DF optimizer, [1] NRC
  float* lr_table[2] = {nullptr, nullptr};
  int32_t lr_table_n[2] = {0, 0};
  // inputs and outputs of the distribution-inspection tools
  int64_t tool_cap = 0;
  float* tool_q = nullptr;       // [tool_cap x 9]
  float* tool_uv = nullptr;      // [tool_cap x 2]
  float* tool_out = nullptr;     // [tool_cap x 4]
  // [0..2]: each pipe stream's end; [3]: the call's start; [4]: a chunk's
  // input copies done; [5]: a chunk's kernels done
  cudaEvent_t pipe_ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// CTAs of the training step's persistent kernels (and weight-gradient partials).
inline int train_ctas(const Context& c) {
  return c.train_ctas > 0 && c.train_ctas < c.num_sms ? c.train_ctas : c.num_sms;
}

// The group's device error flag (set by its kernels' bounded waits).
uint32_t* group_err_flag(gdf_group* g);

// Sets the thread-local message returned by gdf_last_error().
void set_last_error(const char* msg);

// Grid level tables (tcnn encodings/grid.h:967-1012, grid_index :165-188).
bool build_grid_levels(const gdf_grid_config& c, GridLevels* gl, int64_t* n_params);

}  // namespace gdf

// The opaque handle of the C ABI.
struct gdf_ctx {
  gdf::Context c;
};
