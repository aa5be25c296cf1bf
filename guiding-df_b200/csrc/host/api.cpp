// api.cpp -- implementation of the gdf C ABI (include/gdf.h).
//
// Host-side orchestration of the guiding module: configuration presets and
// validation, parameter layout and initialisation, checkpoint files, and the
// launches of the fused kernels. Nothing here computes a query on the CPU;
// every compute entry point launches a CUDA kernel or fails.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <vector>

#include "../kernels/df_kernels.h"
#include "../kernels/nrc_kernels.h"
#include "../kernels/paths_kernels.h"
#include "../kernels/tools_kernels.h"
#include "../kernels/train_kernels.h"
#include "context.h"

using gdf::Context;
using gdf::Net;

namespace {

thread_local std::string g_last_error;

gdf_status fail(gdf_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

gdf_status cuda_fail(cudaError_t e, const char* what) {
  return fail(GDF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GDF_CUDA(call)                                        \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);       \
  } while (0)

int32_t pad16(int32_t v) { return (v + 15) / 16 * 16; }

// PCG32 (M. E. O'Neill, "PCG: a family of simple fast space-efficient
// statistically good algorithms for random number generation", 2014).
struct Pcg32 {
  uint64_t state = 0, inc = 1;
  explicit Pcg32(uint64_t seed, uint64_t seq = 0xda3e39cb94b95bdbULL) {
    inc = (seq << 1u) | 1u;
    next();
    state += seed;
    next();
  }
  uint32_t next() {
    const uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = static_cast<uint32_t>(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
  }
  float uniform() { return static_cast<float>(next() >> 8) * (1.0f / 16777216.0f); }
};

bool valid_grid(const gdf_grid_config& g) {
  return g.n_levels > 0 && g.n_levels <= GDF_MAX_GRID_LEVELS &&
         (g.n_features_per_level == 2 || g.n_features_per_level == 4) &&
         g.log2_hashmap_size > 0 && g.log2_hashmap_size <= 26 && g.base_resolution > 0 &&
         g.per_level_scale >= 1.0f && g.type >= 0 && g.type <= 2 && g.interpolation >= 0 &&
         g.interpolation <= 2;
}

gdf_status validate(const gdf_config& c) {
  if (c.abi_version != GDF_ABI_VERSION) return fail(GDF_ERR_INVALID_ARG, "abi_version mismatch");
  auto bins_ok = [](int b) { return b == 16 || b == 32 || b == 64; };
  if (!bins_ok(c.n_bins_theta) || !bins_ok(c.n_bins_phi))
    return fail(GDF_ERR_INVALID_ARG, "n_bins must be 16, 32 or 64");
  if (c.pdf_interp != GDF_PDF_LINEAR && c.pdf_interp != GDF_PDF_NEAREST)
    return fail(GDF_ERR_INVALID_ARG, "pdf_interp");
  if (!valid_grid(c.grid_theta) || !valid_grid(c.grid_phi))
    return fail(GDF_ERR_INVALID_ARG, "grid config out of range");
  if (std::memcmp(&c.grid_theta, &c.grid_phi, sizeof(gdf_grid_config)) != 0)
    return fail(GDF_ERR_UNSUPPORTED,
                "theta and phi grids must share one configuration (inference gathers both at once)");
  if (c.sh_degree != 4 || c.oneblob_bins != 4 || c.tw_frequencies != 12)
    return fail(GDF_ERR_UNSUPPORTED, "built encodings: SH degree 4, OneBlob 4 bins, TriangleWave 12");
  if (c.mlp_theta.n_neurons != 64 || c.mlp_phi.n_neurons != 64)
    return fail(GDF_ERR_UNSUPPORTED, "only 64-neuron MLPs are built");
  if (c.mlp_theta.n_hidden_layers < 1 || c.mlp_theta.n_hidden_layers > 8 ||
      c.mlp_phi.n_hidden_layers < 1 || c.mlp_phi.n_hidden_layers > 8)
    return fail(GDF_ERR_INVALID_ARG, "n_hidden_layers must be in [1, 8]");
  if (c.nrc_enable) {
    if (c.mlp_nrc.n_neurons != 64 || c.mlp_nrc.n_hidden_layers < 1 || c.mlp_nrc.n_hidden_layers > 8)
      return fail(GDF_ERR_UNSUPPORTED, "NRC MLP must be 64 wide with 1..8 hidden layers");
    if (c.nrc_frequencies != 12 || c.nrc_oneblob_bins != 4)
      return fail(GDF_ERR_UNSUPPORTED, "built NRC encoding: Frequency 12, OneBlob 4");
  }
  for (const gdf_adam_config* a : {&c.adam_df, &c.adam_nrc})
    if (!(a->beta1 >= 0.f && a->beta1 < 1.f && a->beta2 >= 0.f && a->beta2 < 1.f))
      return fail(GDF_ERR_INVALID_ARG, "Adam betas must lie in [0, 1)");
  if (c.precision < GDF_PREC_FP16 || c.precision > GDF_PREC_FP8)
    return fail(GDF_ERR_INVALID_ARG, "precision");
  if (c.precision == GDF_PREC_FP8)
    for (const gdf_mlp_config* m : {&c.mlp_theta, &c.mlp_phi})
      if (m->n_hidden_layers + 1 > gdf::kMaxMlpLayers)
        return fail(GDF_ERR_UNSUPPORTED, "FP8 form: at most 9 hidden layers");
  if (c.max_queries < 0 || c.max_train_batch < 0)
    return fail(GDF_ERR_INVALID_ARG, "negative capacity");
  const int64_t cap = c.max_train_batch > 0 ? c.max_train_batch : 65536;
  if (c.df_batch_size < 128 || c.df_batch_size > cap || c.nrc_batch_size < 128 ||
      c.nrc_batch_size > cap)
    return fail(GDF_ERR_INVALID_ARG, "training batch sizes must be in [128, max_train_batch]");
  if (c.min_train_batch < 1 || c.df_batches_per_frame < 0 || c.nrc_batches_per_frame < 0)
    return fail(GDF_ERR_INVALID_ARG, "min_train_batch / batches_per_frame");
  gdf::DfShape s{c.grid_theta.n_levels, c.grid_theta.n_features_per_level, c.n_bins_theta,
                 c.n_bins_phi, c.pdf_interp == GDF_PDF_LINEAR};
  if (!gdf::df_shape_supported(s))
    return fail(GDF_ERR_UNSUPPORTED, "no fused kernel is built for this (levels, features, bins) shape");
  return GDF_OK;
}

template <typename T>
gdf_status dalloc(T** p, size_t n) {
  if (n == 0) { *p = nullptr; return GDF_OK; }
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(GDF_ERR_OOM_BUDGET, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  return GDF_OK;
}

void free_net(Net& n) {
  cudaFree(n.master); cudaFree(n.w16); cudaFree(n.ema16); cudaFree(n.adam_m);
  cudaFree(n.adam_v); cudaFree(n.adam_step); cudaFree(n.grad); cudaFree(n.blob_ema);
  cudaFree(n.blob_w16); cudaFree(n.blob_f8); cudaFree(n.opt);
  n = Net{};
}

// DF network layout: composite encoding widths (composite.h:187-199) padded
// to 16 (network_with_input_encoding.h:44), FullyFusedMLP matrices
// (fully_fused_mlp.cu:630-668).
gdf_status layout_df_net(const gdf_config& c, int id, Net& n) {
  const gdf_grid_config& g = id == 0 ? c.grid_theta : c.grid_phi;
  const gdf_mlp_config& m = id == 0 ? c.mlp_theta : c.mlp_phi;
  n.present = true;
  n.levels = g.n_levels;
  n.features = g.n_features_per_level;
  int32_t enc = g.n_levels * g.n_features_per_level + c.sh_degree * c.sh_degree + 3 * c.oneblob_bins;
  if (id == 1) enc += c.tw_frequencies;
  n.k0 = pad16(enc);
  n.width = m.n_neurons;
  n.hidden = m.n_hidden_layers;
  n.n_out = id == 0 ? c.n_bins_theta : c.n_bins_phi;
  n.n_out_pad = pad16(n.n_out);
  if (!gdf::build_grid_levels(g, &n.gl, &n.n_grid)) return fail(GDF_ERR_INVALID_ARG, "grid tables");
  n.rows.clear(); n.cols.clear();
  n.rows.push_back(n.width); n.cols.push_back(n.k0);
  for (int l = 1; l < n.hidden; ++l) { n.rows.push_back(n.width); n.cols.push_back(n.width); }
  n.rows.push_back(n.n_out_pad); n.cols.push_back(n.width);
  n.n_mlp = 0;
  for (size_t i = 0; i < n.rows.size(); ++i) n.n_mlp += static_cast<int64_t>(n.rows[i]) * n.cols[i];
  n.n_params = n.n_mlp + n.n_grid;
  n.blob_bytes = static_cast<uint32_t>(n.n_mlp * 2);
  return GDF_OK;
}

// NRC: [Frequency(3 dims x 12 x sin/cos) | OneBlob(6 dims x 4) | Identity(6)]
// padded with ones to 112 (common/configs/nn/base_hashgrid_nrc_df.json).
gdf_status layout_nrc_net(const gdf_config& c, Net& n) {
  n.present = true;
  n.levels = 0; n.features = 0; n.n_grid = 0;
  n.k0 = pad16(3 * c.nrc_frequencies * 2 + 6 * c.nrc_oneblob_bins + 6);
  n.width = c.mlp_nrc.n_neurons;
  n.hidden = c.mlp_nrc.n_hidden_layers;
  n.n_out = 3;
  n.n_out_pad = 16;
  n.rows.clear(); n.cols.clear();
  n.rows.push_back(n.width); n.cols.push_back(n.k0);
  for (int l = 1; l < n.hidden; ++l) { n.rows.push_back(n.width); n.cols.push_back(n.width); }
  n.rows.push_back(n.n_out_pad); n.cols.push_back(n.width);
  n.n_mlp = 0;
  for (size_t i = 0; i < n.rows.size(); ++i) n.n_mlp += static_cast<int64_t>(n.rows[i]) * n.cols[i];
  n.n_params = n.n_mlp;
  n.blob_bytes = static_cast<uint32_t>(n.n_mlp * 2);
  return GDF_OK;
}

gdf_status alloc_net(Net& n) {
  gdf_status s;
  const size_t np = static_cast<size_t>(n.n_params);
  if ((s = dalloc(&n.master, np)) || (s = dalloc(&n.w16, np)) || (s = dalloc(&n.ema16, np)) ||
      (s = dalloc(&n.adam_m, np)) || (s = dalloc(&n.adam_v, np)) ||
      (s = dalloc(&n.adam_step, np)) || (s = dalloc(&n.grad, np)) || (s = dalloc(&n.opt, 1)) ||
      (s = dalloc(&n.blob_ema, static_cast<size_t>(n.n_mlp))) ||
      (s = dalloc(&n.blob_w16, static_cast<size_t>(n.n_mlp))))
    return s;
  if (n.infer_f8) {
    n.f8_bytes = gdf::fp8_blob_bytes(n.rows.data(), n.cols.data(), static_cast<int>(n.rows.size()), &n.f8_pack);
    if ((s = dalloc(&n.blob_f8, n.f8_bytes))) return s;
    n.f8_pack.src = n.ema16;
    n.f8_pack.dst = n.blob_f8;
  }
  return GDF_OK;
}

// Re-packs the tensor-core weight blobs from the fp16 copies.
gdf_status repack(Net& n, cudaStream_t st) {
  cudaError_t e = gdf::launch_pack_mlp(n.ema16, n.blob_ema, n.rows.data(), n.cols.data(),
                                       static_cast<int>(n.rows.size()), st, n.infer_bf16);
  if (e != cudaSuccess) return cuda_fail(e, "pack ema");
  e = gdf::launch_pack_mlp(n.w16, n.blob_w16, n.rows.data(), n.cols.data(),
                           static_cast<int>(n.rows.size()), st, n.train_bf16);
  if (e != cudaSuccess) return cuda_fail(e, "pack w16");
  if (n.infer_f8 && (e = gdf::launch_pack_fp8(n.f8_pack, st)) != cudaSuccess) return cuda_fail(e, "pack fp8");
  return GDF_OK;
}

// Uploads fp32 master weights; fp16 and EMA copies become fp16(master)
// (Trainer::set_params_full_precision, trainer.h:238-250); optimizer state
// is left untouched.
gdf_status upload_params(Net& n, const std::vector<float>& host) {
  std::vector<__half> h16(host.size());
  for (size_t i = 0; i < host.size(); ++i) h16[i] = __float2half_rn(host[i]);
  GDF_CUDA(cudaMemcpy(n.master, host.data(), host.size() * 4, cudaMemcpyHostToDevice));
  GDF_CUDA(cudaMemcpy(n.w16, h16.data(), h16.size() * 2, cudaMemcpyHostToDevice));
  GDF_CUDA(cudaMemcpy(n.ema16, h16.data(), h16.size() * 2, cudaMemcpyHostToDevice));
  gdf_status s = repack(n, nullptr);
  if (s) return s;
  GDF_CUDA(cudaDeviceSynchronize());
  return GDF_OK;
}

// Xavier-uniform MLP matrices (gpu_matrix.h initialize_xavier_uniform,
// fully_fused_mlp.cu:885-904) and U(-1e-4, 1e-4) grid tables
// (grid.h:1364-1369), drawn from PCG32 seeded with `seed`.
gdf_status init_params(Net& n, uint32_t seed, uint32_t stream_id) {
  Pcg32 rng(seed, 0x9e3779b97f4a7c15ULL + stream_id);
  std::vector<float> h(static_cast<size_t>(n.n_params));
  size_t o = 0;
  for (size_t l = 0; l < n.rows.size(); ++l) {
    const float scale = std::sqrt(6.0f / static_cast<float>(n.rows[l] + n.cols[l]));
    const size_t cnt = static_cast<size_t>(n.rows[l]) * n.cols[l];
    for (size_t i = 0; i < cnt; ++i) h[o++] = rng.uniform() * 2.0f * scale - scale;
  }
  for (; o < h.size(); ++o) h[o] = rng.uniform() * 2e-4f - 1e-4f;
  GDF_CUDA(cudaMemset(n.adam_m, 0, h.size() * 4));
  GDF_CUDA(cudaMemset(n.adam_v, 0, h.size() * 4));
  GDF_CUDA(cudaMemset(n.adam_step, 0, h.size() * 4));
  GDF_CUDA(cudaMemset(n.grad, 0, h.size() * 4));
  GDF_CUDA(cudaMemset(n.opt, 0, sizeof(gdf::OptState)));
  return upload_params(n, h);
}

void free_ws(gdf::TrainWorkspace& w) {
  cudaFree(w.fwd);
  for (float*& p : w.partial) cudaFree(p);
  cudaFree(w.sq);
  cudaFree(w.stats);
  cudaFree(w.dropped);
  cudaFree(w.feat[0]);
  cudaFree(w.feat[1]);
  cudaFree(w.dx[0]);
  cudaFree(w.dx[1]);
  cudaFree(w.stat_part);
  w = gdf::TrainWorkspace{};
}

void free_host_stage(Context& c) {
  for (float*& t : c.lr_table) {
    cudaFree(t);
    t = nullptr;
  }
  cudaFree(c.host_q);
  cudaFree(c.host_g);
  cudaFree(c.host_u);
  cudaFree(c.host_wi);
  c.host_q = nullptr;
  c.host_g = nullptr;
  c.host_u = nullptr;
  c.host_wi = nullptr;
  c.host_cap = 0;
  cudaFree(c.tool_q);
  cudaFree(c.tool_uv);
  cudaFree(c.tool_out);
  c.tool_q = c.tool_uv = c.tool_out = nullptr;
  c.tool_cap = 0;
  for (cudaStream_t& s : c.pipe) {
    if (s) cudaStreamDestroy(s);
    s = nullptr;
  }
  for (cudaStream_t& s : c.train_aux) {
    if (s) cudaStreamDestroy(s);
    s = nullptr;
  }
  for (cudaEvent_t& e : c.train_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  for (cudaEvent_t& e : c.pipe_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
}

void free_pw(gdf::PathWorkspace& w) {
  cudaFree(w.mask);
  cudaFree(w.block_counts);
  cudaFree(w.block_offsets);
  cudaFree(w.totals);
  cudaFreeHost(w.totals_host);
  cudaFree(w.df_in);
  cudaFree(w.df_in_phi);
  cudaFree(w.df_target);
  cudaFree(w.nrc_query);
  cudaFree(w.nrc_depth);
  cudaFree(w.nrc_pixel);
  cudaFree(w.nrc_out);
  cudaFree(w.nrc_train_in);
  cudaFree(w.nrc_train_target);
  cudaFree(w.plan);
  cudaFree(w.loss_acc);
  cudaFree(w.frame_loss);
  cudaFree(w.frame_n);
  w = gdf::PathWorkspace{};
}

gdf_status alloc_ws(Context& c) {
  gdf::TrainWorkspace& w = c.ws;
  gdf_status s;
  const int64_t cap = c.cfg.max_train_batch > 0 ? c.cfg.max_train_batch : 65536;
  w.capacity = cap;
  if ((s = dalloc(&w.fwd, static_cast<size_t>(cap) * 4))) return s;
  for (int i = 0; i < 3; ++i)
    if (c.net[i].present &&
        (s = dalloc(&w.partial[i], static_cast<size_t>(c.num_sms) * static_cast<size_t>(c.net[i].n_mlp))))
      return s;
  if ((s = dalloc(&w.sq, 3 * static_cast<size_t>(gdf::kAdamBlocks))) || (s = dalloc(&w.stats, 2)) ||
      (s = dalloc(&w.dropped, 1)))
    return s;
  const size_t feat = static_cast<size_t>((cap + 127) / 128 * 128) * static_cast<size_t>(c.net[0].levels) *
                      static_cast<size_t>(c.net[0].features);
  const size_t dx = static_cast<size_t>(cap) * static_cast<size_t>(c.net[0].levels) *
                    static_cast<size_t>(c.net[0].features);
  // dx[1] (the phi network's own dL/dfeatures) comes with the first
  // training step that runs the two networks' second halves side by side
  if ((s = dalloc(&w.feat[0], feat)) || (s = dalloc(&w.feat[1], feat)) || (s = dalloc(&w.dx[0], dx)) ||
      (s = dalloc(&w.stat_part, gdf::kStatBlocks)))
    return s;
  if (!c.train_aux[0]) {
    for (cudaStream_t& ts : c.train_aux) GDF_CUDA(cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking));
    for (cudaEvent_t& e : c.train_ev) GDF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  return GDF_OK;
}

Net* net_of(Context* c, int32_t id) {
  if (!c || id < 0 || id > 2 || !c->net[id].present) return nullptr;
  return &c->net[id];
}

gdf_status check_ptr(const void* p, const char* name) {
  if (!p) return fail(GDF_ERR_INVALID_ARG, std::string(name) + " is null");
  return GDF_OK;
}

}  // namespace

namespace gdf {

void set_last_error(const char* msg) { g_last_error = msg; }

bool build_grid_levels(const gdf_grid_config& c, GridLevels* gl, int64_t* n_params) {
  std::memset(gl, 0, sizeof(*gl));
  if (c.n_levels > 24) return false;
  gl->n_levels = c.n_levels;
  gl->interp = c.interpolation;
  const float log2_scale = std::log2(c.per_level_scale);
  uint32_t offset = 0;
  for (int i = 0; i < c.n_levels; ++i) {
    const float scale = std::exp2(static_cast<float>(i) * log2_scale) *
                        static_cast<float>(c.base_resolution) - 1.0f;
    const uint32_t res = static_cast<uint32_t>(std::ceil(scale)) + 1u;
    const uint32_t max_params = 0xffffffffu / 2u;
    uint32_t params = std::pow(static_cast<float>(res), 3.0f) > static_cast<float>(max_params)
                          ? max_params
                          : res * res * res;
    params = (params + 7u) / 8u * 8u;
    if (c.type == GDF_GRID_TILED) {
      const uint32_t b = static_cast<uint32_t>(c.base_resolution);
      if (b * b * b < params) params = b * b * b;
    } else if (c.type == GDF_GRID_HASH) {
      const uint32_t t = 1u << c.log2_hashmap_size;
      if (t < params) params = t;
    }
    uint32_t stride = 1, nd = 0;
    for (int d = 0; d < 3 && stride <= params; ++d) {
      ++nd;
      stride *= res;
    }
    gl->scale[i] = scale;
    gl->offset[i] = offset;
    gl->hsize[i] = params;
    gl->res[i] = res;
    gl->ndims[i] = nd;
    gl->hashed[i] = (c.type == GDF_GRID_HASH && params < stride) ? 1u : 0u;
    gl->pow2[i] = (params & (params - 1u)) == 0u ? 1u : 0u;
    offset += params;
  }
  *n_params = static_cast<int64_t>(offset) * c.n_features_per_level;
  return true;
}

}  // namespace gdf

extern "C" {

const char* gdf_last_error(void) { return g_last_error.c_str(); }

const char* gdf_status_string(gdf_status s) {
  switch (s) {
    case GDF_OK: return "ok";
    case GDF_ERR_INVALID_ARG: return "invalid argument";
    case GDF_ERR_OOM_BUDGET: return "out of memory / budget";
    case GDF_ERR_CUDA: return "cuda error";
    case GDF_ERR_TIMEOUT: return "device wait timed out";
    case GDF_ERR_NUMERIC: return "numeric error";
    case GDF_ERR_UNSUPPORTED: return "unsupported configuration";
    case GDF_ERR_STATE: return "invalid state";
  }
  return "unknown";
}

gdf_status gdf_default_config(int32_t preset, gdf_config* cfg) {
  if (!cfg) return fail(GDF_ERR_INVALID_ARG, "cfg is null");
  gdf_config c;
  std::memset(&c, 0, sizeof(c));
  c.abi_version = GDF_ABI_VERSION;
  c.pdf_interp = GDF_PDF_LINEAR;
  c.sh_degree = 4;
  c.oneblob_bins = 4;
  c.tw_frequencies = 12;
  // base_product_df.json optimizer: EMA 0.95 over Adam(3e-2, 0.9, 0.99, 1e-15, l2 1e-6).
  c.adam_df = gdf_adam_config{3e-2f, 0.9f, 0.99f, 1e-15f, 1e-6f, 0.95f};
  c.loss_scale = 1024.f;
  // base_hashgrid_nrc_df.json optimizer: EMA 0.99 over Adam(8e-3, 0.9, 0.99, 1e-8, l2 1e-6).
  c.adam_nrc = gdf_adam_config{8e-3f, 0.9f, 0.99f, 1e-8f, 1e-6f, 0.99f};
  c.nrc_loss_scale = 1024.f;
  c.nrc_frequencies = 12;
  c.nrc_oneblob_bins = 4;
  c.mlp_nrc = gdf_mlp_config{64, 5};
  c.precision = GDF_PREC_FP16;
  c.seed = 7272u;  // KRR_DEFAULT_RND_SEED (src/lib/src/core/config.in.h:15)
  gdf_grid_config hash{GDF_GRID_HASH, 8, 2, 16, 16, 2.0f, GDF_GRID_LINEAR};
  c.min_train_batch = 65536;       // MIN_TRAIN_BATCH_SIZE (parameters.h:55)
  c.df_batches_per_frame = 5;      // batchPerFrame (learnedDistribution.h:138)
  c.nrc_batches_per_frame = 4;     // NRC_ITER_COUNT (parameters.h:65)
  switch (preset) {
    case GDF_PRESET_SMALL:
      c.n_bins_theta = c.n_bins_phi = 32;
      c.grid_theta = c.grid_phi = hash;
      c.mlp_theta = c.mlp_phi = gdf_mlp_config{64, 3};
      c.nrc_enable = 1;
      c.max_queries = 65536;
      c.max_train_batch = 65536;
      c.df_batch_size = c.nrc_batch_size = 65536;
      break;
    case GDF_PRESET_FULL:
      c.n_bins_theta = c.n_bins_phi = 64;
      hash.n_levels = 16;
      hash.log2_hashmap_size = 19;
      c.grid_theta = c.grid_phi = hash;
      c.mlp_theta = c.mlp_phi = gdf_mlp_config{64, 4};
      c.nrc_enable = 1;
      c.max_queries = 1920 * 1080;
      c.max_train_batch = 1048576;
      c.df_batch_size = 262144;
      c.nrc_batch_size = 1048576;  // TRAIN_BATCH_SIZE_NRC (parameters.h:66)
      break;
    case GDF_PRESET_REFERENCE: {
      // common/configs/nn/base_product_df.json + parameters.h:41,48.
      c.n_bins_theta = 16;
      c.n_bins_phi = 32;
      gdf_grid_config dense{GDF_GRID_DENSE, 8, 4, 19, 8, 1.405f, GDF_GRID_SMOOTHSTEP};
      c.grid_theta = c.grid_phi = dense;
      c.mlp_theta = c.mlp_phi = gdf_mlp_config{64, 3};
      c.nrc_enable = 1;
      c.max_queries = 1280 * 720;  // MAX_RESOLUTION (parameters.h:51)
      c.max_train_batch = 1048576;
      c.df_batch_size = 65536 * 8;   // TRAIN_BATCH_SIZE (parameters.h:54)
      c.nrc_batch_size = 1048576;
      break;
    }
    default:
      return fail(GDF_ERR_INVALID_ARG, "unknown preset");
  }
  *cfg = c;
  return GDF_OK;
}

}  // extern "C"

static gdf::DfShape df_shape(const Context& c) {
  return gdf::DfShape{c.cfg.grid_theta.n_levels, c.cfg.grid_theta.n_features_per_level,
                      c.cfg.n_bins_theta, c.cfg.n_bins_phi, c.cfg.pdf_interp == GDF_PDF_LINEAR};
}

static int64_t feat_row_halves(const Context& c) {
  return static_cast<int64_t>(c.cfg.grid_theta.n_levels) * c.cfg.grid_theta.n_features_per_level;
}

// Grows the grid-feature buffer to n_tiles 128-row tiles per network.
static gdf_status ensure_features(Context& c, int64_t n_tiles) {
  if (n_tiles <= c.feat_tiles) return GDF_OK;
  cudaFree(c.feat);
  c.feat = nullptr;
  c.feat_tiles = 0;
  gdf_status s = dalloc(&c.feat, static_cast<size_t>(2 * n_tiles * 128 * feat_row_halves(c)));
  if (s) return s;
  c.feat_tiles = n_tiles;
  return GDF_OK;
}

// Rebuilds the interleaved inference grid from both networks' EMA copies.
static gdf_status refresh_grid_il(Context& c) {
  const Net& t = c.net[0];
  const Net& f = c.net[1];
  cudaError_t e = gdf::launch_interleave_grids(t.ema16 + t.n_mlp, f.ema16 + f.n_mlp, c.grid_il,
                                               t.n_grid / t.features, t.features, nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "interleave grids");
  GDF_CUDA(cudaDeviceSynchronize());
  return GDF_OK;
}

// Both grids' features of n queries (query rows, or shading positions with
// aabb) into the context's buffer; points p at them.
static gdf_status grid_features(Context& c, const float* queries, const gdf_shading* sh,
                                const gdf_aabb& aabb, int64_t n, gdf::DfKernelParams& p,
                                cudaStream_t st, int64_t tile_base = 0) {
  const int64_t tiles = (n + 127) / 128;
  gdf_status s = ensure_features(c, tile_base + tiles);
  if (s) return s;
  gdf::GridFeatParams g;
  std::memset(&g, 0, sizeof(g));
  g.queries = queries;
  g.shading_pos = sh ? sh->pos : nullptr;
  g.aabb = aabb;
  g.n = n;
  g.n_tiles = tiles;
  g.grid_il = c.grid_il;
  g.gl = c.net[0].gl;
  g.bf16 = c.cfg.precision == GDF_PREC_BF16;
  g.feat_theta = c.feat + tile_base * 128 * feat_row_halves(c);
  g.feat_phi = c.feat + (c.feat_tiles + tile_base) * 128 * feat_row_halves(c);
  cudaError_t e = gdf::launch_grid_features(df_shape(c), g, st);
  if (e != cudaSuccess) return cuda_fail(e, "grid_features");
  p.feat_theta = g.feat_theta;
  p.feat_phi = g.feat_phi;
  return GDF_OK;
}

extern "C" {

gdf_status gdf_create(const gdf_config* cfg, gdf_ctx** out) {
  if (!cfg || !out) return fail(GDF_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  gdf_status s = validate(*cfg);
  if (s) return s;
  gdf_ctx* h = new (std::nothrow) gdf_ctx();
  if (!h) return fail(GDF_ERR_OOM_BUDGET, "host allocation failed");
  Context& c = h->c;
  c.cfg = *cfg;
  cudaError_t e = cudaGetDevice(&c.device);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaGetDevice"); }
  cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device);
  auto cleanup = [&](gdf_status st) {
    for (Net& n : c.net) free_net(n);
    free_ws(c.ws);
    free_pw(c.pw);
    cudaFree(c.feat);
    cudaFree(c.grid_il);
    free_host_stage(c);
    cudaFree(c.d_err);
    delete h;
    return st;
  };
  if ((s = layout_df_net(c.cfg, 0, c.net[0])) || (s = layout_df_net(c.cfg, 1, c.net[1])))
    return cleanup(s);
  c.net[0].infer_bf16 = c.net[1].infer_bf16 = c.cfg.precision == GDF_PREC_BF16;
  // the bf16 form trains in bf16 too: the training blob is bf16(fp16 copy)
  c.net[0].train_bf16 = c.net[1].train_bf16 = c.cfg.precision == GDF_PREC_BF16;
  c.net[0].infer_f8 = c.net[1].infer_f8 = c.cfg.precision == GDF_PREC_FP8;
  if (c.cfg.nrc_enable && (s = layout_nrc_net(c.cfg, c.net[2]))) return cleanup(s);
  for (Net& n : c.net)
    if (n.present && (s = alloc_net(n))) return cleanup(s);
  if ((s = dalloc(&c.d_err, 1))) return cleanup(s);
  if ((s = alloc_ws(c))) return cleanup(s);
  if (c.cfg.max_queries > 0 && (s = ensure_features(c, (c.cfg.max_queries + 127) / 128)))
    return cleanup(s);
  if ((s = dalloc(&c.grid_il, static_cast<size_t>(2 * c.net[0].n_grid)))) return cleanup(s);
  for (int t = 0; t < 2; ++t) {
    const gdf_adam_config& a = t == 0 ? c.cfg.adam_df : c.cfg.adam_nrc;
    // past k with beta^k < 2^-27 for both betas, 1 - beta^k is 1.0f and the
    // step size is lr exactly; the table stops two entries after that
    double k = 1.0;
    for (double b : {static_cast<double>(a.beta1), static_cast<double>(a.beta2)})
      if (b > 0.0) k = std::max(k, std::ceil(std::log(std::ldexp(1.0, -27)) / std::log(b)));
    c.lr_table_n[t] = static_cast<int32_t>(std::min(k + 2.0, static_cast<double>(1 << 22)));
    if ((s = dalloc(&c.lr_table[t], static_cast<size_t>(c.lr_table_n[t])))) return cleanup(s);
    e = gdf::launch_adam_lr_table(a.learning_rate, a.beta1, a.beta2, c.lr_table[t], c.lr_table_n[t], nullptr);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "adam lr table"));
  }
  e = cudaMemset(c.d_err, 0, 4);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMemset"));
  for (int i = 0; i < 3; ++i)
    if (c.net[i].present && (s = init_params(c.net[i], c.cfg.seed, static_cast<uint32_t>(i))))
      return cleanup(s);
  if ((s = refresh_grid_il(c))) return cleanup(s);
  *out = h;
  return GDF_OK;
}

gdf_status gdf_destroy(gdf_ctx* ctx) {
  if (!ctx) return GDF_OK;
  cudaDeviceSynchronize();
  for (Net& n : ctx->c.net) free_net(n);
  free_ws(ctx->c.ws);
  free_pw(ctx->c.pw);
  cudaFree(ctx->c.feat);
  cudaFree(ctx->c.grid_il);
  free_host_stage(ctx->c);
  cudaFree(ctx->c.d_err);
  delete ctx;
  return GDF_OK;
}

gdf_status gdf_reset_training(gdf_ctx* ctx, uint32_t seed) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  for (int i = 0; i < 3; ++i) {
    Net& n = ctx->c.net[i];
    if (!n.present) continue;
    gdf_status s = init_params(n, seed, static_cast<uint32_t>(i));
    if (s) return s;
  }
  return refresh_grid_il(ctx->c);
}

gdf_status gdf_ctx_bytes(const gdf_ctx* ctx, int64_t* bytes) {
  if (!ctx || !bytes) return fail(GDF_ERR_INVALID_ARG, "null argument");
  const Context& c = ctx->c;
  int64_t b = 0;
  for (const Net& n : c.net) {
    if (!n.present) continue;
    // master, m, v, step, grad (4 B) + w16, ema16 (2 B) + two MLP blobs
    b += n.n_params * (4 * 5 + 2 * 2) + n.n_mlp * 2 * 2 + n.f8_bytes;
  }
  const int64_t lf = static_cast<int64_t>(c.cfg.grid_theta.n_levels) * c.cfg.grid_theta.n_features_per_level;
  b += c.net[0].n_grid * 2 * 2;                               // interleaved inference grid
  b += c.feat_tiles * 128 * lf * 2 * 2;                       // inference feature tiles
  b += c.ws.capacity * 16 + 3 * static_cast<int64_t>(c.num_sms) * (c.net[0].n_mlp + c.net[1].n_mlp) +
       3 * gdf::kAdamBlocks * 8 + 64 + (c.ws.capacity + 127) / 128 * 128 * lf * 2 * 2 +
       (c.ws.dx[1] ? 2 : 1) * c.ws.capacity * lf * 4 + gdf::kStatBlocks * 8;  // training workspace
  b += (c.lr_table_n[0] + c.lr_table_n[1]) * 4;
  b += c.host_cap * (9 * 4 + 1 + 4 * 4 + 4 * 4) + c.tool_cap * (9 + 2 + 4) * 4;
  b += c.pw.pixels * 2 + c.pw.df_cap * 28 * 4 + c.pw.nrc_cap * (15 + 1 + 1 + 3 + 15 + 3) * 4;
  *bytes = b;
  return GDF_OK;
}

gdf_status gdf_n_params(const gdf_ctx* ctx, int32_t net, int64_t* n_params) {
  Net* n = net_of(const_cast<Context*>(ctx ? &ctx->c : nullptr), net);
  if (!n || !n_params) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id / output pointer");
  *n_params = n->n_params;
  return GDF_OK;
}

gdf_status gdf_set_params(gdf_ctx* ctx, int32_t net, const float* params_host, int64_t n) {
  Net* nt = net_of(ctx ? &ctx->c : nullptr, net);
  if (!nt || !params_host) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id / params");
  if (n != nt->n_params) return fail(GDF_ERR_INVALID_ARG, "parameter count mismatch");
  std::vector<float> h(params_host, params_host + n);
  gdf_status s = upload_params(*nt, h);
  if (s || net == GDF_NET_NRC) return s;
  return refresh_grid_il(ctx->c);
}

gdf_status gdf_get_params(const gdf_ctx* ctx, int32_t net, float* params_host, int64_t n) {
  Net* nt = net_of(const_cast<Context*>(ctx ? &ctx->c : nullptr), net);
  if (!nt || !params_host) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id / params");
  if (n != nt->n_params) return fail(GDF_ERR_INVALID_ARG, "parameter count mismatch");
  GDF_CUDA(cudaDeviceSynchronize());
  GDF_CUDA(cudaMemcpy(params_host, nt->master, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost));
  return GDF_OK;
}

gdf_status gdf_get_inference_params(const gdf_ctx* ctx, int32_t net, float* params_host, int64_t n) {
  Net* nt = net_of(const_cast<Context*>(ctx ? &ctx->c : nullptr), net);
  if (!nt || !params_host) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id / params");
  if (n != nt->n_params) return fail(GDF_ERR_INVALID_ARG, "parameter count mismatch");
  std::vector<__half> h(static_cast<size_t>(n));
  GDF_CUDA(cudaDeviceSynchronize());
  GDF_CUDA(cudaMemcpy(h.data(), nt->ema16, h.size() * 2, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < h.size(); ++i) params_host[i] = __half2float(h[i]);
  return GDF_OK;
}

gdf_status gdf_save_network(const gdf_ctx* ctx, const char* prefix) {
  if (!ctx || !prefix) return fail(GDF_ERR_INVALID_ARG, "null argument");
  const char* names[3] = {"AR_network_theta.bin", "AR_network_phi.bin", "NRC_network.bin"};
  for (int i = 0; i < 3; ++i) {
    const Net& n = ctx->c.net[i];
    if (!n.present) continue;
    std::vector<float> h(static_cast<size_t>(n.n_params));
    gdf_status s = gdf_get_params(ctx, i, h.data(), n.n_params);
    if (s) return s;
    std::ofstream f(std::string(prefix) + names[i], std::ios::binary);
    if (!f.good()) return fail(GDF_ERR_INVALID_ARG, std::string("cannot open ") + prefix + names[i]);
    f.write(reinterpret_cast<const char*>(h.data()), static_cast<std::streamsize>(h.size() * 4));
  }
  return GDF_OK;
}

gdf_status gdf_load_network(gdf_ctx* ctx, const char* prefix) {
  if (!ctx || !prefix) return fail(GDF_ERR_INVALID_ARG, "null argument");
  const char* names[3] = {"AR_network_theta.bin", "AR_network_phi.bin", "NRC_network.bin"};
  for (int i = 0; i < 3; ++i) {
    Net& n = ctx->c.net[i];
    if (!n.present) continue;
    std::ifstream f(std::string(prefix) + names[i], std::ios::binary);
    if (!f.good()) return fail(GDF_ERR_INVALID_ARG, std::string("cannot open ") + prefix + names[i]);
    std::vector<float> h(static_cast<size_t>(n.n_params));
    f.read(reinterpret_cast<char*>(h.data()), static_cast<std::streamsize>(h.size() * 4));
    if (f.gcount() != static_cast<std::streamsize>(h.size() * 4))
      return fail(GDF_ERR_INVALID_ARG, std::string("short file ") + prefix + names[i]);
    gdf_status s = upload_params(n, h);
    if (s) return s;
  }
  return refresh_grid_il(ctx->c);
}

static gdf::DfKernelParams df_params(Context& c) {
  gdf::DfKernelParams p;
  std::memset(&p, 0, sizeof(p));
  const Net& t = c.net[0];
  const Net& f = c.net[1];
  p.grid_theta = t.ema16 + t.n_mlp;
  p.grid_phi = f.ema16 + f.n_mlp;
  const bool f8 = c.cfg.precision == GDF_PREC_FP8;
  p.blob_theta = f8 ? reinterpret_cast<const __half*>(t.blob_f8) : t.blob_ema;
  p.blob_phi = f8 ? reinterpret_cast<const __half*>(f.blob_f8) : f.blob_ema;
  p.blob_theta_bytes = f8 ? t.f8_bytes : t.blob_bytes;
  p.blob_phi_bytes = f8 ? f.f8_bytes : f.blob_bytes;
  p.hidden_theta = t.hidden;
  p.hidden_phi = f.hidden;
  p.gl_theta = t.gl;
  p.gl_phi = f.gl;
  p.err = c.d_err;
  p.bf16 = c.cfg.precision == GDF_PREC_BF16;
  p.fp8 = f8;
  return p;
}



gdf_status gdf_infer(gdf_ctx* ctx, const float* queries, const uint8_t* guided,
                     const float* uniforms, uint64_t philox_seed, uint64_t philox_offset,
                     float* wi, int64_t n, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(queries, "queries")) || (s = check_ptr(wi, "wi"))) return s;
  if (ctx->c.cfg.max_queries > 0 && n > ctx->c.cfg.max_queries)
    return fail(GDF_ERR_INVALID_ARG, "n exceeds max_queries");
  if ((reinterpret_cast<uintptr_t>(wi) & 15u) || (uniforms && (reinterpret_cast<uintptr_t>(uniforms) & 15u)))
    return fail(GDF_ERR_INVALID_ARG, "wi and uniforms must be 16-byte aligned");
  gdf::DfKernelParams p = df_params(ctx->c);
  p.queries = queries;
  p.guided = guided;
  p.uniforms = uniforms;
  p.wi = wi;
  p.n = n;
  p.philox_seed = philox_seed;
  p.philox_offset = philox_offset;
  if ((s = grid_features(ctx->c, queries, nullptr, gdf_aabb{}, n, p, static_cast<cudaStream_t>(stream))))
    return s;
  cudaError_t e = gdf::launch_df_fused(df_shape(ctx->c), gdf::kModeInfer, p, ctx->c.num_sms,
                                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "df_fused (infer)");
  return GDF_OK;
}

gdf_status gdf_infer_ex(gdf_ctx* ctx, const gdf_infer_args* a, void* stream) {
  if (!ctx || !a) return fail(GDF_ERR_INVALID_ARG, "null ctx / args");
  const int64_t n = a->n;
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(a->wi_dev, "wi"))) return s;
  if (a->shading) {
    const gdf_shading& sh = *a->shading;
    if ((s = check_ptr(sh.pos, "shading.pos")) || (s = check_ptr(sh.wo, "shading.wo")) ||
        (s = check_ptr(sh.normal, "shading.normal")) || (s = check_ptr(sh.roughness, "shading.roughness")))
      return s;
  } else if ((s = check_ptr(a->queries_dev, "queries"))) {
    return s;
  }
  if (ctx->c.cfg.max_queries > 0 && n > ctx->c.cfg.max_queries)
    return fail(GDF_ERR_INVALID_ARG, "n exceeds max_queries");
  if ((reinterpret_cast<uintptr_t>(a->wi_dev) & 15u) ||
      (a->uniforms_dev && (reinterpret_cast<uintptr_t>(a->uniforms_dev) & 15u)) ||
      (a->dir_pdf_dev && (reinterpret_cast<uintptr_t>(a->dir_pdf_dev) & 15u)))
    return fail(GDF_ERR_INVALID_ARG, "wi, uniforms and dir_pdf must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(a->cdf_norm_err_dev) & 7u)
    return fail(GDF_ERR_INVALID_ARG, "cdf_norm_err must be 8-byte aligned");
  gdf::DfKernelParams p = df_params(ctx->c);
  p.queries = a->queries_dev;
  if (a->shading) p.shading = *a->shading;
  p.aabb = a->aabb;
  p.guided = a->guided_dev;
  p.uniforms = a->uniforms_dev;
  p.wi = a->wi_dev;
  p.dir_pdf = a->dir_pdf_dev;
  p.norm_err = reinterpret_cast<unsigned long long*>(a->cdf_norm_err_dev);
  p.n = n;
  p.philox_seed = a->philox_seed;
  p.philox_offset = a->philox_offset;
  if ((s = grid_features(ctx->c, a->queries_dev, a->shading, a->aabb, n, p,
                         static_cast<cudaStream_t>(stream))))
    return s;
  if (a->stage_events)
    GDF_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(a->stage_events[0]), static_cast<cudaStream_t>(stream)));
  cudaError_t e = gdf::launch_df_fused(df_shape(ctx->c), gdf::kModeInfer, p, ctx->c.num_sms,
                                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "df_fused (infer)");
  if (a->stage_events)
    GDF_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(a->stage_events[1]), static_cast<cudaStream_t>(stream)));
  return GDF_OK;
}

gdf_status gdf_infer_host(gdf_ctx* ctx, const float* queries_h, const uint8_t* guided_h,
                          const float* uniforms_h, uint64_t philox_seed, uint64_t philox_offset,
                          const float* wi_in_h, float* wi_out_h, int64_t n, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(queries_h, "queries")) || (s = check_ptr(wi_in_h, "wi_in")) ||
      (s = check_ptr(wi_out_h, "wi_out")))
    return s;
  Context& c = ctx->c;
  if (c.cfg.max_queries > 0 && n > c.cfg.max_queries)
    return fail(GDF_ERR_INVALID_ARG, "n exceeds max_queries");
  if (n > c.host_cap) {
    cudaFree(c.host_q);
    cudaFree(c.host_g);
    cudaFree(c.host_u);
    cudaFree(c.host_wi);
    c.host_q = c.host_u = c.host_wi = nullptr;
    c.host_g = nullptr;
    c.host_cap = 0;
    const size_t m = static_cast<size_t>(n);
    if ((s = dalloc(&c.host_q, m * 9)) || (s = dalloc(&c.host_g, m)) || (s = dalloc(&c.host_u, m * 4)) ||
        (s = dalloc(&c.host_wi, m * 4)))
      return s;
    c.host_cap = n;
  }
  if (!c.pipe[0]) {
    for (cudaStream_t& ps : c.pipe) GDF_CUDA(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
    for (cudaEvent_t& e : c.pipe_ev) GDF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if ((s = ensure_features(c, (n + 127) / 128))) return s;
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  GDF_CUDA(cudaEventRecord(c.pipe_ev[3], user));
  for (cudaStream_t ps : c.pipe) GDF_CUDA(cudaStreamWaitEvent(ps, c.pipe_ev[3], 0));
  // Three streams: input copies, kernels, output copies. Each chunk has its
  // own device rows, so the input copies run back to back at the link's
  // rate (they bound the call: the kernels outrun PCIe), a chunk's kernels
  // start when its rows are in, and its output copy when they are done.
  // What remains after the last input copy is the last chunk's kernels and
  // output copy, so chunks are at most 4096 tiles and at most half of what
  // remains, down to 1024 tiles; each copy costs ≈13 µs of set-up, so the
  // guided flags (1 B per query) go in one copy ahead of the chunks.
  cudaStream_t s_in = c.pipe[0], s_run = c.pipe[1], s_out = c.pipe[2];
  constexpr int64_t kChunk = 4096 * 128, kMinChunk = 1024 * 128;
  auto issue = [&]() -> gdf_status {
    if (guided_h) GDF_CUDA(cudaMemcpyAsync(c.host_g, guided_h, static_cast<size_t>(n), cudaMemcpyHostToDevice, s_in));
    int64_t m = 0;
    for (int64_t b = 0; b < n; b += m) {
      const int64_t rest = n - b;
      m = std::min(kChunk, (rest / 2 + 127) / 128 * 128);
      if (m < kMinChunk) m = std::min(rest, kMinChunk);
      GDF_CUDA(cudaMemcpyAsync(c.host_q + b * 9, queries_h + b * 9, static_cast<size_t>(m) * 36,
                               cudaMemcpyHostToDevice, s_in));
      GDF_CUDA(cudaMemcpyAsync(c.host_wi + b * 4, wi_in_h + b * 4, static_cast<size_t>(m) * 16,
                               cudaMemcpyHostToDevice, s_in));
      if (uniforms_h)
        GDF_CUDA(cudaMemcpyAsync(c.host_u + b * 4, uniforms_h + b * 4, static_cast<size_t>(m) * 16,
                                 cudaMemcpyHostToDevice, s_in));
      // one event object per hand-over: each wait takes the record before it
      GDF_CUDA(cudaEventRecord(c.pipe_ev[4], s_in));
      GDF_CUDA(cudaStreamWaitEvent(s_run, c.pipe_ev[4], 0));
      gdf::DfKernelParams p = df_params(c);
      p.queries = c.host_q + b * 9;
      p.guided = guided_h ? c.host_g + b : nullptr;
      p.uniforms = uniforms_h ? c.host_u + b * 4 : nullptr;
      p.wi = c.host_wi + b * 4;
      p.n = m;
      p.philox_seed = philox_seed;
      p.philox_offset = philox_offset;
      p.philox_row_base = b;
      if ((s = grid_features(c, p.queries, nullptr, gdf_aabb{}, m, p, s_run, b / 128))) return s;
      cudaError_t e = gdf::launch_df_fused(df_shape(c), gdf::kModeInfer, p, c.num_sms, s_run);
      if (e != cudaSuccess) return cuda_fail(e, "df_fused (infer_host)");
      GDF_CUDA(cudaEventRecord(c.pipe_ev[5], s_run));
      GDF_CUDA(cudaStreamWaitEvent(s_out, c.pipe_ev[5], 0));
      GDF_CUDA(cudaMemcpyAsync(wi_out_h + b * 4, c.host_wi + b * 4, static_cast<size_t>(m) * 16,
                               cudaMemcpyDeviceToHost, s_out));
    }
    return GDF_OK;
  };
  const gdf_status issued = issue();
  // the three streams join the caller's, also after a failed launch
  for (int i = 0; i < 3; ++i) {
    GDF_CUDA(cudaEventRecord(c.pipe_ev[i], c.pipe[i]));
    GDF_CUDA(cudaStreamWaitEvent(user, c.pipe_ev[i], 0));
  }
  return issued;
}

}  // extern "C"

static gdf_status ensure_tools(Context& c, int64_t n) {
  if (n <= c.tool_cap) return GDF_OK;
  cudaFree(c.tool_q);
  cudaFree(c.tool_uv);
  cudaFree(c.tool_out);
  c.tool_q = c.tool_uv = c.tool_out = nullptr;
  c.tool_cap = 0;
  const size_t m = static_cast<size_t>(n);
  gdf_status s;
  if ((s = dalloc(&c.tool_q, m * 9)) || (s = dalloc(&c.tool_uv, m * 2)) || (s = dalloc(&c.tool_out, m * 4)))
    return s;
  c.tool_cap = n;
  return GDF_OK;
}

static gdf::QueryRow query_row(const float* q) {
  gdf::QueryRow r;
  for (int k = 0; k < 9; ++k) r.v[k] = q[k];
  return r;
}

extern "C" {

gdf_status gdf_pdf_image(gdf_ctx* ctx, const float* query_h, int32_t width, int32_t height,
                         float* image_dev, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  gdf_status s;
  if ((s = check_ptr(query_h, "query")) || (s = check_ptr(image_dev, "image"))) return s;
  if (width < 1 || height < 1 || static_cast<int64_t>(width) * height > (int64_t{1} << 26))
    return fail(GDF_ERR_INVALID_ARG, "image size must be 1 .. 2^26 pixels");
  Context& c = ctx->c;
  const int64_t n = static_cast<int64_t>(width) * height;
  if ((s = ensure_tools(c, n))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = gdf::launch_replicate(query_row(query_h), c.tool_q, c.tool_uv, nullptr, width, height, n, st);
  if (e != cudaSuccess) return cuda_fail(e, "replicate");
  gdf::DfKernelParams p = df_params(c);
  p.queries = c.tool_q;
  p.u_eval = c.tool_uv;
  p.pdf_out = c.tool_out;
  p.n = n;
  if ((s = grid_features(c, c.tool_q, nullptr, gdf_aabb{}, n, p, st))) return s;
  e = gdf::launch_df_fused(df_shape(c), gdf::kModeEval, p, c.num_sms, st);
  if (e != cudaSuccess) return cuda_fail(e, "df_fused (pdf image)");
  e = gdf::launch_pdf_image(c.tool_out, image_dev, n, st);
  if (e != cudaSuccess) return cuda_fail(e, "pdf image");
  return GDF_OK;
}

gdf_status gdf_sample_histogram(gdf_ctx* ctx, const float* query_h, int64_t n_samples, uint64_t seed,
                                int32_t width, int32_t height, uint32_t* counts_dev, float* dirs_dev,
                                void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  gdf_status s;
  if ((s = check_ptr(query_h, "query")) || (s = check_ptr(counts_dev, "counts"))) return s;
  if (n_samples < 0) return fail(GDF_ERR_INVALID_ARG, "n_samples < 0");
  if (width < 1 || height < 1 || static_cast<int64_t>(width) * height > (int64_t{1} << 26))
    return fail(GDF_ERR_INVALID_ARG, "image size must be 1 .. 2^26 pixels");
  Context& c = ctx->c;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GDF_CUDA(cudaMemsetAsync(counts_dev, 0, static_cast<size_t>(width) * height * 4, st));
  constexpr int64_t kChunk = int64_t{1} << 20;
  if ((s = ensure_tools(c, std::min(n_samples, kChunk)))) return s;
  for (int64_t b = 0; b < n_samples; b += kChunk) {
    const int64_t m = std::min(kChunk, n_samples - b);
    cudaError_t e = gdf::launch_replicate(query_row(query_h), c.tool_q, nullptr, c.tool_out, width, height, m, st);
    if (e != cudaSuccess) return cuda_fail(e, "replicate");
    gdf::DfKernelParams p = df_params(c);
    p.queries = c.tool_q;
    p.wi = c.tool_out;
    p.n = m;
    p.philox_seed = seed;
    p.philox_offset = 0;
    p.philox_row_base = b;
    if ((s = grid_features(c, c.tool_q, nullptr, gdf_aabb{}, m, p, st))) return s;
    e = gdf::launch_df_fused(df_shape(c), gdf::kModeInfer, p, c.num_sms, st);
    if (e != cudaSuccess) return cuda_fail(e, "df_fused (sampling)");
    e = gdf::launch_histogram(c.tool_out, m, width, height, counts_dev, dirs_dev ? dirs_dev + b * 2 : nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "histogram");
  }
  return GDF_OK;
}

gdf_status gdf_eval_pdf(gdf_ctx* ctx, const float* queries, const float* u, float* pdf_out,
                        int64_t n, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(queries, "queries")) || (s = check_ptr(u, "u")) || (s = check_ptr(pdf_out, "pdf_out")))
    return s;
  if (reinterpret_cast<uintptr_t>(pdf_out) & 7u) return fail(GDF_ERR_INVALID_ARG, "pdf_out must be 8-byte aligned");
  gdf::DfKernelParams p = df_params(ctx->c);
  p.queries = queries;
  p.u_eval = u;
  p.pdf_out = pdf_out;
  p.n = n;
  if ((s = grid_features(ctx->c, queries, nullptr, gdf_aabb{}, n, p, static_cast<cudaStream_t>(stream))))
    return s;
  cudaError_t e = gdf::launch_df_fused(df_shape(ctx->c), gdf::kModeEval, p, ctx->c.num_sms,
                                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "df_fused (eval)");
  return GDF_OK;
}

gdf_status gdf_post_inference(gdf_ctx* ctx, const float* lt, const float* lp, const uint8_t* guided,
                              const float* uniforms, float* wi, int64_t n, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(lt, "logits_theta")) || (s = check_ptr(lp, "logits_phi")) ||
      (s = check_ptr(uniforms, "uniforms")) || (s = check_ptr(wi, "wi")))
    return s;
  const gdf_config& c = ctx->c.cfg;
  cudaError_t e = gdf::launch_df_post(c.n_bins_theta, c.n_bins_phi, c.pdf_interp == GDF_PDF_LINEAR,
                                      lt, lp, guided, uniforms, wi, n, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "df_post");
  return GDF_OK;
}

static gdf::AdamParams adam_params(Context& c, int id, const gdf_adam_config& a, float loss_scale,
                                    double* sq, const int64_t* n_dev = nullptr) {
  Net& n = c.net[id];
  gdf::AdamParams p;
  std::memset(&p, 0, sizeof(p));
  p.n = n.n_params;
  p.n_mlp = n.n_mlp;
  p.partials = c.ws.partial[id];
  p.n_partials = gdf::train_ctas(c);
  p.grid_grad = n.grad;
  p.master = n.master;
  p.w16 = n.w16;
  p.ema16 = n.ema16;
  p.m = n.adam_m;
  p.v = n.adam_v;
  p.step = n.adam_step;
  p.blob_w16 = n.blob_w16;
  p.blob_ema = n.blob_ema;
  int64_t off = 0;
  p.n_layers = static_cast<int32_t>(n.rows.size());
  for (size_t l = 0; l < n.rows.size(); ++l) {
    p.layer_off[l] = off;
    p.layer_cols[l] = n.cols[l];
    off += static_cast<int64_t>(n.rows[l]) * n.cols[l];
  }
  // the step counter lives on the device; the optimizer kernel advances it
  p.opt = n.opt;
  p.n_dev = n_dev;
  p.loss_scale = loss_scale;
  p.lr = a.learning_rate;
  p.beta1 = a.beta1;
  p.beta2 = a.beta2;
  p.eps = a.epsilon;
  p.l2_reg = a.l2_reg;
  p.ema_decay = a.ema_decay;
  p.sq_partial = sq;
  p.n_blocks = gdf::kAdamBlocks;
  if (id < 2) {
    p.grid_il = c.grid_il;
    p.il_net = id;
    p.il_features = n.features;
  }
  p.lr_table = c.lr_table[id < 2 ? 0 : 1];
  p.lr_table_n = c.lr_table_n[id < 2 ? 0 : 1];
  p.blob_ema_bf16 = n.infer_bf16;
  p.blob_w16_bf16 = n.train_bf16;
  p.err = c.d_err;
  return p;
}

}  // extern "C"

namespace {

// One DF training step (learnedDistribution.cpp:247-288), stream-ordered.
// With n_dev set the batch holds min(*n_dev, n) records, read on the device
// (n bounds the launches), and an empty batch leaves every weight and the
// optimizer step counter untouched; loss_acc (nullable) gets the batch's
// mean loss added on the device.
gdf_status train_step_dev(Context& c, const float* in_theta, const float* in_phi, const float* target,
                          int64_t n, const int64_t* n_dev, double* loss_acc, cudaStream_t st) {
  const gdf::DfShape shape = df_shape(c);
  GDF_CUDA(cudaMemsetAsync(c.ws.dropped, 0, sizeof(unsigned long long), st));

  // 1. forward of both networks with fp16 pdf tables, loss and prefix
  gdf::DfKernelParams p = df_params(c);
  p.grid_theta = c.net[0].w16 + c.net[0].n_mlp;
  p.grid_phi = c.net[1].w16 + c.net[1].n_mlp;
  p.blob_theta = c.net[0].blob_w16;
  p.blob_phi = c.net[1].blob_w16;
  p.blob_theta_bytes = c.net[0].blob_bytes;
  p.blob_phi_bytes = c.net[1].blob_bytes;
  p.bf16 = c.net[0].train_bf16 ? 1 : 0;
  p.fp8 = 0;
  p.feat_theta = c.ws.feat[0];
  p.feat_phi = c.ws.feat[1];
  p.queries = in_theta;
  p.in_phi = in_phi;
  p.target = target;
  p.train_out = c.ws.fwd;
  p.n_dropped = c.ws.dropped;
  p.loss_scale_per_record = c.cfg.loss_scale / static_cast<float>(n);
  p.loss_scale = c.cfg.loss_scale;
  p.n_dev = n_dev;
  p.n = n;
  gdf::TrainFeatParams tf;
  std::memset(&tf, 0, sizeof(tf));
  tf.in_theta = in_theta;
  tf.in_phi = in_phi;
  tf.target = target;
  tf.n = n;
  tf.n_dev = n_dev;
  tf.n_tiles = (n + 127) / 128;
  tf.grid_theta = p.grid_theta;
  tf.grid_phi = p.grid_phi;
  tf.gl_theta = c.net[0].gl;
  tf.gl_phi = c.net[1].gl;
  tf.feat_theta = c.ws.feat[0];
  tf.feat_phi = c.ws.feat[1];
  tf.bf16 = p.bf16;
  cudaError_t e = gdf::launch_train_features(shape, tf, st);
  if (e != cudaSuccess) return cuda_fail(e, "train_features");
  e = gdf::launch_df_fused(shape, gdf::kModeTrainFeat, p, gdf::train_ctas(c), st);
  if (e != cudaSuccess) return cuda_fail(e, "df_fused (train forward)");

  // 2.-3. backward of each network, then its optimizer step. The theta
  // backward runs first; then the phi backward (one CTA per SM: its weight
  // gradients fill the TMEM; launched first) on one stream beside the theta
  // grid backward (fp32 atomics, a different bound) on a second stream,
  // which then runs the theta optimizer beside the phi grid backward. Each
  // network has its own dL/dfeatures buffer; both streams join the caller's
  // stream before the statistics. (The phi stream at high priority measured
  // the same: 1.222 against 1.227 ms.)
  auto backward = [&](int id, cudaStream_t sb) -> gdf_status {
    Net& nt = c.net[id];
    gdf::DfBwdParams b;
    std::memset(&b, 0, sizeof(b));
    b.in = id == 0 ? in_theta : in_phi;
    b.in_stride = id == 0 ? 9 : 10;
    b.target = target;
    b.fwd = c.ws.fwd;
    b.n = n;
    b.n_dev = n_dev;
    b.blob = nt.blob_w16;
    b.blob_bytes = nt.blob_bytes;
    b.grid = nt.w16 + nt.n_mlp;
    b.feat = c.ws.feat[id];
    b.dx = c.ws.dx[c.train_one_stream ? 0 : id];
    b.dx_rows = c.ws.capacity;
    b.grid_grad = nt.grad + nt.n_mlp;
    b.wgrad_partial = c.ws.partial[id];
    b.n_mlp = nt.n_mlp;
    b.hidden = nt.hidden;
    b.err = c.d_err;
    b.gl = nt.gl;
    b.bf16 = nt.train_bf16 ? 1 : 0;
    const cudaError_t eb = gdf::launch_df_train_bwd(shape, id == 1, b, gdf::train_ctas(c), sb);
    if (eb != cudaSuccess) return cuda_fail(eb, "df_train_bwd");
    return GDF_OK;
  };
  auto grid_and_optimizer = [&](int id, cudaStream_t sb) -> gdf_status {
    Net& nt = c.net[id];
    gdf::GridScatterParams g;
    std::memset(&g, 0, sizeof(g));
    g.in = id == 0 ? in_theta : in_phi;
    g.in_stride = id == 0 ? 9 : 10;
    g.fwd = c.ws.fwd;
    g.n = n;
    g.n_dev = n_dev;
    g.dx = c.ws.dx[c.train_one_stream ? 0 : id];
    g.dx_rows = c.ws.capacity;
    g.grid_grad = nt.grad + nt.n_mlp;
    g.gl = nt.gl;
    cudaError_t eg = gdf::launch_grid_scatter(nt.levels, nt.features, g, sb);
    if (eg != cudaSuccess) return cuda_fail(eg, "grid_scatter");
    gdf::AdamParams a = adam_params(c, id, c.cfg.adam_df, c.cfg.loss_scale,
                                    c.ws.sq + static_cast<size_t>(id) * gdf::kAdamBlocks, n_dev);
    a.grid_grad = nt.grad + nt.n_mlp;
    eg = gdf::launch_adam_ema(a, sb);
    if (eg != cudaSuccess) return cuda_fail(eg, "adam_ema");
    if (nt.infer_f8 && (eg = gdf::launch_pack_fp8(nt.f8_pack, sb)) != cudaSuccess) return cuda_fail(eg, "pack fp8");
    return GDF_OK;
  };
  gdf_status sg;
  if ((sg = backward(0, st))) return sg;
  if (c.train_one_stream) {  // one stream: both networks share dx[0]
    if ((sg = grid_and_optimizer(0, st)) || (sg = backward(1, st)) || (sg = grid_and_optimizer(1, st))) return sg;
  } else {
    if (!c.ws.dx[1] && (sg = dalloc(&c.ws.dx[1], static_cast<size_t>(c.ws.capacity) *
                                                     static_cast<size_t>(c.net[0].levels * c.net[0].features))))
      return sg;
    cudaStream_t s_phi = c.train_aux[0], s_theta = c.train_aux[1];
    GDF_CUDA(cudaEventRecord(c.train_ev[0], st));
    GDF_CUDA(cudaStreamWaitEvent(s_phi, c.train_ev[0], 0));
    GDF_CUDA(cudaStreamWaitEvent(s_theta, c.train_ev[0], 0));
    if (!(sg = backward(1, s_phi)) && !(sg = grid_and_optimizer(0, s_theta))) sg = grid_and_optimizer(1, s_phi);
    // both streams join the caller's, also after a failed launch
    GDF_CUDA(cudaEventRecord(c.train_ev[1], s_phi));
    GDF_CUDA(cudaEventRecord(c.train_ev[2], s_theta));
    GDF_CUDA(cudaStreamWaitEvent(st, c.train_ev[1], 0));
    GDF_CUDA(cudaStreamWaitEvent(st, c.train_ev[2], 0));
    if (sg) return sg;
  }
  // 4. FP64 loss and gradient-norm reductions
  e = gdf::launch_train_stats_mb(c.ws.fwd, n, n_dev, c.ws.sq, 2 * gdf::kAdamBlocks, c.ws.stat_part, c.ws.stats,
                                 loss_acc, st);
  if (e != cudaSuccess) return cuda_fail(e, "train_stats");
  return GDF_OK;
}

}  // namespace

extern "C" {

gdf_status gdf_train_step(gdf_ctx* ctx, const float* in_theta, const float* in_phi,
                          const float* target, int64_t n, gdf_train_stats* stats, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  if (n <= 0) return fail(GDF_ERR_INVALID_ARG, "n must be positive");
  if (n > c.ws.capacity) return fail(GDF_ERR_INVALID_ARG, "n exceeds max_train_batch");
  gdf_status s;
  if ((s = check_ptr(in_theta, "in_theta")) || (s = check_ptr(in_phi, "in_phi")) ||
      (s = check_ptr(target, "target")))
    return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = train_step_dev(c, in_theta, in_phi, target, n, nullptr, nullptr, st))) return s;
  if (stats) {
    double h[2];
    unsigned long long dropped = 0;
    GDF_CUDA(cudaMemcpyAsync(h, c.ws.stats, sizeof(h), cudaMemcpyDeviceToHost, st));
    GDF_CUDA(cudaMemcpyAsync(&dropped, c.ws.dropped, sizeof(dropped), cudaMemcpyDeviceToHost, st));
    GDF_CUDA(cudaStreamSynchronize(st));
    stats->loss = h[0] / static_cast<double>(n);
    stats->grad_norm = std::sqrt(h[1]);
    stats->n_records = n;
    stats->n_dropped = static_cast<int64_t>(dropped);
  }
  return GDF_OK;
}

gdf_status gdf_get_optimizer_state(const gdf_ctx* ctx, int32_t net, float* m, float* v,
                                   uint32_t* steps, int64_t n, uint32_t* opt_step) {
  Net* nt = net_of(const_cast<Context*>(ctx ? &ctx->c : nullptr), net);
  if (!nt) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id");
  if (n != nt->n_params) return fail(GDF_ERR_INVALID_ARG, "parameter count mismatch");
  GDF_CUDA(cudaDeviceSynchronize());
  if (m) GDF_CUDA(cudaMemcpy(m, nt->adam_m, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost));
  if (v) GDF_CUDA(cudaMemcpy(v, nt->adam_v, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost));
  if (steps) GDF_CUDA(cudaMemcpy(steps, nt->adam_step, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost));
  if (opt_step) {
    gdf::OptState o;
    GDF_CUDA(cudaMemcpy(&o, nt->opt, sizeof(o), cudaMemcpyDeviceToHost));
    *opt_step = o.step;
  }
  return GDF_OK;
}

gdf_status gdf_set_optimizer_state(gdf_ctx* ctx, int32_t net, const float* m, const float* v,
                                   const uint32_t* steps, int64_t n, uint32_t opt_step) {
  Net* nt = net_of(ctx ? &ctx->c : nullptr, net);
  if (!nt) return fail(GDF_ERR_INVALID_ARG, "bad ctx / net id");
  if (n != nt->n_params) return fail(GDF_ERR_INVALID_ARG, "parameter count mismatch");
  if (m) GDF_CUDA(cudaMemcpy(nt->adam_m, m, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice));
  if (v) GDF_CUDA(cudaMemcpy(nt->adam_v, v, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice));
  if (steps) GDF_CUDA(cudaMemcpy(nt->adam_step, steps, static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice));
  GDF_CUDA(cudaMemcpy(&nt->opt->step, &opt_step, sizeof(opt_step), cudaMemcpyHostToDevice));
  GDF_CUDA(cudaDeviceSynchronize());
  return GDF_OK;
}

gdf_status gdf_nrc_query(gdf_ctx* ctx, const float* in, float* out, int64_t m, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  if (!c.net[2].present) return fail(GDF_ERR_STATE, "NRC is disabled in this context");
  if (m < 0) return fail(GDF_ERR_INVALID_ARG, "m < 0");
  if (m == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(in, "in")) || (s = check_ptr(out, "out"))) return s;
  gdf::NrcParams p;
  std::memset(&p, 0, sizeof(p));
  p.in = in;
  p.out = out;
  p.n = m;
  p.blob = c.net[2].blob_ema;
  p.blob_bytes = c.net[2].blob_bytes;
  p.hidden = c.net[2].hidden;
  p.err = c.d_err;
  cudaError_t e = gdf::launch_nrc_query(p, c.num_sms, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "nrc_query");
  return GDF_OK;
}

gdf_status gdf_nrc_train_step(gdf_ctx* ctx, const float* in, const float* target, int64_t m,
                              gdf_train_stats* stats, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  if (!c.net[2].present) return fail(GDF_ERR_STATE, "NRC is disabled in this context");
  if (m <= 0) return fail(GDF_ERR_INVALID_ARG, "m must be positive");
  if (m > c.ws.capacity) return fail(GDF_ERR_INVALID_ARG, "m exceeds max_train_batch");
  gdf_status s;
  if ((s = check_ptr(in, "in")) || (s = check_ptr(target, "target"))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Net& n = c.net[2];
  GDF_CUDA(cudaMemsetAsync(c.ws.dropped, 0, sizeof(unsigned long long), st));
  gdf::NrcTrainParams p;
  std::memset(&p, 0, sizeof(p));
  p.in = in;
  p.target = target;
  p.n = m;
  p.blob = n.blob_w16;
  p.blob_bytes = n.blob_bytes;
  p.hidden = n.hidden;
  p.wgrad_partial = c.ws.partial[2];
  p.n_mlp = n.n_mlp;
  p.loss_scale = c.cfg.nrc_loss_scale;
  p.n_total = static_cast<float>(m * 3);
  p.loss_out = c.ws.fwd;
  p.n_dropped = c.ws.dropped;
  p.err = c.d_err;
  cudaError_t e = gdf::launch_nrc_train_bwd(p, gdf::train_ctas(c), st);
  if (e != cudaSuccess) return cuda_fail(e, "nrc_train_bwd");
  gdf::AdamParams a = adam_params(c, 2, c.cfg.adam_nrc, c.cfg.nrc_loss_scale, c.ws.sq + 2 * gdf::kAdamBlocks);
  a.grid_grad = nullptr;
  e = gdf::launch_adam_ema(a, st);
  if (e != cudaSuccess) return cuda_fail(e, "adam_ema (nrc)");
  e = gdf::launch_train_stats_mb(c.ws.fwd, m, nullptr, c.ws.sq + 2 * gdf::kAdamBlocks, gdf::kAdamBlocks,
                                 c.ws.stat_part, c.ws.stats, nullptr, st);
  if (e != cudaSuccess) return cuda_fail(e, "train_stats (nrc)");
  if (stats) {
    double h[2];
    unsigned long long dropped = 0;
    GDF_CUDA(cudaMemcpyAsync(h, c.ws.stats, sizeof(h), cudaMemcpyDeviceToHost, st));
    GDF_CUDA(cudaMemcpyAsync(&dropped, c.ws.dropped, sizeof(dropped), cudaMemcpyDeviceToHost, st));
    GDF_CUDA(cudaStreamSynchronize(st));
    // NRC::trainStep reports reduce(L) / batch (nrc.cpp:166)
    stats->loss = h[0] / static_cast<double>(m);
    stats->grad_norm = std::sqrt(h[1]);
    stats->n_records = m;
    stats->n_dropped = static_cast<int64_t>(dropped);
  }
  return GDF_OK;
}

}  // extern "C"

// ------------------------------------------------ records from the path tracer

namespace {

int64_t train_pixels(const gdf_train_pixels& px) {
  return px.stride > 0 ? px.max_queue_size / px.stride : 0;
}

gdf_status check_px(const gdf_path_state* st, const gdf_aabb* aabb, const gdf_train_pixels* px) {
  if (!st || !aabb || !px) return fail(GDF_ERR_INVALID_ARG, "null state / aabb / pixels");
  if (px->stride == 0 || px->max_queue_size < 0)
    return fail(GDF_ERR_INVALID_ARG, "train pixel stride must be >= 1 and queue size >= 0");
  if (px->max_queue_size > INT32_MAX) return fail(GDF_ERR_INVALID_ARG, "max_queue_size > 2^31 - 1");
  if (!st->cur_depth) return fail(GDF_ERR_INVALID_ARG, "cur_depth is null");
  return GDF_OK;
}

// Scratch of the count/scan/emit passes for n training pixels.
gdf_status ensure_scratch(Context& c, int64_t n) {
  gdf::PathWorkspace& w = c.pw;
  if (!w.totals) {
    gdf_status s;
    if ((s = dalloc(&w.totals, 2))) return s;
    if (cudaMallocHost(&w.totals_host, 2 * sizeof(int64_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(GDF_ERR_OOM_BUDGET, "pinned host allocation failed");
    }
  }
  if (n <= w.pixels) return GDF_OK;
  cudaFree(w.mask);
  cudaFree(w.block_counts);
  cudaFree(w.block_offsets);
  w.mask = nullptr;
  w.block_counts = nullptr;
  w.block_offsets = nullptr;
  w.pixels = 0;
  const int64_t nb = gdf::produce_blocks(n);
  gdf_status s;
  if ((s = dalloc(&w.mask, static_cast<size_t>(n))) ||
      (s = dalloc(&w.block_counts, static_cast<size_t>(2 * nb))) ||
      (s = dalloc(&w.block_offsets, static_cast<size_t>(2 * nb))))
    return s;
  w.pixels = n;
  return GDF_OK;
}

gdf_status ensure_df_records(Context& c, int64_t cap) {
  gdf::PathWorkspace& w = c.pw;
  if (cap <= w.df_cap) return GDF_OK;
  cudaFree(w.df_in);
  cudaFree(w.df_in_phi);
  cudaFree(w.df_target);
  w.df_in = w.df_in_phi = w.df_target = nullptr;
  w.df_cap = 0;
  gdf_status s;
  if ((s = dalloc(&w.df_in, static_cast<size_t>(cap) * 9)) ||
      (s = dalloc(&w.df_in_phi, static_cast<size_t>(cap) * 10)) ||
      (s = dalloc(&w.df_target, static_cast<size_t>(cap) * 9)))
    return s;
  w.df_cap = cap;
  return GDF_OK;
}

gdf_status ensure_plan(Context& c, int32_t batches) {
  gdf::PathWorkspace& w = c.pw;
  gdf_status s;
  if (!w.loss_acc && ((s = dalloc(&w.loss_acc, 1)) || (s = dalloc(&w.frame_loss, 1)) ||
                      (s = dalloc(&w.frame_n, 1))))
    return s;
  if (batches <= w.plan_len && w.plan) return GDF_OK;
  cudaFree(w.plan);
  w.plan = nullptr;
  w.plan_len = 0;
  if ((s = dalloc(&w.plan, static_cast<size_t>(batches) + 1))) return s;
  w.plan_len = batches;
  return GDF_OK;
}

gdf_status ensure_nrc_rows(Context& c, int64_t cap) {
  gdf::PathWorkspace& w = c.pw;
  if (cap <= w.nrc_cap) return GDF_OK;
  cudaFree(w.nrc_query);
  cudaFree(w.nrc_depth);
  cudaFree(w.nrc_pixel);
  cudaFree(w.nrc_out);
  cudaFree(w.nrc_train_in);
  cudaFree(w.nrc_train_target);
  w.nrc_query = w.nrc_out = w.nrc_train_in = w.nrc_train_target = nullptr;
  w.nrc_depth = w.nrc_pixel = nullptr;
  w.nrc_cap = 0;
  w.nrc_rows = 0;
  const size_t n = static_cast<size_t>(cap);
  gdf_status s;
  if ((s = dalloc(&w.nrc_query, n * 15)) || (s = dalloc(&w.nrc_depth, n)) ||
      (s = dalloc(&w.nrc_pixel, n)) || (s = dalloc(&w.nrc_out, n * 3)) ||
      (s = dalloc(&w.nrc_train_in, n * 15)) || (s = dalloc(&w.nrc_train_target, n * 3)))
    return s;
  w.nrc_cap = cap;
  return GDF_OK;
}

// One producer pass; counts[] receive the full list sizes (synchronises).
// Launches the record producer; the counts stay on the device (c.pw.totals).
gdf_status produce_dev(Context& c, const gdf_path_state& st, const gdf_aabb& aabb,
                       const gdf_train_pixels& px, int kind, gdf::ProduceParams p, cudaStream_t s) {
  const int64_t n = train_pixels(px);
  gdf_status rc = ensure_scratch(c, n);
  if (rc) return rc;
  p.st = st;
  p.aabb = aabb;
  p.n_train = n;
  p.offset = px.offset;
  p.stride = px.stride;
  p.bins_theta = c.cfg.n_bins_theta;
  p.linear = c.cfg.pdf_interp == GDF_PDF_LINEAR;
  p.mask = c.pw.mask;
  p.block_counts = c.pw.block_counts;
  p.block_offsets = c.pw.block_offsets;
  p.totals = c.pw.totals;
  cudaError_t e = gdf::launch_produce(p, kind, s);
  if (e != cudaSuccess) return cuda_fail(e, "record producer");
  return GDF_OK;
}

// The record producer with its counts read back to the host.
gdf_status produce(Context& c, const gdf_path_state& st, const gdf_aabb& aabb,
                   const gdf_train_pixels& px, int kind, gdf::ProduceParams p,
                   int64_t counts[2], cudaStream_t s) {
  gdf_status rc = produce_dev(c, st, aabb, px, kind, p, s);
  if (rc) return rc;
  GDF_CUDA(cudaMemcpyAsync(c.pw.totals_host, c.pw.totals, 2 * sizeof(int64_t),
                           cudaMemcpyDeviceToHost, s));
  GDF_CUDA(cudaStreamSynchronize(s));
  counts[0] = c.pw.totals_host[0];
  counts[1] = c.pw.totals_host[1];
  return GDF_OK;
}

gdf_status nrc_query_rows(Context& c, const float* in, float* out, int64_t m, cudaStream_t s) {
  if (m == 0) return GDF_OK;
  gdf::NrcParams q;
  std::memset(&q, 0, sizeof(q));
  q.in = in;
  q.out = out;
  q.n = m;
  q.blob = c.net[2].blob_ema;
  q.blob_bytes = c.net[2].blob_bytes;
  q.hidden = c.net[2].hidden;
  q.err = c.d_err;
  cudaError_t e = gdf::launch_nrc_query(q, c.num_sms, s);
  if (e != cudaSuccess) return cuda_fail(e, "nrc_query");
  return GDF_OK;
}

}  // namespace

extern "C" {

gdf_status gdf_prepare_queries(const gdf_shading* sh, const gdf_aabb* aabb, float* queries,
                               int64_t n, void* stream) {
  if (!sh || !aabb) return fail(GDF_ERR_INVALID_ARG, "null shading / aabb");
  if (n < 0) return fail(GDF_ERR_INVALID_ARG, "n < 0");
  if (n == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(sh->pos, "shading.pos")) || (s = check_ptr(sh->wo, "shading.wo")) ||
      (s = check_ptr(sh->normal, "shading.normal")) || (s = check_ptr(sh->roughness, "shading.roughness")) ||
      (s = check_ptr(queries, "queries")))
    return s;
  cudaError_t e = gdf::launch_prepare_queries(*sh, *aabb, queries, n, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "prepare_queries");
  return GDF_OK;
}

gdf_status gdf_build_train_records(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                                   const gdf_train_pixels* px, float* in_theta, float* in_phi,
                                   float* target, int64_t capacity, int64_t* count_host,
                                   void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  gdf_status s;
  if ((s = check_px(state, aabb, px))) return s;
  if (capacity < 0) return fail(GDF_ERR_INVALID_ARG, "capacity < 0");
  if (capacity > 0 && ((s = check_ptr(in_theta, "in_theta")) || (s = check_ptr(in_phi, "in_phi")) ||
                       (s = check_ptr(target, "target"))))
    return s;
  gdf::ProduceParams p;
  std::memset(&p, 0, sizeof(p));
  p.out_a0 = in_theta;
  p.out_a1 = in_phi;
  p.out_a2 = target;
  p.cap_a = capacity;
  int64_t counts[2];
  if ((s = produce(ctx->c, *state, *aabb, *px, gdf::kRecordsDf, p, counts,
                   static_cast<cudaStream_t>(stream))))
    return s;
  if (count_host) *count_host = counts[0];
  if (counts[0] > capacity) return fail(GDF_ERR_INVALID_ARG, "more records than capacity");
  return GDF_OK;
}

gdf_status gdf_build_nrc_records(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                                 const gdf_train_pixels* px, int32_t with_training,
                                 float* query_in, int32_t* query_depth, int32_t* query_pixel,
                                 int64_t query_capacity, float* train_in, float* train_target,
                                 int64_t train_capacity, int64_t* counts_host, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  gdf_status s;
  if ((s = check_px(state, aabb, px))) return s;
  if (query_capacity < 0 || train_capacity < 0) return fail(GDF_ERR_INVALID_ARG, "capacity < 0");
  if (query_capacity > 0 && ((s = check_ptr(query_in, "query_in")) ||
                             (s = check_ptr(query_depth, "query_depth")) ||
                             (s = check_ptr(query_pixel, "query_pixel"))))
    return s;
  if (with_training && train_capacity > 0 &&
      ((s = check_ptr(train_in, "train_in")) || (s = check_ptr(train_target, "train_target"))))
    return s;
  gdf::ProduceParams p;
  std::memset(&p, 0, sizeof(p));
  p.out_a0 = query_in;
  p.a_depth = query_depth;
  p.a_pixel = query_pixel;
  p.cap_a = query_capacity;
  p.out_b0 = train_in;
  p.out_b1 = train_target;
  p.cap_b = with_training ? train_capacity : 0;
  int64_t counts[2];
  if ((s = produce(ctx->c, *state, *aabb, *px,
                   with_training ? gdf::kRecordsNrcTrain : gdf::kRecordsNrcQuery, p, counts,
                   static_cast<cudaStream_t>(stream))))
    return s;
  if (counts_host) {
    counts_host[0] = counts[0];
    counts_host[1] = counts[1];
  }
  if (counts[0] > query_capacity || counts[1] > p.cap_b)
    return fail(GDF_ERR_INVALID_ARG, "more rows than capacity");
  return GDF_OK;
}

gdf_status gdf_apply_nrc(gdf_ctx* ctx, gdf_path_state* state, const float* nrc_out,
                         const int32_t* depth, const int32_t* pixel, int64_t m, void* stream) {
  if (!ctx || !state) return fail(GDF_ERR_INVALID_ARG, "null ctx / state");
  if (m < 0) return fail(GDF_ERR_INVALID_ARG, "m < 0");
  if (m == 0) return GDF_OK;
  gdf_status s;
  if ((s = check_ptr(nrc_out, "nrc_out")) || (s = check_ptr(depth, "depth")) ||
      (s = check_ptr(pixel, "pixel")) || (s = check_ptr(state->cur_depth, "cur_depth")))
    return s;
  cudaError_t e = gdf::launch_apply_nrc(*state, nrc_out, depth, pixel, m, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "apply_nrc");
  return GDF_OK;
}

gdf_status gdf_nrc_train_paths(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                               const gdf_train_pixels* px, float* loss_host,
                               int64_t* n_samples_host, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  if (!c.net[2].present) return fail(GDF_ERR_STATE, "NRC is disabled in this context");
  gdf_status s;
  if ((s = check_px(state, aabb, px))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t cap = train_pixels(*px) * GDF_MAX_TRAIN_DEPTH;
  if ((s = ensure_nrc_rows(c, cap))) return s;
  gdf::ProduceParams p;
  std::memset(&p, 0, sizeof(p));
  p.out_a0 = c.pw.nrc_query;
  p.a_depth = c.pw.nrc_depth;
  p.a_pixel = c.pw.nrc_pixel;
  p.cap_a = c.pw.nrc_cap;
  p.out_b0 = c.pw.nrc_train_in;
  p.out_b1 = c.pw.nrc_train_target;
  p.cap_b = c.pw.nrc_cap;
  int64_t counts[2];
  if ((s = produce(c, *state, *aabb, *px, gdf::kRecordsNrcTrain, p, counts, st))) return s;
  c.pw.nrc_rows = counts[0];
  const int64_t n = counts[1];
  if (n_samples_host) *n_samples_host = n;
  // NRC::trainStep batch loop (nrc.cpp:129-168), including its use of the
  // rounded local batch size as the row offset.
  const int64_t bs = c.cfg.nrc_batch_size;
  const int64_t batches = std::max<int64_t>(n / bs + 1, c.cfg.nrc_batches_per_frame);
  const int64_t eff = std::min<int64_t>(n / batches, bs);
  double loss_sum = 0.0;
  for (int64_t it = 0; it < batches; ++it) {
    int64_t local = std::min<int64_t>(n - it * eff, eff);
    local -= local % 128;
    if (local < c.cfg.min_train_batch) break;
    gdf_train_stats ts;
    if ((s = gdf_nrc_train_step(ctx, c.pw.nrc_train_in + it * local * 15,
                                c.pw.nrc_train_target + it * local * 3, local, &ts, stream)))
      return s;
    loss_sum += ts.loss;
  }
  if (loss_host) *loss_host = static_cast<float>(loss_sum / static_cast<double>(batches));
  return GDF_OK;
}

gdf_status gdf_nrc_substitute_paths(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                                    const gdf_train_pixels* px, int32_t skip_generation,
                                    void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  if (!c.net[2].present) return fail(GDF_ERR_STATE, "NRC is disabled in this context");
  gdf_status s;
  if ((s = check_px(state, aabb, px))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!skip_generation) {
    const int64_t cap = train_pixels(*px) * GDF_MAX_TRAIN_DEPTH;
    if ((s = ensure_nrc_rows(c, cap))) return s;
    gdf::ProduceParams p;
    std::memset(&p, 0, sizeof(p));
    p.out_a0 = c.pw.nrc_query;
    p.a_depth = c.pw.nrc_depth;
    p.a_pixel = c.pw.nrc_pixel;
    p.cap_a = c.pw.nrc_cap;
    int64_t counts[2];
    if ((s = produce(c, *state, *aabb, *px, gdf::kRecordsNrcQuery, p, counts, st))) return s;
    c.pw.nrc_rows = counts[0];
  }
  const int64_t m = c.pw.nrc_rows;
  if ((s = nrc_query_rows(c, c.pw.nrc_query, c.pw.nrc_out, m, st))) return s;
  if ((s = gdf_apply_nrc(ctx, state, c.pw.nrc_out, c.pw.nrc_depth, c.pw.nrc_pixel, m, stream)))
    return s;
  c.pw.nrc_rows = 0;  // inferenceBuffer clear() (nrc.cpp:216)
  GDF_CUDA(cudaStreamSynchronize(st));
  return GDF_OK;
}

gdf_status gdf_train_paths_async(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                                 const gdf_train_pixels* px, float* loss_dev, int64_t* n_samples_dev,
                                 void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  gdf_status s;
  if ((s = check_px(state, aabb, px))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t cap = train_pixels(*px) * GDF_MAX_TRAIN_DEPTH;
  const int32_t per_frame = c.cfg.df_batches_per_frame;
  if ((s = ensure_df_records(c, cap)) || (s = ensure_plan(c, std::max<int32_t>(per_frame, 1)))) return s;
  gdf::ProduceParams p;
  std::memset(&p, 0, sizeof(p));
  p.out_a0 = c.pw.df_in;
  p.out_a1 = c.pw.df_in_phi;
  p.out_a2 = c.pw.df_target;
  p.cap_a = c.pw.df_cap;
  if ((s = produce_dev(c, *state, *aabb, *px, gdf::kRecordsDf, p, st))) return s;
  // LearnedDistribution::trainStep batch loop (learnedDistribution.cpp:226-290)
  // with the record count on the device: every batch the loop can reach is
  // launched, sized by the plan, and one past the count trains nothing.
  const int64_t bs = c.cfg.df_batch_size;
  cudaError_t e = gdf::launch_df_batch_plan(c.pw.totals, bs, per_frame, c.cfg.min_train_batch, c.pw.plan,
                                            c.pw.loss_acc, st);
  if (e != cudaSuccess) return cuda_fail(e, "batch plan");
  for (int32_t it = 0; it < per_frame; ++it) {
    const int64_t o = it * bs;
    if (o >= c.pw.df_cap) break;  // the count never exceeds the record capacity
    const int64_t bound = std::min<int64_t>(bs, c.pw.df_cap - o);
    if ((s = train_step_dev(c, c.pw.df_in + o * 9, c.pw.df_in_phi + o * 10, c.pw.df_target + o * 9, bound,
                            c.pw.plan + 1 + it, c.pw.loss_acc, st)))
      return s;
  }
  e = gdf::launch_df_frame_finish(c.pw.plan, c.pw.loss_acc, c.pw.totals, loss_dev, n_samples_dev, st);
  if (e != cudaSuccess) return cuda_fail(e, "frame finish");
  return GDF_OK;
}

gdf_status gdf_train_paths(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                           const gdf_train_pixels* px, float* loss_host, int64_t* n_samples_host,
                           void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  Context& c = ctx->c;
  gdf_status s;
  if ((s = check_px(state, aabb, px)) || (s = ensure_plan(c, std::max<int32_t>(c.cfg.df_batches_per_frame, 1))))
    return s;
  if ((s = gdf_train_paths_async(ctx, state, aabb, px, c.pw.frame_loss, c.pw.frame_n, stream))) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float loss = 0.f;
  int64_t n = 0;
  GDF_CUDA(cudaMemcpyAsync(&loss, c.pw.frame_loss, sizeof(loss), cudaMemcpyDeviceToHost, st));
  GDF_CUDA(cudaMemcpyAsync(&n, c.pw.frame_n, sizeof(n), cudaMemcpyDeviceToHost, st));
  GDF_CUDA(cudaStreamSynchronize(st));
  if (loss_host) *loss_host = loss;
  if (n_samples_host) *n_samples_host = n;
  return GDF_OK;
}

gdf_status gdf_sync_status(gdf_ctx* ctx, void* stream) {
  if (!ctx) return fail(GDF_ERR_INVALID_ARG, "ctx is null");
  GDF_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  uint32_t err = 0;
  GDF_CUDA(cudaMemcpy(&err, ctx->c.d_err, 4, cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(ctx->c.d_err, 0, 4);
    return fail(GDF_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(err) + ")");
  }
  return GDF_OK;
}

}  // extern "C"
