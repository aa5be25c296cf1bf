// group.cpp -- grouped inference over many contexts (gdf_group_*): one
// grid-feature launch and one persistent fused launch for all jobs,
// replayed from a CUDA graph, with the warpgroups per CTA and the feature
// kernel's block size chosen by timing the candidates on the job set.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../kernels/group_kernels.h"
#include "context.h"

namespace {

gdf_status gfail(gdf_status s, const std::string& msg) {
  gdf::set_last_error(msg.c_str());
  return s;
}

gdf_status gcuda(cudaError_t e, const char* what) {
  cudaGetLastError();
  return gfail(GDF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GDF_GCUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return gcuda(e_, #call);       \
  } while (0)

struct Plan {
  int levels = 0, features = 0;
  bool linear = false, bf16 = false;
  int wgs = 0, fblock = 0;
  uint32_t bt = 0, bp = 0;
  gdf::GridLevels gl{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the feature launch, whose grid follows the call's row count
  cudaGraphNode_t feat_node = nullptr;
  cudaKernelNodeParams feat_params{};
  // the fused launch, whose grid follows the group's SM cap
  cudaGraphNode_t fused_node = nullptr;
  cudaKernelNodeParams fused_params{};
  unsigned fused_grid = 0;  // as captured: one CTA per SM
};

}  // namespace

struct gdf_group {
  int device = 0;
  int num_sms = 148;
  int sm_cap = 0;  // CTAs of the fused launch (0: one per SM)
  int32_t max_jobs = 0;
  gdf::GroupHeader* d_hdr = nullptr;
  gdf::GroupJobDev* d_jobs = nullptr;
  // pinned staging of the job table, two slots so a call never overwrites
  // a table whose copy is still queued
  uint8_t* h_stage[2] = {nullptr, nullptr};
  cudaEvent_t copied[2] = {nullptr, nullptr};
  int slot = 0;
  __half* feat = nullptr;  // stream-ordered allocation (cudaMallocAsync)
  int64_t feat_tiles = 0;
  cudaEvent_t last_launch = nullptr;  // after the group's last replay
  bool launched = false;
  uint32_t* d_err = nullptr;
  // per-job completion: warps done per job (device), and per job the
  // sequence number of the last call that finished it (host-mapped)
  uint32_t* d_job_tiles_done = nullptr;
  uint32_t* h_job_flag = nullptr;
  uint32_t* d_job_flag = nullptr;
  uint32_t seq = 0;               // sequence number of the last call
  bool track = false;             // job completion reported (gdf_group_track_jobs)
  std::vector<int64_t> job_n;     // the last call's job sizes
  cudaStream_t cap_stream = nullptr;
  std::vector<Plan> plans;
  // (levels, features, jobs, log2 tiles) -> (warpgroups, feature block)
  std::map<std::tuple<int, int, int, int>, std::pair<int, int>> tuned;
  float* tune_wi = nullptr;
  int64_t tune_cap = 0;
  int last_wgs = 0, last_fblock = 0;
  float last_tune_ms[4] = {0.f, 0.f, 0.f, 0.f};
  int pinned_wgs = 0, pinned_fblock = 0;  // set: skip tuning
};

namespace {

size_t stage_bytes(int32_t max_jobs) {
  return sizeof(gdf::GroupHeader) + static_cast<size_t>(max_jobs) * sizeof(gdf::GroupJobDev);
}

void drop_plans(gdf_group* g) {
  for (Plan& p : g->plans) {
    if (p.exec) cudaGraphExecDestroy(p.exec);
    if (p.graph) cudaGraphDestroy(p.graph);
  }
  g->plans.clear();
}

// Grows the feature buffer. Its only reader is the group's own last replay
// (calls on one group are ordered), so the growth waits for that replay
// alone and frees and allocates stream-ordered: work on other streams (a
// server's training steps) is not waited for.
gdf_status ensure_feat(gdf_group* g, int64_t tiles, int lf, cudaStream_t st) {
  if (tiles <= g->feat_tiles) return GDF_OK;
  if (g->launched) GDF_GCUDA(cudaEventSynchronize(g->last_launch));
  drop_plans(g);
  if (g->feat) cudaFreeAsync(g->feat, st);
  g->feat = nullptr;
  g->feat_tiles = 0;
  const int64_t cap = tiles + tiles / 4 + 64;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&g->feat),
                                  static_cast<size_t>(2 * cap * 128 * lf) * sizeof(__half), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return gfail(GDF_ERR_OOM_BUDGET, "grouped feature buffer");
  }
  g->feat_tiles = cap;
  return GDF_OK;
}

struct JobSet {
  int32_t n_jobs = 0;
  int levels, features;
  bool linear, bf16;
  uint32_t bt = 0, bp = 0;
  int64_t total_tiles = 0;
  gdf::GridLevels gl{};
};

gdf_status check_jobs(const gdf_job* jobs, int32_t n, JobSet* js) {
  for (int32_t i = 0; i < n; ++i) {
    const gdf_job& j = jobs[i];
    if (!j.ctx) return gfail(GDF_ERR_INVALID_ARG, "job without a context");
    if (j.n < 0) return gfail(GDF_ERR_INVALID_ARG, "job with n < 0");
    if (j.n > 0 && (!j.queries_dev || !j.wi_dev)) return gfail(GDF_ERR_INVALID_ARG, "job without queries / wi");
    if ((reinterpret_cast<uintptr_t>(j.wi_dev) & 15u) ||
        (j.uniforms_dev && (reinterpret_cast<uintptr_t>(j.uniforms_dev) & 15u)))
      return gfail(GDF_ERR_INVALID_ARG, "wi and uniforms must be 16-byte aligned");
    const gdf::Context& c = j.ctx->c;
    const int levels = c.cfg.grid_theta.n_levels, features = c.cfg.grid_theta.n_features_per_level;
    const bool linear = c.cfg.pdf_interp == GDF_PDF_LINEAR, bf16 = c.cfg.precision == GDF_PREC_BF16;
    if (c.cfg.precision == GDF_PREC_FP8)
      return gfail(GDF_ERR_UNSUPPORTED, "grouped launches take the FP16 and BF16 forms");
    if (i == 0) {
      js->levels = levels;
      js->features = features;
      js->linear = linear;
      js->bf16 = bf16;
      js->gl = c.net[0].gl;
    } else if (levels != js->levels || features != js->features || linear != js->linear ||
               bf16 != js->bf16 || std::memcmp(&c.net[0].gl, &js->gl, sizeof(gdf::GridLevels)) != 0) {
      return gfail(GDF_ERR_UNSUPPORTED,
                   "grouped jobs must share the grid configuration, pdf interpolation and precision");
    }
    js->bt = std::max(js->bt, c.net[0].blob_bytes);
    js->bp = std::max(js->bp, c.net[1].blob_bytes);
    js->total_tiles += (j.n + 127) / 128;
  }
  gdf::GroupShape s{js->levels, js->features, js->linear, js->bf16};
  if (!gdf::group_shape_supported(s)) return gfail(GDF_ERR_UNSUPPORTED, "no grouped kernel for this grid shape");
  return GDF_OK;
}

// Writes the table for `wgs` warpgroups per CTA into a staging slot and
// queues its copy to the device; wi_override (nullable) redirects every
// job's guiding data to one scratch buffer (tuning runs).
gdf_status upload_table(gdf_group* g, const gdf_job* jobs, int32_t n, int wgs, float* wi_override,
                        uint32_t seq, cudaStream_t st) {
  const int k = g->slot;
  g->slot ^= 1;
  GDF_GCUDA(cudaEventSynchronize(g->copied[k]));
  auto* hdr = reinterpret_cast<gdf::GroupHeader*>(g->h_stage[k]);
  auto* tab = reinterpret_cast<gdf::GroupJobDev*>(g->h_stage[k] + sizeof(gdf::GroupHeader));
  int64_t tile = 0, super = 0, wi_off = 0;
  for (int32_t i = 0; i < n; ++i) {
    const gdf_job& j = jobs[i];
    const gdf::Context& c = j.ctx->c;
    gdf::GroupJobDev& d = tab[i];
    d.blob_theta = c.net[0].blob_ema;
    d.blob_phi = c.net[1].blob_ema;
    d.blob_theta_bytes = c.net[0].blob_bytes;
    d.blob_phi_bytes = c.net[1].blob_bytes;
    d.hidden_theta = c.net[0].hidden;
    d.hidden_phi = c.net[1].hidden;
    d.bins_theta = c.cfg.n_bins_theta;
    d.bins_phi = c.cfg.n_bins_phi;
    d.grid_il = c.grid_il;
    d.queries = j.queries_dev;
    d.guided = j.guided_dev;
    d.uniforms = j.uniforms_dev;
    d.wi = wi_override ? wi_override + wi_off * 4 : j.wi_dev;
    d.n = j.n;
    d.seed = j.philox_seed;
    d.offset = j.philox_offset;
    d.tile_begin = tile;
    d.super_begin = super;
    const int64_t tiles = (j.n + 127) / 128;
    tile += tiles;
    super += (tiles + wgs - 1) / wgs;
    wi_off += (j.n + 3) / 4 * 4;
  }
  hdr->n_jobs = n;
  hdr->seq = seq;
  hdr->track = g->track ? 1u : 0u;
  hdr->pad = 0u;
  hdr->total_tiles = tile;
  hdr->n_super = super;
  GDF_GCUDA(cudaMemcpyAsync(g->d_hdr, hdr, sizeof(gdf::GroupHeader), cudaMemcpyHostToDevice, st));
  GDF_GCUDA(cudaMemcpyAsync(g->d_jobs, tab, static_cast<size_t>(n) * sizeof(gdf::GroupJobDev),
                            cudaMemcpyHostToDevice, st));
  GDF_GCUDA(cudaEventRecord(g->copied[k], st));
  return GDF_OK;
}

int64_t feature_blocks(const JobSet& js, int fblock) {
  return js.total_tiles * 128 * (js.levels * js.features / 8) / fblock;
}

gdf_status get_plan(gdf_group* g, const JobSet& js, int wgs, int fblock, size_t* out) {
  for (size_t i = 0; i < g->plans.size(); ++i) {
    const Plan& p = g->plans[i];
    if (p.levels == js.levels && p.features == js.features && p.linear == js.linear && p.bf16 == js.bf16 &&
        p.wgs == wgs && p.fblock == fblock && p.bt == js.bt && p.bp == js.bp &&
        std::memcmp(&p.gl, &js.gl, sizeof(gdf::GridLevels)) == 0) {
      *out = i;
      return GDF_OK;
    }
  }
  const gdf::GroupShape shape{js.levels, js.features, js.linear, js.bf16};
  gdf::GroupParams prm;
  std::memset(&prm, 0, sizeof(prm));
  prm.hdr = g->d_hdr;
  prm.jobs = g->d_jobs;
  prm.feat_theta = g->feat;
  prm.feat_phi = g->feat + g->feat_tiles * 128 * js.levels * js.features;
  prm.gl = js.gl;
  prm.max_blob_theta = js.bt;
  prm.max_blob_phi = js.bp;
  prm.err = g->d_err;
  prm.job_tiles_done = g->d_job_tiles_done;
  prm.job_flag = g->d_job_flag;
  const size_t smem = gdf::group_fused_smem_bytes(shape, wgs, js.bt, js.bp);
  if (smem > 227u * 1024u) return gfail(GDF_ERR_UNSUPPORTED, "grouped kernel shared memory exceeds 227 KB");
  cudaGraph_t graph = nullptr;
  GDF_GCUDA(cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeRelaxed));
  cudaError_t e1 = gdf::launch_group_features(shape, prm, static_cast<int>(feature_blocks(js, fblock)), fblock,
                                              g->cap_stream);
  cudaError_t e2 = gdf::launch_group_fused(shape, wgs, prm, g->num_sms, g->cap_stream);
  cudaError_t e3 = cudaStreamEndCapture(g->cap_stream, &graph);
  if (e1 != cudaSuccess) return gcuda(e1, "grouped features (capture)");
  if (e2 != cudaSuccess) return gcuda(e2, "grouped fused (capture)");
  if (e3 != cudaSuccess) return gcuda(e3, "end capture");
  Plan p;
  p.graph = graph;
  size_t n_roots = 1;
  cudaError_t e4 = cudaGraphGetRootNodes(graph, &p.feat_node, &n_roots);
  if (e4 == cudaSuccess && n_roots != 1) e4 = cudaErrorInvalidValue;
  if (e4 == cudaSuccess) e4 = cudaGraphKernelNodeGetParams(p.feat_node, &p.feat_params);
  if (e4 == cudaSuccess) {
    cudaGraphNode_t nodes[2];
    size_t n_nodes = 2;
    e4 = cudaGraphGetNodes(graph, nodes, &n_nodes);
    if (e4 == cudaSuccess && n_nodes != 2) e4 = cudaErrorInvalidValue;
    if (e4 == cudaSuccess) p.fused_node = nodes[0] == p.feat_node ? nodes[1] : nodes[0];
    if (e4 == cudaSuccess) e4 = cudaGraphKernelNodeGetParams(p.fused_node, &p.fused_params);
    p.fused_grid = p.fused_params.gridDim.x;
  }
  if (e4 == cudaSuccess) e4 = cudaGraphInstantiate(&p.exec, graph, 0);
  if (e4 != cudaSuccess) {
    cudaGraphDestroy(graph);
    return gcuda(e4, "graph instantiate");
  }
  p.levels = js.levels;
  p.features = js.features;
  p.linear = js.linear;
  p.bf16 = js.bf16;
  p.wgs = wgs;
  p.fblock = fblock;
  p.bt = js.bt;
  p.bp = js.bp;
  p.gl = js.gl;
  g->plans.push_back(p);
  *out = g->plans.size() - 1;
  return GDF_OK;
}

// Sizes the feature launch to the job set and replays the plan's graph
// (parameter updates apply to launches queued after them).
gdf_status launch_plan(gdf_group* g, size_t plan, const JobSet& js, cudaStream_t st) {
  Plan& p = g->plans[plan];
  p.feat_params.gridDim = dim3(static_cast<unsigned>(feature_blocks(js, p.fblock)));
  GDF_GCUDA(cudaGraphExecKernelNodeSetParams(p.exec, p.feat_node, &p.feat_params));
  GDF_GCUDA(cudaMemsetAsync(g->d_job_tiles_done, 0, static_cast<size_t>(js.n_jobs) * 4, st));
  const unsigned grid = g->sm_cap > 0 ? std::min(p.fused_grid, static_cast<unsigned>(g->sm_cap)) : p.fused_grid;
  if (p.fused_params.gridDim.x != grid) {
    p.fused_params.gridDim = dim3(grid);
    GDF_GCUDA(cudaGraphExecKernelNodeSetParams(p.exec, p.fused_node, &p.fused_params));
  }
  GDF_GCUDA(cudaGraphLaunch(p.exec, st));
  GDF_GCUDA(cudaEventRecord(g->last_launch, st));
  g->launched = true;
  return GDF_OK;
}

// Times each (warpgroups, feature block) candidate on the job set, writing
// into scratch copies of the guiding data, and keeps the fastest.
gdf_status autotune(gdf_group* g, const gdf_job* jobs, int32_t n, const JobSet& js, cudaStream_t st,
                    std::pair<int, int>* best) {
  int64_t total = 0;
  for (int32_t i = 0; i < n; ++i) total += (jobs[i].n + 3) / 4 * 4;
  if (total > g->tune_cap) {
    GDF_GCUDA(cudaStreamSynchronize(st));
    cudaFree(g->tune_wi);
    g->tune_wi = nullptr;
    g->tune_cap = 0;
    if (cudaMalloc(&g->tune_wi, static_cast<size_t>(total) * 16) != cudaSuccess) {
      cudaGetLastError();
      return gfail(GDF_ERR_OOM_BUDGET, "grouped tuning scratch");
    }
    g->tune_cap = total;
  }
  // candidates are timed on the whole device, whatever the launch cap
  struct Uncap {
    gdf_group* g;
    int cap;
    ~Uncap() { g->sm_cap = cap; }
  } uncap{g, g->sm_cap};
  g->sm_cap = 0;
  const std::pair<int, int> cand[4] = {{4, 256}, {4, 128}, {2, 256}, {2, 128}};
  cudaEvent_t a, b;
  GDF_GCUDA(cudaEventCreate(&a));
  GDF_GCUDA(cudaEventCreate(&b));
  float best_ms = 1e30f;
  gdf_status s = GDF_OK;
  for (int k = 0; k < 4 && s == GDF_OK; ++k) {
    int64_t off = 0;
    for (int32_t i = 0; i < n; ++i) {
      if (jobs[i].n > 0)
        GDF_GCUDA(cudaMemcpyAsync(g->tune_wi + off * 4, jobs[i].wi_dev, static_cast<size_t>(jobs[i].n) * 16,
                                  cudaMemcpyDeviceToDevice, st));
      off += (jobs[i].n + 3) / 4 * 4;
    }
    size_t plan = 0;
    // sequence number 0: a timing run marks no job done
    if ((s = upload_table(g, jobs, n, cand[k].first, g->tune_wi, 0u, st))) break;
    if ((s = get_plan(g, js, cand[k].first, cand[k].second, &plan))) break;
    if ((s = launch_plan(g, plan, js, st))) break;  // warm-up
    GDF_GCUDA(cudaEventRecord(a, st));
    if ((s = launch_plan(g, plan, js, st))) break;
    GDF_GCUDA(cudaEventRecord(b, st));
    GDF_GCUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    GDF_GCUDA(cudaEventElapsedTime(&ms, a, b));
    g->last_tune_ms[k] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      *best = cand[k];
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return s;
}

}  // namespace

extern "C" {

gdf_status gdf_group_create(int32_t max_jobs, gdf_group** out) {
  if (!out || max_jobs < 1 || max_jobs > 4096) return gfail(GDF_ERR_INVALID_ARG, "max_jobs must be in [1, 4096]");
  *out = nullptr;
  gdf_group* g = new (std::nothrow) gdf_group();
  if (!g) return gfail(GDF_ERR_OOM_BUDGET, "host allocation failed");
  auto bail = [&](gdf_status s) {
    gdf_group_destroy(g);
    return s;
  };
  g->max_jobs = max_jobs;
  if (cudaGetDevice(&g->device) != cudaSuccess) return bail(gcuda(cudaGetLastError(), "cudaGetDevice"));
  cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device);
  if (cudaMalloc(&g->d_hdr, sizeof(gdf::GroupHeader)) != cudaSuccess ||
      cudaMalloc(&g->d_jobs, static_cast<size_t>(max_jobs) * sizeof(gdf::GroupJobDev)) != cudaSuccess ||
      cudaMalloc(&g->d_err, 4) != cudaSuccess ||
      cudaMalloc(&g->d_job_tiles_done, static_cast<size_t>(max_jobs) * 4) != cudaSuccess ||
      cudaHostAlloc(&g->h_job_flag, static_cast<size_t>(max_jobs) * 4, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&g->d_job_flag, g->h_job_flag, 0) != cudaSuccess) {
    cudaGetLastError();
    return bail(gfail(GDF_ERR_OOM_BUDGET, "grouped job table"));
  }
  std::memset(g->h_job_flag, 0, static_cast<size_t>(max_jobs) * 4);
  for (int k = 0; k < 2; ++k) {
    if (cudaMallocHost(&g->h_stage[k], stage_bytes(max_jobs)) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->copied[k], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return bail(gfail(GDF_ERR_OOM_BUDGET, "grouped staging"));
    }
  }
  if (cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->last_launch, cudaEventDisableTiming) != cudaSuccess ||
      cudaMemset(g->d_err, 0, 4) != cudaSuccess)
    return bail(gcuda(cudaGetLastError(), "grouped set-up"));
  *out = g;
  return GDF_OK;
}

gdf_status gdf_group_destroy(gdf_group* g) {
  if (!g) return GDF_OK;
  cudaDeviceSynchronize();
  drop_plans(g);
  cudaFree(g->d_hdr);
  cudaFree(g->d_jobs);
  cudaFree(g->d_err);
  cudaFree(g->d_job_tiles_done);
  if (g->h_job_flag) cudaFreeHost(g->h_job_flag);
  if (g->feat) cudaFreeAsync(g->feat, nullptr);
  cudaFree(g->tune_wi);
  if (g->last_launch) cudaEventDestroy(g->last_launch);
  for (int k = 0; k < 2; ++k) {
    if (g->h_stage[k]) cudaFreeHost(g->h_stage[k]);
    if (g->copied[k]) cudaEventDestroy(g->copied[k]);
  }
  if (g->cap_stream) cudaStreamDestroy(g->cap_stream);
  delete g;
  return GDF_OK;
}

gdf_status gdf_group_infer(gdf_group* g, const gdf_job* jobs, int32_t n_jobs, void* stream) {
  if (!g || !jobs) return gfail(GDF_ERR_INVALID_ARG, "null group / jobs");
  if (n_jobs < 1 || n_jobs > g->max_jobs) return gfail(GDF_ERR_INVALID_ARG, "n_jobs out of [1, max_jobs]");
  JobSet js{};
  gdf_status s = check_jobs(jobs, n_jobs, &js);
  if (s) return s;
  js.n_jobs = n_jobs;
  if (++g->seq == 0u) g->seq = 1u;  // 0 is the timing runs' number
  g->job_n.assign(static_cast<size_t>(n_jobs), 0);
  for (int32_t i = 0; i < n_jobs; ++i) g->job_n[static_cast<size_t>(i)] = jobs[i].n;
  if (js.total_tiles == 0) return GDF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((s = ensure_feat(g, js.total_tiles, js.levels * js.features, st))) return s;
  const auto key = std::make_tuple(js.levels, js.features, static_cast<int>(n_jobs),
                                   static_cast<int>(std::ceil(std::log2(static_cast<double>(js.total_tiles)))));
  auto it = g->tuned.find(key);
  std::pair<int, int> cfg;
  if (g->pinned_wgs) {
    cfg = {g->pinned_wgs, g->pinned_fblock};
  } else if (it == g->tuned.end()) {
    if ((s = autotune(g, jobs, n_jobs, js, st, &cfg))) return s;
    g->tuned[key] = cfg;
  } else {
    cfg = it->second;
  }
  g->last_wgs = cfg.first;
  g->last_fblock = cfg.second;
  size_t plan = 0;
  if ((s = upload_table(g, jobs, n_jobs, cfg.first, nullptr, g->seq, st))) return s;
  if ((s = get_plan(g, js, cfg.first, cfg.second, &plan))) return s;
  return launch_plan(g, plan, js, st);
}

gdf_status gdf_group_set_shape(gdf_group* g, int32_t warpgroups, int32_t feature_block) {
  if (!g) return gfail(GDF_ERR_INVALID_ARG, "null group");
  if (warpgroups == 0) {
    g->pinned_wgs = g->pinned_fblock = 0;
    return GDF_OK;
  }
  if ((warpgroups != 2 && warpgroups != 4) || (feature_block != 128 && feature_block != 256))
    return gfail(GDF_ERR_INVALID_ARG, "launch shape must be 2 or 4 warpgroups x 128 or 256 threads");
  g->pinned_wgs = warpgroups;
  g->pinned_fblock = feature_block;
  return GDF_OK;
}

gdf_status gdf_group_tuning(const gdf_group* g, int32_t* warpgroups, int32_t* feature_block, float* tuned_ms) {
  if (!g) return gfail(GDF_ERR_INVALID_ARG, "null group");
  if (warpgroups) *warpgroups = g->last_wgs;
  if (feature_block) *feature_block = g->last_fblock;
  if (tuned_ms)
    for (int k = 0; k < 4; ++k) tuned_ms[k] = g->last_tune_ms[k];
  return GDF_OK;
}

gdf_status gdf_group_track_jobs(gdf_group* g, int32_t on) {
  if (!g) return gfail(GDF_ERR_INVALID_ARG, "null group");
  g->track = on != 0;
  return GDF_OK;
}

int32_t gdf_group_job_done(const gdf_group* g, int32_t job) {
  if (!g || !g->track || job < 0 || static_cast<size_t>(job) >= g->job_n.size()) return 0;
  if (g->job_n[static_cast<size_t>(job)] == 0) return 1;
  return *reinterpret_cast<const volatile uint32_t*>(g->h_job_flag + job) == g->seq ? 1 : 0;
}

gdf_status gdf_group_set_sm_cap(gdf_group* g, int32_t ctas) {
  if (!g) return gfail(GDF_ERR_INVALID_ARG, "null group");
  if (ctas < 0) return gfail(GDF_ERR_INVALID_ARG, "ctas must be >= 0");
  g->sm_cap = ctas;
  return GDF_OK;
}

gdf_status gdf_group_sync_status(gdf_group* g, void* stream) {
  if (!g) return gfail(GDF_ERR_INVALID_ARG, "null group");
  GDF_GCUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  uint32_t err = 0;
  GDF_GCUDA(cudaMemcpy(&err, g->d_err, 4, cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(g->d_err, 0, 4);
    return gfail(GDF_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(err) + ")");
  }
  return GDF_OK;
}

}  // extern "C"

namespace gdf {

uint32_t* group_err_flag(gdf_group* g) { return g->d_err; }

}  // namespace gdf
