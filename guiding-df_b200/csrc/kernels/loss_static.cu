// loss_static.cu -- training-loss evaluation that allocates no device memory.
//
// Some callers cannot allocate device memory at the moment they want the
// loss: a renderer whose device memory is a fixed arena handed out at start-
// up, or a host application that forbids cudaMalloc/cudaFree once its frame
// loop runs. gdf_train_loss_static serves them: it runs the forward half of
// the training step (theta/phi networks, fp16 pdf tables, divergence loss per
// record) and the FP64 mean, keeping every intermediate in one fixed-size
// array that is part of the library image instead of allocated memory.
//
// The scratch array is a file-scope __device__ variable: each GPU that loads
// the library holds its kStaticScratchBytes until the process exits. Host code
// must not pass the variable itself to a kernel (on the host it only names a
// host-side shadow); its device address is looked up with
// cudaGetSymbolAddress the first time the entry point runs on a device, with
// that device current, and cached per device.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../host/context.h"
#include "df_kernels.h"
#include "train_kernels.h"

namespace gdf {
namespace {

// Largest batch the static scratch holds: 4 floats per record.
constexpr int64_t kStaticMaxRecords = 65536;
constexpr size_t kFwdBytes = static_cast<size_t>(kStaticMaxRecords) * 4 * sizeof(float);
// [per-record forward outputs | 2 doubles of reduction output | dropped counter]
constexpr size_t kStaticScratchBytes = kFwdBytes + 256;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (set-up on first use).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

__global__ void finalize_loss_kernel(const double* stats, const unsigned long long* dropped, int64_t n,
                                     double* loss_out, int64_t* dropped_out) {
  loss_out[0] = stats[0] / static_cast<double>(n);
  dropped_out[0] = static_cast<int64_t>(dropped[0]);
}

}  // namespace
}  // namespace gdf

extern "C" gdf_status gdf_train_loss_static(gdf_ctx* ctx, const float* in_theta, const float* in_phi,
                                            const float* target, int64_t n, double* loss_out,
                                            int64_t* dropped_out, void* stream) {
  using namespace gdf;
  if (!ctx) { set_last_error("ctx is null"); return GDF_ERR_INVALID_ARG; }
  if (!in_theta || !in_phi || !target || !loss_out || !dropped_out) {
    set_last_error("gdf_train_loss_static: null input or output pointer");
    return GDF_ERR_INVALID_ARG;
  }
  if (n <= 0 || n > kStaticMaxRecords) {
    set_last_error(("gdf_train_loss_static: n must be in [1, " + std::to_string(kStaticMaxRecords) +
                    "], the capacity of its static scratch")
                       .c_str());
    return GDF_ERR_INVALID_ARG;
  }
  Context& c = ctx->c;
  // The scratch address is looked up on the current device, the weights live
  // on the context's: the two must be the same device.
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess || cur != c.device) {
    set_last_error(("gdf_train_loss_static: the current device (" + std::to_string(cur) +
                    ") is not the context's device (" + std::to_string(c.device) + ")")
                       .c_str());
    return GDF_ERR_INVALID_ARG;
  }
  // its forward gathers the grid itself and runs fp16 operands only: the
  // bf16 form's training weights are bf16
  if (c.net[0].train_bf16) {
    set_last_error("gdf_train_loss_static: not available for the bf16 precision form");
    return GDF_ERR_UNSUPPORTED;
  }
  void* base = nullptr;
  e = scratch_address(&base);
  if (e != cudaSuccess) {
    set_last_error((std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e)).c_str());
    return GDF_ERR_CUDA;
  }
  float* fwd = static_cast<float*>(base);
  double* stats = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kFwdBytes);
  unsigned long long* dropped =
      reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(base) + kFwdBytes + 64);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The array keeps the previous call's contents: the counter must restart at 0.
  e = cudaMemsetAsync(dropped, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) {
    set_last_error((std::string("cudaMemsetAsync: ") + cudaGetErrorString(e)).c_str());
    return GDF_ERR_CUDA;
  }
  const Net& t = c.net[0];
  const Net& f = c.net[1];
  DfKernelParams p{};
  p.queries = in_theta;
  p.in_phi = in_phi;
  p.target = target;
  p.train_out = fwd;
  p.n_dropped = dropped;
  p.loss_scale_per_record = c.cfg.loss_scale / static_cast<float>(n);
  p.n = n;
  p.grid_theta = t.w16 + t.n_mlp;
  p.grid_phi = f.w16 + f.n_mlp;
  p.blob_theta = t.blob_w16;
  p.blob_phi = f.blob_w16;
  p.blob_theta_bytes = t.blob_bytes;
  p.blob_phi_bytes = f.blob_bytes;
  p.hidden_theta = t.hidden;
  p.hidden_phi = f.hidden;
  p.gl_theta = t.gl;
  p.gl_phi = f.gl;
  p.err = c.d_err;
  const DfShape shape{c.cfg.grid_theta.n_levels, c.cfg.grid_theta.n_features_per_level, c.cfg.n_bins_theta,
                      c.cfg.n_bins_phi, c.cfg.pdf_interp == GDF_PDF_LINEAR};
  e = launch_df_fused(shape, kModeTrainFwd, p, c.num_sms, st);
  if (e == cudaSuccess) e = launch_train_stats(fwd, n, nullptr, 0, stats, st);
  if (e == cudaSuccess) {
    finalize_loss_kernel<<<1, 1, 0, st>>>(stats, dropped, n, loss_out, dropped_out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_last_error((std::string("gdf_train_loss_static: ") + cudaGetErrorString(e)).c_str());
    return GDF_ERR_CUDA;
  }
  return GDF_OK;
}
