// ref_cpu.cpp -- the CPU baseline of the guided-inference path: the
// reference's own interpolation and sampling code compiled for the host,
// fed by a scalar fp32 forward of the same encodings and MLPs.
//
// TEST / BASELINE INFRASTRUCTURE ONLY: the product never links this file.
// Built by oracle/build_ref.py (build_cpu_baseline), once per bin
// configuration, into oracle/_ref/libgdf_refcpu_<theta>x<phi>.so, from:
//   - the reference's unmodified src/render/guided/train.h (with AR.h,
//     guideditem.h, workqueue.h), reached through the directory of links that
//     oracle/build_ref_gpu.py makes (oracle/ref_gpu/parameters_shadow.h as
//     parameters.h, bin counts GDF_REF_BINS_THETA / GDF_REF_BINS_PHI), with
//     oracle/ref_stub/ as the framework headers: its kernels
//     thetaPostInference and phiPostInference (train.h:896-929) run here as
//     host loops over the thread index;
//   - the C oracle's encodings (go_df_encode) and its plain fp32 MLP forward
//     (go_mlp_forward_f32): the reference has no CPU path of its own for
//     tiny-cuda-nn's encodings and networks.
// Per chunk of queries the sequence is learnedDistribution.cpp:167-206's:
// theta encode + MLP, thetaPostInference (softmax x N, sample u_theta,
// condition the phi input), phi encode + MLP, phiPostInference (softmax x N,
// sample u_phi, pdf_theta / pdf_phi into the guiding data). OpenMP threads
// take whole chunks.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

#include "train.h"

extern "C" {
#include "gdf_oracle.h"
}

thread_local krr_stub_idx krr_stub_threadIdx, krr_stub_blockIdx, krr_stub_blockDim;

using namespace krr;

namespace {

constexpr int kChunk = 1024;

template <typename Fn>
void for_threads(int64_t n, Fn&& fn) {
  krr_stub_blockIdx.x = 0;
  krr_stub_blockDim.x = 1;
  for (int64_t i = 0; i < n; ++i) {
    krr_stub_threadIdx.x = static_cast<unsigned>(i);
    fn();
  }
}

}  // namespace

extern "C" {

void refcpu_bins(int32_t* theta, int32_t* phi) {
  *theta = (int32_t)N_DIM_OUTPUT;
  *phi = (int32_t)N_DIM_OUTPUT_PHI;
}

// Guided inference of n queries [n x 9] on the host: wi [n x 4] in/out
// (slots 2, 3 hold the caller's sign), guided [n] (NULL = all), uniforms
// [n x 4] (theta main, theta fallback, phi main, phi fallback). The weights
// are the fp16-rounded parameters of both networks in tcnn order.
// Returns -1 when the config's bin counts differ from this build's.
int refcpu_infer(const go_df_config* c, const float* p_theta16, const float* p_phi16, const float* queries,
                 const uint8_t* guided, const float* uniforms, float* wi, int64_t n, int n_threads) {
  if (c->n_bins_theta != (int)N_DIM_OUTPUT || c->n_bins_phi != (int)N_DIM_OUTPUT_PHI || c->pdf_interp != 0)
    return -1;
  go_grid gt, gp;
  go_grid_init(&gt, &c->grid_theta);
  go_grid_init(&gp, &c->grid_phi);
  const int k0t = go_df_input_width(c, 0), k0p = go_df_input_width(c, 1);
  const int64_t n_chunks = (n + kChunk - 1) / kChunk;
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
  {
    std::vector<float> x(256), lt((size_t)kChunk * N_DIM_OUTPUT), lp((size_t)kChunk * N_DIM_OUTPUT_PHI),
        in_phi((size_t)kChunk * N_DIM_INPUT_PHI);
    std::vector<ScatterRayWorkItem> items(kChunk);
    std::vector<PCGSampler> samplers(kChunk);
    std::vector<AuxInfo> aux(kChunk);
    for (int i = 0; i < kChunk; ++i) items[i].pixelId = (unsigned)i;
#pragma omp for schedule(dynamic, 1)
    for (int64_t ch = 0; ch < n_chunks; ++ch) {
      const int64_t i0 = ch * kChunk;
      const int m = (int)std::min<int64_t>(kChunk, n - i0);
      for (int i = 0; i < m; ++i) {
        const float* q = queries + (i0 + i) * 9;
        go_df_encode(c, &gt, 0, p_theta16, q, 0.f, x.data());
        go_mlp_forward_f32(p_theta16, k0t, c->width, c->hidden_theta, N_DIM_OUTPUT, x.data(),
                           lt.data() + (size_t)i * N_DIM_OUTPUT);
        std::memcpy(in_phi.data() + (size_t)i * N_DIM_INPUT_PHI, q, 9 * sizeof(float));
        samplers[i].seq = uniforms + (i0 + i) * 4;
        samplers[i].pos = 0;
        aux[i].guided_pass = guided ? guided[i0 + i] != 0 : true;
      }
      ScatterRayQueue queue;
      queue.items_ = items.data();
      queue.size_ = m;
      PixelStateBuffer ps;
      ps.sampler = samplers.data();
      float* w = wi + i0 * 4;
      for_threads(m, [&] {
        thetaPostInference<float, N_DIM_OUTPUT, N_DIM_OUTPUT, N_DIM_OUTPUT>((size_t)m, lt.data(), in_phi.data(),
                                                                            &queue, &ps, aux.data(), w);
      });
      for (int i = 0; i < m; ++i) {
        samplers[i].pos = 2;  // phi draws are slots 2-3 of a query's uniforms
        go_df_encode(c, &gp, 1, p_phi16, queries + (i0 + i) * 9, in_phi[(size_t)i * N_DIM_INPUT_PHI + 9],
                     x.data());
        go_mlp_forward_f32(p_phi16, k0p, c->width, c->hidden_phi, N_DIM_OUTPUT_PHI, x.data(),
                           lp.data() + (size_t)i * N_DIM_OUTPUT_PHI);
      }
      for_threads(m, [&] {
        phiPostInference<float, N_DIM_OUTPUT, N_DIM_OUTPUT, N_DIM_OUTPUT_PHI, N_DIM_OUTPUT_PHI, N_DIM_OUTPUT_PHI>(
            (size_t)m, lt.data(), lp.data(), &queue, &ps, aux.data(), w);
      });
    }
  }
  return 0;
}

}  // extern "C"
