// ref_pin.cpp -- the reference's own DF functions compiled for the host.
//
// TEST INFRASTRUCTURE ONLY. This translation unit #includes, unmodified,
// src/render/guided/train.h (and through it AR.h, guideditem.h, workqueue.h,
// parameters.h) from the reference tree, with oracle/ref_stub/ standing in
// for the framework headers. The functions below call the reference's code
// and expose it with C linkage so tests can compare the oracle restatement
// against it bit for bit. Built by oracle/build_ref.py into oracle/_ref/.
//
// The reference fixes N_DIM_OUTPUT = 16, N_DIM_OUTPUT_PHI = 32 and
// AR_LINEAR_INTERPOLATION = 1 (parameters.h:20,41,48); templated functions
// are instantiated here for 16/32/64 bins.
//
// train.cu (the record producers and the NRC substitution kernels) is
// included too; its kernels run here as host loops over the thread index.
// The record buffers of train.h keep their storage pointers private and
// allocate with cudaMalloc in their constructors, so this file opens their
// members (`private` read as `public`, after every system header is in) and
// points them at host arrays instead.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#define private public
#include "train.cu"
#undef private

thread_local krr_stub_idx krr_stub_threadIdx, krr_stub_blockIdx, krr_stub_blockDim;

using namespace krr;

namespace {

// Runs `fn` as the host execution of a 1-D kernel of n threads.
template <typename Fn>
void for_threads(int64_t n, Fn&& fn) {
  krr_stub_blockIdx.x = 0;
  krr_stub_blockDim.x = 1;
  for (int64_t i = 0; i < n; ++i) {
    krr_stub_threadIdx.x = static_cast<unsigned>(i);
    fn();
  }
}

template <int N>
void softmax_n(float* v) {
  krr_stub_threadIdx.x = 0;
  krr_stub_blockIdx.x = 0;
  krr_stub_blockDim.x = 1;
  softmaxMultFactor_F<float, N, N, N>(1, v);
}

// sample_dir_guided_inputs_F for one row with a scripted sampler.
template <bool IS_THETA, int N>
float sample_one(const float* pdf, float u_main, float u_fallback) {
  ScatterRayWorkItem item;
  item.pixelId = 0;
  ScatterRayQueue q;
  q.items_ = &item;
  q.size_ = 1;
  const float seq[2] = {u_main, u_fallback};
  PCGSampler s;
  s.seq = seq;
  PixelStateBuffer ps;
  ps.sampler = &s;
  AuxInfo aux;
  aux.guided_pass = true;
  float wi[4] = {-1.f, -1.f, 1.f, 1.f};
  krr_stub_threadIdx.x = 0;
  krr_stub_blockIdx.x = 0;
  krr_stub_blockDim.x = 1;
  sample_dir_guided_inputs_F<IS_THETA, N, N>(1, &q, &ps, pdf, &aux, wi);
  return IS_THETA ? wi[0] : wi[1];
}

template <int N, bool IS_THETA>
void grads_linear(float u, float other, float prefix, const __half* pdfs, __half* out) {
  AutoRegressive::compute_gradients_specialized_linear_interpolation<N, IS_THETA>(u, other, prefix, pdfs, out);
}

// LearnedDistribution::getDistribution (learnedDistribution.h:72-82) for the
// training layout (N_DIM_WI floats per record).
struct LearnedDistributionView {
  template <typename T, bool isNEE = true, bool isTrain = true>
  static AutoRegressive getDistribution(T* data, size_t idx, uint /*padding*/ = 0) {
    return AutoRegressive(data + idx * N_DIM_WI);
  }
};

// The oracle's path-state view (go_paths in gdf_oracle.h): per field one
// array [depth][pixel][components], plus the per-pixel depth counter.
struct PinPaths {
  int64_t n;
  void *L, *thp, *Le, *pos, *dir, *wi_pdf, *mis_weight, *delta, *miss, *bsdf_val, *wo, *normal, *roughness,
      *diffuse, *specular;
  void* cur_depth;
};

// GuidedPixelStateBuffer (workqueue.h:15) over the oracle's arrays.
GuidedPixelStateBuffer state_of(const PinPaths* s) {
  GuidedPixelStateBuffer g;
  const int64_t n = s->n;
  for (int d = 0; d < (int)MAX_TRAIN_DEPTH; ++d) {
    auto& r = g.records[d];
    r.L = reinterpret_cast<Color*>(s->L) + d * n;
    r.thp = reinterpret_cast<Color*>(s->thp) + d * n;
    r.Le = reinterpret_cast<Color*>(s->Le) + d * n;
    r.pos = reinterpret_cast<Vector3f*>(s->pos) + d * n;
    r.dir = reinterpret_cast<Vector2f*>(s->dir) + d * n;
    r.wiPdf = reinterpret_cast<float*>(s->wi_pdf) + d * n;
    r.misWeight = reinterpret_cast<float*>(s->mis_weight) + d * n;
    r.delta = reinterpret_cast<bool*>(s->delta) + d * n;
    r.miss = reinterpret_cast<bool*>(s->miss) + d * n;
    r.bsdfVal = reinterpret_cast<Color*>(s->bsdf_val) + d * n;
    r.wo = reinterpret_cast<Vector2f*>(s->wo) + d * n;
    r.normal = reinterpret_cast<Vector2f*>(s->normal) + d * n;
    r.roughness = reinterpret_cast<float*>(s->roughness) + d * n;
    r.diffuse = reinterpret_cast<Vector3f*>(s->diffuse) + d * n;
    r.specular = reinterpret_cast<Vector3f*>(s->specular) + d * n;
  }
  g.curDepth = reinterpret_cast<uint*>(s->cur_depth);
  return g;
}

AABB box_of(const float* a) {
  AABB b;
  b.mn = Vector3f(a[0], a[1], a[2]);
  b.mx = Vector3f(a[3], a[4], a[5]);
  return b;
}

}  // namespace

extern "C" {

// normalizeSpatialCoord, warp_direction_for_sh and warp_roughness_for_ob
// (train.h:272-276, 1243-1249) for n points: out [n x 7] =
// (pos'[3], wo'[3], roughness').
void ref_input_warps(const float* pos, const float* wo, const float* rough, int64_t n, const float* aabb,
                     float* out) {
  const AABB box = box_of(aabb);
  for (int64_t i = 0; i < n; ++i) {
    const Vector3f p = normalizeSpatialCoord(Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), box);
    const Vector3f w = warp_direction_for_sh(Vector3f(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]));
    for (int k = 0; k < 3; ++k) {
      out[7 * i + k] = p[k];
      out[7 * i + 3 + k] = w[k];
    }
    out[7 * i + 6] = warp_roughness_for_ob(rough[i]);
  }
}

// AutoRegressive::pdf / sample (AR.h:25-48) of n guiding records [n x 4]
// (two-sided: slots 2, 3 positive): out [n x 4] = (solid-angle pdf, wi).
void ref_autoregressive(const float* wi4, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    float rec[4] = {wi4[4 * i], wi4[4 * i + 1], wi4[4 * i + 2], wi4[4 * i + 3]};
    AutoRegressive ar(rec);
    const Vector3f w = ar.sample();
    out[4 * i] = ar.pdf();
    out[4 * i + 1] = w[0];
    out[4 * i + 2] = w[1];
    out[4 * i + 3] = w[2];
  }
}

// generate_inference_data_AR (train.cu:334-362) over n shading points:
// theta inputs [n x 9] and the first 9 floats of the phi inputs [n x 10].
void ref_generate_inference_data(const float* pos, const float* wo, const float* nrm, const float* rough,
                                 int64_t n, const float* aabb, float* out_theta, float* out_phi) {
  std::vector<ScatterRayWorkItem> items(n);
  for (int64_t i = 0; i < n; ++i) {
    items[i].sd.pos = Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    items[i].sd.wo = Vector3f(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    items[i].sd.frame.N = Vector3f(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    items[i].sd.roughness = rough[i];
    items[i].pixelId = (unsigned)i;
  }
  ScatterRayQueue q;
  q.items_ = items.data();
  q.size_ = (int)n;
  const AABB box = box_of(aabb);
  for_threads(n, [&] { generate_inference_data_AR((size_t)n, &q, nullptr, out_theta, out_phi, box); });
}

// generate_training_data_AR (train.cu:6-96) over training pixels
// offset + i * stride, i < n_train: records appended in thread order (pixel,
// then depth). Returns the record count; at most cap are written.
int64_t ref_generate_training_data(const PinPaths* s, const float* aabb, int64_t n_train, uint32_t offset,
                                   uint32_t stride, float* in_theta, float* in_phi, float* target, int64_t cap) {
  GuidedPixelStateBuffer g = state_of(s);
  TrainBufferDuoInputs<GuidedInput, GuidedInputPhi, GuidedOutput> buf;
  buf.mInputs1 = reinterpret_cast<GuidedInput*>(in_theta);
  buf.mInputs2 = reinterpret_cast<GuidedInputPhi*>(in_phi);
  buf.mOutputs = reinterpret_cast<GuidedOutput*>(target);
  buf.mMaxSize = (int)cap;
  static_assert(sizeof(GuidedInput) == 9 * sizeof(float) && sizeof(GuidedInputPhi) == 10 * sizeof(float) &&
                    sizeof(GuidedOutput) == 9 * sizeof(float), "record layouts");
  const AABB box = box_of(aabb);
  for_threads(n_train, [&] { generate_training_data_AR((size_t)n_train, offset, stride, &buf, &g, box); });
  return buf.mSize.load();
}

// generate_training_data_nrc_with_inference (train.cu:156-220) when
// with_training != 0, else generate_NRCinput_from_training_data
// (train.cu:222-262, OPTIMIZE_ON_NRC = 4): the NRC query rows with their
// (depth, pixel), and the NRC training rows; decrements the depth counters.
// counts = (query rows, training rows).
void ref_generate_nrc_records(PinPaths* s, const float* aabb, int64_t n_train, uint32_t offset, uint32_t stride,
                              int with_training, float* q_in, int32_t* q_depth, int32_t* q_pixel, int64_t q_cap,
                              float* t_in, float* t_target, int64_t t_cap, int64_t* counts) {
  GuidedPixelStateBuffer g = state_of(s);
  NRCInputBuffer<GuidedInputNRC> qb;
  qb.mData = reinterpret_cast<GuidedInputNRC*>(q_in);
  qb.mDepths = q_depth;
  qb.mPixelIds = q_pixel;
  qb.mMaxSize = (int)q_cap;
  TrainBuffer<GuidedInputNRC, GuidedOutputNRC> tb;
  tb.mInputs = reinterpret_cast<GuidedInputNRC*>(t_in);
  tb.mOutputs = reinterpret_cast<GuidedOutputNRC*>(t_target);
  tb.mMaxSize = (int)t_cap;
  static_assert(sizeof(GuidedInputNRC) == 15 * sizeof(float) && sizeof(GuidedOutputNRC) == 3 * sizeof(float),
                "NRC record layouts");
  const AABB box = box_of(aabb);
  if (with_training)
    for_threads(n_train, [&] {
      generate_training_data_nrc_with_inference((size_t)n_train, offset, stride, &tb, &qb, &g, box);
    });
  else
    for_threads(n_train, [&] { generate_NRCinput_from_training_data((size_t)n_train, offset, stride, &qb, &g, box); });
  counts[0] = qb.mSize.load();
  counts[1] = tb.mSize.load();
}

// apply_NRCoutput_to_training_data then divide_training_data_by_NRCoutput
// (train.cu:265-308; OPTIMIZE_ON_NRC = 4) for m NRC outputs [m x 3] at
// (depth, pixel); modifies the radiance records in place.
void ref_apply_nrc(PinPaths* s, const float* out, const int32_t* depth, const int32_t* pixel, int64_t m) {
  GuidedPixelStateBuffer g = state_of(s);
  for_threads(m, [&] { apply_NRCoutput_to_training_data((size_t)m, depth, pixel, out, &g); });
  for_threads(m, [&] { divide_training_data_by_NRCoutput((size_t)m, depth, pixel, out, &g); });
}

int ref_softmax_times_n(float* v, int n) {
  switch (n) {
    case 16: softmax_n<16>(v); return 0;
    case 32: softmax_n<32>(v); return 0;
    case 64: softmax_n<64>(v); return 0;
  }
  return -1;
}

float ref_sample_dir(const float* pdf, int n, int is_theta, float u_main, float u_fallback) {
  switch (n) {
    case 16: return is_theta ? sample_one<true, 16>(pdf, u_main, u_fallback) : sample_one<false, 16>(pdf, u_main, u_fallback);
    case 32: return is_theta ? sample_one<true, 32>(pdf, u_main, u_fallback) : sample_one<false, 32>(pdf, u_main, u_fallback);
    case 64: return is_theta ? sample_one<true, 64>(pdf, u_main, u_fallback) : sample_one<false, 64>(pdf, u_main, u_fallback);
  }
  return -1.f;
}

// sample_pdf called the way compute_AR_pdf_combined_F does: idx = u * N.
float ref_sample_pdf(const float* pdf, float u, int n, int is_theta) {
  return is_theta ? sample_pdf<float, true>(pdf, u * static_cast<float>(n), n)
                  : sample_pdf<float, false>(pdf, u * static_cast<float>(n), n);
}

// add_theta_to_input_F (N_DIM_OUTPUT = 16): the phi network's theta input.
float ref_theta_condition16(float u_theta) {
  float wi[4] = {u_theta, 0.f, 1.f, 1.f};
  float in[N_DIM_INPUT_PHI] = {};
  krr_stub_threadIdx.x = 0;
  krr_stub_blockIdx.x = 0;
  krr_stub_blockDim.x = 1;
  add_theta_to_input_F<float, false>(1, wi, in);
  return in[N_DIM_INPUT_PHI - 1];
}

// AutoRegressive::compute_gradients_specialized_linear_interpolation.
int ref_grads_linear(float u, float pdf_other, float prefix, const uint16_t* pdfs_bits, int n, int is_theta,
                     uint16_t* out_bits) {
  const __half* p = reinterpret_cast<const __half*>(pdfs_bits);
  __half* o = reinterpret_cast<__half*>(out_bits);
  switch (n) {
    case 16: is_theta ? grads_linear<16, true>(u, pdf_other, prefix, p, o) : grads_linear<16, false>(u, pdf_other, prefix, p, o); return 0;
    case 32: is_theta ? grads_linear<32, true>(u, pdf_other, prefix, p, o) : grads_linear<32, false>(u, pdf_other, prefix, p, o); return 0;
    case 64: is_theta ? grads_linear<64, true>(u, pdf_other, prefix, p, o) : grads_linear<64, false>(u, pdf_other, prefix, p, o); return 0;
  }
  return -1;
}

// combine_AR_pdf_and_dl_doutput (train.h:932-965) over n records with the
// reference's 16 (theta) / 32 (phi) bins. target rows: dir2, L3, wiPdf, bsdf3.
void ref_combine(const float* target, int64_t n, const uint16_t* pdf_theta_bits, const uint16_t* pdf_phi_bits,
                 uint16_t* dl_theta_bits, uint16_t* dl_phi_bits, float* likelihood, float loss_scale) {
  static_assert(sizeof(GuidedOutput) == 9 * sizeof(float), "GuidedOutput layout");
  GuidedOutput* out = reinterpret_cast<GuidedOutput*>(const_cast<float*>(target));
  precision_t* pt = reinterpret_cast<precision_t*>(const_cast<uint16_t*>(pdf_theta_bits));
  precision_t* pp = reinterpret_cast<precision_t*>(const_cast<uint16_t*>(pdf_phi_bits));
  precision_t* dt = reinterpret_cast<precision_t*>(dl_theta_bits);
  precision_t* dp = reinterpret_cast<precision_t*>(dl_phi_bits);
  for_threads(n, [&] {
    combine_AR_pdf_and_dl_doutput<LearnedDistributionView>(static_cast<size_t>(n), out, pt, pp, dt, dp,
                                                           likelihood, loss_scale);
  });
}

}  // extern "C"
