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
#include "train.h"

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

}  // namespace

extern "C" {

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
