// df_math.cuh -- per-query math of the DF guiding path: input encodings and
// the softmax / CDF / inversion-sampling / pdf-interpolation epilogue.
//
// Everything here is written for one thread = one query with register
// arrays indexed only by compile-time constants (data-dependent lookups are
// unrolled selects), so no value spills to local memory. Files including
// this header are compiled with -fmad=false: the float sequences below then
// round exactly like the reference's operation order, and the explicit
// fmaf() calls stand for the products nvcc contracts in the reference.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>

#include "grid_levels.h"

namespace gdf {

constexpr float kEps = 1e-5f;  // M_EPSILON (krrmath/constants.h:19)

// 2^x by the SFU (ex2.approx.ftz.f32; subnormal results flush to zero).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// grid_index (grid.h:165-188) with the CoherentPrime hash (grid.h:112-129).
__device__ __forceinline__ uint32_t grid_entry(const GridLevels& g, int l, uint32_t x,
                                               uint32_t y, uint32_t z) {
  uint32_t index;
  if (g.hashed[l]) {
    index = x ^ (y * 2654435761u) ^ (z * 805459861u);
  } else {
    const uint32_t r = g.res[l];
    index = x;
    if (g.ndims[l] > 1) index += y * r;
    if (g.ndims[l] > 2) index += z * r * r;
  }
  return g.pow2[l] ? (index & (g.hsize[l] - 1u)) : (index % g.hsize[l]);
}

// kernel_grid forward (grid.h:220-349): per level, trilinear (or smoothstep /
// nearest) interpolation of F features over the 8 cell corners. Accumulation
// in fp32 (tcnn accumulates the corner sum in fp16).
template <int L, int F>
__device__ __forceinline__ void grid_encode(const GridLevels& g, const __half* __restrict__ table,
                                            float px, float py, float pz, float* out) {
#pragma unroll
  for (int l = 0; l < L; ++l) {
    const float scale = g.scale[l];
    float fr[3];
    uint32_t pg[3];
    const float pin[3] = {px, py, pz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float p = fmaf(pin[d], scale, 0.5f);
      const float t = floorf(p);
      pg[d] = static_cast<uint32_t>(static_cast<int>(t));
      p -= t;
      if (g.interp == 1) p = p * p * (3.0f - 2.0f * p);
      fr[d] = p;
    }
    const __half* tab = table + static_cast<size_t>(g.offset[l]) * F;
    float acc[F];
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] = 0.f;
    if (g.interp == 2) {
      const uint32_t e = grid_entry(g, l, pg[0], pg[1], pg[2]);
#pragma unroll
      for (int f = 0; f < F; ++f) acc[f] = __half2float(tab[static_cast<size_t>(e) * F + f]);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        float w = 1.f;
        const uint32_t x = pg[0] + (c & 1), y = pg[1] + ((c >> 1) & 1), z = pg[2] + ((c >> 2) & 1);
        w *= (c & 1) ? fr[0] : 1.f - fr[0];
        w *= (c & 2) ? fr[1] : 1.f - fr[1];
        w *= (c & 4) ? fr[2] : 1.f - fr[2];
        const uint32_t e = grid_entry(g, l, x, y, z);
        if constexpr (F == 2) {
          const uint32_t raw = __ldg(reinterpret_cast<const unsigned int*>(tab) + e);
          const float2 v = __half22float2(*reinterpret_cast<const __half2*>(&raw));
          acc[0] += w * v.x;
          acc[1] += w * v.y;
        } else {
          const uint2 raw = __ldg(reinterpret_cast<const uint2*>(tab) + e);
          const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
          const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
          acc[0] += w * a.x;
          acc[1] += w * a.y;
          acc[2] += w * b.x;
          acc[3] += w * b.y;
        }
      }
    }
#pragma unroll
    for (int f = 0; f < F; ++f) out[l * F + f] = acc[f];
  }
}

// Real spherical harmonics of degree 4 of (2v - 1) (tcnn encodings/
// spherical_harmonics.h:46-150). Coefficients are the closed forms
// sqrt(k) / (m sqrt(pi)).
namespace shc {
constexpr double kInvSqrtPi = 0.56418958354775628694807945156077;
constexpr double s3 = 1.7320508075688772935274463415059, s5 = 2.2360679774997896964091736687313,
                 s7 = 2.6457513110645905905016157536393, s15 = 3.8729833462074168851792653997824,
                 s42 = 6.4807406984078602309659674360879, s70 = 8.3666002653407554797817202578519,
                 s105 = 10.246950765959598383221038680521;
constexpr float c0 = float(kInvSqrtPi / 2), c1 = float(s3 * kInvSqrtPi / 2),
                c4 = float(s15 * kInvSqrtPi / 2), c6a = float(3 * s5 * kInvSqrtPi / 4),
                c6b = float(s5 * kInvSqrtPi / 4), c8 = float(s15 * kInvSqrtPi / 4),
                c9 = float(s70 * kInvSqrtPi / 8), c10 = float(s105 * kInvSqrtPi / 2),
                c11 = float(s42 * kInvSqrtPi / 8), c12 = float(s7 * kInvSqrtPi / 4),
                c14 = float(s105 * kInvSqrtPi / 4);
}  // namespace shc

__device__ __forceinline__ void sh4_encode(float vx, float vy, float vz, float* o) {
  using namespace shc;
  const float x = vx * 2.f - 1.f, y = vy * 2.f - 1.f, z = vz * 2.f - 1.f;
  const float xy = x * y, xz = x * z, yz = y * z, x2 = x * x, y2 = y * y, z2 = z * z;
  o[0] = c0;
  o[1] = -c1 * y;
  o[2] = c1 * z;
  o[3] = -c1 * x;
  o[4] = c4 * xy;
  o[5] = -c4 * yz;
  o[6] = c6a * z2 - c6b;
  o[7] = -c4 * xz;
  o[8] = c8 * x2 - c8 * y2;
  o[9] = c9 * y * (-3.0f * x2 + y2);
  o[10] = c10 * xy * z;
  o[11] = c11 * y * (1.0f - 5.0f * z2);
  o[12] = c12 * z * (5.0f * z2 - 3.0f);
  o[13] = c11 * x * (1.0f - 5.0f * z2);
  o[14] = c14 * z * (x2 - y2);
  o[15] = c9 * x * (-x2 + 3.0f * y2);
}

// quartic_cdf (tcnn common_device.h:492-497).
__device__ __forceinline__ float quartic_cdf(float x, float inv_radius) {
  const float u = x * inv_radius, u2 = u * u, u4 = u2 * u2;
  return fmaxf(0.0f, fminf(1.0f, (15.0f / 16.0f) * u * (1.0f - (2.0f / 3.0f) * u2 +
                                                          (1.0f / 5.0f) * u4) + 0.5f));
}

// The three wrapped kernel CDFs of one bin boundary, q(d) + q(d - 1) +
// q(d + 1) summed left to right (oneblob.h:116-120), for d = boundary - x.
// With 4 bins and x in [0, 1] (so d in [-1, 1]), |4 (d - 1)| >= 1.25 unless
// d > 0.6875 and |4 (d + 1)| >= 1.25 unless d < -0.6875; the quartic is
// monotone and already -0.023 / 1.023 at u = -1.25 / 1.25, so those terms
// are exactly 0 and 1 after the clamp, and only one of the two wrapped
// terms needs evaluating: the same float sum with 2 evaluations instead of 3.
template <int NB>
__device__ __forceinline__ float oneblob_boundary(float d, bool in_unit) {
  const float nb = static_cast<float>(NB);
  if (NB == 4 && in_unit) {
    const float qw = quartic_cdf(d > 0.f ? d - 1.0f : d + 1.0f, nb);
    const float t1 = d > 0.6875f ? qw : 0.0f;
    const float t2 = d < -0.6875f ? qw : 1.0f;
    return quartic_cdf(d, nb) + t1 + t2;
  }
  return quartic_cdf(d, nb) + quartic_cdf(d - 1.0f, nb) + quartic_cdf(d + 1.0f, nb);
}

// kernel_one_blob_soa (tcnn encodings/oneblob.h:99-127) for one input dim.
template <int NB>
__device__ __forceinline__ void oneblob_encode(float x, float* o) {
  const float nb = static_cast<float>(NB);
  const bool in_unit = x >= 0.0f && x <= 1.0f;
  float left = oneblob_boundary<NB>(-x, in_unit);
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    const float rb = static_cast<float>(k + 1) / nb;
    const float right = oneblob_boundary<NB>(rb - x, in_unit);
    o[k] = right - left;
    left = right;
  }
}

// triangle_wave_encoding (tcnn encodings/triangle_wave.h:46-80).
template <int NF>
__device__ __forceinline__ void triangle_wave_encode(float x, float* o) {
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    const float xs = ldexpf(x, j - 1);
    const float val = xs + j * 0.25f;
    o[j] = fabsf(val - floorf(val) - 0.5f) * 4.f - 1.f;
  }
}

// frequency_encoding (tcnn encodings/frequency.h:46-95): sin/cos pairs.
template <int NF>
__device__ __forceinline__ void frequency_encode(float x, float* o) {
  constexpr float kPi = 3.14159265358979323846f;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const float xs = ldexpf(x, f);
    o[2 * f] = sinf(fmaf(xs, kPi, 0.0f));
    o[2 * f + 1] = sinf(fmaf(xs, kPi, kPi / 2.0f));
  }
}

// ------------------------------------------------------------- epilogue

// softmax2 (src/render/guided/train.h:845-862) then x N (softmaxMultFactor_F,
// train.h:872-881). The running max starts at 0.
template <int N>
__device__ __forceinline__ void softmax2_times_n(float (&v)[N]) {
  float mx = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) mx = fmaxf(mx, v[i]);
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) s += expf(v[i] - mx);
  const float ls = logf(s);
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = expf(v[i] - mx - ls);
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] *= static_cast<float>(N);
}

// softmaxMultFactor<__half> of the training forward (train.h:872-893 with
// T = fp16): fp16 logits, softmax2 rounded to fp16, times N in fp16 (exact
// for power-of-two N). In place, results as float.
template <int N>
__device__ __forceinline__ void softmax_table_fp16(float (&v)[N]) {
  float mx = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    v[i] = __half2float(__float2half_rn(v[i]));
    mx = fmaxf(mx, v[i]);
  }
  float s = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) s += __expf(v[i] - mx);
  const float ls = __logf(s);
#pragma unroll
  for (int i = 0; i < N; ++i)
    v[i] = __half2float(__float2half_rn(__half2float(__float2half_rn(__expf(v[i] - mx - ls))) *
                                        static_cast<float>(N)));
}

template <int N>
__device__ __forceinline__ int safe_floor(float v) {
  const int f = static_cast<int>(floorf(v));
  return f < N - 1 ? f : N - 1;
}

// Unrolled select of pdf[idx] for a data-dependent idx in [0, N).
template <int N>
__device__ __forceinline__ float select_bin(const float (&pdf)[N], int idx) {
  float r = pdf[0];
#pragma unroll
  for (int i = 1; i < N; ++i) r = (idx == i) ? pdf[i] : r;
  return r;
}

// sample_pdf (train.h:655-681).
template <int N, bool LINEAR>
__device__ __forceinline__ float sample_pdf(const float (&pdf)[N], float u) {
  float idx = u * static_cast<float>(N);
  if constexpr (!LINEAR) {
    return select_bin<N>(pdf, safe_floor<N>(idx));
  } else {
    idx -= 0.5f;
    int f = safe_floor<N>(idx);
    int c = f + 1;
    float w = idx - static_cast<float>(f);
    if (f < 0) { f = N - 1; w = 1.0f; }
    if (c > N - 1) { c = 0; w = 0.0f; }
    return (1.0f - w) * select_bin<N>(pdf, f) + w * select_bin<N>(pdf, c);
  }
}

// add_theta_to_input_F (train.h:794-812): the phi network's theta input.
template <int N, bool LINEAR>
__device__ __forceinline__ float theta_condition(float u) {
  const int fl = safe_floor<N>(u * static_cast<float>(N));
  if constexpr (!LINEAR) {
    return static_cast<float>(fl) / static_cast<float>(N);
  } else {
    const float w = u * static_cast<float>(N) - static_cast<float>(fl);
    return (static_cast<float>(fl) + w) / static_cast<float>(N);
  }
}

// sample_dir_guided_inputs_F (train.h:416-520) with the CDF walk of
// search_sorted_cdf_linearinterpolation (train.h:362-397) or
// search_sorted_cdf_nearest (train.h:346-359). The walk is unrolled over all
// bins and latches the first segment with u < cdf, which is the reference's
// early exit without divergence.
template <int N, bool LINEAR>
__device__ __forceinline__ float sample_dir(const float (&pdf)[N], float u, float u2) {
  const float inv_n = 1.f / static_cast<float>(N);
  float cm1 = 0.f, ci = 0.f;
  int seg = N;
  bool found = false;
  float lo = pdf[N - 1], hi = pdf[N - 1];
  if constexpr (LINEAR) {
    float run = pdf[0] * 0.5f / static_cast<float>(N);
    if (u < run) {
      found = true; seg = 0; cm1 = 0.f; ci = run; lo = pdf[0]; hi = pdf[0];
    }
    float prev = run;
#pragma unroll
    for (int i = 1; i < N; ++i) {
      const float c = prev + (pdf[i - 1] + pdf[i]) / static_cast<float>(2 * N);
      if (!found && u < c) {
        found = true; seg = i; cm1 = prev; ci = c; lo = pdf[i - 1]; hi = pdf[i];
      }
      prev = c;
    }
    if (!found) {
      cm1 = prev;
      ci = prev + pdf[N - 1] * 0.5f / static_cast<float>(N);
    }
    int idx_m1 = seg - 1;
    float v = static_cast<float>(idx_m1) + 0.5f;
    float ecm = 1.f, v_off = 0.f;
    if (idx_m1 < 0) { v_off = 0.5f; ecm = 0.5f; }
    else if (seg > N - 1) { ecm = 0.5f; }
    const float m = (hi - lo) * static_cast<float>(N);
    const float B = lo * (1 + v) - hi * v;
    v += v_off;
    const float A = m * 0.5f;
    float d;
    if (fabsf(A) < kEps) {
      const float v_diff = u - cm1;
      const float v_cdf_diff = ci - cm1;
      const float w = v_cdf_diff > kEps ? v_diff / v_cdf_diff : u2;
      d = (v + w * ecm) * inv_n;
    } else {
      const float C = -(m * 0.5f) * (v * v * inv_n * inv_n) - (B * v * inv_n) + cm1 - u;
      const float delta = B * B - 4 * A * C;
      if (delta < kEps) {
        d = (v + u2 * ecm) * inv_n;
      } else {
        const float sq = sqrtf(delta);
        const float s0 = (-B + sq) / (2 * A);
        const float s1 = (-B - sq) / (2 * A);
        d = A >= 0 ? fmaxf(s0, s1) : fminf(s0, s1);
      }
    }
    return fminf(d, 1.f - kEps);
  } else {
    float prev = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const float c = prev + pdf[i] / static_cast<float>(N);
      if (!found && u < c) { found = true; seg = i; cm1 = prev; ci = c; }
      prev = c;
    }
    if (!found) { cm1 = prev; ci = prev; }
    const float v_diff = u - cm1;
    const float v_cdf_diff = ci - cm1;
    const float w = v_cdf_diff > kEps ? v_diff / v_cdf_diff : u2;
    const float d = (static_cast<float>(seg) + w) / static_cast<float>(N);
    return fminf(d, 1.f - kEps);
  }
}

// Inversion inside the segment found by the CDF walk (train.h:453-519):
// seg is the index of the first boundary above u (0 = the leading half-bin,
// N = the trailing one), cm1/ci the CDF at the segment's ends, lo/hi the pdf
// at its ends.
template <int N, bool LINEAR>
__device__ __forceinline__ float invert_segment(int seg, float cm1, float ci, float lo, float hi, float u,
                                                float u2) {
  const float inv_n = 1.f / static_cast<float>(N);
  if constexpr (LINEAR) {
    int idx_m1 = seg - 1;
    float v = static_cast<float>(idx_m1) + 0.5f;
    float ecm = 1.f, v_off = 0.f;
    if (idx_m1 < 0) { v_off = 0.5f; ecm = 0.5f; }
    else if (seg > N - 1) { ecm = 0.5f; }
    const float m = (hi - lo) * static_cast<float>(N);
    const float B = lo * (1 + v) - hi * v;
    v += v_off;
    const float A = m * 0.5f;
    float d;
    if (fabsf(A) < kEps) {
      const float v_diff = u - cm1;
      const float v_cdf_diff = ci - cm1;
      const float w = v_cdf_diff > kEps ? v_diff / v_cdf_diff : u2;
      d = (v + w * ecm) * inv_n;
    } else {
      const float C = -(m * 0.5f) * (v * v * inv_n * inv_n) - (B * v * inv_n) + cm1 - u;
      const float delta = B * B - 4 * A * C;
      if (delta < kEps) {
        d = (v + u2 * ecm) * inv_n;
      } else {
        const float sq = sqrtf(delta);
        const float s0 = (-B + sq) / (2 * A);
        const float s1 = (-B - sq) / (2 * A);
        d = A >= 0 ? fmaxf(s0, s1) : fminf(s0, s1);
      }
    }
    return fminf(d, 1.f - kEps);
  } else {
    const float v_diff = u - cm1;
    const float v_cdf_diff = ci - cm1;
    const float w = v_cdf_diff > kEps ? v_diff / v_cdf_diff : u2;
    const float d = (static_cast<float>(seg) + w) / static_cast<float>(N);
    return fminf(d, 1.f - kEps);
  }
}

struct SampleResult {
  float u;    // sampled (guided) or given square coordinate
  float pdf;  // interpolated pdf at u
};

// sample_dir_guided_inputs_F (train.h:416-520) followed by sample_pdf
// (train.h:655-681) in one pass over the bins.
//
// The CDF is non-decreasing, so the reference's early-exit search for the
// first boundary above u equals counting the boundaries b_i <= u; the walk
// latches the values of the last counted boundary (its index, CDF, and the
// pdf at both ends of the next segment) without a "found" flag. Rows that
// are not guided count bins up to the given direction's floor(N u - 1/2)
// instead, so the same latched pair serves the pdf interpolation of every
// row; a guided sample whose rounding puts it outside its segment falls back
// to indexed reads.
// Neumaier's compensated summation step (Neumaier 1974, the improved Kahan
// sum): s + c carries the running sum with the rounding error of each
// addition kept in c.
__device__ __forceinline__ void neumaier_add(float& s, float& c, float x) {
  const float t = s + x;
  c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
  s = t;
}

// COMP: the CDF boundaries accumulate with neumaier_add (the BF16 / FP8
// inference forms); without it they follow the reference's plain float sum.
template <int N, bool LINEAR, bool COMP = false>
__device__ __forceinline__ SampleResult sample_and_pdf(const float (&pdf)[N], bool guided, float u_given,
                                                       float u, float u2) {
  const float nf = static_cast<float>(N);
  SampleResult r;
  if constexpr (LINEAR) {
    const int f_given = safe_floor<N>(u_given * nf - 0.5f);
    int seg = 0;
    float cm1 = 0.f, lo = pdf[0], hi = pdf[0];
    float b = pdf[0] * 0.5f / nf;  // b_0: end of the leading half-bin
    float bc = 0.f;                 // its compensation (COMP)
    const float b0 = b;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (i > 0) {
        const float term = (pdf[i - 1] + pdf[i]) / static_cast<float>(2 * N);
        if constexpr (COMP) neumaier_add(b, bc, term);
        else b = b + term;
      }
      const float bv = COMP ? b + bc : b;
      const bool cond = guided ? (bv <= u) : (i <= f_given);
      if (cond) {
        seg = i + 1;
        cm1 = bv;
        lo = pdf[i];
        hi = pdf[i + 1 < N ? i + 1 : N - 1];
      }
    }
    float d = u_given;
    if (guided) {
      const float ci = seg == 0 ? b0 : (seg < N ? cm1 + (lo + hi) / static_cast<float>(2 * N)
                                                : cm1 + pdf[N - 1] * 0.5f / nf);
      d = invert_segment<N, true>(seg, cm1, ci, lo, hi, u, u2);
    }
    r.u = d;
    // sample_pdf (train.h:656-676): bins f = floor(N d - 1/2) and f + 1,
    // the leading half-bin reads pdf[0], the trailing one pdf[N-1]
    const float x = d * nf - 0.5f;
    const int f = safe_floor<N>(x);
    if (f == seg - 1) {
      r.pdf = f < 0 ? lo : (f + 1 > N - 1 ? lo : (1.0f - (x - static_cast<float>(f))) * lo +
                                                     (x - static_cast<float>(f)) * hi);
    } else {
      r.pdf = sample_pdf<N, true>(pdf, d);
    }
  } else {
    const int f_given = safe_floor<N>(u_given * nf);
    int seg = 0;
    float cm1 = 0.f, cur = pdf[0];
    float c = 0.f, cc = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if constexpr (COMP) neumaier_add(c, cc, pdf[i] / nf);
      else c = c + pdf[i] / nf;
      const float cv = COMP ? c + cc : c;
      const bool cond = guided ? (cv <= u) : (i < f_given);
      if (cond) {
        seg = i + 1;
        cm1 = cv;
        cur = pdf[i + 1 < N ? i + 1 : N - 1];
      }
    }
    float d = u_given;
    if (guided) {
      const float ci = seg < N ? cm1 + cur / nf : cm1;
      d = invert_segment<N, false>(seg, cm1, ci, 0.f, 0.f, u, u2);
    }
    r.u = d;
    const int f = safe_floor<N>(d * nf);  // sample_pdf, nearest (train.h:679)
    r.pdf = (f == (seg < N ? seg : N - 1)) ? cur : select_bin<N>(pdf, f);
  }
  return r;
}

// ------------------------------------------------------------ Philox RNG
// Philox4x32-10 (Salmon et al., SC'11): four uniforms per query, counter
// (row, offset), key = seed. Uniforms use the 23-bit mantissa trick of
// PCGSampler::nextFloat (src/lib/src/core/sampler.h:77-86).
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t (&o)[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  o[0] = c0; o[1] = c1; o[2] = c2; o[3] = c3;
}

__device__ __forceinline__ float u32_to_uniform(uint32_t x) {
  return __uint_as_float((x >> 9) | 0x3f800000u) - 1.0f;
}

}  // namespace gdf
