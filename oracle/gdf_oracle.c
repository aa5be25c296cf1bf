/*
 * gdf_oracle.c -- CPU oracle of the guiding-df DF/NRC inference path.
 *
 * TEST INFRASTRUCTURE ONLY (checker for tests/, smoke() and the CPU
 * baseline of bench.py). Never linked into the product library.
 *
 * Compiled with -ffp-contract=off so that the float restatements keep the
 * reference's rounding sequence; where the reference's device code computes
 * a*b+c that nvcc contracts (pos_fract, frequency encoding), fmaf is written
 * explicitly so both sides round once.
 */
#include "gdf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define GO_EPS 1e-5f /* M_EPSILON, src/lib/src/core/math/include/krrmath/constants.h:19 */
#define GO_PI_F 3.14159265358979323846f
#define GO_PI 3.14159265358979323846

/* ------------------------------------------------------------ fp16 bits */

/* IEEE binary16 round-to-nearest-even from a double (single rounding). */
static uint16_t f64_to_f16(double x) {
  uint16_t sign = signbit(x) ? 0x8000u : 0u;
  if (isnan(x)) return 0x7e00u;
  double a = fabs(x);
  if (a >= 65520.0) return sign | 0x7c00u; /* rounds to infinity */
  double q;
  if (a >= 6.103515625e-05) { /* 2^-14, normal range */
    int e;
    frexp(a, &e);            /* a = m * 2^e, m in [0.5, 1) */
    q = ldexp(1.0, e - 11);  /* quantum of a 10-bit mantissa at exponent e-1 */
  } else {
    q = ldexp(1.0, -24);     /* subnormal quantum */
  }
  double r = nearbyint(a / q) * q; /* default rounding mode: ties to even */
  if (r == 0.0) return sign;
  if (r < 6.103515625e-05) return sign | (uint16_t)(r / ldexp(1.0, -24));
  if (r >= 65520.0) return sign | 0x7c00u;
  int e;
  double m = frexp(r, &e); /* r = m 2^e, m in [0.5,1) -> exponent e-1 */
  int field = (e - 1) + 15;
  uint16_t mant = (uint16_t)((m * 2.0 - 1.0) * 1024.0 + 0.5);
  if (field >= 31) return sign | 0x7c00u;
  return sign | (uint16_t)(field << 10) | mant;
}

uint16_t go_f32_to_f16(float x) { return f64_to_f16((double)x); }

float go_f16_to_f32(uint16_t h) {
  uint32_t sign = (h & 0x8000u) << 16;
  uint32_t exp = (h >> 10) & 0x1fu;
  uint32_t mant = h & 0x3ffu;
  float v;
  if (exp == 0) {
    v = ldexpf((float)mant, -24);
  } else if (exp == 31) {
    v = mant ? NAN : INFINITY;
  } else {
    v = ldexpf((float)(mant | 0x400u), (int)exp - 25);
  }
  union { float f; uint32_t u; } cv;
  cv.f = v;
  cv.u |= sign;
  return cv.f;
}

float go_round_f16(double x) { return go_f16_to_f32(f64_to_f16(x)); }

/* ------------------------------------------------------------- Philox */

/* Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11: multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
 * increments 0x9E3779B9 / 0xBB67AE85, 10 rounds. */
void go_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* PCGSampler::nextFloat bit trick (src/lib/src/core/sampler.h:77-86):
 * 23 high bits into the mantissa of 1.0f, minus 1. */
float go_u32_to_uniform(uint32_t x) {
  union { uint32_t u; float f; } cv;
  cv.u = (x >> 9) | 0x3f800000u;
  return cv.f - 1.0f;
}

void go_philox_uniforms(uint64_t seed, uint64_t offset, int64_t n, float* out) {
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int64_t i = 0; i < n; ++i) {
    uint32_t ctr[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)offset,
                       (uint32_t)(offset >> 32)};
    uint32_t r[4];
    go_philox4x32_10(ctr, key, r);
    for (int k = 0; k < 4; ++k) out[i * 4 + k] = go_u32_to_uniform(r[k]);
  }
}

/* -------------------------------------------------------------- grid */

static uint32_t next_multiple_u32(uint32_t v, uint32_t m) { return (v + m - 1) / m * m; }

/* GridEncodingTemplated constructor (tcnn/include/tiny-cuda-nn/encodings/
 * grid.h:967-1012) with grid_scale / grid_resolution (grid.h:194-203).
 * The scale table is evaluated once on the host and shared with the device
 * kernels, so both sides use the same per-level scale. */
int go_grid_init(go_grid* g, const go_grid_config* c) {
  memset(g, 0, sizeof(*g));
  g->c = *c;
  if (c->n_levels <= 0 || c->n_levels > GO_MAX_LEVELS) return -1;
  const float log2_scale = log2f(c->per_level_scale);
  uint32_t offset = 0;
  for (int i = 0; i < c->n_levels; ++i) {
    const float scale = exp2f((float)i * log2_scale) * (float)c->base_resolution - 1.0f;
    const uint32_t res = (uint32_t)ceilf(scale) + 1u;
    const uint32_t max_params = 0xffffffffu / 2u;
    uint32_t params = powf((float)res, 3.0f) > (float)max_params ? max_params : res * res * res;
    params = next_multiple_u32(params, 8u);
    if (c->type == 2) { /* Tiled */
      uint32_t b = (uint32_t)c->base_resolution;
      if (b * b * b < params) params = b * b * b;
    } else if (c->type == 0) { /* Hash */
      uint32_t t = 1u << c->log2_hashmap_size;
      if (t < params) params = t;
    }
    g->scale[i] = scale;
    g->resolution[i] = res;
    g->offset[i] = offset;
    offset += params;
  }
  g->offset[c->n_levels] = offset;
  g->n_params = (int64_t)offset * c->n_features_per_level;
  return 0;
}

/* grid_index (grid.h:165-188) with prime_hash<3, COHERENT> (grid.h:112-129):
 * primes {1, 2654435761, 805459861} for CoherentPrime. */
static uint32_t grid_index(const go_grid* g, uint32_t hashmap_size, uint32_t res,
                           const uint32_t p[3]) {
  uint32_t stride = 1, index = 0;
  for (int d = 0; d < 3 && stride <= hashmap_size; ++d) {
    index += p[d] * stride;
    stride *= res;
  }
  if (g->c.type == 0 && hashmap_size < stride) {
    index = (p[0] * 1u) ^ (p[1] * 2654435761u) ^ (p[2] * 805459861u);
  }
  return index % hashmap_size;
}

/* kernel_grid (grid.h:220-392), forward values only; pos_fract
 * (common_device.h:403-432) with the FMA the device code rounds once. */
void go_grid_encode(const go_grid* g, const float* table, const float pos[3], double* out) {
  const int F = g->c.n_features_per_level;
  for (int l = 0; l < g->c.n_levels; ++l) {
    const float scale = g->scale[l];
    const uint32_t res = g->resolution[l];
    const uint32_t hsize = g->offset[l + 1] - g->offset[l];
    const float* tab = table + (size_t)g->offset[l] * F;
    float fr[3];
    uint32_t pg[3];
    for (int d = 0; d < 3; ++d) {
      float p = fmaf(pos[d], scale, 0.5f);
      float t = floorf(p);
      pg[d] = (uint32_t)(int)t;
      p -= t;
      if (g->c.interpolation == 1) p = p * p * (3.0f - 2.0f * p); /* smoothstep */
      fr[d] = p;
    }
    if (g->c.interpolation == 2) { /* Nearest */
      uint32_t idx = grid_index(g, hsize, res, pg);
      for (int f = 0; f < F; ++f) out[l * F + f] = tab[(size_t)idx * F + f];
      continue;
    }
    double acc[8] = {0};
    for (int c = 0; c < 8; ++c) {
      double w = 1.0;
      uint32_t q[3];
      for (int d = 0; d < 3; ++d) {
        if (c & (1 << d)) { w *= fr[d]; q[d] = pg[d] + 1; }
        else { w *= 1.0 - (double)fr[d]; q[d] = pg[d]; }
      }
      uint32_t idx = grid_index(g, hsize, res, q);
      for (int f = 0; f < F; ++f) acc[f] += w * (double)tab[(size_t)idx * F + f];
    }
    for (int f = 0; f < F; ++f) out[l * F + f] = acc[f];
  }
}

/* kernel_sh (tcnn/include/tiny-cuda-nn/encodings/spherical_harmonics.h:46-150)
 * for degree <= 4: real spherical harmonics of (2v - 1); the constants are the
 * closed forms sqrt(.)/(k sqrt(pi)) written next to each term there. */
void go_sh_encode(int degree, const float dir01[3], double* out) {
  const double x = (double)(dir01[0] * 2.f - 1.f);
  const double y = (double)(dir01[1] * 2.f - 1.f);
  const double z = (double)(dir01[2] * 2.f - 1.f);
  const double sp = sqrt(GO_PI);
  const double xy = x * y, xz = x * z, yz = y * z, x2 = x * x, y2 = y * y, z2 = z * z;
  out[0] = 1.0 / (2.0 * sp);
  if (degree <= 1) return;
  out[1] = -sqrt(3.0) * y / (2.0 * sp);
  out[2] = sqrt(3.0) * z / (2.0 * sp);
  out[3] = -sqrt(3.0) * x / (2.0 * sp);
  if (degree <= 2) return;
  out[4] = sqrt(15.0) * xy / (2.0 * sp);
  out[5] = -sqrt(15.0) * yz / (2.0 * sp);
  out[6] = sqrt(5.0) * (3.0 * z2 - 1.0) / (4.0 * sp);
  out[7] = -sqrt(15.0) * xz / (2.0 * sp);
  out[8] = sqrt(15.0) * (x2 - y2) / (4.0 * sp);
  if (degree <= 3) return;
  out[9] = sqrt(70.0) * y * (-3.0 * x2 + y2) / (8.0 * sp);
  out[10] = sqrt(105.0) * xy * z / (2.0 * sp);
  out[11] = sqrt(42.0) * y * (1.0 - 5.0 * z2) / (8.0 * sp);
  out[12] = sqrt(7.0) * z * (5.0 * z2 - 3.0) / (4.0 * sp);
  out[13] = sqrt(42.0) * x * (1.0 - 5.0 * z2) / (8.0 * sp);
  out[14] = sqrt(105.0) * z * (x2 - y2) / (4.0 * sp);
  out[15] = sqrt(70.0) * x * (-x2 + 3.0 * y2) / (8.0 * sp);
}

/* quartic_cdf (tcnn/include/tiny-cuda-nn/common_device.h:492-497). */
static double quartic_cdf(double x, double inv_radius) {
  const double u = x * inv_radius, u2 = u * u, u4 = u2 * u2;
  double v = (15.0 / 16.0) * u * (1.0 - (2.0 / 3.0) * u2 + (1.0 / 5.0) * u4) + 0.5;
  return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

/* kernel_one_blob_soa (tcnn/include/tiny-cuda-nn/encodings/oneblob.h:99-127):
 * wrapped quartic kernel integrated over each of n_bins bins. */
void go_oneblob_encode(int n_bins, const float* x, int n_dims, double* out) {
  const double nb = (double)n_bins;
  for (int j = 0; j < n_dims; ++j) {
    const double xv = x[j];
    double left = quartic_cdf(-xv, nb) + quartic_cdf(-xv - 1.0, nb) + quartic_cdf(-xv + 1.0, nb);
    for (int k = 0; k < n_bins; ++k) {
      const double rb = (double)(k + 1) / nb;
      const double right = quartic_cdf(rb - xv, nb) + quartic_cdf(rb - xv - 1.0, nb) +
                           quartic_cdf(rb - xv + 1.0, nb);
      out[j * n_bins + k] = right - left;
      left = right;
    }
  }
}

/* triangle_wave_encoding (tcnn/include/tiny-cuda-nn/encodings/triangle_wave.h:46-80). */
void go_triangle_wave_encode(int n_freq, float x, double* out) {
  for (int j = 0; j < n_freq; ++j) {
    const double xs = ldexp((double)x, j - 1);
    const double val = xs + j * 0.25;
    out[j] = fabs(val - floor(val) - 0.5) * 4.0 - 1.0;
  }
}

/* frequency_encoding (tcnn/include/tiny-cuda-nn/encodings/frequency.h:46-95):
 * per input dim, [sin, cos](2^f pi x) for f < n_freq, interleaved. */
void go_frequency_encode(int n_freq, const float* x, int n_dims, double* out) {
  for (int j = 0; j < n_dims * n_freq * 2; ++j) {
    const int dim = j / (n_freq * 2);
    const int f = (j / 2) % n_freq;
    const double arg = ldexp((double)x[dim], f) * GO_PI + (j % 2) * (GO_PI / 2.0);
    out[j] = sin(arg);
  }
}

/* --------------------------------------------------------- networks */

static int32_t pad16(int32_t v) { return (v + 15) / 16 * 16; }

/* Composite encoding widths (tcnn/include/tiny-cuda-nn/encodings/composite.h:
 * 187-199, 395-406) padded to the FullyFusedMLP alignment of 16
 * (network_with_input_encoding.h:44, encoding.h:85-87). */
int32_t go_df_input_width(const go_df_config* c, int net) {
  const go_grid_config* gc = net == 0 ? &c->grid_theta : &c->grid_phi;
  int32_t w = gc->n_levels * gc->n_features_per_level + c->sh_degree * c->sh_degree +
              3 * c->oneblob_bins;
  if (net == 1) w += c->tw_frequencies;
  return pad16(w);
}

static int32_t df_bins(const go_df_config* c, int net) {
  return net == 0 ? c->n_bins_theta : c->n_bins_phi;
}

/* FullyFusedMLP weight matrices (tcnn/src/fully_fused_mlp.cu:630-668). */
int64_t go_df_mlp_params(const go_df_config* c, int net) {
  const int64_t w = c->width;
  const int64_t h = net == 0 ? c->hidden_theta : c->hidden_phi;
  return w * go_df_input_width(c, net) + (h - 1) * w * w + (int64_t)pad16(df_bins(c, net)) * w;
}

int64_t go_df_n_params(const go_df_config* c, int net) {
  go_grid g;
  go_grid_init(&g, net == 0 ? &c->grid_theta : &c->grid_phi);
  return go_df_mlp_params(c, net) + g.n_params;
}

int32_t go_nrc_input_width(const go_nrc_config* c) {
  return pad16(3 * c->frequencies * 2 + 6 * c->oneblob_bins + 6);
}

int64_t go_nrc_n_params(const go_nrc_config* c) {
  const int64_t w = c->width;
  return w * go_nrc_input_width(c) + (c->hidden - 1) * w * w + 16 * w;
}

/* Composite input of the theta (9 dims) or phi (10 dims) network:
 * [grid(pos) | SH(wo') | OneBlob(n_theta', n_phi', r') | (phi: TriangleWave(theta'))
 *  | padding], base_product_df.json order; the last nested encoding takes the
 * alignment padding: TriangleWave writes ones (triangle_wave.h:65), OneBlob
 * (theta) writes them at the wrong rows (below). Values rounded to fp16. */
void go_df_encode(const go_df_config* c, const go_grid* g, int net, const float* params16,
                  const float* q, float theta_cond, float* out) {
  const int32_t k0 = go_df_input_width(c, net);
  double tmp[256];
  int o = 0;
  const float* table = params16 + go_df_mlp_params(c, net);
  go_grid_encode(g, table, q, tmp + o);
  o += g->c.n_levels * g->c.n_features_per_level;
  go_sh_encode(c->sh_degree, q + 3, tmp + o);
  o += c->sh_degree * c->sh_degree;
  const int ob = o;
  go_oneblob_encode(c->oneblob_bins, q + 6, 3, tmp + o);
  o += 3 * c->oneblob_bins;
  if (net == 1) {
    go_triangle_wave_encode(c->tw_frequencies, theta_cond, tmp + o);
    o += c->tw_frequencies;
    for (; o < k0; ++o) tmp[o] = 1.0;
  } else {
    /* OneBlob is the theta composite's last encoding and takes its alignment
       padding; tcnn's OneBlob writes that padding (encodings/oneblob.h:223-226,
       SoA layout) from n_dims_to_encode (3) rows into its own output: outputs
       [3, 3 + pad) read 1 and the pad columns stay as allocated, 0. */
    const int pad = k0 - o;
    for (; o < k0; ++o) tmp[o] = 0.0;
    for (int j = 3; j < 3 + pad; ++j) tmp[ob + j] = 1.0;
  }
  for (int i = 0; i < k0; ++i) out[i] = go_store(tmp[i]);
}

/* NRC composite (common/configs/nn/base_hashgrid_nrc_df.json):
 * [Frequency(pos, 12) | OneBlob(dims 3..8, 4) | Identity(dims 9..14) | 1.0 pad]. */
void go_nrc_encode(const go_nrc_config* c, const float* q15, float* out) {
  const int32_t k0 = go_nrc_input_width(c);
  double tmp[256];
  int o = 0;
  go_frequency_encode(c->frequencies, q15, 3, tmp + o);
  o += 3 * c->frequencies * 2;
  go_oneblob_encode(c->oneblob_bins, q15 + 3, 6, tmp + o);
  o += 6 * c->oneblob_bins;
  for (int j = 0; j < 6; ++j) tmp[o++] = q15[9 + j];
  for (; o < k0; ++o) tmp[o] = 1.0;
  for (int i = 0; i < k0; ++i) out[i] = go_round_f16(tmp[i]);
}

/* kernel_mlp_fused (tcnn/src/fully_fused_mlp.cu:500-556): ReLU hidden layers,
 * linear output, no biases; hidden activations stored as fp16. */
/* Number format of the DF networks' stored MLP inputs and activations:
 * 0 = fp16 (the reference's precision_t), 1 = bf16 (round to nearest
 * even), 2 = unrounded (kept in fp32 beside the FP64 accumulation: the
 * reference point of the precision comparison), 3 = the FP8 form (fp16
 * first and output matrices, e4m3 hidden matrices: mlp_forward_fp8). */
static int g_storage = 0;
void go_set_storage(int fmt) { g_storage = fmt; }

float go_round_bf16(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x; /* inf / nan */
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

float go_store(double x) {
  if (g_storage == 1) return go_round_bf16((float)x);
  if (g_storage == 2) return (float)x;
  return go_round_f16(x);
}

/* Accumulation model of go_mlp_forward: 0 = FP64 (checker), 1 = sequential
 * FP32 (an emulation of a tensor-core kernel's accumulation, used only to
 * calibrate test tolerances). */
static int g_acc32 = 0;
void go_set_accumulation(int acc32) { g_acc32 = acc32; }

static double dot_acc(const float* a, const float* b, int k) {
  if (g_acc32) {
    float acc = 0.f;
    for (int i = 0; i < k; ++i) acc += a[i] * b[i];
    return acc;
  }
  double acc = 0.0;
  for (int i = 0; i < k; ++i) acc += (double)a[i] * (double)b[i];
  return acc;
}

/* OCP E4M3 (4 exponent bits, bias 7, 3 mantissa bits, no infinities,
 * largest finite 448) rounded to nearest even from a double, saturating
 * to +-448 (cvt.rn.satfinite.e4m3x2.f32 semantics for finite inputs). */
double go_round_e4m3(double x) {
  if (isnan(x) || x == 0.0) return x;
  const double a = fabs(x);
  int e;
  frexp(a, &e);             /* a = m * 2^e, m in [0.5, 1): leading exponent e-1 */
  int lead = e - 1;
  if (lead < -6) lead = -6; /* subnormals: quantum 2^-9 */
  const double q = ldexp(1.0, lead - 3);
  double r = nearbyint(a / q) * q;
  if (r > 448.0) r = 448.0;
  return copysign(r, x);
}

/* Exponent k of the largest power of two with amax * 2^k <= 448, clamped
 * to [-100, 100]; 0 for a zero or non-finite amax. */
int go_e4m3_scale_exp(double amax) {
  if (amax == 0.0 || !isfinite(amax)) return 0;
  int e;
  const double m = frexp(amax, &e); /* amax = (2m) * 2^(e-1), 2m in [1, 2) */
  const int k = (m <= 0.875 ? 8 : 7) - (e - 1);
  return k < -100 ? -100 : (k > 100 ? 100 : k);
}

/* The FP8 inference form: matrix 0 over the fp16 inputs with fp16 weights;
 * each 64x64 hidden matrix W as e4m3(W * 2^kw), kw from max|W|, over the
 * row's activations e4m3(h * 2^kr), kr from the row's max, the product
 * descaled by 2^-(kw+kr); ReLU before each quantisation; the last hidden
 * activations rounded to fp16 for the fp16 output matrix. */
static void mlp_forward_fp8(const float* w16, int k0, int width, int n_hidden, int n_out_pad,
                            const float* x16, float* out) {
  double acc[256], v[256];
  float qa[256], h16[256];
  static __thread float qw[256 * 256];
  const float* w = w16;
  for (int o = 0; o < width; ++o) acc[o] = dot_acc(w + (size_t)o * k0, x16, k0);
  w += (size_t)width * k0;
  double d = 1.0;
  for (int l = 1; l <= n_hidden; ++l) {
    double amax = 0.0;
    for (int o = 0; o < width; ++o) {
      const double y = acc[o] * d;
      v[o] = y > 0.0 ? y : 0.0; /* NaN -> 0 */
      if (v[o] > amax) amax = v[o];
    }
    if (l < n_hidden) {
      const int kr = go_e4m3_scale_exp(amax);
      for (int o = 0; o < width; ++o) qa[o] = (float)go_round_e4m3(ldexp(v[o], kr));
      double wmax = 0.0;
      for (int i = 0; i < width * width; ++i)
        if (fabs((double)w[i]) > wmax) wmax = fabs((double)w[i]);
      const int kw = go_e4m3_scale_exp(wmax);
      for (int i = 0; i < width * width; ++i) qw[i] = (float)go_round_e4m3(ldexp((double)w[i], kw));
      for (int o = 0; o < width; ++o) acc[o] = dot_acc(qw + (size_t)o * width, qa, width);
      d = ldexp(1.0, -(kw + kr));
      w += (size_t)width * width;
    } else {
      for (int o = 0; o < width; ++o) h16[o] = go_round_f16(v[o]);
      for (int o = 0; o < n_out_pad; ++o) out[o] = (float)dot_acc(w + (size_t)o * width, h16, width);
    }
  }
}

void go_mlp_forward(const float* w16, int k0, int width, int n_hidden, int n_out_pad,
                    const float* x16, float* out, float* hidden_out) {
  if (g_storage == 3 && !hidden_out) {
    mlp_forward_fp8(w16, k0, width, n_hidden, n_out_pad, x16, out);
    return;
  }
  float h[256], hn[256];
  memcpy(h, x16, sizeof(float) * (size_t)k0);
  int k = k0;
  const float* w = w16;
  for (int l = 0; l < n_hidden; ++l) {
    for (int o = 0; o < width; ++o) {
      const double acc = dot_acc(w + (size_t)o * k, h, k);
      hn[o] = go_store(acc > 0.0 ? acc : 0.0);
    }
    w += (size_t)width * k;
    k = width;
    memcpy(h, hn, sizeof(float) * (size_t)width);
    if (hidden_out) memcpy(hidden_out + (size_t)l * width, h, sizeof(float) * (size_t)width);
  }
  for (int o = 0; o < n_out_pad; ++o) out[o] = (float)dot_acc(w + (size_t)o * k, h, k);
}

/* fp32 variant of the same forward for the CPU baseline. */
static void mlp_forward_f32(const float* w16, int k0, int width, int n_hidden, int n_out,
                            const float* x16, float* out) {
  float h[256], hn[256];
  memcpy(h, x16, sizeof(float) * (size_t)k0);
  int k = k0;
  const float* w = w16;
  for (int l = 0; l < n_hidden; ++l) {
    for (int o = 0; o < width; ++o) {
      float acc = 0.f;
      const float* row = w + (size_t)o * k;
      for (int i = 0; i < k; ++i) acc += row[i] * h[i];
      hn[o] = acc > 0.f ? acc : 0.f;
    }
    w += (size_t)width * k;
    k = width;
    memcpy(h, hn, sizeof(float) * (size_t)width);
  }
  for (int o = 0; o < n_out; ++o) {
    float acc = 0.f;
    const float* row = w + (size_t)o * k;
    for (int i = 0; i < k; ++i) acc += row[i] * h[i];
    out[o] = acc;
  }
}

void go_mlp_forward_f32(const float* w16, int k0, int width, int n_hidden, int n_out,
                        const float* x16, float* out) {
  mlp_forward_f32(w16, k0, width, n_hidden, n_out, x16, out);
}

/* ------------------------------------------------------ DF epilogue */

/* softmax2 (src/render/guided/train.h:845-862) followed by the x N factor of
 * softmaxMultFactor_F (train.h:872-881); max starts at 0. */
void go_softmax2_times_n(float* v, int n) {
  float mx = 0.0f;
  for (int i = 0; i < n; ++i) mx = fmaxf(mx, v[i]);
  float s = 0.0f;
  for (int i = 0; i < n; ++i) s += expf(v[i] - mx);
  const float ls = logf(s);
  for (int i = 0; i < n; ++i) v[i] = expf(v[i] - mx - ls);
  for (int i = 0; i < n; ++i) v[i] *= (float)n;
}

/* search_sorted_cdf_linearinterpolation (train.h:362-397) and
 * search_sorted_cdf_nearest (train.h:346-359). */
static int search_cdf(const float* pdf, int n, int linear, float u, float* cm1, float* ci) {
  *cm1 = 0.0f;
  int i = 0;
  if (linear) {
    *ci = pdf[0] * 0.5f / (float)n;
    if (u < *ci) return 0;
    *cm1 = *ci;
    for (i = 1; i < n; ++i) {
      *ci = *cm1 + (pdf[i - 1] + pdf[i]) / (float)(2 * n);
      if (u < *ci) return i;
      *cm1 = *ci;
    }
    *ci = *cm1 + pdf[n - 1] * 0.5f / (float)n;
    return n;
  }
  for (i = 0; i < n; ++i) {
    *ci = *cm1 + pdf[i] / (float)n;
    if (u < *ci) break;
    *cm1 = *ci;
  }
  return i;
}

/* sample_dir_guided_inputs_F (train.h:416-520) for one row. Returns the
 * segment index; *out_edge_gap = min distance of u to the segment's CDF
 * edges (used by tests to skip ties at bin edges). */
int go_sample_dir(const float* pdf, int n, int linear, float u_main, float u_fallback,
                  float* out_dir, float* out_edge_gap) {
  float cm1, ci;
  const float inv_n = 1.f / (float)n;
  const int seg = search_cdf(pdf, n, linear, u_main, &cm1, &ci);
  if (out_edge_gap) {
    float a = fabsf(u_main - cm1), b = fabsf(ci - u_main);
    *out_edge_gap = a < b ? a : b;
  }
  if (!linear) {
    const float v_diff = u_main - cm1;
    const float v_cdf_diff = ci - cm1;
    const float w = v_cdf_diff > GO_EPS ? v_diff / v_cdf_diff : u_fallback;
    const float d = ((float)seg + w) / (float)n;
    *out_dir = fminf(d, 1.f - GO_EPS);
    return seg;
  }
  int idx = seg;
  int idx_m1 = idx - 1;
  float v = (float)idx_m1 + 0.5f;
  float ecm = 1.f;
  float v_off = 0.f;
  if (idx_m1 < 0) {
    idx_m1 = idx;
    v_off = 0.5f;
    ecm = 0.5f;
  } else if (idx > n - 1) {
    idx = idx_m1;
    ecm = 0.5f;
  }
  const float m = (pdf[idx] - pdf[idx_m1]) * (float)n;
  const float B = pdf[idx_m1] * (1 + v) - pdf[idx] * v;
  v += v_off;
  const float A = m * 0.5f;
  if (fabsf(A) < GO_EPS) {
    const float v_diff = u_main - cm1;
    const float v_cdf_diff = ci - cm1;
    const float w = v_cdf_diff > GO_EPS ? v_diff / v_cdf_diff : u_fallback;
    const float d = (v + w * ecm) * inv_n;
    *out_dir = fminf(d, 1.f - GO_EPS);
    return seg;
  }
  const float C = -(m * 0.5f) * (v * v * inv_n * inv_n) - (B * v * inv_n) + cm1 - u_main;
  const float delta = B * B - 4 * A * C;
  float d;
  if (delta < GO_EPS) {
    d = (v + u_fallback * ecm) * inv_n;
  } else {
    const float sq = sqrtf(delta);
    const float s0 = (-B + sq) / (2 * A);
    const float s1 = (-B - sq) / (2 * A);
    d = A >= 0 ? fmaxf(s0, s1) : fminf(s0, s1);
  }
  *out_dir = fminf(d, 1.f - GO_EPS);
  return seg;
}

/* Double twin of go_sample_dir (error reporting against FP64). */
double go_sample_dir_f64(const float* pdf, int n, int linear, double u, double u2) {
  double cm1 = 0.0, ci = 0.0;
  int seg = 0;
  if (linear) {
    ci = pdf[0] * 0.5 / n;
    if (!(u < ci)) {
      cm1 = ci;
      for (seg = 1; seg < n; ++seg) {
        ci = cm1 + ((double)pdf[seg - 1] + pdf[seg]) / (2.0 * n);
        if (u < ci) break;
        cm1 = ci;
      }
      if (seg == n) ci = cm1 + pdf[n - 1] * 0.5 / n;
    }
  } else {
    for (seg = 0; seg < n; ++seg) {
      ci = cm1 + (double)pdf[seg] / n;
      if (u < ci) break;
      cm1 = ci;
    }
  }
  double d;
  if (!linear) {
    double w = (ci - cm1) > 1e-5 ? (u - cm1) / (ci - cm1) : u2;
    d = (seg + w) / n;
  } else {
    int idx = seg, im1 = seg - 1;
    double v = im1 + 0.5, ecm = 1.0, off = 0.0;
    if (im1 < 0) { im1 = idx; off = 0.5; ecm = 0.5; }
    else if (idx > n - 1) { idx = im1; ecm = 0.5; }
    const double m = ((double)pdf[idx] - pdf[im1]) * n;
    const double B = pdf[im1] * (1 + v) - pdf[idx] * v;
    v += off;
    const double A = m * 0.5;
    if (fabs(A) < 1e-5) {
      double w = (ci - cm1) > 1e-5 ? (u - cm1) / (ci - cm1) : u2;
      d = (v + w * ecm) / n;
    } else {
      const double C = -(m * 0.5) * (v * v / n / n) - (B * v / n) + cm1 - u;
      const double delta = B * B - 4 * A * C;
      if (delta < 1e-5) d = (v + u2 * ecm) / n;
      else {
        const double sq = sqrt(delta);
        const double s0 = (-B + sq) / (2 * A), s1 = (-B - sq) / (2 * A);
        d = A >= 0 ? (s0 > s1 ? s0 : s1) : (s0 < s1 ? s0 : s1);
      }
    }
  }
  return d < 1.0 - 1e-5 ? d : 1.0 - 1e-5;
}

static int safe_floor(float v, int n) {
  int f = (int)floorf(v);
  return f < n - 1 ? f : n - 1;
}

/* sample_pdf (train.h:655-681): linear blend with nearest in the outer
 * half-bins (no wrap), or nearest bin. */
float go_sample_pdf(const float* pdf, float u, int n, int linear) {
  float idx = u * (float)n;
  if (!linear) return pdf[safe_floor(idx, n)];
  idx -= 0.5f;
  int f = safe_floor(idx, n);
  int c = f + 1;
  float w = idx - (float)f;
  if (f < 0) { f = n - 1; w = 1.0f; }
  if (c > n - 1) { c = 0; w = 0.0f; }
  return (1.0f - w) * pdf[f] + w * pdf[c];
}

/* add_theta_to_input_F (train.h:794-812). */
float go_theta_condition(float u_theta, int n, int linear) {
  const int fl = safe_floor(u_theta * (float)n, n);
  if (!linear) return (float)fl / (float)n;
  const float w = u_theta * (float)n - (float)fl;
  return ((float)fl + w) / (float)n;
}

/* One row of thetaPostInference (train.h:896-911). */
static void theta_post(const go_df_config* c, float* pdf, int guided, const float* u, float* wi,
                       float* gap) {
  const int nb = c->n_bins_theta, lin = c->pdf_interp == 0;
  go_softmax2_times_n(pdf, nb);
  if (guided) go_sample_dir(pdf, nb, lin, u[0], u[1], &wi[0], gap);
  else if (gap) *gap = 1.0f;
}

/* One row of phiPostInference (train.h:914-929) + compute_AR_pdf_combined_F
 * (train.h:730-751). */
static void phi_post(const go_df_config* c, const float* pdf_t, float* pdf_p, int guided,
                     const float* u, float* wi, float* gap) {
  const int nbp = c->n_bins_phi, lin = c->pdf_interp == 0;
  go_softmax2_times_n(pdf_p, nbp);
  if (guided) go_sample_dir(pdf_p, nbp, lin, u[2], u[3], &wi[1], gap);
  else if (gap) *gap = 1.0f;
  wi[2] *= go_sample_pdf(pdf_t, wi[0], c->n_bins_theta, lin);
  wi[3] *= go_sample_pdf(pdf_p, wi[1], nbp, lin);
}

void go_post_inference(const go_df_config* c, const float* logits_theta, const float* logits_phi,
                       const uint8_t* guided, const float* uniforms, float* wi, float* edge_gap,
                       int64_t n) {
  const int nbt = c->n_bins_theta, nbp = c->n_bins_phi;
  for (int64_t i = 0; i < n; ++i) {
    float pt[128], pp[128];
    memcpy(pt, logits_theta + i * nbt, sizeof(float) * (size_t)nbt);
    memcpy(pp, logits_phi + i * nbp, sizeof(float) * (size_t)nbp);
    const int g = guided ? guided[i] != 0 : 1;
    theta_post(c, pt, g, uniforms + i * 4, wi + i * 4, edge_gap ? edge_gap + i * 2 : 0);
    phi_post(c, pt, pp, g, uniforms + i * 4, wi + i * 4, edge_gap ? edge_gap + i * 2 + 1 : 0);
  }
}

static void infer_impl(const go_df_config* c, const float* p_theta, const float* p_phi,
                       const float* queries, const uint8_t* guided, const float* uniforms,
                       float* wi, float* edge_gap, int64_t n, int n_threads, int fast) {
  go_grid gt, gp;
  go_grid_init(&gt, &c->grid_theta);
  go_grid_init(&gp, &c->grid_phi);
  const int k0t = go_df_input_width(c, 0), k0p = go_df_input_width(c, 1);
  const int nbt = c->n_bins_theta, nbp = c->n_bins_phi, lin = c->pdf_interp == 0;
  (void)n_threads;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < n; ++i) {
    float x[256], logit_t[128], logit_p[128];
    const float* q = queries + i * 9;
    float* w = wi + i * 4;
    const int g = guided ? guided[i] != 0 : 1;
    go_df_encode(c, &gt, 0, p_theta, q, 0.f, x);
    if (fast) mlp_forward_f32(p_theta, k0t, c->width, c->hidden_theta, nbt, x, logit_t);
    else go_mlp_forward(p_theta, k0t, c->width, c->hidden_theta, pad16(nbt), x, logit_t, 0);
    theta_post(c, logit_t, g, uniforms + i * 4, w, edge_gap ? edge_gap + i * 2 : 0);
    const float cond = go_theta_condition(w[0], nbt, lin);
    go_df_encode(c, &gp, 1, p_phi, q, cond, x);
    if (fast) mlp_forward_f32(p_phi, k0p, c->width, c->hidden_phi, nbp, x, logit_p);
    else go_mlp_forward(p_phi, k0p, c->width, c->hidden_phi, pad16(nbp), x, logit_p, 0);
    phi_post(c, logit_t, logit_p, g, uniforms + i * 4, w, edge_gap ? edge_gap + i * 2 + 1 : 0);
  }
}

void go_infer(const go_df_config* c, const float* p_theta, const float* p_phi,
              const float* queries, const uint8_t* guided, const float* uniforms, float* wi,
              float* edge_gap, int64_t n, int n_threads) {
  infer_impl(c, p_theta, p_phi, queries, guided, uniforms, wi, edge_gap, n, n_threads, 0);
}

void go_infer_fp32(const go_df_config* c, const float* p_theta, const float* p_phi,
                   const float* queries, const uint8_t* guided, const float* uniforms,
                   float* wi, int64_t n, int n_threads) {
  infer_impl(c, p_theta, p_phi, queries, guided, uniforms, wi, 0, n, n_threads, 1);
}

void go_eval_pdf(const go_df_config* c, const float* p_theta, const float* p_phi,
                 const float* queries, const float* u, float* pdf_out, int64_t n,
                 int n_threads) {
  go_grid gt, gp;
  go_grid_init(&gt, &c->grid_theta);
  go_grid_init(&gp, &c->grid_phi);
  const int k0t = go_df_input_width(c, 0), k0p = go_df_input_width(c, 1);
  const int nbt = c->n_bins_theta, nbp = c->n_bins_phi, lin = c->pdf_interp == 0;
  (void)n_threads;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < n; ++i) {
    float x[256], lt[128], lp[128];
    const float* q = queries + i * 9;
    go_df_encode(c, &gt, 0, p_theta, q, 0.f, x);
    go_mlp_forward(p_theta, k0t, c->width, c->hidden_theta, pad16(nbt), x, lt, 0);
    go_softmax2_times_n(lt, nbt);
    const float cond = go_theta_condition(u[i * 2], nbt, lin);
    go_df_encode(c, &gp, 1, p_phi, q, cond, x);
    go_mlp_forward(p_phi, k0p, c->width, c->hidden_phi, pad16(nbp), x, lp, 0);
    go_softmax2_times_n(lp, nbp);
    pdf_out[i * 2] = go_sample_pdf(lt, u[i * 2], nbt, lin);
    pdf_out[i * 2 + 1] = go_sample_pdf(lp, u[i * 2 + 1], nbp, lin);
  }
}

void go_nrc_query(const go_nrc_config* c, const float* params16, const float* in15, float* out3,
                  int64_t m, int n_threads) {
  const int k0 = go_nrc_input_width(c);
  (void)n_threads;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < m; ++i) {
    float x[256], o[16];
    go_nrc_encode(c, in15 + i * 15, x);
    go_mlp_forward(params16, k0, c->width, c->hidden, 16, x, o, 0);
    out3[i * 3 + 0] = o[0];
    out3[i * 3 + 1] = o[1];
    out3[i * 3 + 2] = o[2];
  }
}

/* Per-row pdf tables (softmax x N) of both networks, the phi net conditioned
 * on u_theta[i]; diagnostics for tests. */
void go_df_pdf_tables(const go_df_config* c, const float* p_theta, const float* p_phi,
                      const float* queries, const float* u_theta, float* pdf_theta,
                      float* pdf_phi, int64_t n) {
  go_grid gt, gp;
  go_grid_init(&gt, &c->grid_theta);
  go_grid_init(&gp, &c->grid_phi);
  const int k0t = go_df_input_width(c, 0), k0p = go_df_input_width(c, 1);
  const int nbt = c->n_bins_theta, nbp = c->n_bins_phi, lin = c->pdf_interp == 0;
  for (int64_t i = 0; i < n; ++i) {
    float x[256], lt[128], lp[128];
    const float* q = queries + i * 9;
    go_df_encode(c, &gt, 0, p_theta, q, 0.f, x);
    go_mlp_forward(p_theta, k0t, c->width, c->hidden_theta, pad16(nbt), x, lt, 0);
    go_softmax2_times_n(lt, nbt);
    go_df_encode(c, &gp, 1, p_phi, q, go_theta_condition(u_theta[i], nbt, lin), x);
    go_mlp_forward(p_phi, k0p, c->width, c->hidden_phi, pad16(nbp), x, lp, 0);
    go_softmax2_times_n(lp, nbp);
    memcpy(pdf_theta + i * nbt, lt, sizeof(float) * (size_t)nbt);
    memcpy(pdf_phi + i * nbp, lp, sizeof(float) * (size_t)nbp);
  }
}
