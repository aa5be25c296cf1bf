/*
 * gdf_oracle_paths.c -- CPU oracle of the record producers and of the NRC
 * target substitution.
 *
 * TEST INFRASTRUCTURE ONLY (checker for tests/). Never linked into the
 * product library.
 *
 * Restates, in float with the reference's float constants
 * (krrmath/constants.h:10-19):
 *   - generate_inference_data_AR      src/render/guided/train.cu:334-362
 *   - generate_training_data_AR       train.cu:6-96
 *   - generate_training_data_nrc_with_inference  train.cu:156-214
 *   - generate_NRCinput_from_training_data        train.cu:216-262
 *   - apply_NRCoutput_to_training_data / divide_training_data_by_NRCoutput
 *     train.cu:265-308 with GuidedPixelStateBuffer::
 *     replaceIndirectRadianceSkipDelta / divideRadiance (workqueue.h:100-129)
 *   - AutoRegressive::pdf / sample (AR.h:25-48), the consumer view of a
 *     guiding record
 *   - normalizeSpatialCoord (train.h:272-276), warp_direction_for_sh /
 *     warp_roughness_for_ob (train.h:1243-1249), sphericalToCartesian,
 *     cartesianToSphericalNormalized, uniformSphereToSquare
 *     (util/math_utils.h:183-240), AABB::inflate (krrmath/aabb.h:25-28).
 * The reference appends records atomically in no fixed order; the oracle
 * emits them by training pixel, then depth.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "gdf_oracle.h"

#define P_PI 3.14159265358979323846f
#define P_2PI 6.28318530717958647693f
#define P_INV_PI 0.318309886183790671538f
#define P_INV_2PI 0.15915494309189533577f
#define P_EPS 1e-5f
#define P_MAXD 5 /* MAX_TRAIN_DEPTH (parameters.h:24) */

typedef struct { float c[3], d[3]; } frame_t;

static frame_t scene_frame(const float aabb[6]) {
  const float d0 = aabb[3] - aabb[0], d1 = aabb[4] - aabb[1], d2 = aabb[5] - aabb[2];
  const float infl = sqrtf((d0 * d0 + d1 * d1) + d2 * d2) * 0.005f;
  frame_t f;
  for (int k = 0; k < 3; ++k) {
    const float lo = aabb[k] - infl, hi = aabb[3 + k] + infl;
    f.c[k] = (lo + hi) / 2.0f;
    f.d[k] = hi - lo;
  }
  return f;
}

static void normalize_spatial(const float* p, const frame_t* f, float* o) {
  for (int k = 0; k < 3; ++k) o[k] = 0.5f + (p[k] - f->c[k]) / f->d[k];
}

static void sph_to_cart(float t, float p, float* o) {
  const float st = sinf(t), ct = cosf(t), sp = sinf(p), cp = cosf(p);
  o[0] = st * cp;
  o[1] = st * sp;
  o[2] = ct;
}

static void normalized(const float* v, float* o) {
  const float z = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
  if (z > 0.0f) {
    const float s = sqrtf(z);
    for (int k = 0; k < 3; ++k) o[k] = v[k] / s;
  } else {
    for (int k = 0; k < 3; ++k) o[k] = v[k];
  }
}

static void warp_sh(const float* v, float* o) {
  for (int k = 0; k < 3; ++k) o[k] = (v[k] + 1.0f) * 0.5f;
}

static float warp_rough(float r) { return 1.0f - expf(-r); }

static int any_nan(const float* v, int n) {
  for (int k = 0; k < n; ++k)
    if (isnan(v[k])) return 1;
  return 0;
}

void go_prepare_queries(const float* pos, const float* wo, const float* nrm, const float* rough,
                        const float aabb[6], float* q, int64_t n) {
  const frame_t f = scene_frame(aabb);
  for (int64_t i = 0; i < n; ++i) {
    float* r = q + i * 9;
    normalize_spatial(pos + i * 3, &f, r);
    float w[3];
    normalized(wo + i * 3, w);
    warp_sh(w, r + 3);
    float nn[3];
    normalized(nrm + i * 3, nn);
    const float z = nn[2] < -1.0f ? -1.0f : (nn[2] > 1.0f ? 1.0f : nn[2]);
    const float theta = acosf(z);
    float phi = atan2f(nn[1], nn[0]);
    if (phi < 0.0f) phi += P_2PI;
    /* math_utils.h:194: sph[0] / M_PI with the C library's double M_PI
       (defined before krrmath/constants.h, whose float M_PI is #ifndef'd) */
    r[6] = (float)((double)theta / 3.14159265358979323846);
    r[7] = phi / P_2PI;
    r[8] = warp_rough(rough[i]);
  }
}

void go_autoregressive(const float* wi4, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    const float* w = wi4 + i * 4;
    /* AR.h:25-43: pdf = |pdf_theta| * |pdf_phi| * squareToUniformSpherePdf() */
    out[i * 4] = fabsf(w[2]) * fabsf(w[3]) * 0.07957747154594766788f;
    /* squareToUniformSphere (math_utils.h:226-231) */
    const float z = 1.0f - 2.0f * w[0];
    const float t = 1.0f - z * z;
    const float r = sqrtf(t > 0.0f ? t : 0.0f);
    const float phi = P_2PI * w[1];
    out[i * 4 + 1] = r * cosf(phi);
    out[i * 4 + 2] = r * sinf(phi);
    out[i * 4 + 3] = z;
  }
}

/* Host copy of GuidedPixelStateBuffer: field arrays [depth][pixel][k]. */
#define F3(a, d, p) ((a) + ((int64_t)(d) * s->n + (p)) * 3)
#define F2(a, d, p) ((a) + ((int64_t)(d) * s->n + (p)) * 2)
#define F1(a, d, p) ((a) + (int64_t)(d) * s->n + (p))

static void local_radiance(const go_paths* s, int d, int64_t p, float* L) {
  const float* l = F3(s->L, d, p);
  const float* t = F3(s->thp, d, p);
  const float mis = *F1(s->mis_weight, d, p);
  for (int c = 0; c < 3; ++c) L[c] = (t[c] > P_EPS ? l[c] / t[c] : 0.0f) * mis;
}

static void vertex_inputs(const go_paths* s, int d, int64_t p, const frame_t* f, float* in) {
  normalize_spatial(F3(s->pos, d, p), f, in);
  float v[3];
  sph_to_cart(F2(s->wo, d, p)[0], F2(s->wo, d, p)[1], v);
  warp_sh(v, in + 3);
  in[6] = F2(s->normal, d, p)[0] * P_INV_PI;
  in[7] = F2(s->normal, d, p)[1] * P_INV_2PI;
  in[8] = warp_rough(*F1(s->roughness, d, p));
}

int64_t go_build_df_records(const go_paths* s, const float aabb[6], int64_t n_train, uint32_t offset,
                            uint32_t stride, int bins, int linear, float* in, float* in_phi,
                            float* target, int64_t cap) {
  const frame_t f = scene_frame(aabb);
  int64_t k = 0;
  for (int64_t i = 0; i < n_train; ++i) {
    const int64_t p = (int64_t)(offset + (uint32_t)i * stride);
    const int depth = (int)s->cur_depth[p];
    for (int d = 0; d < depth && d < P_MAXD; ++d) {
      if (*F1(s->delta, d, p)) continue;
      float x[9];
      vertex_inputs(s, d, p, &f, x);
      float v[3], wi[2];
      sph_to_cart(F2(s->dir, d, p)[0], F2(s->dir, d, p)[1], v);
      {
        float vn[3];
        normalized(v, vn);
        const float phi = atan2f(vn[1], vn[0]) * P_INV_2PI;
        wi[0] = (1.0f - vn[2]) * 0.5f;
        wi[1] = phi < 0.0f ? phi + 1.0f : phi;
      }
      int fl = (int)floorf(wi[0] * (float)bins);
      if (fl > bins - 1) fl = bins - 1;
      float theta;
      if (linear) {
        const float w = wi[0] * (float)bins - (float)fl;
        theta = ((float)fl + w) / (float)bins;
      } else {
        theta = (float)fl / (float)bins;
      }
      float L[3];
      local_radiance(s, d, p, L);
      const float* bv = F3(s->bsdf_val, d, p);
      const float wpdf = *F1(s->wi_pdf, d, p);
      if (any_nan(x, 3) || any_nan(wi, 2) || any_nan(x + 3, 3) || isnan(wpdf) || wpdf == 0.0f ||
          any_nan(L, 3))
        continue;
      if (k < cap) {
        memcpy(in + k * 9, x, sizeof(x));
        memcpy(in_phi + k * 10, x, sizeof(x));
        in_phi[k * 10 + 9] = theta;
        float* o = target + k * 9;
        o[0] = wi[0];
        o[1] = wi[1];
        for (int c = 0; c < 3; ++c) o[2 + c] = L[c] * bv[c];
        o[5] = wpdf;
        /* GuidedOutput::bsdfVal is value-initialised and never assigned
           (train.cu:21-81); bsdfVal enters only through L */
        for (int c = 0; c < 3; ++c) o[6 + c] = 0.0f;
      }
      ++k;
    }
  }
  return k;
}

void go_build_nrc_records(go_paths* s, const float aabb[6], int64_t n_train, uint32_t offset,
                          uint32_t stride, int with_training, float* q_in, int32_t* q_depth,
                          int32_t* q_pixel, int64_t q_cap, float* t_in, float* t_target,
                          int64_t t_cap, int64_t* counts) {
  const frame_t f = scene_frame(aabb);
  int64_t kq = 0, kt = 0;
  for (int64_t i = 0; i < n_train; ++i) {
    const int64_t p = (int64_t)(offset + (uint32_t)i * stride);
    const int depth = (int)s->cur_depth[p];
    for (int d = 0; d < depth && d < P_MAXD; ++d) {
      if (*F1(s->delta, d, p) || *F1(s->miss, d, p)) continue;
      float x[15];
      vertex_inputs(s, d, p, &f, x);
      memcpy(x + 9, F3(s->diffuse, d, p), 3 * sizeof(float));
      memcpy(x + 12, F3(s->specular, d, p), 3 * sizeof(float));
      int ok = !(any_nan(x, 3) || any_nan(x + 3, 3));
      float L[3] = {0.f, 0.f, 0.f};
      if (with_training) {
        local_radiance(s, d, p, L);
        const float* bv = F3(s->bsdf_val, d, p);
        const float den = *F1(s->wi_pdf, d, p) + P_EPS;
        for (int c = 0; c < 3; ++c) L[c] = L[c] * bv[c] / den;
        ok = ok && !any_nan(L, 3);
      }
      if (!ok) continue;
      if (kq < q_cap) {
        memcpy(q_in + kq * 15, x, sizeof(x));
        q_depth[kq] = d;
        q_pixel[kq] = (int32_t)p;
      }
      ++kq;
      if (with_training && d < depth - 1) {
        if (kt < t_cap) {
          memcpy(t_in + kt * 15, x, sizeof(x));
          memcpy(t_target + kt * 3, L, sizeof(L));
        }
        ++kt;
      }
    }
    s->cur_depth[p] = s->cur_depth[p] - 1u;
  }
  counts[0] = kq;
  counts[1] = kt;
}

static int valid_record(const go_paths* s, int64_t p, int d) {
  return d >= 0 && d < P_MAXD && (uint32_t)d < s->cur_depth[p];
}

void go_apply_nrc(go_paths* s, const float* out, const int32_t* depth, const int32_t* pixel,
                  int64_t m) {
  for (int64_t i = 0; i < m; ++i) { /* replaceIndirectRadianceSkipDelta(p, d - 1, o) */
    const int64_t p = pixel[i];
    const int initial = depth[i] - 1;
    if (initial >= P_MAXD) continue;
    int d = initial;
    while (d >= 0 && *F1(s->delta, d, p)) --d;
    if (!valid_record(s, p, d)) continue;
    float* L = F3(s->L, d, p);
    const float* t = F3(s->thp, initial, p);
    const float* e = F3(s->Le, initial, p);
    for (int c = 0; c < 3; ++c) L[c] = t[c] * (out[i * 3 + c] + e[c]);
  }
  for (int64_t i = 0; i < m; ++i) { /* divideRadiance(p, d, o) */
    const int64_t p = pixel[i];
    const int d = depth[i];
    if (!valid_record(s, p, d)) continue;
    float* L = F3(s->L, d, p);
    for (int c = 0; c < 3; ++c) {
      const float o = out[i * 3 + c];
      if (o > P_EPS) L[c] = L[c] / o;
    }
  }
}
