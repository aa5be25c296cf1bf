/*
 * gdf_oracle_train.c -- CPU oracle of the DF / NRC training step.
 *
 * TEST INFRASTRUCTURE ONLY (checker for tests/). Never linked into the
 * product library.
 *
 * Restates, for one batch:
 *   - the forward with fp16 network outputs and fp16 pdf tables
 *     (softmaxMultFactor, src/render/guided/learnedDistribution.cpp:255,262;
 *     train.h:872-881);
 *   - combine_AR_pdf_and_dl_doutput (train.h:932-965) with the analytic
 *     Jacobians of AutoRegressive::compute_gradients_specialized_* (AR.h:51-104);
 *   - the FullyFusedMLP backward (tcnn/src/fully_fused_mlp.cu:755-850: ReLU
 *     masks on the fp16 forward activations, weight gradients G = dY^T X) and
 *     the grid backward (tcnn encodings/grid.h:395-520), accumulated in FP64;
 *   - RelativeL2Luminance (tcnn losses/relative_l2_luminance.h:40-86) for NRC;
 *   - Adam (tcnn optimizers/adam.h:48-117) followed by EMA
 *     (tcnn optimizers/ema.h:63-130).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gdf_oracle.h"

#define GO_EPS 1e-5f
#define GO_INV_4PI 0.0795774715459476678844f /* M_INV_4PI */

static int32_t pad16i(int32_t v) { return (v + 15) / 16 * 16; }
static float h16(float x) { return go_round_f16(x); }
/* a backward storage point of the MLP operand format (go_set_storage: fp16,
 * the reference's; bf16 for the bf16 training form) */
static float hst(float x) { return go_store(x); }

/* fp16 pdf table of one network from its fp32 logits: logits stored as fp16
 * (tcnn output precision), softmax2 in float stored as fp16, times N in fp16
 * (exact for N a power of two). */
static void train_pdf_table(const float* logits, int n, float* table) {
  float z[128];
  float mx = 0.0f;
  for (int i = 0; i < n; ++i) { z[i] = h16(logits[i]); mx = fmaxf(mx, z[i]); }
  float s = 0.0f;
  for (int i = 0; i < n; ++i) s += expf(z[i] - mx);
  const float ls = logf(s);
  for (int i = 0; i < n; ++i) table[i] = h16(h16(expf(z[i] - mx - ls)) * (float)n);
}

/* compute_gradients_specialized_linear_interpolation / _nearest (AR.h:51-104):
 * dL/dlogit_i = prefix * pdf_other * N * dpdf(u)/dlogit_i, stored as fp16. */
static void dlogits(const float* table, int n, int linear, float u, float pdf_other, float prefix,
                    float* out) {
  const float inv_res = 1.0f / (float)n;
  const float multiplier = prefix * pdf_other * (float)n;
  if (linear) {
    const float idx = u * (float)n - 0.5f;
    int f = (int)floorf(idx);
    if (f > n - 1) f = n - 1;
    int c = f + 1;
    float w = idx - (float)f;
    if (f < 0) { f = n - 1; w = 1.0f; }
    if (c > n - 1) { c = 0; w = 0.0f; }
    const float p0 = table[f] * inv_res, p1 = table[c] * inv_res;
    for (int i = 0; i < n; ++i) {
      const float pi = table[i] * inv_res;
      const float j0 = f == i ? p0 * (1.0f - p0) : -p0 * pi;
      const float j1 = c == i ? p1 * (1.0f - p1) : -p1 * pi;
      out[i] = hst(multiplier * ((1.0f - w) * j0 + w * j1));
    }
  } else {
    int f = (int)(u * (float)n);
    if (f > n - 1) f = n - 1;
    const float p0 = table[f] * inv_res;
    for (int i = 0; i < n; ++i) {
      const float pi = table[i] * inv_res;
      out[i] = hst(multiplier * (f == i ? p0 * (1.0f - p0) : -p0 * pi));
    }
  }
}

/* Exported for the reference pin: dL/dlogits of one row from a pdf table. */
void go_dlogits(const float* table, int n, int linear, float u, float pdf_other, float prefix, float* out) {
  dlogits(table, n, linear, u, pdf_other, prefix, out);
}

/* combine_AR_pdf_and_dl_doutput (train.h:932-965) on given fp16 pdf tables
 * (values as float): likelihood and fp16 dL/dlogits of both networks. */
void go_combine(const float* target, int64_t n, const float* tab_theta, int nbt, const float* tab_phi,
                int nbp, int linear, float loss_scale, float* dl_theta, float* dl_phi, float* likelihood) {
  const float scale = loss_scale / (float)n;
  for (int64_t i = 0; i < n; ++i) {
    const float* tg = target + i * 9;
    const float* tt = tab_theta + i * nbt;
    const float* tp = tab_phi + i * nbp;
    const float pt = go_sample_pdf(tt, tg[0], nbt, linear);
    const float pp = go_sample_pdf(tp, tg[1], nbp, linear);
    const float li = (tg[2] + tg[3] + tg[4]) / 3.0f;
    const float wi_pdf = tg[5] + GO_EPS;
    const float pdf_tr = GO_INV_4PI;
    const float guided = fabsf(pt) * fabsf(pp) * pdf_tr * (1.f / pdf_tr) + GO_EPS;
    const float prefix = -li / wi_pdf / guided * scale;
    likelihood[i] = -li / wi_pdf * logf(guided);
    dlogits(tt, nbt, linear, tg[0], fabsf(pp), prefix, dl_theta + i * nbt);
    dlogits(tp, nbp, linear, tg[1], fabsf(pt), prefix, dl_phi + i * nbp);
  }
}

static int finite_row(const float* a, int n) {
  for (int i = 0; i < n; ++i)
    if (isnan(a[i])) return 0;
  return 1;
}

/* MLP forward keeping the fp16 activations; out = fp32 logits. */
static void mlp_fwd_save(const float* w16, int k0, int width, int n_hidden, int n_out_pad,
                         const float* x16, float* hidden /* n_hidden x width */, float* out) {
  go_mlp_forward(w16, k0, width, n_hidden, n_out_pad, x16, out, hidden);
}

/* Backward of one row: dY (n_out_pad, fp16 values) -> accumulate weight
 * gradients into g (fp64, tcnn order) and return dX (k0, fp64). */
static void mlp_bwd_row(const float* w16, int k0, int width, int n_hidden, int n_out_pad,
                        const float* x16, const float* hidden, const float* dy, double* g,
                        double* dx) {
  double d[256], dn[256];
  /* offsets of each matrix */
  int64_t off[16];
  off[0] = 0;
  int64_t o = (int64_t)width * k0;
  for (int l = 1; l < n_hidden; ++l) { off[l] = o; o += (int64_t)width * width; }
  off[n_hidden] = o;
  /* output layer */
  const float* hl = hidden + (size_t)(n_hidden - 1) * width;
  for (int r = 0; r < n_out_pad; ++r)
    for (int c = 0; c < width; ++c) g[off[n_hidden] + (int64_t)r * width + c] += (double)dy[r] * hl[c];
  for (int c = 0; c < width; ++c) {
    double acc = 0.0;
    for (int r = 0; r < n_out_pad; ++r) acc += (double)dy[r] * w16[off[n_hidden] + (int64_t)r * width + c];
    d[c] = hl[c] > 0.0f ? (double)hst(acc) : 0.0; /* backward activations stored as fp16 (bf16) */
  }
  for (int l = n_hidden - 1; l >= 1; --l) {
    const float* hp = hidden + (size_t)(l - 1) * width;
    for (int r = 0; r < width; ++r)
      for (int c = 0; c < width; ++c) g[off[l] + (int64_t)r * width + c] += d[r] * hp[c];
    for (int c = 0; c < width; ++c) {
      double acc = 0.0;
      for (int r = 0; r < width; ++r) acc += d[r] * w16[off[l] + (int64_t)r * width + c];
      dn[c] = hp[c] > 0.0f ? (double)hst(acc) : 0.0;
    }
    memcpy(d, dn, sizeof(double) * (size_t)width);
  }
  for (int r = 0; r < width; ++r)
    for (int c = 0; c < k0; ++c) g[(int64_t)r * k0 + c] += d[r] * x16[c];
  for (int c = 0; c < k0; ++c) {
    double acc = 0.0;
    for (int r = 0; r < width; ++r) acc += d[r] * w16[(int64_t)r * k0 + c];
    dx[c] = acc;
  }
}

/* grid_index / kernel_grid_backward scatter (grid.h:395-520), FP64. */
static uint32_t grid_idx(const go_grid* g, uint32_t hsize, uint32_t res, const uint32_t p[3]) {
  uint32_t stride = 1, index = 0;
  for (int d = 0; d < 3 && stride <= hsize; ++d) { index += p[d] * stride; stride *= res; }
  if (g->c.type == 0 && hsize < stride) index = p[0] ^ (p[1] * 2654435761u) ^ (p[2] * 805459861u);
  return index % hsize;
}

static void grid_bwd_row(const go_grid* g, const float pos[3], const double* dy, double* grad) {
  const int F = g->c.n_features_per_level;
  for (int l = 0; l < g->c.n_levels; ++l) {
    const float scale = g->scale[l];
    const uint32_t res = g->resolution[l], hsize = g->offset[l + 1] - g->offset[l];
    float fr[3];
    uint32_t pg[3];
    for (int d = 0; d < 3; ++d) {
      float p = fmaf(pos[d], scale, 0.5f);
      float t = floorf(p);
      pg[d] = (uint32_t)(int)t;
      p -= t;
      if (g->c.interpolation == 1) p = p * p * (3.0f - 2.0f * p);
      fr[d] = p;
    }
    double* gl = grad + (size_t)g->offset[l] * F;
    if (g->c.interpolation == 2) {
      uint32_t e = grid_idx(g, hsize, res, pg);
      for (int f = 0; f < F; ++f) gl[(size_t)e * F + f] += dy[l * F + f];
      continue;
    }
    for (int c = 0; c < 8; ++c) {
      double w = 1.0;
      uint32_t q[3];
      for (int d = 0; d < 3; ++d) {
        if (c & (1 << d)) { w *= fr[d]; q[d] = pg[d] + 1; }
        else { w *= 1.0 - (double)fr[d]; q[d] = pg[d]; }
      }
      uint32_t e = grid_idx(g, hsize, res, q);
      for (int f = 0; f < F; ++f) gl[(size_t)e * F + f] += w * dy[l * F + f];
    }
  }
}

/* One DF training batch: forward (fp16 tables), loss, dL/dlogits and the
 * gradients of every parameter of both networks (scaled by loss_scale like
 * the reference's fp16 gradient buffers; FP64).
 *   in_theta [n x 9], in_phi [n x 10], target [n x 9] (dir2, L3, wiPdf, bsdf3)
 *   w16_theta / w16_phi: fp16-rounded training weights (tcnn order)
 *   grad_theta / grad_phi (FP64, zeroed by the caller)
 *   likelihood [n] (float, reference semantics), dlog_theta/phi (nullable). */
int64_t go_df_train_grads(const go_df_config* c, const float* w16_theta, const float* w16_phi,
                          const float* in_theta, const float* in_phi, const float* target,
                          int64_t n, float loss_scale, double* grad_theta, double* grad_phi,
                          float* likelihood, float* pdf_out, float* dlog_theta, float* dlog_phi) {
  go_grid gt, gp;
  go_grid_init(&gt, &c->grid_theta);
  go_grid_init(&gp, &c->grid_phi);
  const int k0t = go_df_input_width(c, 0), k0p = go_df_input_width(c, 1);
  const int nbt = c->n_bins_theta, nbp = c->n_bins_phi, lin = c->pdf_interp == 0;
  const int w = c->width;
  const int64_t mlp_t = go_df_mlp_params(c, 0), mlp_p = go_df_mlp_params(c, 1);
  int64_t dropped = 0;
  const float scale = loss_scale / (float)n;
  for (int64_t i = 0; i < n; ++i) {
    const float* qt = in_theta + i * 9;
    const float* qp = in_phi + i * 10;
    const float* tg = target + i * 9;
    /* generate_training_data_AR validity filter (train.cu:77-81) */
    if (!finite_row(qt, 9) || !finite_row(qp, 10) || !finite_row(tg, 9) || tg[5] == 0.0f) {
      likelihood[i] = 0.0f;
      if (pdf_out) { pdf_out[i * 2] = 0.f; pdf_out[i * 2 + 1] = 0.f; }
      if (dlog_theta) memset(dlog_theta + i * nbt, 0, sizeof(float) * (size_t)nbt);
      if (dlog_phi) memset(dlog_phi + i * nbp, 0, sizeof(float) * (size_t)nbp);
      ++dropped;
      continue;
    }
    float xt[256], xp[256], ht[8 * 64], hp[8 * 64], lt[128], lp[128], tt[128], tp[128];
    go_df_encode(c, &gt, 0, w16_theta, qt, 0.f, xt);
    go_df_encode(c, &gp, 1, w16_phi, qp, qp[9], xp);
    mlp_fwd_save(w16_theta, k0t, w, c->hidden_theta, pad16i(nbt), xt, ht, lt);
    mlp_fwd_save(w16_phi, k0p, w, c->hidden_phi, pad16i(nbp), xp, hp, lp);
    train_pdf_table(lt, nbt, tt);
    train_pdf_table(lp, nbp, tp);
    /* combine_AR_pdf_and_dl_doutput (train.h:932-965) */
    const float pt = go_sample_pdf(tt, tg[0], nbt, lin);
    const float pp = go_sample_pdf(tp, tg[1], nbp, lin);
    const float li = (tg[2] + tg[3] + tg[4]) / 3.0f;
    const float wi_pdf = tg[5] + GO_EPS;
    const float pdf_tr = GO_INV_4PI;
    const float guided = fabsf(pt) * fabsf(pp) * pdf_tr * (1.f / pdf_tr) + GO_EPS;
    const float prefix = -li / wi_pdf / guided * scale;
    likelihood[i] = -li / wi_pdf * logf(guided);
    if (pdf_out) { pdf_out[i * 2] = pt; pdf_out[i * 2 + 1] = pp; }
    float dt[128], dp[128];
    memset(dt, 0, sizeof(dt));
    memset(dp, 0, sizeof(dp));
    dlogits(tt, nbt, lin, tg[0], fabsf(pp), prefix, dt);
    dlogits(tp, nbp, lin, tg[1], fabsf(pt), prefix, dp);
    if (dlog_theta) memcpy(dlog_theta + i * nbt, dt, sizeof(float) * (size_t)nbt);
    if (dlog_phi) memcpy(dlog_phi + i * nbp, dp, sizeof(float) * (size_t)nbp);
    double dxt[256], dxp[256];
    mlp_bwd_row(w16_theta, k0t, w, c->hidden_theta, pad16i(nbt), xt, ht, dt, grad_theta, dxt);
    mlp_bwd_row(w16_phi, k0p, w, c->hidden_phi, pad16i(nbp), xp, hp, dp, grad_phi, dxp);
    grid_bwd_row(&gt, qt, dxt, grad_theta + mlp_t);
    grid_bwd_row(&gp, qp, dxp, grad_phi + mlp_p);
  }
  return dropped;
}

/* NRC batch: relative L2 luminance loss (relative_l2_luminance.h:40-86) over
 * the 3 real outputs of the 16-wide padded output; gradients scaled by
 * loss_scale (FP64). loss_out[i] = sum over channels of the values. */
void go_nrc_train_grads(const go_nrc_config* c, const float* w16, const float* in15,
                        const float* target3, int64_t m, float loss_scale, double* grad,
                        float* loss_out) {
  const int k0 = go_nrc_input_width(c);
  const float n_total = (float)(m * 3);
  for (int64_t i = 0; i < m; ++i) {
    float x[256], h[8 * 64], y[16], dy[16];
    go_nrc_encode(c, in15 + i * 15, x);
    mlp_fwd_save(w16, k0, c->width, c->hidden, 16, x, h, y);
    float yh[16];
    for (int k = 0; k < 16; ++k) yh[k] = h16(y[k]); /* fp16 network output */
    const float lum = 0.299f * yh[0] + 0.587f * yh[1] + 0.114f * yh[2];
    const float denom = lum * lum + 0.01f;
    float lsum = 0.f;
    for (int k = 0; k < 16; ++k) {
      if (k < 3) {
        const float diff = yh[k] - target3[i * 3 + k];
        lsum += diff * diff / denom / 1.0f / n_total;
        const float gr = 2 * diff / denom / 1.0f;
        dy[k] = h16(loss_scale * gr / n_total);
      } else {
        dy[k] = 0.f;
      }
    }
    loss_out[i] = lsum;
    double dx[256];
    mlp_bwd_row(w16, k0, c->width, c->hidden, 16, x, h, dy, grad, dx);
  }
}

/* Adam (adam.h:48-117) + EMA (ema.h:63-130) over one network's parameters.
 * step = the optimizer's global step after increment (m_current_step).
 * Parameters at index >= n_matrix with a zero gradient are skipped by Adam
 * (non-matrix params); EMA runs over all. master/ema/m/v/steps updated. */
void go_adam_ema(int64_t n, int64_t n_matrix, const double* grad_scaled, float loss_scale,
                 float lr, float beta1, float beta2, float eps, float l2_reg, float ema_decay,
                 uint32_t step, float* master, float* w16, float* ema16, float* m1, float* m2,
                 uint32_t* steps) {
  const float debias_old = 1.0f - (float)pow((double)ema_decay, (double)(step - 1));
  const float debias_new = 1.0f / (1.0f - (float)pow((double)ema_decay, (double)step));
  for (int64_t i = 0; i < n; ++i) {
    float g = (float)grad_scaled[i] / loss_scale;
    int skip = i >= n_matrix && g == 0.0f;
    if (!skip) {
      const float wf = master[i];
      if (i < n_matrix) g += l2_reg * wf;
      const float g2 = g * g;
      const float fm = m1[i] = beta1 * m1[i] + (1 - beta1) * g;
      const float sm = m2[i] = beta2 * m2[i] + (1 - beta2) * g2;
      const uint32_t cs = ++steps[i];
      float l = lr * sqrtf(1 - powf(beta2, (float)cs)) / (1 - powf(beta1, (float)cs));
      const float eff = fminf(fmaxf(l / (sqrtf(sm) + eps), 0.0f), 3.402823466e38f);
      const float nw = wf - eff * fm;
      master[i] = nw;
      w16[i] = h16(nw);
    }
    ema16[i] = h16((ema16[i] * ema_decay * debias_old + w16[i] * (1 - ema_decay)) * debias_new);
  }
}
