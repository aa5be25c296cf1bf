/*
 * gdf_oracle.h -- CPU oracle of the guiding-df DF/NRC hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm used as the checker by tests/, by __graft_entry__.smoke() and by
 * bench.py's cpu_baseline leg. The product library never links or calls it.
 *
 * Every function cites the reference file:line it restates. Paths are
 * relative to the guiding-df project root; `tcnn/` = src/ext/tcnn.
 *
 * Pinning. tests/test_reference_pin.py checks the DF epilogue and training
 * restatements bit for bit against the reference's own train.h / AR.h
 * compiled for the host (oracle/build_ref.py -> oracle/_ref/); the encodings
 * and MLP against analytic identities (tests/test_oracle.py).
 *
 * Precision model. The checker computes in FP64 with fp16 rounding at the
 * storage points the product kernels use (fp16 parameters, fp16 encoded
 * inputs, fp16 hidden activations, fp32 logits). The DF epilogue
 * (softmax / CDF / inversion sampling / pdf interpolation) is restated in
 * fp32 with the reference's operation order (compiled without FMA
 * contraction) so that its discrete decisions follow the reference's float
 * behaviour; a double twin reports the error of the float epilogue.
 */
#ifndef GDF_ORACLE_H_
#define GDF_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GO_MAX_LEVELS 24

typedef struct go_grid_config {
  int32_t type, n_levels, n_features_per_level, log2_hashmap_size, base_resolution;
  float per_level_scale;
  int32_t interpolation;
} go_grid_config;

/* Per-level tables of tcnn GridEncodingTemplated (tcnn/include/tiny-cuda-nn/
 * encodings/grid.h:967-1012). */
typedef struct go_grid {
  go_grid_config c;
  float scale[GO_MAX_LEVELS];
  uint32_t resolution[GO_MAX_LEVELS];
  uint32_t offset[GO_MAX_LEVELS + 1]; /* in entries (features / F) */
  int64_t n_params;
} go_grid;

typedef struct go_df_config {
  int32_t n_bins_theta, n_bins_phi, pdf_interp; /* 0 linear, 1 nearest */
  go_grid_config grid_theta, grid_phi;
  int32_t sh_degree, oneblob_bins, tw_frequencies;
  int32_t width, hidden_theta, hidden_phi;
} go_df_config;

typedef struct go_nrc_config {
  int32_t frequencies, oneblob_bins, width, hidden;
} go_nrc_config;

/* ---- scalar helpers ---- */
uint16_t go_f32_to_f16(float x);
float go_f16_to_f32(uint16_t h);
float go_round_f16(double x);
void go_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float go_u32_to_uniform(uint32_t x);
void go_philox_uniforms(uint64_t seed, uint64_t offset, int64_t n, float* out /* n x 4 */);

/* ---- encodings ---- */
int go_grid_init(go_grid* g, const go_grid_config* c);
void go_grid_encode(const go_grid* g, const float* table, const float pos[3], double* out);
void go_sh_encode(int degree, const float dir01[3], double* out);
void go_oneblob_encode(int n_bins, const float* x, int n_dims, double* out);
void go_triangle_wave_encode(int n_freq, float x, double* out);
void go_frequency_encode(int n_freq, const float* x, int n_dims, double* out);

/* Network layout (tcnn order: MLP matrices, then encoding parameters). */
int32_t go_df_input_width(const go_df_config* c, int net);  /* padded encoded width */
int64_t go_df_mlp_params(const go_df_config* c, int net);
int64_t go_df_n_params(const go_df_config* c, int net);
int32_t go_nrc_input_width(const go_nrc_config* c);
int64_t go_nrc_n_params(const go_nrc_config* c);

/* Encoded network input (fp16-rounded, padded) for one query. */
void go_df_encode(const go_df_config* c, const go_grid* g, int net, const float* params16,
                  const float* q, float theta_cond, float* out);
void go_nrc_encode(const go_nrc_config* c, const float* q15, float* out);

/* MLP forward, fp16 weights/activations, fp64 accumulation, fp32 outputs. */
void go_mlp_forward(const float* w16, int k0, int width, int n_hidden, int n_out_pad,
                    const float* x16, float* out, float* hidden_out /* nullable, n_hidden x width */);

void go_set_accumulation(int acc32);
/* The same forward in plain fp32 (sequential sums), the CPU baseline's MLP. */
void go_mlp_forward_f32(const float* w16, int k0, int width, int n_hidden, int n_out,
                        const float* x16, float* out);

/* ---- DF epilogue, reference float semantics ---- */
void go_softmax2_times_n(float* v, int n);
int go_sample_dir(const float* pdf, int n, int linear, float u_main, float u_fallback,
                  float* out_dir, float* out_edge_gap);
float go_sample_pdf(const float* pdf, float u, int n, int linear);
float go_theta_condition(float u_theta, int n, int linear);
double go_sample_dir_f64(const float* pdf, int n, int linear, double u_main, double u_fallback);

/* Epilogue on given logits: thetaPostInference + phiPostInference. */
void go_post_inference(const go_df_config* c, const float* logits_theta, const float* logits_phi,
                       const uint8_t* guided, const float* uniforms, float* wi, float* edge_gap,
                       int64_t n);

/* Full inference (gdf_infer semantics). params are fp16-rounded, tcnn order.
 * edge_gap (nullable, n x 2) receives the distance of the main uniform to
 * the nearest CDF edge of the sampled segment. */
void go_infer(const go_df_config* c, const float* params_theta16, const float* params_phi16,
              const float* queries, const uint8_t* guided, const float* uniforms, float* wi,
              float* edge_gap, int64_t n, int n_threads);

/* Same forward as go_infer but with the fp32 throughput-oriented MLP (CPU
 * baseline; not a checker). */
void go_infer_fp32(const go_df_config* c, const float* params_theta16,
                   const float* params_phi16, const float* queries, const uint8_t* guided,
                   const float* uniforms, float* wi, int64_t n, int n_threads);

/* pdf evaluation at given directions (gdf_eval_pdf semantics). */
void go_eval_pdf(const go_df_config* c, const float* params_theta16, const float* params_phi16,
                 const float* queries, const float* u, float* pdf_out, int64_t n, int n_threads);

/* Per-row softmax x N tables of both networks (phi conditioned on u_theta). */
void go_df_pdf_tables(const go_df_config* c, const float* p_theta, const float* p_phi,
                      const float* queries, const float* u_theta, float* pdf_theta,
                      float* pdf_phi, int64_t n);

/* NRC query (gdf_nrc_query semantics). */
void go_nrc_query(const go_nrc_config* c, const float* params16, const float* in15, float* out3,
                  int64_t m, int n_threads);


/* Storage format of the DF networks' MLP inputs/activations: 0 fp16,
 * 1 bf16, 2 unrounded. */
void go_set_storage(int fmt);
float go_round_bf16(float x);
double go_round_e4m3(double x);
int go_e4m3_scale_exp(double amax);
float go_store(double x);

/* ---- path records (gdf_oracle_paths.c) ---------------------------------- */
/* Host copy of GuidedPixelStateBuffer: each field is [5][n][k] (depth-major). */
typedef struct go_paths {
  int64_t n; /* pixels */
  float *L, *thp, *Le, *pos, *dir, *wi_pdf, *mis_weight;
  uint8_t *delta, *miss;
  float *bsdf_val, *wo, *normal, *roughness, *diffuse, *specular;
  uint32_t* cur_depth;
} go_paths;

void go_prepare_queries(const float* pos, const float* wo, const float* nrm, const float* rough,
                        const float aabb[6], float* q, int64_t n);
int64_t go_build_df_records(const go_paths* s, const float aabb[6], int64_t n_train, uint32_t offset,
                            uint32_t stride, int bins, int linear, float* in, float* in_phi,
                            float* target, int64_t cap);
void go_build_nrc_records(go_paths* s, const float aabb[6], int64_t n_train, uint32_t offset,
                          uint32_t stride, int with_training, float* q_in, int32_t* q_depth,
                          int32_t* q_pixel, int64_t q_cap, float* t_in, float* t_target,
                          int64_t t_cap, int64_t* counts);
void go_apply_nrc(go_paths* s, const float* out, const int32_t* depth, const int32_t* pixel,
                  int64_t m);
/* AutoRegressive view of guiding records [n x 4]: out [n x 4] =
 * (solid-angle pdf, world direction). */
void go_autoregressive(const float* wi4, int64_t n, float* out);

#ifdef __cplusplus
}
#endif
#endif
