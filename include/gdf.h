/*
 * gdf.h -- C ABI of the B200-native neural path-guiding module (Distribution
 * Factorization, DF) and its Neural Radiance Cache (NRC).
 *
 * The entry points replace the guiding-module interface of guiding-df
 * (pedrovfigueiredo/guiding-df):
 *   - LearnedDistribution  src/render/guided/learnedDistribution.h:37-168
 *   - NRC                  src/render/guided/nrc.h:30-97
 * Each declaration below cites the reference member it stands in for.
 *
 * Conventions
 *   - Every function returns gdf_status; nothing throws across the ABI.
 *     gdf_last_error() returns a thread-local message for the last failure.
 *   - Buffers named *_dev are device pointers owned by the caller; the
 *     library owns network weights, optimizer state and workspaces.
 *   - `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 *     Work is stream-ordered; no entry point below synchronises the device
 *     except where the comment says "synchronises".
 *   - Query layout (one row per query, fp32), identical to the reference's
 *     inference input buffer (train.cu:334-362, guideditem.h:53-72):
 *       [0..2] position normalised to [0,1]^3
 *       [3..5] outgoing direction warped to [0,1]^3, (wo + 1) / 2
 *       [6]    shading-normal theta / pi, [7] shading-normal phi / (2 pi)
 *       [8]    1 - exp(-roughness)
 *   - Guiding-data layout, identical to the reference's inferenceWiBuffer
 *     (parameters.h:44): [u_theta, u_phi, pdf_theta, pdf_phi] per query.
 */
#ifndef GDF_H_
#define GDF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GDF_ABI_VERSION 2
#define GDF_MAX_GRID_LEVELS 24
/* MAX_TRAIN_DEPTH (parameters.h:24): path vertices recorded per pixel. */
#define GDF_MAX_TRAIN_DEPTH 5

typedef enum gdf_status {
  GDF_OK = 0,
  GDF_ERR_INVALID_ARG = 1,  /* malformed config, bad size or null pointer    */
  GDF_ERR_OOM_BUDGET = 2,   /* allocation refused by the HBM budget / device */
  GDF_ERR_CUDA = 3,         /* a CUDA runtime call failed                    */
  GDF_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up            */
  GDF_ERR_NUMERIC = 5,      /* NaN/Inf detected where the contract forbids it */
  GDF_ERR_UNSUPPORTED = 6,  /* configuration outside what the kernels build  */
  GDF_ERR_STATE = 7         /* call order violated (e.g. no parameters yet)  */
} gdf_status;

/* Interpolation of the per-bin PDF (parameters.h:20 AR_LINEAR_INTERPOLATION). */
typedef enum gdf_pdf_interp { GDF_PDF_LINEAR = 0, GDF_PDF_NEAREST = 1 } gdf_pdf_interp;

/* tiny-cuda-nn GridType / InterpolationType (encodings/grid.h:944-1000). */
typedef enum gdf_grid_type { GDF_GRID_HASH = 0, GDF_GRID_DENSE = 1, GDF_GRID_TILED = 2 } gdf_grid_type;
typedef enum gdf_grid_interp {
  GDF_GRID_LINEAR = 0, GDF_GRID_SMOOTHSTEP = 1, GDF_GRID_NEAREST = 2
} gdf_grid_interp;

/* Arithmetic type of the MLP layers (tensor-core operands); accumulation is fp32. */
typedef enum gdf_precision { GDF_PREC_FP16 = 0, GDF_PREC_BF16 = 1, GDF_PREC_FP8 = 2 } gdf_precision;

/* Network ids for parameter access. */
typedef enum gdf_net { GDF_NET_THETA = 0, GDF_NET_PHI = 1, GDF_NET_NRC = 2 } gdf_net;

typedef struct gdf_grid_config {
  int32_t type;                 /* gdf_grid_type                         */
  int32_t n_levels;             /* grid.h:1457 n_levels                  */
  int32_t n_features_per_level; /* 2 or 4                                */
  int32_t log2_hashmap_size;    /* hash table entries per level = 2^this */
  int32_t base_resolution;
  float per_level_scale;
  int32_t interpolation;        /* gdf_grid_interp                       */
} gdf_grid_config;

typedef struct gdf_mlp_config {
  int32_t n_neurons;       /* only 64 is built                                */
  int32_t n_hidden_layers; /* tcnn semantics: hidden layers incl. the first  */
} gdf_mlp_config;

typedef struct gdf_adam_config {
  float learning_rate, beta1, beta2, epsilon, l2_reg;
  float ema_decay;  /* EmaOptimizer decay (optimizers/ema.h)           */
} gdf_adam_config;

typedef struct gdf_config {
  int32_t abi_version;     /* must be GDF_ABI_VERSION                      */
  int32_t n_bins_theta;    /* N_DIM_OUTPUT      (parameters.h:41): 16/32/64 */
  int32_t n_bins_phi;      /* N_DIM_OUTPUT_PHI  (parameters.h:48): 16/32/64 */
  int32_t pdf_interp;      /* gdf_pdf_interp                               */
  gdf_grid_config grid_theta, grid_phi; /* the positional grid of each net */
  int32_t sh_degree;       /* SphericalHarmonics degree (4)                */
  int32_t oneblob_bins;    /* OneBlob n_bins (4)                           */
  int32_t tw_frequencies;  /* TriangleWave n_frequencies of the phi net (12) */
  gdf_mlp_config mlp_theta, mlp_phi;
  gdf_adam_config adam_df;  /* base_product_df.json optimizer               */
  float loss_scale;         /* TRAIN_LOSS_SCALE (parameters.h:45) = 1024     */
  int32_t nrc_enable;
  int32_t nrc_frequencies;  /* Frequency n_frequencies (12)                 */
  int32_t nrc_oneblob_bins; /* OneBlob n_bins (4)                           */
  gdf_mlp_config mlp_nrc;
  gdf_adam_config adam_nrc; /* base_hashgrid_nrc_df.json optimizer          */
  float nrc_loss_scale;     /* TRAIN_LOSS_SCALE_NRC (parameters.h:62) = 1024 */
  int32_t precision;        /* gdf_precision of the DF MLP layers: FP16 (the
                               reference), BF16 (inference and training),
                               FP8 (inference; training stays fp16)         */
  uint32_t seed;            /* parameter initialisation seed (7272)          */
  int64_t max_queries;      /* capacity of one inference call                */
  int64_t max_train_batch;  /* capacity of one training call                 */
  /* Frame-level training loops (gdf_train_paths, gdf_nrc_train_paths):
   * LearnedDistribution batchSize / batchPerFrame (learnedDistribution.h:138-139),
   * NRC batchSize / batchPerFrame (nrc.h:80-81), MIN_TRAIN_BATCH_SIZE
   * (parameters.h:55). Batch sizes must not exceed max_train_batch. */
  int64_t df_batch_size;
  int64_t nrc_batch_size;
  int64_t min_train_batch;
  int32_t df_batches_per_frame;
  int32_t nrc_batches_per_frame;
} gdf_config;

typedef enum gdf_preset {
  GDF_PRESET_SMALL = 0,     /* 65,536 queries: hash 8x2, 2^16, 64x3, 32 bins    */
  GDF_PRESET_FULL = 1,      /* 1920x1080 queries: hash 16x2, 2^19, 64x4, 64 bins */
  GDF_PRESET_REFERENCE = 2  /* common/configs/nn/base_product_df.json exactly   */
} gdf_preset;

typedef struct gdf_ctx gdf_ctx;

/* Per-call statistics of the last training step. */
typedef struct gdf_train_stats {
  double loss;          /* mean divergence loss of the batch (FP64 reduction) */
  double grad_norm;     /* L2 norm of the unscaled parameter gradient (FP64)  */
  int64_t n_records;    /* records used                                       */
  int64_t n_dropped;    /* records rejected as non-finite                     */
} gdf_train_stats;

/* ------------------------------------------------------------------ setup */

/* Fills *cfg with one of the presets. */
gdf_status gdf_default_config(int32_t preset, gdf_config* cfg);

/* LearnedDistribution::resetNetwork (learnedDistribution.cpp:64) and
 * NRC::resetNetwork (nrc.cpp:35): validates the config, allocates weights,
 * optimizer state and workspaces on the current device, initialises the
 * weights (Xavier-uniform MLP, U(-1e-4, 1e-4) grid) and zeroes the Adam/EMA
 * state. Synchronises. */
gdf_status gdf_create(const gdf_config* cfg, gdf_ctx** out);
gdf_status gdf_destroy(gdf_ctx* ctx);

/* LearnedDistribution::resetTraining (learnedDistribution.h:44): re-draws the
 * weights from `seed` and clears optimizer + EMA state. Synchronises. */
gdf_status gdf_reset_training(gdf_ctx* ctx, uint32_t seed);

/* Number of parameters of one network, in tcnn order: MLP weight matrices
 * (first, hidden..., output; each row-major [out][in], output rows padded to
 * a multiple of 16) followed by the grid encoding's tables
 * (network_with_input_encoding.h set_params order). */
gdf_status gdf_n_params(const gdf_ctx* ctx, int32_t net, int64_t* n_params);

/* Trainer::set_params_full_precision (trainer.h:238) through
 * LearnedDistribution::loadNetwork (learnedDistribution.cpp:340): copies fp32
 * host parameters; the fp16 training copy and the EMA inference copy are both
 * set to fp16(params). Synchronises. */
gdf_status gdf_set_params(gdf_ctx* ctx, int32_t net, const float* params_host, int64_t n);

/* Trainer::params_full_precision read-back used by saveNetwork
 * (learnedDistribution.cpp:295): fp32 master parameters. Synchronises. */
gdf_status gdf_get_params(const gdf_ctx* ctx, int32_t net, float* params_host, int64_t n);

/* Read-back of the fp16 EMA weights that inference uses (trainer.h:317-332),
 * widened to fp32. Synchronises. */
gdf_status gdf_get_inference_params(const gdf_ctx* ctx, int32_t net, float* params_host, int64_t n);

/* saveNetwork / loadNetwork (learnedDistribution.cpp:295-384, nrc.cpp:62-112):
 * raw fp32 parameter dumps `<prefix>AR_network_theta.bin`,
 * `<prefix>AR_network_phi.bin` and, with NRC enabled, `<prefix>NRC_network.bin`. */
gdf_status gdf_save_network(const gdf_ctx* ctx, const char* path_prefix);
gdf_status gdf_load_network(gdf_ctx* ctx, const char* path_prefix);

/* -------------------------------------------------------------- inference */

/* LearnedDistribution::inferenceStep (learnedDistribution.cpp:167-206) with
 * thetaPostInference / phiPostInference (train.h:896-929) fused into one
 * kernel: encode -> theta MLP -> softmax x N -> sample u_theta (guided rows)
 * -> phi MLP conditioned on u_theta -> softmax x N -> sample u_phi (guided
 * rows) -> pdf_theta(wi[0]), pdf_phi(wi[1]) multiplied into wi[2], wi[3].
 *
 *   queries_dev  [n x 9] fp32, layout above
 *   guided_dev   [n] uint8, nonzero = guided_pass (guideditem.h:109); NULL = all
 *   uniforms_dev [n x 4] fp32 in [0,1): theta main, theta fallback, phi main,
 *                phi fallback (the sampler.get1D() draws of train.h:438,482,494);
 *                NULL = draw them in-kernel with Philox4x32-10 keyed by
 *                (philox_seed) at counter (row, philox_offset)
 *   wi_dev       [n x 4] fp32 in/out: slots 0,1 hold the BSDF-sampled square
 *                direction of non-guided rows; slots 2,3 hold the caller's
 *                sign (+1/-1) that the pdfs multiply into.
 * Inference uses the EMA weights, like tcnn's inference params. The
 * context's inference workspace is shared by its calls: calls on one
 * context must be ordered (one stream); concurrent streams need separate
 * contexts. */
gdf_status gdf_infer(gdf_ctx* ctx, const float* queries_dev, const uint8_t* guided_dev,
                     const float* uniforms_dev, uint64_t philox_seed, uint64_t philox_offset,
                     float* wi_dev, int64_t n, void* stream);

/* Scene bounds (krr AABB, aabb.h:11-33): positions are normalised by
 * normalizeSpatialCoord (train.h:272-276) against this box inflated by
 * 0.005 x its diagonal length. */
typedef struct gdf_aabb {
  float lo[3];
  float hi[3];
} gdf_aabb;

/* Raw shading points of a wavefront (the ShadingData fields that
 * generate_inference_data_AR, train.cu:334-362, reads). Device arrays. */
typedef struct gdf_shading {
  const float* pos;       /* [n x 3] world-space position (sd.pos)        */
  const float* wo;        /* [n x 3] outgoing direction (sd.wo, any length) */
  const float* normal;    /* [n x 3] shading normal (sd.frame.N)          */
  const float* roughness; /* [n]     (sd.roughness)                        */
} gdf_shading;

/* gdf_infer with the optional stages either side of it:
 *   - shading != NULL: the queries are built in-kernel from raw shading
 *     points and `aabb` (generate_inference_data_AR, train.cu:334-362), so
 *     the 9-float rows never reach memory; queries_dev is then ignored;
 *   - dir_pdf_dev != NULL: also writes, per query, the consumer view of
 *     the result (AutoRegressive, AR.h:25-48): the unit direction
 *     squareToUniformSphere(u_theta, u_phi) (math_utils.h:226-231) and the
 *     solid-angle pdf |wi[2]| * |wi[3]| / (4 pi), as [x, y, z, pdf];
 *   - cdf_norm_err_dev != NULL: the CDF normalisation check, in FP64: for
 *     every row and both distributions, |1 - sum_i p_i / N| over the N bin
 *     pdfs the sampling uses (summed in double), max-merged into
 *     *cdf_norm_err_dev (8-byte aligned; the caller sets it to 0 first). */
typedef struct gdf_infer_args {
  const float* queries_dev;
  const gdf_shading* shading;
  gdf_aabb aabb;
  const uint8_t* guided_dev;
  const float* uniforms_dev;
  uint64_t philox_seed;
  uint64_t philox_offset;
  float* wi_dev;
  float* dir_pdf_dev;
  int64_t n;
  double* cdf_norm_err_dev;
  /* nullable: two cudaEvent_t that the call records on `stream`, after the
   * grid-feature launch and after the fused launch, so that a caller can
   * time each kernel (no counterpart in the reference) */
  void* const* stage_events;
} gdf_infer_args;
gdf_status gdf_infer_ex(gdf_ctx* ctx, const gdf_infer_args* args, void* stream);

/* gdf_infer on HOST buffers, for callers whose queries live in host memory:
 * the inputs are copied in, inferred and the guiding data copied back in
 * chunks of at most 524,288 queries pipelined over three internal streams
 * (input copies, kernels, output copies), so the transfers overlap the
 * kernels. Results are identical to gdf_infer on the
 * same data (the in-kernel Philox counter continues across chunks).
 *   queries_h [n x 9], guided_h [n] (nullable), uniforms_h [n x 4]
 *   (nullable), wi_in_h / wi_out_h [n x 4] (may alias); page-locked host
 *   memory lets the copies run asynchronously.
 * Ordered after prior work on `stream`; work on `stream` issued afterwards
 * runs after it. The host buffers must stay valid until then. */
gdf_status gdf_infer_host(gdf_ctx* ctx, const float* queries_h, const uint8_t* guided_h,
                          const float* uniforms_h, uint64_t philox_seed, uint64_t philox_offset,
                          const float* wi_in_h, float* wi_out_h, int64_t n, void* stream);

/* compute_AR_pdf_combined_F (train.h:730-751) for given square directions:
 * pdf_out_dev[i] = {pdf_theta(u[i].x), pdf_phi(u[i].y)} of the learned
 * distribution at query i (the phi net is conditioned on u[i].x). */
gdf_status gdf_eval_pdf(gdf_ctx* ctx, const float* queries_dev, const float* u_dev,
                        float* pdf_out_dev, int64_t n, void* stream);

/* The DF epilogue alone on given logits, i.e. thetaPostInference +
 * phiPostInference (train.h:896-929) without the networks: softmax x N,
 * inversion sampling of guided rows and pdf evaluation into wi. logits are
 * [n x n_bins] fp32 row-major per net. */
gdf_status gdf_post_inference(gdf_ctx* ctx, const float* logits_theta_dev,
                              const float* logits_phi_dev, const uint8_t* guided_dev,
                              const float* uniforms_dev, float* wi_dev, int64_t n,
                              void* stream);

/* LearnedDistribution::mouseOverInference (learnedDistribution.cpp:486-583)
 * for one query row query_h[9] (host): the solid-angle pdf
 * pdf_theta * pdf_phi / (4 pi) of the learned distribution at the centre of
 * every pixel of a width x height image over the square of directions
 * (pixel (x, y) at u = (x + 1/2) / width, v = (y + 1/2) / height,
 * integrator.cpp:721-731), row-major into image_dev. At most 2^26 pixels. */
gdf_status gdf_pdf_image(gdf_ctx* ctx, const float* query_h, int32_t width, int32_t height,
                         float* image_dev, void* stream);

/* LearnedDistribution::mouseOverSampling (learnedDistribution.cpp:585-654)
 * with the integrator's binning (integrator.cpp:782-827): n_samples
 * directions drawn from the learned distribution of query_h[9] (every draw
 * guided, Philox uniforms keyed by seed, counter = sample index), counted
 * into counts_dev[height][width] by pixel ((int)(u width), (int)(v height));
 * counts are zeroed first. dirs_dev [n_samples x 2] (nullable) receives the
 * samples. */
gdf_status gdf_sample_histogram(gdf_ctx* ctx, const float* query_h, int64_t n_samples, uint64_t seed,
                                int32_t width, int32_t height, uint32_t* counts_dev, float* dirs_dev,
                                void* stream);

/* --------------------------------------------------------------- training */

/* One iteration of LearnedDistribution::trainStep (learnedDistribution.cpp:
 * 230-289) on a batch of n records: theta/phi forward with fp16 pdfs
 * (softmaxMultFactor), divergence loss and dL/dlogits
 * (combine_AR_pdf_and_dl_doutput, train.h:932-965), backward through both
 * MLPs and grids, Adam + EMA (optimizers/adam.h:48, ema.h:102).
 *   in_theta_dev [n x 9]  GuidedInput
 *   in_phi_dev   [n x 10] GuidedInputPhi (slot 9 = theta condition)
 *   target_dev   [n x 9]  GuidedOutput: dir[2], L[3], wiPdf, bsdfVal[3]
 * stats_host (nullable) receives the loss; filling it synchronises. */
gdf_status gdf_train_step(gdf_ctx* ctx, const float* in_theta_dev, const float* in_phi_dev,
                          const float* target_dev, int64_t n, gdf_train_stats* stats_host,
                          void* stream);

/* Optimizer state of one network (Adam first/second moments, per-parameter
 * step counters, optimizer step) for exact resume. The reference saves only
 * the fp32 weights (learnedDistribution.cpp:295-384); tcnn keeps these in
 * AdamOptimizer (optimizers/adam.h:250-290). Any output pointer may be NULL.
 * Synchronises. */
gdf_status gdf_get_optimizer_state(const gdf_ctx* ctx, int32_t net, float* m_host, float* v_host,
                                   uint32_t* steps_host, int64_t n, uint32_t* opt_step);
gdf_status gdf_set_optimizer_state(gdf_ctx* ctx, int32_t net, const float* m_host,
                                   const float* v_host, const uint32_t* steps_host, int64_t n,
                                   uint32_t opt_step);

/* Mean divergence loss of a batch, like the loss gdf_train_step reports
 * (same forward kernel, same FP64 reduction), without updating anything
 * and without allocating: every intermediate lives in a fixed array that is
 * part of the library image, for callers that cannot allocate device memory
 * while they run (a renderer with a fixed arena, a host that forbids
 * cudaMalloc after start-up). No counterpart in the reference.
 *   - n <= 65536 records (the array's capacity, 1 MiB + 256 B held on every
 *     GPU that loads the library until exit); larger n -> GDF_ERR_INVALID_ARG;
 *   - loss_out_dev: one double (mean loss), dropped_out_dev: one int64
 *     (records rejected by the validity filter), both device pointers;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) and keeps it for the life of the process; make
 *     that first call before any stream capture, and do not reset the
 *     device (cudaDeviceReset) while the library is loaded;
 *   - the current device must be the context's (else GDF_ERR_INVALID_ARG);
 *   - not for the BF16 precision form (GDF_ERR_UNSUPPORTED);
 *   - all calls share the one array: calls whose work overlaps on the GPU
 *     (other streams, other threads) race; order them on one stream. */
gdf_status gdf_train_loss_static(gdf_ctx* ctx, const float* in_theta_dev, const float* in_phi_dev,
                                 const float* target_dev, int64_t n, double* loss_out_dev,
                                 int64_t* dropped_out_dev, void* stream);

/* ------------------------------------------------------------ grouped */

/* One job of a grouped inference: a context (its own networks) and one
 * wavefront of queries, with the arguments of gdf_infer. */
typedef struct gdf_job {
  gdf_ctx* ctx;
  const float* queries_dev;   /* [n x 9]                                  */
  const uint8_t* guided_dev;  /* [n] or NULL                              */
  const float* uniforms_dev;  /* [n x 4] or NULL (Philox: seed, offset)    */
  uint64_t philox_seed;
  uint64_t philox_offset;
  float* wi_dev;              /* [n x 4] in/out                           */
  int64_t n;
} gdf_job;

typedef struct gdf_group gdf_group;

/* A grouped inference engine for up to max_jobs jobs per call, on the
 * current device. No counterpart in the reference, which guides one render
 * job (LearnedDistribution::inferenceStep, learnedDistribution.cpp:167-206);
 * a grouped call gives every job exactly what gdf_infer gives it. */
gdf_status gdf_group_create(int32_t max_jobs, gdf_group** out);
gdf_status gdf_group_destroy(gdf_group* g);

/* Inference of all jobs in one grid-feature launch and one persistent fused
 * launch, replayed from a CUDA graph built on first use of a configuration
 * (the job table is read from device memory, so later calls with other jobs
 * reuse it). Jobs must share the grid configuration, pdf interpolation and
 * precision; bin counts may differ. The first call for a new job-set
 * signature (grid shape, job count, log2 of the tile count) times the
 * candidate launch shapes (2 or 4 warpgroups per CTA x 128- or 256-thread
 * feature blocks) on scratch copies of the guiding data and keeps the
 * fastest; that call synchronises `stream`. Calls on one group are ordered
 * (one feature buffer); a call that needs a larger buffer waits for the
 * group's previous call to finish (only that; other streams run on). Jobs
 * must not share wi buffers. */
gdf_status gdf_group_infer(gdf_group* g, const gdf_job* jobs, int32_t n_jobs, void* stream);

/* The launch shape chosen for the last call and the candidates' times (ms)
 * of the last tuning, in the order (4,256), (4,128), (2,256), (2,128). */
gdf_status gdf_group_tuning(const gdf_group* g, int32_t* warpgroups, int32_t* feature_block,
                            float* tuned_ms);

/* Fixes the launch shape (warpgroups 2 or 4, feature block 128 or 256)
 * and skips tuning; warpgroups = 0 returns to tuning. */
gdf_status gdf_group_set_shape(gdf_group* g, int32_t warpgroups, int32_t feature_block);

/* Turns per-job completion reports on (1) or off (0, the default) for the
 * group's later calls: each warp of the fused kernel then counts its rows
 * with an atomic after a memory fence (about 4 % of a launch's time). No
 * counterpart in the reference. */
gdf_status gdf_group_track_jobs(gdf_group* g, int32_t on);

/* With tracking on: 1 once job `job` of the group's last gdf_group_infer
 * call has all its guiding data written (visible to the host and to later
 * work on any stream), 0 while it has not, or for a job index outside that
 * call; always 0 with tracking off. Jobs
 * early in the table finish first, so small jobs listed first come back before the
 * launch ends; polls host memory, never synchronises. No counterpart in
 * the reference. */
int32_t gdf_group_job_done(const gdf_group* g, int32_t job);

/* Caps the CTAs of the group's persistent fused launches at `ctas` (0: one
 * per SM, the default), so that later calls leave the other SMs to work on
 * other streams; results do not depend on the cap. */
gdf_status gdf_group_set_sm_cap(gdf_group* g, int32_t ctas);

/* gdf_sync_status for the group's kernels. */
gdf_status gdf_group_sync_status(gdf_group* g, void* stream);

/* ------------------------------------------------------------- serving */

/* Device memory held by a context: networks, optimizer state, workspaces. */
gdf_status gdf_ctx_bytes(const gdf_ctx* ctx, int64_t* bytes);

typedef enum gdf_request_kind { GDF_REQ_INFER = 0, GDF_REQ_TRAIN = 1 } gdf_request_kind;

/* One request to a server: gdf_infer (queries_dev, guided_dev,
 * uniforms_dev, philox_*, wi_dev) or gdf_train_step (in_theta_dev,
 * in_phi_dev, target_dev) on one registered instance. The buffers stay
 * owned by the caller and must stay valid until gdf_server_wait returns. */
typedef struct gdf_request {
  int32_t kind;               /* gdf_request_kind */
  gdf_ctx* instance;
  int64_t n;
  const float* queries_dev;
  const uint8_t* guided_dev;
  const float* uniforms_dev;
  uint64_t philox_seed;
  uint64_t philox_offset;
  float* wi_dev;
  const float* in_theta_dev;
  const float* in_phi_dev;
  const float* target_dev;
} gdf_request;

typedef struct gdf_server_config {
  int32_t device;
  int32_t slots;              /* concurrent device streams (1..64)            */
  int32_t max_batch;          /* inference requests per grouped launch        */
  int32_t max_train_slots;    /* slots training may hold at once (0: slots-1) */
  int64_t hbm_budget_bytes;   /* resident instances + in-flight requests      */
  int32_t train_sm_reserve;   /* SMs training's persistent kernels leave free,
                                 and the CTAs inference launches get while
                                 training runs (0: none reserved)            */
} gdf_server_config;

typedef struct gdf_server_stats {
  int64_t requests, queries, pending, resident_bytes;
  double p50_ms, p99_ms, max_ms;   /* submit -> completion latency            */
  double queries_per_s;            /* completed queries / first submit..last completion */
} gdf_server_stats;

typedef struct gdf_server gdf_server;

/* A request server over resident instances (no counterpart in the
 * reference, which guides one job per process). A scheduler thread admits
 * requests in arrival order as stream slots and budget allow -- per
 * instance, a training request runs after every earlier request and
 * before every later one, while the inference requests between two
 * training requests may run together (they only read the networks; give
 * them distinct output buffers) -- batches all
 * inference requests admitted together into one grouped launch
 * (gdf_group_infer) and runs training requests on streams of their own, so
 * their work overlaps on the device. Instances must share the grid
 * configuration, pdf interpolation and precision, and must not be used
 * directly while registered. */
gdf_status gdf_server_create(const gdf_server_config* cfg, gdf_server** out);
gdf_status gdf_server_destroy(gdf_server* s);
/* Registers a context; its gdf_ctx_bytes count against the budget. */
gdf_status gdf_server_add_instance(gdf_server* s, gdf_ctx* ctx);
gdf_status gdf_server_submit(gdf_server* s, const gdf_request* r, uint64_t* ticket);
/* Blocks until the request completed; training requests fill stats. */
gdf_status gdf_server_wait(gdf_server* s, uint64_t ticket, gdf_train_stats* stats, double* latency_ms);
/* Latency percentiles and throughput of the requests completed since the
 * last reset. */
gdf_status gdf_server_get_stats(gdf_server* s, gdf_server_stats* out, int32_t reset);

/* -------------------------------------------------------------------- NRC */

/* NRC::inferenceStep (nrc.cpp:172-181): in [m x 15] fp32 (GuidedInputNRC,
 * guideditem.h:89-93) -> out [m x 3] fp32 RGB radiance, EMA weights. */
gdf_status gdf_nrc_query(gdf_ctx* ctx, const float* in_dev, float* out_dev, int64_t m,
                         void* stream);

/* One iteration of NRC::trainStep (nrc.cpp:132-167) on m records with
 * RelativeL2Luminance loss (losses/relative_l2_luminance.h:40-86) and
 * Adam + EMA. target [m x 3] fp32. */
gdf_status gdf_nrc_train_step(gdf_ctx* ctx, const float* in_dev, const float* target_dev,
                              int64_t m, gdf_train_stats* stats_host, void* stream);

/* ------------------------------------------- records from the path tracer */

/* One depth of GuidedPixelStateBuffer (workqueue.h:16-145): the
 * RadianceRecordItem fields (guideditem.h:23-44) as device arrays indexed
 * by pixel id. Angles are (theta, phi) in radians as the reference stores
 * them. L is read and written (NRC target substitution); the rest is read. */
typedef struct gdf_record_fields {
  float* L;                 /* [n x 3] accumulated radiance               */
  const float* thp;         /* [n x 3] throughput                          */
  const float* Le;          /* [n x 3] emission at the vertex              */
  const float* pos;         /* [n x 3] world-space vertex position         */
  const float* dir;         /* [n x 2] scattered direction wi              */
  const float* wi_pdf;      /* [n]     pdf of wi                            */
  const float* mis_weight;  /* [n]                                          */
  const uint8_t* delta;     /* [n]     sampled from a delta lobe           */
  const uint8_t* miss;      /* [n]     NRC alignment record of a miss      */
  const float* bsdf_val;    /* [n x 3]                                      */
  const float* wo;          /* [n x 2] outgoing direction                  */
  const float* normal;      /* [n x 2] shading normal                      */
  const float* roughness;   /* [n]                                          */
  const float* diffuse;     /* [n x 3]                                      */
  const float* specular;    /* [n x 3]                                      */
} gdf_record_fields;

typedef struct gdf_path_state {
  gdf_record_fields depth[GDF_MAX_TRAIN_DEPTH];
  uint32_t* cur_depth;      /* [n] curDepth; NRC record building decrements it */
} gdf_path_state;

/* The training pixels of a frame: pixel = offset + i * stride for
 * i < max_queue_size / stride (learnedDistribution.cpp:218-222). */
typedef struct gdf_train_pixels {
  int64_t max_queue_size;
  uint32_t offset;  /* trainPixelOffset */
  uint32_t stride;  /* trainPixelStride, >= 1 */
} gdf_train_pixels;

/* generate_inference_data_AR (train.cu:334-362) alone: shading points ->
 * the 9-float query rows described at the top of this file. */
gdf_status gdf_prepare_queries(const gdf_shading* shading, const gdf_aabb* aabb,
                               float* queries_dev, int64_t n, void* stream);

/* generate_training_data_AR (train.cu:6-96): one GuidedInput,
 * GuidedInputPhi and GuidedOutput per non-delta, finite vertex of each
 * training pixel. Records are ordered by training pixel, then depth (the
 * reference appends them atomically in no fixed order). At most `capacity`
 * records are written; *count_host receives the full count and
 * GDF_ERR_INVALID_ARG is returned when it exceeds capacity. Synchronises. */
gdf_status gdf_build_train_records(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                                   const gdf_train_pixels* px, float* in_theta_dev,
                                   float* in_phi_dev, float* target_dev, int64_t capacity,
                                   int64_t* count_host, void* stream);

/* NRC record building, ordered like gdf_build_train_records:
 *   with_training = 1: generate_training_data_nrc_with_inference
 *     (train.cu:156-214): query rows for every non-delta, non-miss vertex and
 *     training rows (GuidedInputNRC + RGB target) for all but the last;
 *   with_training = 0: generate_NRCinput_from_training_data
 *     (train.cu:216-262): query rows only.
 * Both decrement cur_depth of every training pixel, like the reference.
 * query_depth/query_pixel receive each query row's depth and pixel id.
 * counts_host[0] = query rows, counts_host[1] = training rows. Synchronises. */
gdf_status gdf_build_nrc_records(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                                 const gdf_train_pixels* px, int32_t with_training,
                                 float* query_in_dev, int32_t* query_depth_dev,
                                 int32_t* query_pixel_dev, int64_t query_capacity,
                                 float* train_in_dev, float* train_target_dev,
                                 int64_t train_capacity, int64_t* counts_host, void* stream);

/* apply_NRCoutput_to_training_data + divide_training_data_by_NRCoutput
 * (train.cu:265-308) for OPTIMIZE_ON_NRC 4 (parameters.h:19): for every
 * query row (depth d, pixel p, NRC output o), first
 *   replaceIndirectRadianceSkipDelta(p, d-1, o)   (workqueue.h:122-129)
 * for all rows, then divideRadiance(p, d, o) (workqueue.h:104-111). Rows
 * may come in any order. */
gdf_status gdf_apply_nrc(gdf_ctx* ctx, gdf_path_state* state, const float* nrc_out_dev,
                         const int32_t* query_depth_dev, const int32_t* query_pixel_dev,
                         int64_t m, void* stream);

/* NRC::trainStep (nrc.cpp:114-170): builds the NRC query and training rows
 * into library buffers (with_training = 1 above, cur_depth decremented),
 * then runs its batch loop of gdf_nrc_train_step. *loss_host = the mean of
 * the batch losses over the loop's batch count; *n_samples_host = training
 * rows. The query rows are kept for gdf_nrc_substitute_paths. Synchronises. */
gdf_status gdf_nrc_train_paths(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                               const gdf_train_pixels* px, float* loss_host,
                               int64_t* n_samples_host, void* stream);

/* NRC::inferenceStepFromTrainingData (nrc.cpp:183-217): builds the query
 * rows unless skip_generation (then the rows of the last
 * gdf_nrc_train_paths are used), queries the NRC and substitutes the
 * targets in state (gdf_apply_nrc). Synchronises. */
gdf_status gdf_nrc_substitute_paths(gdf_ctx* ctx, gdf_path_state* state, const gdf_aabb* aabb,
                                    const gdf_train_pixels* px, int32_t skip_generation,
                                    void* stream);

/* LearnedDistribution::trainStep (learnedDistribution.cpp:208-293): builds
 * the records (gdf_build_train_records) into library buffers and runs the
 * batch loop of gdf_train_step. *loss_host = sum of batch losses / batch
 * count; *n_samples_host = records built. Synchronises once, at the end, to
 * read the two results (gdf_train_paths_async without the read-back). */
gdf_status gdf_train_paths(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                           const gdf_train_pixels* px, float* loss_host, int64_t* n_samples_host,
                           void* stream);

/* gdf_train_paths, stream-ordered: the record count stays on the device,
 * every batch the loop can reach (df_batches_per_frame) is launched with
 * its size read on the device, and a batch past the count, or below
 * min_train_batch, trains nothing (no optimizer step). No host
 * synchronisation and no allocation once the buffers for this pixel count
 * exist (a first call allocates them), so the call can be captured in a
 * CUDA graph. loss_dev (float) and n_samples_dev (int64), device pointers,
 * receive the two results; either may be null. The reference reads the
 * count back (learnedDistribution.cpp:225-226); this entry point has no
 * counterpart there. */
gdf_status gdf_train_paths_async(gdf_ctx* ctx, const gdf_path_state* state, const gdf_aabb* aabb,
                                 const gdf_train_pixels* px, float* loss_dev, int64_t* n_samples_dev,
                                 void* stream);

/* ----------------------------------------------------------------- errors */

/* Synchronises `stream` and reports device-side failures of the kernels
 * launched on it: GDF_ERR_TIMEOUT when a bounded device wait gave up (the
 * error word is then cleared), GDF_ERR_CUDA for an asynchronous CUDA error.
 * The reference has no counterpart (it aborts on CUDA errors,
 * src/lib/src/core/device/cuda.h:58-60). */
gdf_status gdf_sync_status(gdf_ctx* ctx, void* stream);

const char* gdf_last_error(void);
const char* gdf_status_string(gdf_status s);

#ifdef __cplusplus
}
#endif

#endif  /* GDF_H_ */
