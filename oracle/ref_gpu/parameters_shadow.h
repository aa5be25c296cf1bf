// parameters_shadow.h -- compile-time configuration of the reference guided
// path, for the reference GPU harness (TEST INFRASTRUCTURE ONLY).
//
// The reference fixes its bin counts in src/render/guided/parameters.h:41-48
// (theta 16, phi 2 x 16) and its wavefront capacity at :51 (1280 x 720).
// The harness compiles the unmodified train.h / AR.h / train.cu once per
// bin configuration; oracle/build_ref_gpu.py exposes this header to them
// under the name parameters.h (through a directory of symbolic links to the
// reference files), so every name the reference's header declares is
// declared here with the reference's value, except:
//   N_DIM_OUTPUT      = GDF_REF_BINS_THETA  (reference: 16)
//   N_DIM_OUTPUT_PHI  = GDF_REF_BINS_PHI    (reference: 2 * N_DIM_OUTPUT)
//   MAX_RESOLUTION    = 1920 * 1080         (reference: 1280 * 720; the
//                                            1080p wavefront needs more)
#pragma once
#include "common.h"

#ifndef GDF_REF_BINS_THETA
#error "GDF_REF_BINS_THETA must be defined"
#endif
#ifndef GDF_REF_BINS_PHI
#error "GDF_REF_BINS_PHI must be defined"
#endif

template <uint32_t dim, uint32_t multiple> struct padded_dim_compiletime {
  static const uint32_t value = (dim + multiple - 1) / multiple * multiple;
};

#define GUIDED_AUXILIARY_INPUT 1
#define GUIDED_PRODUCT_SAMPLING 1
#define OPTIMIZE_ON_NRC 4
#define AR_LINEAR_INTERPOLATION 1
#define RENDER_NOISY_ONLY 0

constexpr unsigned int MAX_TRAIN_DEPTH = 5;
constexpr unsigned int NETWORK_ALIGNMENT = 16;
constexpr unsigned int N_DIM_SPATIAL_INPUT = 3;
constexpr unsigned int N_DIM_DIRECTIONAL_INPUT = GUIDED_PRODUCT_SAMPLING ? 3 : 0;
constexpr unsigned int N_DIM_AUXILIARY_INPUT = 3;
constexpr unsigned int N_WI_PER_PIXEL = 1;
constexpr unsigned int N_DIM_INPUT = N_DIM_DIRECTIONAL_INPUT + N_DIM_SPATIAL_INPUT + N_DIM_AUXILIARY_INPUT;

constexpr unsigned int N_DIM_OUTPUT = GDF_REF_BINS_THETA;
constexpr unsigned int N_DIM_PADDED_OUTPUT = padded_dim_compiletime<N_DIM_OUTPUT, 16>::value;
constexpr unsigned int N_DIM_WI = 4;
constexpr float TRAIN_LOSS_SCALE = 1024.f;

constexpr unsigned int N_DIM_INPUT_PHI = 1 + N_DIM_INPUT;
constexpr unsigned int N_DIM_OUTPUT_PHI = GDF_REF_BINS_PHI;
constexpr unsigned int N_DIM_PADDED_OUTPUT_PHI = padded_dim_compiletime<N_DIM_OUTPUT_PHI, 16>::value;

constexpr unsigned int MAX_RESOLUTION = 1920 * 1080;
constexpr int TRAIN_BUFFER_SIZE = MAX_TRAIN_DEPTH * MAX_RESOLUTION;
constexpr size_t TRAIN_BATCH_SIZE = 65'536 * 8;
constexpr size_t MIN_TRAIN_BATCH_SIZE = 65'536;
constexpr int MAX_INFERENCE_NUM = MAX_RESOLUTION;

constexpr unsigned int LOSS_GRAPH_SIZE = 256;
constexpr unsigned int MOUSEOVER_SAMPLING_N_SAMPLERS = 20'000'000;

constexpr unsigned int N_DIM_INPUT_NRC = 15;
constexpr unsigned int N_DIM_OUTPUT_NRC = 3;
constexpr unsigned int N_DIM_PADDED_OUTPUT_NRC = 16;
constexpr float TRAIN_LOSS_SCALE_NRC = 1024.f;
constexpr unsigned int NRC_ITER_COUNT = 4;
constexpr unsigned int TRAIN_BATCH_SIZE_NRC = 1'048'576;

constexpr int N_TRAIN_ITER_NRC = -1;
constexpr int START_TRAIN_ITER_NRC = 0;
