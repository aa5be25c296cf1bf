// Stand-in for tiny-cuda-nn/common.h: the network precision type (fp16).
#pragma once
#include <cuda_fp16.h>
#define TCNN_PRAGMA_UNROLL
namespace tcnn { using network_precision_t = __half; }
