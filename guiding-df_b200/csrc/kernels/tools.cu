// tools.cu -- batch workloads that inspect one learned distribution: its pdf
// image over the square of directions and a histogram of samples drawn from
// it (LearnedDistribution::mouseOverInference and mouseOverSampling,
// src/render/guided/learnedDistribution.cpp:386-656, and the integrator's
// binning of the samples, integrator.cpp:720-735 and 782-830). The networks
// run through the regular kernels; these kernels only lay out the inputs
// and reduce the outputs.
#include <cuda_runtime.h>

#include "../device/records.cuh"
#include "tools_kernels.h"

namespace gdf {
namespace {

// Query row i = q; for images also the pixel centre of pixel i
// (x, y) = (i % W, i / W): u = x / W + 0.5 / W, v = y / H + 0.5 / H
// (integrator.cpp:724-730).
__global__ void replicate_kernel(const QueryRow q, float* __restrict__ rows, float* __restrict__ uv,
                                 float* __restrict__ wi, int32_t width, int32_t height, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int k = 0; k < 9; ++k) rows[i * 9 + k] = q.v[k];
  if (uv) {
    const int x = static_cast<int>(i % width), y = static_cast<int>(i / width);
    float u = static_cast<float>(x) / static_cast<float>(width);
    float v = static_cast<float>(y) / static_cast<float>(height);
    u += 0.5f / static_cast<float>(width);
    v += 0.5f / static_cast<float>(height);
    uv[i * 2] = u;
    uv[i * 2 + 1] = v;
  }
  if (wi) *reinterpret_cast<float4*>(wi + i * 4) = make_float4(0.f, 0.f, 1.f, 1.f);
}

// image = pdf_theta * pdf_phi * squareToUniformSpherePdf (learnedDistribution.cpp:472-480)
__global__ void pdf_image_kernel(const float* __restrict__ pdf2, float* __restrict__ image, int64_t n) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  image[i] = pdf2[i * 2] * pdf2[i * 2 + 1] * rec::kInv4Pi;
}

// pixel (int)(u W), (int)(v H); samples outside the image are skipped
// (integrator.cpp:815-827)
__global__ void histogram_kernel(const float* __restrict__ wi, int64_t n, int32_t width, int32_t height,
                                 uint32_t* __restrict__ counts, float* __restrict__ dirs) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float u = wi[i * 4], v = wi[i * 4 + 1];
  if (dirs) {
    dirs[i * 2] = u;
    dirs[i * 2 + 1] = v;
  }
  const int x = static_cast<int>(u * static_cast<float>(width));
  const int y = static_cast<int>(v * static_cast<float>(height));
  if (x >= width || y >= height || x < 0 || y < 0) return;
  atomicAdd(counts + static_cast<int64_t>(y) * width + x, 1u);
}

inline unsigned blocks(int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

}  // namespace

cudaError_t launch_replicate(const QueryRow& q, float* rows, float* uv, float* wi, int32_t width,
                             int32_t height, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  replicate_kernel<<<blocks(n), 256, 0, st>>>(q, rows, uv, wi, width, height, n);
  return cudaGetLastError();
}

cudaError_t launch_pdf_image(const float* pdf2, float* image, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  pdf_image_kernel<<<blocks(n), 256, 0, st>>>(pdf2, image, n);
  return cudaGetLastError();
}

cudaError_t launch_histogram(const float* wi, int64_t n, int32_t width, int32_t height, uint32_t* counts,
                             float* dirs, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  histogram_kernel<<<blocks(n), 256, 0, st>>>(wi, n, width, height, counts, dirs);
  return cudaGetLastError();
}

}  // namespace gdf
