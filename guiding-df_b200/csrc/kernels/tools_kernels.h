// tools_kernels.h -- host-side declarations of the distribution-inspection kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gdf {

struct QueryRow {
  float v[9];
};

// rows[i] = q; uv[i] = centre of pixel i of a width x height image
// (nullable); wi[i] = (0, 0, +1, +1) (nullable).
cudaError_t launch_replicate(const QueryRow& q, float* rows, float* uv, float* wi, int32_t width,
                             int32_t height, int64_t n, cudaStream_t st);
// image[i] = pdf2[i].x * pdf2[i].y / (4 pi)
cudaError_t launch_pdf_image(const float* pdf2, float* image, int64_t n, cudaStream_t st);
// counts[pixel of (wi[i].x, wi[i].y)] += 1; dirs[i] = (wi[i].x, wi[i].y) (nullable)
cudaError_t launch_histogram(const float* wi, int64_t n, int32_t width, int32_t height, uint32_t* counts,
                             float* dirs, cudaStream_t st);

}  // namespace gdf
