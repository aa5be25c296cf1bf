// records.cuh -- transforms from path-tracer records to network inputs.
//
// Restates, in fp32 with the reference's float constants
// (krrmath/constants.h:10-19):
//   normalizeSpatialCoord        render/guided/train.h:272-276
//   warp_direction_for_sh        render/guided/train.h:1243-1245
//   warp_roughness_for_ob        render/guided/train.h:1247-1249
//   sphericalToCartesian         util/math_utils.h:198-208
//   cartesianToSphericalNormalized util/math_utils.h:183-196
//   squareToUniformSphere / uniformSphereToSquare  util/math_utils.h:226-240
// Transcendentals use CUDA's full-precision sinf/cosf/acosf/atan2f/expf.
#pragma once

#include <cstdint>

#include "../../../include/gdf.h"

namespace gdf {
namespace rec {

constexpr float kPi = 3.14159265358979323846f;
constexpr float k2Pi = 6.28318530717958647693f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kInv2Pi = 0.15915494309189533577f;
constexpr float kInv4Pi = 0.0795774715459476678844f;
constexpr float kEpsilon = 1e-5f;  // M_EPSILON

// Centre and diagonal of the scene box after AABB::inflate by 0.005 x the
// diagonal length (aabb.h:25-28; Eigen AlignedBox center() / diagonal()).
struct SceneFrame {
  float c[3];
  float d[3];
};

__device__ __forceinline__ SceneFrame scene_frame(const gdf_aabb& b) {
  const float d0 = b.hi[0] - b.lo[0], d1 = b.hi[1] - b.lo[1], d2 = b.hi[2] - b.lo[2];
  const float infl = sqrtf((d0 * d0 + d1 * d1) + d2 * d2) * 0.005f;
  SceneFrame f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float lo = b.lo[k] - infl, hi = b.hi[k] + infl;
    f.c[k] = (lo + hi) / 2.0f;
    f.d[k] = hi - lo;
  }
  return f;
}

__device__ __forceinline__ void normalize_spatial(const float p[3], const SceneFrame& f, float o[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = 0.5f + (p[k] - f.c[k]) / f.d[k];
}

__device__ __forceinline__ void warp_direction_for_sh(const float v[3], float o[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = (v[k] + 1.0f) * 0.5f;
}

__device__ __forceinline__ float warp_roughness_for_ob(float r) { return 1.0f - expf(-r); }

__device__ __forceinline__ void spherical_to_cartesian(float theta, float phi, float o[3]) {
  const float st = sinf(theta), ct = cosf(theta), sp = sinf(phi), cp = cosf(phi);
  o[0] = st * cp;
  o[1] = st * sp;
  o[2] = ct;
}

// Eigen normalized(): v / sqrt(|v|^2) when |v|^2 > 0, else v unchanged.
__device__ __forceinline__ void normalized(const float v[3], float o[3]) {
  const float z = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
  if (z > 0.0f) {
    const float s = sqrtf(z);
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = v[k] / s;
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = v[k];
  }
}

__device__ __forceinline__ void cartesian_to_spherical_normalized(const float v[3], float o[2]) {
  float vn[3];
  normalized(v, vn);
  const float z = vn[2] < -1.0f ? -1.0f : (vn[2] > 1.0f ? 1.0f : vn[2]);  // safe_acos
  const float theta = acosf(z);
  float phi = atan2f(vn[1], vn[0]);
  if (phi < 0.0f) phi += k2Pi;
  // cartesianToSphericalNormalized divides theta by M_PI, which the C math
  // header defines as a double before krrmath/constants.h could define its
  // float one, so that quotient is a double rounded to float; M_2PI is
  // krrmath's float constant.
  o[0] = (float)((double)theta / 3.14159265358979323846);
  o[1] = phi / k2Pi;
}

__device__ __forceinline__ void uniform_sphere_to_square(const float v[3], float o[2]) {
  float vn[3];
  normalized(v, vn);
  const float phi = atan2f(vn[1], vn[0]) * kInv2Pi;
  o[0] = (1.0f - vn[2]) * 0.5f;
  o[1] = phi < 0.0f ? phi + 1.0f : phi;
}

__device__ __forceinline__ void square_to_uniform_sphere(float u0, float u1, float o[3]) {
  const float z = 1.0f - 2.0f * u0;
  const float rr = 1.0f - z * z;
  const float r = sqrtf(rr > 0.0f ? rr : 0.0f);  // safe_sqrt
  const float phi = k2Pi * u1;
  o[0] = r * cosf(phi);
  o[1] = r * sinf(phi);
  o[2] = z;
}

// generate_inference_data_AR (train.cu:344-361): one shading point -> the
// 9-float query row.
__device__ __forceinline__ void shading_to_query(const float pos[3], const float wo[3],
                                                 const float nrm[3], float rough,
                                                 const SceneFrame& f, float q[9]) {
  normalize_spatial(pos, f, q);
  float won[3];
  normalized(wo, won);
  warp_direction_for_sh(won, q + 3);
  cartesian_to_spherical_normalized(nrm, q + 6);
  q[8] = warp_roughness_for_ob(rough);
}

__device__ __forceinline__ bool any_nan(const float* v, int n) {
  bool r = false;
  for (int k = 0; k < n; ++k) r |= isnan(v[k]);
  return r;
}

}  // namespace rec
}  // namespace gdf
