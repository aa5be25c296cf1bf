// Stand-in for the krr math utilities the DF functions call: spherical
// coordinates and the square <-> uniform-sphere maps (the formulas of the
// reference's src/lib/src/util/math_utils.h:183-243). Host and device.
#pragma once
#include "../common.h"
namespace krr {
namespace utils {
KRR_CALLABLE Vector2f cartesianToSpherical(const Vector3f& v) {
  const Vector3f n = v.normalized();
  Vector2f s(acosf(fminf(1.f, fmaxf(-1.f, n[2]))), atan2f(n[1], n[0]));
  if (s[1] < 0) s[1] += M_2PI;
  return s;
}
KRR_CALLABLE Vector2f cartesianToSphericalNormalized(const Vector3f& v) {
  const Vector2f s = cartesianToSpherical(v);
  return Vector2f(float(s[0] / M_PI), float(s[1] / M_2PI));
}
KRR_CALLABLE Vector3f sphericalToCartesian(float t, float p) {
  return Vector3f(sinf(t) * cosf(p), sinf(t) * sinf(p), cosf(t));
}
KRR_CALLABLE Vector3f squareToUniformSphere(Vector2f u) {
  const float z = 1 - 2 * u[0];
  const float r = sqrtf(fmaxf(0.f, 1 - z * z));
  const float phi = M_2PI * u[1];
  return Vector3f(r * cosf(phi), r * sinf(phi), z);
}
KRR_CALLABLE Vector2f uniformSphereToSquare(Vector3f v) {
  const Vector3f n = v.normalized();
  float phi = atan2f(n[1], n[0]) * M_INV_2PI;
  return Vector2f((1.f - n[2]) * 0.5f, phi < 0.f ? phi + 1.f : phi);
}
KRR_CALLABLE float squareToUniformSpherePdf() { return M_INV_4PI; }
}  // namespace utils
using utils::cartesianToSpherical;
using utils::sphericalToCartesian;
}  // namespace krr
