// Stand-in for render/shared.h: shading data and BSDF sample records.
#pragma once
#include "../common.h"
namespace krr {
namespace shader {}
enum BSDFType : unsigned { BSDF_SMOOTH = 1u };
struct Frame { Vector3f N; };
struct ShadingData {
  Vector3f pos, wo;
  Frame frame;
  float roughness = 0.f;
  Vector3f diffuse, specular;
  bool isTwoSided() const { return true; }
  unsigned getBsdfType() const { return BSDF_SMOOTH; }
};
struct BSDFSample { Vector3f wi; float pdf = 0.f; };
struct PCGSampler {
  // the reference's sampler returns its next uniform; here a fixed script
  const float* seq = nullptr;
  int pos = 0;
  float get1D() { return seq[pos++]; }
};
class Sampler {
 public:
  Sampler(PCGSampler* s) : s_(s) {}
  float get1D() { return s_->get1D(); }
 private:
  PCGSampler* s_;
};
}  // namespace krr
