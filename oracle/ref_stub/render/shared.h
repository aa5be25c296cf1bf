// Stand-in for render/shared.h: shading data, BSDF sample records and the
// per-pixel sampler.
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
  KRR_STUB_HD bool isTwoSided() const { return true; }
  KRR_STUB_HD unsigned getBsdfType() const { return BSDF_SMOOTH; }
};
struct BSDFSample { Vector3f wi; float pdf = 0.f; };
struct PCGSampler {
  // The reference's PCG sampler returns its next uniform (sampler.h:77-86);
  // here each pixel's sampler walks a scripted sequence of uniforms, so both
  // sides of a comparison consume identical random numbers.
  const float* seq = nullptr;
  int pos = 0;
  KRR_STUB_HD float get1D() { return seq[pos++]; }
};
class Sampler {
 public:
  KRR_STUB_HD Sampler(PCGSampler* s) : s_(s) {}
  KRR_STUB_HD float get1D() { return s_->get1D(); }
 private:
  PCGSampler* s_;
};
}  // namespace krr
