// Stand-in for the generated render/guided/guideditem_soa.h: structure-of-
// arrays views of the guided records (included inside namespace krr).
// Indexing a record array gathers one RadianceRecordItem, as the generated
// SOA accessor does; a field left null reads as zero.
template <> struct SOA<RadianceRecordItem> {
  Color* L = nullptr; Color* thp = nullptr; Color* Le = nullptr; Vector3f* pos = nullptr;
  Vector2f* dir = nullptr; float* wiPdf = nullptr; float* bsdfPdf = nullptr; float* misWeight = nullptr;
  bool* delta = nullptr; bool* miss = nullptr; bool* isTwoSided = nullptr; Color* bsdfVal = nullptr;
  Vector2f* wo = nullptr; Vector2f* normal = nullptr; float* roughness = nullptr;
  Vector3f* diffuse = nullptr; Vector3f* specular = nullptr;
  KRR_STUB_HD RadianceRecordItem operator[](int i) const {
    RadianceRecordItem r{};
#define KRR_STUB_GET(f) if (f) r.f = f[i]
    KRR_STUB_GET(L); KRR_STUB_GET(thp); KRR_STUB_GET(Le); KRR_STUB_GET(pos); KRR_STUB_GET(dir);
    KRR_STUB_GET(wiPdf); KRR_STUB_GET(bsdfPdf); KRR_STUB_GET(misWeight); KRR_STUB_GET(delta);
    KRR_STUB_GET(miss); KRR_STUB_GET(isTwoSided); KRR_STUB_GET(bsdfVal); KRR_STUB_GET(wo);
    KRR_STUB_GET(normal); KRR_STUB_GET(roughness); KRR_STUB_GET(diffuse); KRR_STUB_GET(specular);
#undef KRR_STUB_GET
    return r;
  }
};
template <> struct SOA<GuidedPixelState> {
  SOA() = default;
  SOA(int, Allocator) {}
  SOA<RadianceRecordItem> records[MAX_TRAIN_DEPTH];
  uint* curDepth = nullptr;
};
