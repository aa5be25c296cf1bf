// Stand-in for the generated render/guided/guideditem_soa.h: structure-of-
// arrays views of the guided records (included inside namespace krr).
template <> struct SOA<RadianceRecordItem> {
  Color* L = nullptr; Color* thp = nullptr; Color* Le = nullptr; Vector3f* pos = nullptr;
  Vector2f* dir = nullptr; float* wiPdf = nullptr; float* bsdfPdf = nullptr; float* misWeight = nullptr;
  bool* delta = nullptr; bool* miss = nullptr; bool* isTwoSided = nullptr; Color* bsdfVal = nullptr;
  Vector2f* wo = nullptr; Vector2f* normal = nullptr; float* roughness = nullptr;
  Vector3f* diffuse = nullptr; Vector3f* specular = nullptr;
};
template <> struct SOA<GuidedPixelState> {
  SOA() = default;
  SOA(int, Allocator) {}
  SOA<RadianceRecordItem> records[MAX_TRAIN_DEPTH];
  uint* curDepth = nullptr;
};
