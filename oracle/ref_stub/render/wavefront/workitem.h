// Stand-in for render/wavefront/workitem.h: the scatter-ray work items and
// the per-pixel state the DF sampling reads.
#pragma once
#include "../../common.h"
#include "../shared.h"
namespace krr {
template <typename T> struct SOA;
struct ScatterRayWorkItem { ShadingData sd; unsigned pixelId = 0; };
}
