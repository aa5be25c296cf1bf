// Stand-in for raytracing.h: the ray type referenced by the guided records.
#pragma once
#include "common.h"
namespace krr { struct Ray { Vector3f origin, dir; }; }
