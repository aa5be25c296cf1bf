// Stand-in for render/wavefront/workqueue.h: a fixed-size work queue, the
// structure-of-arrays template and the pixel-state buffer.
#pragma once
#include "../../common.h"
#include "workitem.h"
namespace krr {
template <typename T> class WorkQueue {
 public:
  WorkQueue() = default;
  WorkQueue(int n, Allocator) : cap_(n) {}
  int push(const T& w) { items_[size_] = w; return size_++; }
  int size() const { return size_; }
  T& operator[](int i) { return items_[i]; }
  const T& operator[](int i) const { return items_[i]; }
  T* items_ = nullptr;
  int size_ = 0, cap_ = 0;
};
using ScatterRayQueue = WorkQueue<ScatterRayWorkItem>;
struct PixelStateBuffer { PCGSampler* sampler = nullptr; };
}  // namespace krr
