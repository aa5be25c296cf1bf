// Stand-in for render/wavefront/workqueue.h: a fixed-size work queue, the
// structure-of-arrays template and the pixel-state buffer. Indexing a queue
// yields a proxy that converts to the work item, as the reference's SOA
// queues do (train.cu:341 names the conversion operator explicitly).
#pragma once
#include "../../common.h"
#include "workitem.h"
namespace krr {
template <typename T> struct WorkItemRef {
  const T* p;
  KRR_STUB_HD operator T() const { return *p; }
};
template <typename T> class WorkQueue {
 public:
  WorkQueue() = default;
  WorkQueue(int n, Allocator) : cap_(n) {}
  KRR_STUB_HD int push(const T& w) { items_[size_] = w; return size_++; }
  KRR_STUB_HD int size() const { return size_; }
  KRR_STUB_HD WorkItemRef<T> operator[](int i) const { return WorkItemRef<T>{items_ + i}; }
  T* items_ = nullptr;
  int size_ = 0, cap_ = 0;
};
using ScatterRayQueue = WorkQueue<ScatterRayWorkItem>;
struct PixelStateBuffer { PCGSampler* sampler = nullptr; };
}  // namespace krr
