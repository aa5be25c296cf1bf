// Stand-in for the krr framework's common.h: namespace macros, call-site
// qualifiers, and the small vector / colour / box types the guided-path
// headers use.
//
// Two modes. Compiled by g++ (ref_pin.cpp) the device bodies run on the host:
// `__global__` is empty and the thread indices are thread-local globals set
// by the caller. Compiled by nvcc (oracle/ref_gpu/harness.cu) the same types
// are __host__ __device__ and the reference's kernels run on the GPU.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>

#define KRR_NAMESPACE_BEGIN namespace krr {
#define KRR_NAMESPACE_END }

#if defined(__CUDACC__)
#define KRR_STUB_HD __host__ __device__
#define KRR_HOST __host__
#define KRR_DEVICE __device__
#define KRR_HOST_DEVICE __host__ __device__
#define KRR_CALLABLE __host__ __device__ inline
#define KRR_DEVICE_FUNCTION __device__ inline
#define DCHECK_LT(a, b)
#define DCHECK_GT(a, b)
#else
#define KRR_STUB_HD
#define KRR_HOST
#define KRR_DEVICE
#define KRR_HOST_DEVICE
#define KRR_CALLABLE inline
#define KRR_DEVICE_FUNCTION inline
#define DCHECK_LT(a, b) assert((a) < (b))
#define DCHECK_GT(a, b) assert((a) > (b))
#ifndef __global__
#define __global__
#endif
// Thread indices of the host execution of device bodies (set by the caller).
struct krr_stub_idx { unsigned x = 0, y = 0, z = 0; };
extern thread_local krr_stub_idx krr_stub_threadIdx, krr_stub_blockIdx, krr_stub_blockDim;
#define threadIdx krr_stub_threadIdx
#define blockIdx krr_stub_blockIdx
#define blockDim krr_stub_blockDim
#endif
#define CUDA_SYNC_CHECK()
#ifndef TCNN_PRAGMA_UNROLL
#define TCNN_PRAGMA_UNROLL
#endif

namespace krr {
using std::abs;
using std::isnan;
using std::max;
using std::min;
typedef unsigned int uint;

template <int N>
struct VecN {
  float v[N];
  KRR_STUB_HD VecN() { for (int i = 0; i < N; ++i) v[i] = 0.f; }
  KRR_STUB_HD explicit VecN(float a) { for (int i = 0; i < N; ++i) v[i] = a; }
  KRR_STUB_HD float& operator[](int i) { return v[i]; }
  KRR_STUB_HD float operator[](int i) const { return v[i]; }
  KRR_STUB_HD bool hasNaN() const { for (int i = 0; i < N; ++i) if (isnan(v[i])) return true; return false; }
  KRR_STUB_HD float mean() const { float s = 0.f; for (int i = 0; i < N; ++i) s += v[i]; return s / N; }
  KRR_STUB_HD float norm() const { float s = 0.f; for (int i = 0; i < N; ++i) s += v[i] * v[i]; return sqrtf(s); }
  KRR_STUB_HD static VecN Zero() { return VecN(0.f); }
  KRR_STUB_HD static VecN Ones() { return VecN(1.f); }
  KRR_STUB_HD static VecN Constant(float a) { return VecN(a); }
  static constexpr int dim = N;
};
template <int N> KRR_STUB_HD VecN<N> operator+(VecN<N> a, const VecN<N>& b) { for (int i = 0; i < N; ++i) a[i] += b[i]; return a; }
template <int N> KRR_STUB_HD VecN<N> operator-(VecN<N> a, const VecN<N>& b) { for (int i = 0; i < N; ++i) a[i] -= b[i]; return a; }
template <int N> KRR_STUB_HD VecN<N> operator*(VecN<N> a, const VecN<N>& b) { for (int i = 0; i < N; ++i) a[i] *= b[i]; return a; }
template <int N> KRR_STUB_HD VecN<N> operator/(VecN<N> a, const VecN<N>& b) { for (int i = 0; i < N; ++i) a[i] /= b[i]; return a; }
template <int N> KRR_STUB_HD VecN<N> operator*(VecN<N> a, float s) { for (int i = 0; i < N; ++i) a[i] *= s; return a; }
template <int N> KRR_STUB_HD VecN<N> operator*(float s, VecN<N> a) { for (int i = 0; i < N; ++i) a[i] *= s; return a; }
template <int N> KRR_STUB_HD VecN<N> operator/(VecN<N> a, float s) { for (int i = 0; i < N; ++i) a[i] /= s; return a; }
template <int N> KRR_STUB_HD VecN<N>& operator+=(VecN<N>& a, const VecN<N>& b) { a = a + b; return a; }
template <int N> KRR_STUB_HD VecN<N>& operator*=(VecN<N>& a, const VecN<N>& b) { a = a * b; return a; }
template <int N> KRR_STUB_HD VecN<N>& operator/=(VecN<N>& a, const VecN<N>& b) { a = a / b; return a; }
template <int N> KRR_STUB_HD VecN<N>& operator*=(VecN<N>& a, float s) { a = a * s; return a; }
template <int N> KRR_STUB_HD VecN<N>& operator/=(VecN<N>& a, float s) { a = a / s; return a; }

struct Vector2f : VecN<2> {
  KRR_STUB_HD Vector2f() = default;
  KRR_STUB_HD Vector2f(const VecN<2>& o) : VecN<2>(o) {}
  KRR_STUB_HD Vector2f(float a, float b) { v[0] = a; v[1] = b; }
};
struct Vector3f : VecN<3> {
  KRR_STUB_HD Vector3f() = default;
  KRR_STUB_HD Vector3f(const VecN<3>& o) : VecN<3>(o) {}
  KRR_STUB_HD explicit Vector3f(float a) : VecN<3>(a) {}
  KRR_STUB_HD Vector3f(float a, float b, float c) { v[0] = a; v[1] = b; v[2] = c; }
  KRR_STUB_HD Vector3f(const float3& f) { v[0] = f.x; v[1] = f.y; v[2] = f.z; }
  KRR_STUB_HD Vector3f normalized() const { return *this / norm(); }
};
struct Color : VecN<3> {
  KRR_STUB_HD Color() = default;
  KRR_STUB_HD Color(const VecN<3>& o) : VecN<3>(o) {}
  KRR_STUB_HD explicit Color(float a) : VecN<3>(a) {}
  KRR_STUB_HD Color(float a, float b, float c) { v[0] = a; v[1] = b; v[2] = c; }
  KRR_STUB_HD static Color Zero() { return Color(0.f); }
};
struct Vector2i { int v[2]; KRR_STUB_HD int operator[](int i) const { return v[i]; } };

struct AABB {
  Vector3f mn, mx;
  KRR_STUB_HD void inflate(float d) { for (int i = 0; i < 3; ++i) { mn[i] -= d; mx[i] += d; } }
  KRR_STUB_HD Vector3f diagonal() const { return mx - mn; }
  KRR_STUB_HD Vector3f center() const { return (mn + mx) * 0.5f; }
};

template <typename T> class atomic {
 public:
  KRR_STUB_HD void store(T x) { v_ = x; }
  KRR_STUB_HD T load() const { return v_; }
#if defined(__CUDA_ARCH__)
  __device__ T fetch_add(T x) { return atomicAdd(&v_, x); }
#else
  T fetch_add(T x) { T o = v_; v_ += x; return o; }
#endif
  KRR_STUB_HD operator T() const { return v_; }
 private:
  T v_{};
};

struct Allocator {};
}  // namespace krr

#define M_EPSILON 1e-5f
#ifndef M_PI
#define M_PI 3.14159265358979323846f
#endif
#define M_2PI 6.28318530717958647693f
#define M_INV_PI 0.318309886183790671538f
#define M_INV_2PI 0.15915494309189533577f
#define M_INV_4PI 0.07957747154594766788f
#define M_4PI 12.5663706143591729538f
