// Packed values of several right-hand sides: Pack<F, R> holds one value per
// system of a group that is solved in lockstep on one mesh, so one load,
// store or shared-memory access moves all R systems' values of a node and the
// element operator's index and factor traffic is shared by the R systems.
// Scalars (R = 1) keep their own type; the helpers below let the same kernel
// code run on both.
#pragma once

#include <cuda_runtime.h>

namespace bp {

template <class F, int R>
struct alignas(sizeof(F) * R <= 16 ? sizeof(F) * R : 16) Pack {
  F v[R];
  Pack() = default;
  __host__ __device__ __forceinline__ explicit Pack(F a) {
#pragma unroll
    for (int l = 0; l < R; ++l) v[l] = a;
  }
};

template <class F, int R>
__device__ __forceinline__ Pack<F, R> operator+(const Pack<F, R>& a, const Pack<F, R>& b) {
  Pack<F, R> c;
#pragma unroll
  for (int l = 0; l < R; ++l) c.v[l] = a.v[l] + b.v[l];
  return c;
}
template <class F, int R>
__device__ __forceinline__ Pack<F, R> operator-(const Pack<F, R>& a, const Pack<F, R>& b) {
  Pack<F, R> c;
#pragma unroll
  for (int l = 0; l < R; ++l) c.v[l] = a.v[l] - b.v[l];
  return c;
}
template <class F, int R>
__device__ __forceinline__ Pack<F, R> operator*(F a, const Pack<F, R>& b) {
  Pack<F, R> c;
#pragma unroll
  for (int l = 0; l < R; ++l) c.v[l] = a * b.v[l];
  return c;
}
template <class F, int R>
__device__ __forceinline__ Pack<F, R>& operator+=(Pack<F, R>& a, const Pack<F, R>& b) {
#pragma unroll
  for (int l = 0; l < R; ++l) a.v[l] += b.v[l];
  return a;
}

template <class T>
struct PackTraits {
  using F = T;
  static constexpr int R = 1;
};
template <class F_, int R_>
struct PackTraits<Pack<F_, R_>> {
  using F = F_;
  static constexpr int R = R_;
};

// lane l of a value (l = 0 for scalars)
template <class T>
__device__ __forceinline__ typename PackTraits<T>::F lane(const T& a, int) {
  return a;
}
template <class F, int R>
__device__ __forceinline__ F lane(const Pack<F, R>& a, int l) {
  return a.v[l];
}

// read-only load through the non-coherent path: the compiler may move it
// ahead of the kernel's stores (which never alias the array read)
__device__ __forceinline__ double ldg_val(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ldg_val(const float* p) { return __ldg(p); }
__device__ __forceinline__ Pack<float, 2> ldg_val(const Pack<float, 2>* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  Pack<float, 2> r;
  r.v[0] = v.x;
  r.v[1] = v.y;
  return r;
}
__device__ __forceinline__ Pack<float, 4> ldg_val(const Pack<float, 4>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  Pack<float, 4> r;
  r.v[0] = v.x;
  r.v[1] = v.y;
  r.v[2] = v.z;
  r.v[3] = v.w;
  return r;
}

// lane l of a value set to x
template <class T>
__device__ __forceinline__ void lane_set(T& a, int, T x) {
  a = x;
}
template <class F, int R>
__device__ __forceinline__ void lane_set(Pack<F, R>& a, int l, F x) {
  a.v[l] = x;
}

// acc[l] += a_l * b_l in FP64
template <class T>
__device__ __forceinline__ void lane_dot(double* acc, const T& a, const T& b) {
  acc[0] += (double)a * (double)b;
}
template <class F, int R>
__device__ __forceinline__ void lane_dot(double* acc, const Pack<F, R>& a, const Pack<F, R>& b) {
#pragma unroll
  for (int l = 0; l < R; ++l) acc[l] += (double)a.v[l] * (double)b.v[l];
}

template <class T>
__device__ __forceinline__ T pack_zero() {
  return T(0);
}

}  // namespace bp
