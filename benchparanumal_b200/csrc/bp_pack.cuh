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
