// Shared device helpers for the sparse-coding kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define SC_INF_F (__int_as_float(0x7f800000))

namespace sc {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

template <typename T> __device__ __forceinline__ T inf();
template <> __device__ __forceinline__ float inf<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double inf<double>() { return __longlong_as_double(0x7ff0000000000000ll); }

// Four consecutive elements starting at a 4-element-aligned address, as one
// (float) or two (double) vector loads.
template <typename T> struct Vec4 { T v[4]; };

__device__ __forceinline__ Vec4<float> ld4(const float* p) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  return Vec4<float>{{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Vec4<double> ld4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return Vec4<double>{{a.x, a.y, b.x, b.y}};
}
// Read-only path through L1/L2 (the Gram matrix and the correlations).
__device__ __forceinline__ Vec4<float> ldg4(const float* p) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  return Vec4<float>{{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Vec4<double> ldg4(const double* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p + 2));
  return Vec4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const Vec4<float>& q) {
  *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ void st4(double* p, const Vec4<double>& q) {
  *reinterpret_cast<double2*>(p) = make_double2(q.v[0], q.v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(q.v[2], q.v[3]);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Arg-min of (key, idx) pairs, ties resolved to the smaller idx.  Keys are
// compared as given (callers pass magnitudes); NaN keys never win.
template <typename T>
__device__ __forceinline__ void warp_argmin(T& key, int& idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    if (k2 < key || (k2 == key && i2 < idx)) { key = k2; idx = i2; }
  }
}

// Arg-max of (key, idx), ties to the smaller idx (BLAS i?amax / first max).
template <typename T>
__device__ __forceinline__ void warp_argmax(T& key, int& idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    if (k2 > key || (k2 == key && i2 < idx)) { key = k2; idx = i2; }
  }
}

// Arg-min with ties resolved to the LARGER idx: the reference's "ratio <=
// step_max" scan keeps the last index among equal ratios.
template <typename T>
__device__ __forceinline__ void warp_argmin_last(T& key, int& idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    if (k2 < key || (k2 == key && i2 > idx)) { key = k2; idx = i2; }
  }
}

}  // namespace sc
