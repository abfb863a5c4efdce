// Shared device helpers for the sparse-coding kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <map>
#include <mutex>
#include <tuple>

#define SC_INF_F (__int_as_float(0x7f800000))

namespace sc {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

template <typename T> __device__ __forceinline__ T inf();
template <> __device__ __forceinline__ float inf<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double inf<double>() { return __longlong_as_double(0x7ff0000000000000ll); }

// Four consecutive elements starting at a 4-element-aligned address, as one
// (float) or two (double) vector loads.
// a * b rounded on its own, never contracted with a following add into one
// FMA: the reference's scalar updates (built without FMA contraction) round
// the product first, and the L1COEFFS stop compares their sum with the
// constraint at rounding level.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

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

// d = a * b + c on a pair of floats with one packed FP32x2 instruction.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
      "mov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

// Column accumulation acc[0..3] += g[0..3] * u: packed pairs in single
// precision, plain FMAs in double precision.
__device__ __forceinline__ void axpy4(float* acc, const Vec4<float>& g, float u) {
  const float2 uu = make_float2(u, u);
  const float2 lo = fma2(make_float2(g.v[0], g.v[1]), uu, make_float2(acc[0], acc[1]));
  const float2 hi = fma2(make_float2(g.v[2], g.v[3]), uu, make_float2(acc[2], acc[3]));
  acc[0] = lo.x; acc[1] = lo.y; acc[2] = hi.x; acc[3] = hi.y;
}
__device__ __forceinline__ void axpy4(double* acc, const Vec4<double>& g, double u) {
#pragma unroll
  for (int e = 0; e < 4; ++e) acc[e] += g.v[e] * u;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Order-preserving map of a float to an unsigned key: a < b (as floats, no
// NaN) exactly when key(a) < key(b) (as unsigned).
__device__ __forceinline__ unsigned float_key(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Warp-uniform results of the arg-reductions below (every lane gets them).
template <typename T> struct ArgRes { T val; int idx; };

// (min key, first index among the minima, the value carried by that entry)
// over the warp; keys must be non-NaN.  Single precision uses the warp
// reduction instructions on order-preserving key bits; double precision a
// butterfly of shuffles.
__device__ __forceinline__ ArgRes<float> warp_argmin_first(float key, int idx, float carry) {
  const unsigned kb = float_key(key);
  const unsigned mn = __reduce_min_sync(kFull, kb);
  const int wi = (int)__reduce_min_sync(kFull, kb == mn ? (unsigned)idx : 0xffffffffu);
  const unsigned who = __ballot_sync(kFull, kb == mn && idx == wi);
  const float v = __shfl_sync(kFull, carry, __ffs(who) - 1);
  return ArgRes<float>{v, wi};
}
__device__ __forceinline__ ArgRes<double> warp_argmin_first(double key, int idx, double carry) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    const double c2 = __shfl_xor_sync(kFull, carry, o);
    if (k2 < key || (k2 == key && i2 < idx)) { key = k2; idx = i2; carry = c2; }
  }
  return ArgRes<double>{__shfl_sync(kFull, carry, 0), __shfl_sync(kFull, idx, 0)};
}
// (min key, LAST index among the minima); idx -1 marks "no candidate".
__device__ __forceinline__ ArgRes<float> warp_argmin_last_u(float key, int idx) {
  const unsigned kb = float_key(key);
  const unsigned mn = __reduce_min_sync(kFull, kb);
  const int wi = __reduce_max_sync(kFull, kb == mn ? idx : -1);
  const float v = __shfl_sync(kFull, key, __ffs(__ballot_sync(kFull, kb == mn)) - 1);
  return ArgRes<float>{v, wi};
}
__device__ __forceinline__ ArgRes<double> warp_argmin_last_u(double key, int idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    if (k2 < key || (k2 == key && i2 > idx)) { key = k2; idx = i2; }
  }
  return ArgRes<double>{__shfl_sync(kFull, key, 0), __shfl_sync(kFull, idx, 0)};
}
// (max key, first index among the maxima).
__device__ __forceinline__ int warp_argmax_first(float key, int idx) {
  const unsigned kb = float_key(key);
  const unsigned mx = __reduce_max_sync(kFull, kb);
  return (int)__reduce_min_sync(kFull, kb == mx ? (unsigned)idx : 0xffffffffu);
}
__device__ __forceinline__ int warp_argmax_first(double key, int idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double k2 = __shfl_xor_sync(kFull, key, o);
    const int i2 = __shfl_xor_sync(kFull, idx, o);
    if (k2 > key || (k2 == key && i2 < idx)) { key = k2; idx = i2; }
  }
  return __shfl_sync(kFull, idx, 0);
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

// Persistent-grid size for a kernel whose blocks loop over a work counter:
// grid > 0 is kept; otherwise as many blocks as fit on the device at once.
template <typename Kern>
inline cudaError_t fill_grid(Kern k, int threads, size_t smem, int* grid) {
  if (*grid > 0) return cudaSuccess;
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
  if (e != cudaSuccess) return e;
  *grid = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  return cudaSuccess;
}

// Lets kernel `k` launch with `smem` bytes of dynamic shared memory.  The
// function attribute is process-wide, not per launch: it is always set to the
// device's full opt-in size (less the kernel's static shared memory), the
// same value from every caller, so that a thread launching this kernel with a
// large size never races with another thread lowering the limit for a smaller
// one.  Also prefers the largest shared-memory carveout.
template <typename Kern>
inline cudaError_t allow_smem(Kern k, size_t smem) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void*)k);
  if (e != cudaSuccess) return e;
  const int limit = optin - (int)fa.sharedSizeBytes;
  if (smem > (size_t)limit) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

// Of two builds of one kernel, the second compiled with a register bound,
// the one that keeps more CTAs resident per SM with `smem` bytes of dynamic
// shared memory; the unbounded build on ties (the bound only costs spills
// when shared memory or threads limit residency anyway).
// The answer is kept per (kernel, threads, shared memory, device).
template <typename Kern>
inline Kern more_resident(Kern plain, Kern bounded, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t, int>, bool> memo;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return plain;
  const auto key = std::make_tuple((const void*)plain, threads, smem, dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second ? bounded : plain;
  }
  int a = 0, b = 0;
  if (allow_smem(plain, smem) != cudaSuccess || allow_smem(bounded, smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, plain, threads, smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, bounded, threads, smem) != cudaSuccess)
    return plain;
  std::lock_guard<std::mutex> lk(mu);
  memo[key] = b > a;
  return b > a ? bounded : plain;
}

}  // namespace sc
