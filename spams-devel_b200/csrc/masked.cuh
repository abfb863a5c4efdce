// Gram products of the masked variants (lasso_mask / omp_mask,
// decomp/decomp.h:406-519 and :1466-1561), formed on the fly for a signal
// whose observed rows are a strict subset of the m rows.  The reference
// copies the observed rows of D and x (Matrix::copyMask,
// linalg/linalg.h:4082-4107) and codes with the Gram of those rows plus a
// ridge on the diagonal; here the kernels never form that K x K matrix: an
// entry G_m(a, b) is a masked dot product of two atoms, and a product
// G_m(:, A) u is Dᵀ (mask ∘ (D_A u)) plus the ridge on the active rows.
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace sc {

// G_m(a, b) (+ ridge when a == b) over the observed rows; every lane of the
// warp returns the same value.
template <typename T>
__device__ __forceinline__ T masked_gram(const MaskArgs<T>& mk, const uint8_t* mrow, int a,
                                         int b) {
  const T* da = mk.D + (size_t)a * mk.m;
  const T* db = mk.D + (size_t)b * mk.m;
  T s = 0;
  for (int r = (int)(threadIdx.x & 31); r < mk.m; r += 32)
    if (mrow[r]) s += da[r] * db[r];
  s = warp_sum(s);
  return a == b ? s + mk.ridge : s;
}

// A += G_m(:, ind[0:len]) u over the lane's rows (r = 128 v + 4 lane + e),
// u[j] at u[j * ustride].  w: this warp's mpad-vector of global scratch.
template <typename T, int NV>
__device__ __forceinline__ void masked_gram_times(const MaskArgs<T>& mk, const uint8_t* mrow,
                                                  T* w, int Kp, const int* ind, const T* u,
                                                  int ustride, int len, T (&A)[NV][4]) {
  const int lane = threadIdx.x & 31;
  // w = mask ∘ (D_ind u)
  for (int r = lane; r < mk.m; r += 32) {
    T s = 0;
    if (mrow[r])
      for (int j = 0; j < len; ++j) s += mk.D[(size_t)ind[j] * mk.m + r] * u[(size_t)j * ustride];
    w[r] = s;
  }
  __syncwarp();
  // A += Dᵀ w, one coalesced row of Dᵀ per observed row
  for (int r = 0; r < mk.m; ++r) {
    const T wr = w[r];
    if (wr == T(0)) continue;
    const T* dt = mk.Dt + (size_t)r * Kp + lane * 4;
#pragma unroll
    for (int v = 0; v < NV; ++v) axpy4(A[v], ldg4(dt + v * 128), wr);
  }
  // the ridge sits on the diagonal of G_m
  for (int j = 0; j < len; ++j) {
    const int c = ind[j];
    const T add = mk.ridge * u[(size_t)j * ustride];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (v * 128 + lane * 4 + e == c) A[v][e] += add;
  }
  __syncwarp();  // w is rewritten at the next step
}

// CTA-collective form for the CTA-per-signal kernels (every thread of the CTA
// calls it): A += G_m(:, ind[0:len]) u over this warp's rows
// (r = rbase + 128 v + 4 lane + e); w: the CTA's mpad-vector of scratch.  The
// same sums in the same order as masked_gram_times, so both kernel families
// give the same bits.
template <typename T, int NV, int W>
__device__ __forceinline__ void masked_gram_times_cta(const MaskArgs<T>& mk, const uint8_t* mrow,
                                                      T* w, int Kp, int rbase, const int* ind,
                                                      const T* u, int ustride, int len,
                                                      T (&A)[NV][4]) {
  const int lane = threadIdx.x & 31;
  for (int r = threadIdx.x; r < mk.m; r += W * 32) {
    T s = 0;
    if (mrow[r])
      for (int j = 0; j < len; ++j) s += mk.D[(size_t)ind[j] * mk.m + r] * u[(size_t)j * ustride];
    w[r] = s;
  }
  __syncthreads();
  for (int r = 0; r < mk.m; ++r) {
    const T wr = w[r];
    if (wr == T(0)) continue;
    const T* dt = mk.Dt + (size_t)r * Kp + rbase + lane * 4;
#pragma unroll
    for (int v = 0; v < NV; ++v) axpy4(A[v], ldg4(dt + v * 128), wr);
  }
  for (int j = 0; j < len; ++j) {
    const int c = ind[j];
    const T add = mk.ridge * u[(size_t)j * ustride];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (rbase + v * 128 + lane * 4 + e == c) A[v][e] += add;
  }
  __syncthreads();  // w is rewritten at the next step
}

}  // namespace sc
