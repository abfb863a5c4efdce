// FP64 refactor of the LARS inverse Gram.  In single precision the
// homotopy's inverse of the active set's Gram, G_AA^-1, is kept up to date by
// rank-one Schur updates (coreLARS2, decomp/decomp.h:1749-1771); when the new
// atom's pivot g_ii - g_iᵀ G_AA^-1 g_i is small against g_ii the update
// loses digits.  The refactor recomputes the inverse from G in double
// instead: Cholesky G_AA = L Lᵀ, L^-1 by forward substitution, then
// G_AA^-1 = L^-T L^-1, rounded once into the single-precision rows.
#pragma once
#include "common.cuh"

namespace sc {

constexpr int kRefactorMax = 32;  // active sets refactored up to this size
constexpr double kRefactorPivot = 1e-3;  // relative pivot that triggers it

// Warp-collective: inv (n x n, leading dimension ldi) = G_AA^-1 for the atoms
// ind[0..n), n <= kRefactorMax; A and B are this warp's 2 x 32 x 32 doubles of
// global scratch.  Returns false and writes nothing when G_AA is not
// positive definite in double.
template <typename T>
__device__ __noinline__ bool refactor_inverse(const T* __restrict__ G, int Kp, const int* ind, int n, T* inv,
                                 int ldi, double* A, double* B) {
  const int lane = threadIdx.x & 31;
  constexpr int ld = kRefactorMax;
  if (lane < n)
    for (int c = 0; c <= lane; ++c) A[lane * ld + c] = (double)G[(size_t)ind[c] * Kp + ind[lane]];
  __syncwarp();
  // Cholesky, lower triangle in place; lane r owns row r
  for (int k = 0; k < n; ++k) {
    double piv = A[k * ld + k];
    if (!(piv > 0.0)) return false;  // warp-uniform
    piv = sqrt(piv);
    __syncwarp();
    if (lane == k) A[k * ld + k] = piv;
    if (lane > k && lane < n) A[lane * ld + k] /= piv;
    __syncwarp();
    if (lane > k && lane < n) {
      const double lk = A[lane * ld + k];
      for (int c = k + 1; c <= lane; ++c) A[lane * ld + c] -= lk * A[c * ld + k];
    }
    __syncwarp();
  }
  // B = L^-1 (lower); lane c computes column c
  if (lane < n) {
    B[lane * ld + lane] = 1.0 / A[lane * ld + lane];
    for (int r = lane + 1; r < n; ++r) {
      double s = 0;
      for (int k = lane; k < r; ++k) s += A[r * ld + k] * B[k * ld + lane];
      B[r * ld + lane] = -s / A[r * ld + r];
    }
  }
  __syncwarp();
  // inv(a, b) = sum_{r >= max(a, b)} B(r, a) B(r, b); lane a writes row a
  if (lane < n)
    for (int b = 0; b < n; ++b) {
      double s = 0;
      for (int r = lane > b ? lane : b; r < n; ++r) s += B[r * ld + lane] * B[r * ld + b];
      inv[(size_t)lane * ldi + b] = (T)s;
    }
  __syncwarp();
  return true;
}

}  // namespace sc
