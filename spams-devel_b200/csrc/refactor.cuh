// FP64 refactor of the single-precision active-set state.
//
// LARS (coreLARS2, decomp/decomp.h:1749-1771) keeps the inverse of the active
// set's Gram, G_AA^-1, up to date by rank-one Schur updates; OMP (coreORMP,
// :576-598) keeps the inverse Cholesky factor Un (Un^T G_AA Un = I) by
// appending one column per selected atom.  When the new atom's pivot (LARS:
// g_ii - g_i^T G_AA^-1 g_i against g_ii; OMP: the atom's residual norm,
// against its unit norm) is small, single-precision updates lose digits.
// The refactor recomputes the state from G in double instead: Cholesky
// G_AA = L L^T and L^-1 by rows, then
//   LARS  G_AA^-1 = L^-T L^-1
//   OMP   Un = L^-T, RUn = Un^T (D^T x)_A, ||r||^2 = ||x||^2 - ||RUn||^2
// rounded once into the single-precision state.
#pragma once
#include "common.cuh"

namespace sc {

constexpr int kRefactorMax = 96;        // active sets refactored up to this size
constexpr double kRefactorPivot = 1e-3; // relative pivot that triggers it
// Scratch of one refactor unit (a warp of the warp kernels, a CTA of the CTA
// kernels): cap x cap doubles for active sets of up to `cap` atoms.
__host__ __device__ inline int refactor_cap(int Lcap) {
  return Lcap < kRefactorMax ? Lcap : kRefactorMax;
}

// Warp-collective.  S (n x n doubles, row-major, ld n) = L^-1, the inverse of
// the lower Cholesky factor of G_AA for the atoms ind[0..n) of G (Kp x Kp,
// column-major, symmetric), n <= kRefactorMax.  Returns false (warp-uniform)
// when G_AA is not positive definite in double; S is then scratch.
template <typename T>
__device__ __noinline__ bool chol_inverse64(const T* __restrict__ G, int Kp, const int* ind, int n,
                                            double* S) {
  const int lane = threadIdx.x & 31;
  for (int r = lane; r < n; r += 32) {
    const T* gr = G + (size_t)ind[r] * Kp;
    for (int c = 0; c <= r; ++c) S[r * n + c] = (double)gr[ind[c]];
  }
  __syncwarp();
  // right-looking Cholesky, lower triangle in place; rows spread over lanes
  for (int k = 0; k < n; ++k) {
    const double piv = S[k * n + k];
    if (!(piv > 0.0)) return false;  // every lane reads the same value
    const double d = sqrt(piv);
    __syncwarp();
    for (int r = k + 1 + lane; r < n; r += 32) S[r * n + k] /= d;
    if (lane == 0) S[k * n + k] = d;
    __syncwarp();
    for (int r = k + 1 + lane; r < n; r += 32) {
      const double lk = S[r * n + k];
      for (int c = k + 1; c <= r; ++c) S[r * n + c] -= lk * S[c * n + k];
    }
    __syncwarp();
  }
  // L^-1 row by row: Linv(i, j) = -(sum_{j <= k < i} L(i, k) Linv(k, j)) / L(i, i),
  // the row's entries computed from the untouched row of L, then stored
  for (int i = 0; i < n; ++i) {
    const double dii = S[i * n + i];
    double t[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int j = lane + 32 * q;
      double s = 0.0;
      if (j < i)
        for (int k = j; k < i; ++k) s += S[i * n + k] * S[k * n + j];
      t[q] = -s / dii;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int j = lane + 32 * q;
      if (j < i) S[i * n + j] = t[q];
    }
    if (lane == 0) S[i * n + i] = 1.0 / dii;
    __syncwarp();
  }
  return true;
}

// Warp-collective: inv (n x n, leading dimension ldi) = G_AA^-1 for the atoms
// ind[0..n) (the LARS state); S: n x n doubles of scratch.  False, with inv
// untouched, when G_AA is not positive definite in double.
template <typename T>
__device__ __noinline__ bool refactor_inverse(const T* __restrict__ G, int Kp, const int* ind,
                                              int n, T* inv, int ldi, double* S) {
  if (!chol_inverse64<T>(G, Kp, ind, n, S)) return false;
  const int lane = threadIdx.x & 31;
  // inv(a, b) = sum_{r >= max(a, b)} Linv(r, a) Linv(r, b)
  for (int a = lane; a < n; a += 32)
    for (int b = 0; b < n; ++b) {
      double s = 0.0;
      for (int r = a > b ? a : b; r < n; ++r) s += S[r * n + a] * S[r * n + b];
      inv[(size_t)a * ldi + b] = (T)s;
    }
  __syncwarp();
  return true;
}

// Warp-collective refactor of the OMP state for the atoms ind[0..n):
// Un (row-major, ld ldu, upper triangle) = L^-T and RUn[k] = sum_l Un(l, k) d_l
// with d = D^T x (dtx, by atom), from double-precision sums.  Returns
// ||x||^2 - sum_k RUn[k]^2 (every lane), or NaN, with the state untouched,
// when G_AA is not positive definite in double.
template <typename T>
__device__ __noinline__ double refactor_un(const T* __restrict__ G, int Kp, const int* ind, int n,
                                           const T* __restrict__ dtx, T xnorm2, T* Un, int ldu,
                                           T* RUn, double* S) {
  if (!chol_inverse64<T>(G, Kp, ind, n, S)) return __longlong_as_double(0x7ff8000000000000ll);
  const int lane = threadIdx.x & 31;
  // Un(r, c) = Linv(c, r) for r <= c; RUn[c] = sum_{l <= c} Linv(c, l) d_l
  double part = 0.0;
  for (int c = lane; c < n; c += 32) {
    double s = 0.0;
    for (int r = 0; r <= c; ++r) {
      const double v = S[c * n + r];
      Un[(size_t)r * ldu + c] = (T)v;
      s += v * (double)dtx[ind[r]];
    }
    RUn[c] = (T)s;
    part += s * s;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
  __syncwarp();
  return (double)xnorm2 - part;
}

}  // namespace sc
