// Double-precision refinement of the final active-set coefficients.
//
// The homotopy (or OMP) picks the active set A and the signs; its float32
// coefficients carry the error of the correlations it started from (the BF16
// hi/lo tensor-core products are accurate to ~1e-5 relative).  The solution
// on a fixed active set is known in closed form:
//   LARS-Lasso  G_AA a = D_A^T x - level s_A   (the equicorrelation condition
//               of coreLARS2's path, decomp/decomp.h:1706-1915; level = lambda1
//               when the path stopped at lambda1 in PENALTY mode)
//   OMP         G_AA a = D_A^T x               (coreORMP's least-squares fit on
//               the selected atoms, decomp/decomp.h:538-640)
// so one warp per signal recomputes D_A^T x from the inputs with double
// accumulation, factors G_AA by Cholesky in double and solves.
#include "common.cuh"
#include "kernels.h"

namespace sc {

constexpr int RF_MAX = 32;  // active sets refined (larger ones keep their values)

__global__ void __launch_bounds__(128)
refine_kernel(const float* __restrict__ D, int m, const float* __restrict__ X,
              const float* __restrict__ G, int Kp, const int* __restrict__ slab_ind,
              float* __restrict__ slab_val, int L, const int* __restrict__ cnt,
              const float* __restrict__ level, int64_t n) {
  __shared__ double sA[4][RF_MAX][RF_MAX + 1];
  __shared__ double sb[4][RF_MAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t sig = (int64_t)blockIdx.x * 4 + w;
  if (sig >= n) return;
  const int s = cnt[sig];
  if (s <= 0 || s > RF_MAX) return;
  const int* ind = slab_ind + (size_t)sig * L;
  float* val = slab_val + (size_t)sig * L;
  const float* x = X + (size_t)sig * m;
  double (*A)[RF_MAX + 1] = sA[w];
  double* b = sb[w];
  // right-hand side: D_A^T x - level * sign(a)
  bool ok = true;
  for (int j = 0; j < s; ++j) {
    const float* d = D + (size_t)ind[j] * m;
    double p = 0;
    for (int r = lane; r < m; r += 32) p += (double)d[r] * (double)x[r];
    p = warp_sum(p);
    if (lane == 0) {
      const float a = val[j];
      double rhs = p;
      if (level) {
        if (a == 0.f) ok = false;
        rhs -= (double)level[sig] * (a > 0.f ? 1.0 : -1.0);
      }
      b[j] = rhs;
    }
  }
  ok = __shfl_sync(kFull, (int)ok, 0);
  if (!ok) return;
  // G_AA (ridge included), lower triangle used
  for (int i = lane; i < s; i += 32)
    for (int j = 0; j <= i; ++j) A[i][j] = (double)G[(size_t)ind[j] * Kp + ind[i]];
  __syncwarp();
  // Cholesky, lanes own rows
  for (int k = 0; k < s; ++k) {
    double piv = A[k][k];
    if (!(piv > 0)) { ok = false; break; }  // uniform: every lane reads the same value
    piv = sqrt(piv);
    __syncwarp();
    if (lane == 0) A[k][k] = piv;
    for (int i = k + 1 + lane; i < s; i += 32) A[i][k] /= piv;
    __syncwarp();
    for (int i = k + 1 + lane; i < s; i += 32) {
      const double lik = A[i][k];
      for (int j = k + 1; j <= i; ++j) A[i][j] -= lik * A[j][k];
    }
    __syncwarp();
  }
  if (!ok) return;
  if (lane == 0) {
    // forward and back substitution
    for (int i = 0; i < s; ++i) {
      double t = b[i];
      for (int j = 0; j < i; ++j) t -= A[i][j] * b[j];
      b[i] = t / A[i][i];
    }
    for (int i = s - 1; i >= 0; --i) {
      double t = b[i];
      for (int j = i + 1; j < s; ++j) t -= A[j][i] * b[j];
      b[i] = t / A[i][i];
    }
  }
  __syncwarp();
  for (int j = lane; j < s; j += 32) val[j] = (float)b[j];
}

cudaError_t launch_refine(const float* D, int m, const float* X, const float* G, int Kp,
                          const int* slab_ind, float* slab_val, int L, const int* cnt,
                          const float* level, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  refine_kernel<<<(unsigned)((n + 3) / 4), 128, 0, st>>>(D, m, X, G, Kp, slab_ind, slab_val, L,
                                                         cnt, level, n);
  return cudaGetLastError();
}

}  // namespace sc
