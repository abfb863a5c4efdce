// Double-precision solves on the final active sets.
//
// Two users:
//  * refinement of single-precision codes: the homotopy (or OMP) picks the
//    active set A and the signs; its float32 coefficients carry the error of
//    the correlations it started from, while the solution on a fixed active
//    set is known in closed form:
//      LARS-Lasso  G_AA a = D_A^T x - level s_A   (the equicorrelation condition
//                  of coreLARS2's path, decomp/decomp.h:1706-1915; level =
//                  lambda1 when the path stopped at lambda1 in PENALTY mode)
//      OMP         G_AA a = D_A^T x               (coreORMP's least-squares fit
//                  on the selected atoms, decomp/decomp.h:538-640)
//  * the `ols` option of the Cholesky lasso (coreLARS, decomp/decomp.h:1087-1091):
//    the final orthogonal projection, i.e. the least-squares fit G_AA a = D_A^T x
//    on the support of the path (G with its ridge).
// One warp per signal recomputes D_A^T x from the inputs with double
// accumulation, factors G_AA by Cholesky in double and solves.  Active sets
// of up to RF_SMEM atoms keep G_AA in shared memory; larger ones are queued to
// a second pass whose warps use a global scratch slab each.
#include "common.cuh"
#include "kernels.h"

namespace sc {

constexpr int RF_SMEM = 32;
constexpr int RF_WARPS = 4;

template <typename T>
__device__ void refine_one(const T* __restrict__ D, int m, const T* __restrict__ x,
                           const T* __restrict__ qcol, const T* __restrict__ G, int Kp,
                           const int* ind, T* val, int s, const T* level_p, double* A, int lda,
                           double* b) {
  const int lane = threadIdx.x & 31;
  bool ok = true;
  for (int j = 0; j < s; ++j) {
    double p = 0;
    if (qcol) {  // correlations given by the caller (D^T X, the (Q, q) form)
      p = (double)qcol[ind[j]];
    } else {
      const T* d = D + (size_t)ind[j] * m;
      for (int r = lane; r < m; r += 32) p += (double)d[r] * (double)x[r];
      p = warp_sum(p);
    }
    if (lane == 0) {
      const T a = val[j];
      double rhs = p;
      if (level_p) {
        if (a == T(0)) ok = false;
        rhs -= (double)(*level_p) * (a > T(0) ? 1.0 : -1.0);
      }
      b[j] = rhs;
    }
  }
  ok = __shfl_sync(kFull, (int)ok, 0);
  if (!ok) return;
  for (int i = lane; i < s; i += 32)
    for (int j = 0; j <= i; ++j) A[(size_t)i * lda + j] = (double)G[(size_t)ind[j] * Kp + ind[i]];
  __syncwarp();
  // Cholesky (lower), lanes own rows; every lane reads the same pivot
  for (int k = 0; k < s; ++k) {
    double piv = A[(size_t)k * lda + k];
    if (!(piv > 0)) { ok = false; break; }
    piv = sqrt(piv);
    __syncwarp();
    if (lane == 0) A[(size_t)k * lda + k] = piv;
    for (int i = k + 1 + lane; i < s; i += 32) A[(size_t)i * lda + k] /= piv;
    __syncwarp();
    for (int i = k + 1 + lane; i < s; i += 32) {
      const double lik = A[(size_t)i * lda + k];
      for (int j = k + 1; j <= i; ++j) A[(size_t)i * lda + j] -= lik * A[(size_t)j * lda + k];
    }
    __syncwarp();
  }
  if (!ok) return;
  if (lane == 0) {
    for (int i = 0; i < s; ++i) {
      double t = b[i];
      for (int j = 0; j < i; ++j) t -= A[(size_t)i * lda + j] * b[j];
      b[i] = t / A[(size_t)i * lda + i];
    }
    for (int i = s - 1; i >= 0; --i) {
      double t = b[i];
      for (int j = i + 1; j < s; ++j) t -= A[(size_t)j * lda + i] * b[j];
      b[i] = t / A[(size_t)i * lda + i];
    }
  }
  __syncwarp();
  for (int j = lane; j < s; j += 32) val[j] = (T)b[j];
}

// Pass 1: one warp per signal, active sets up to RF_SMEM atoms in shared
// memory; larger ones are appended to big_list.
template <typename T>
__global__ void __launch_bounds__(RF_WARPS * 32)
refine_kernel(const T* __restrict__ D, int m, const T* __restrict__ X, const T* __restrict__ Q,
              int ldq, const T* __restrict__ G,
              int Kp, const int* __restrict__ slab_ind, T* __restrict__ slab_val, int L,
              const int* __restrict__ cnt, const T* __restrict__ level, int64_t n,
              int64_t* big_list, int* big_count) {
  __shared__ double sA[RF_WARPS][RF_SMEM][RF_SMEM + 1];
  __shared__ double sb[RF_WARPS][RF_SMEM];
  const int w = threadIdx.x >> 5;
  const int64_t sig = (int64_t)blockIdx.x * RF_WARPS + w;
  if (sig >= n) return;
  const int s = cnt[sig];
  if (s <= 0) return;
  if (s > RF_SMEM) {
    if ((threadIdx.x & 31) == 0) big_list[atomicAdd(big_count, 1)] = sig;
    return;
  }
  refine_one<T>(D, m, X ? X + (size_t)sig * m : nullptr, Q ? Q + (size_t)sig * ldq : nullptr, G,
                Kp, slab_ind + (size_t)sig * L, slab_val + (size_t)sig * L, s,
                level ? level + sig : nullptr, &sA[w][0][0], RF_SMEM + 1, sb[w]);
}

// Pass 2: the queued signals, a global L x (L+1) slab of doubles per warp.
template <typename T>
__global__ void __launch_bounds__(RF_WARPS * 32)
refine_big_kernel(const T* __restrict__ D, int m, const T* __restrict__ X,
                  const T* __restrict__ Q, int ldq, const T* __restrict__ G, int Kp, const int* __restrict__ slab_ind,
                  T* __restrict__ slab_val, int L, const int* __restrict__ cnt,
                  const T* __restrict__ level, const int64_t* big_list, const int* big_count,
                  unsigned* counter, double* scratch) {
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * RF_WARPS + (threadIdx.x >> 5);
  double* A = scratch + (size_t)gw * ((size_t)L * (L + 1) + L);
  double* b = A + (size_t)L * (L + 1);
  const int total = *big_count;
  for (;;) {
    int job = 0;
    if (lane == 0) job = (int)atomicAdd(counter, 1u);
    job = __shfl_sync(kFull, job, 0);
    if (job >= total) break;
    const int64_t sig = big_list[job];
    refine_one<T>(D, m, X ? X + (size_t)sig * m : nullptr, Q ? Q + (size_t)sig * ldq : nullptr,
                  G, Kp, slab_ind + (size_t)sig * L, slab_val + (size_t)sig * L, cnt[sig],
                  level ? level + sig : nullptr, A, L + 1, b);
    __syncwarp();
  }
}

size_t refine_scratch_bytes(int L, int grid) {
  return (size_t)grid * RF_WARPS * ((size_t)L * (L + 1) + L) * sizeof(double);
}

template <typename T>
cudaError_t launch_refine(const T* D, int m, const T* X, const T* Q, int ldq, const T* G, int Kp,
                          const int* slab_ind,
                          T* slab_val, int L, const int* cnt, const T* level, int64_t n,
                          int64_t* big_list, int* big_count, unsigned* counter, double* scratch,
                          int big_grid, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(big_count, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return e;
  refine_kernel<T><<<(unsigned)((n + RF_WARPS - 1) / RF_WARPS), RF_WARPS * 32, 0, st>>>(
      D, m, X, Q, ldq, G, Kp, slab_ind, slab_val, L, cnt, level, n, big_list, big_count);
  e = cudaGetLastError();
  if (e != cudaSuccess || L <= RF_SMEM) return e;
  refine_big_kernel<T><<<big_grid, RF_WARPS * 32, 0, st>>>(D, m, X, Q, ldq, G, Kp, slab_ind,
                                                           slab_val, L, cnt, level, big_list,
                                                           big_count, counter, scratch);
  return cudaGetLastError();
}

template cudaError_t launch_refine<float>(const float*, int, const float*, const float*, int,
                                          const float*, int, const int*, float*, int, const int*,
                                          const float*, int64_t, int64_t*, int*, unsigned*,
                                          double*, int, cudaStream_t);
template cudaError_t launch_refine<double>(const double*, int, const double*, const double*, int,
                                           const double*, int, const int*, double*, int,
                                           const int*, const double*, int64_t, int64_t*, int*,
                                           unsigned*, double*, int, cudaStream_t);

}  // namespace sc
