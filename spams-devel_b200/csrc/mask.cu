// Preparation of the masked variants (lasso_mask / omp_mask): the transposed
// dictionary that the kernels' masked Gram products read, and per signal the
// masked signal, its observation class and its scaled parameter.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace sc {

namespace {

// Dt (Kp x m, column-major) = Dᵀ with zero rows K..Kp-1.
template <typename T>
__global__ void transpose_pad_kernel(const T* __restrict__ D, int m, int K, int Kp,
                                     T* __restrict__ Dt) {
  const int64_t tot = (int64_t)Kp * m;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % Kp);
    const int r = (int)(i / Kp);
    Dt[i] = k < K ? D[(size_t)k * m + r] : T(0);
  }
}

// One warp per signal: unobserved rows of x set to zero (Vector::copyMask,
// linalg/linalg.h:4082-4090, keeps only the observed ones), flag 0 / 1 / 2
// for none / some / all rows observed, and the parameter the reference scales
// by the observed fraction: value * count / m (decomp/decomp.h:481, 1535)
// when some rows are observed and `scale` is set, value otherwise.
template <typename T>
__global__ void mask_prep_kernel(T* __restrict__ X, int m, int64_t n,
                                 const uint8_t* __restrict__ mask, int8_t* __restrict__ flag,
                                 const T* __restrict__ vbase, T base, int scale,
                                 T* __restrict__ out) {
  const int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  const uint8_t* mk = mask + (size_t)j * m;
  T* x = X + (size_t)j * m;
  int count = 0;
  for (int r = lane; r < m; r += 32) {
    if (mk[r]) ++count;
    else x[r] = T(0);
  }
  for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(kFull, count, o);
  if (lane == 0) {
    const int f = count == 0 ? 0 : (count == m ? 2 : 1);
    flag[j] = (int8_t)f;
    const T v = vbase ? vbase[j] : base;
    out[j] = (f == 1 && scale) ? (v * T(count)) / T(m) : v;
  }
}

}  // namespace

template <typename T>
cudaError_t launch_transpose_pad(const T* D, int m, int K, int Kp, T* Dt, cudaStream_t st) {
  const int64_t tot = (int64_t)Kp * m;
  if (tot <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, 148 * 16);
  transpose_pad_kernel<T><<<blocks, 256, 0, st>>>(D, m, K, Kp, Dt);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_mask_prep(T* X, int m, int64_t n, const uint8_t* mask, int8_t* flag,
                             const T* vbase, T base, int scale, T* out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  mask_prep_kernel<T><<<(unsigned)((n + 7) / 8), 256, 0, st>>>(X, m, n, mask, flag, vbase, base,
                                                               scale, out);
  return cudaGetLastError();
}

template cudaError_t launch_transpose_pad<float>(const float*, int, int, int, float*, cudaStream_t);
template cudaError_t launch_transpose_pad<double>(const double*, int, int, int, double*,
                                                  cudaStream_t);
template cudaError_t launch_mask_prep<float>(float*, int, int64_t, const uint8_t*, int8_t*,
                                             const float*, float, int, float*, cudaStream_t);
template cudaError_t launch_mask_prep<double>(double*, int, int64_t, const uint8_t*, int8_t*,
                                              const double*, double, int, double*, cudaStream_t);

}  // namespace sc
