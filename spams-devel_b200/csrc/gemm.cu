// Dense products on the CUDA cores (FP32 / FP64): the correlation D^T X and
// the Gram D^T D of the plain numerical form, and small helpers.
//
// Reference: ProdMatrix (linalg/linalg.h:1021-1067, 5101-5190) computes the
// Gram with syrk (Matrix::XtX, :1967-1972) and the correlation per column
// with gemv (Matrix::multTrans, :1751-1756).  Here both are one "A^T B" GEMM
// over column-major operands whose contraction dimension (the signal length
// m) is contiguous, tiled 128 x 128 x 16 per CTA with 8 x 8 outputs a thread.
#include "common.cuh"
#include "kernels.h"

namespace sc {

constexpr int GB_M = 128, GB_N = 128;

template <typename T>
__global__ void __launch_bounds__(256)
gemm_tn_kernel(const T* __restrict__ A, int lda, int Ka, const T* __restrict__ B,
               int ldb, int64_t n, int m, T* __restrict__ C, int ldc, int Kp) {
  // contraction tile: 16 (FP32) or 8 (FP64) so both stay in 48 KB static smem
  constexpr int GB_K = sizeof(T) == 4 ? 16 : 8;
  constexpr int LCS = 256 / GB_K;  // columns loaded per pass
  constexpr int Q = GB_M / LCS;    // passes per tile
  __shared__ T As[2][GB_K][GB_M + 4];
  __shared__ T Bs[2][GB_K][GB_N + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int k0 = blockIdx.y * GB_M;          // output rows (atoms)
  const int64_t i0 = (int64_t)blockIdx.x * GB_N;  // output columns (signals)
  if (k0 >= Kp) return;

  // loader mapping: GB_K consecutive threads read consecutive r of one column
  const int lr = tid % GB_K;
  const int lc = tid / GB_K;

  T acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0;

  T ra[Q], rb[Q];
  auto load = [&](int r0) {
    const int r = r0 + lr;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int kk = k0 + lc + LCS * q;
      ra[q] = (r < m && kk < Ka) ? A[(size_t)kk * lda + r] : T(0);
      const int64_t ii = i0 + lc + LCS * q;
      rb[q] = (r < m && ii < n) ? B[(size_t)ii * ldb + r] : T(0);
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      As[buf][lr][lc + LCS * q] = ra[q];
      Bs[buf][lr][lc + LCS * q] = rb[q];
    }
  };

  const int ntiles = (m + GB_K - 1) / GB_K;
  if (ntiles == 0) goto write_out;
  load(0);
  store(0);
  __syncthreads();
  for (int t = 0; t < ntiles; ++t) {
    const int buf = t & 1;
    if (t + 1 < ntiles) load((t + 1) * GB_K);
#pragma unroll
    for (int kk = 0; kk < GB_K; ++kk) {
      T av[8], bv[8];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        av[a] = As[buf][kk][ty * 4 + a];
        av[a + 4] = As[buf][kk][64 + ty * 4 + a];
        bv[a] = Bs[buf][kk][tx * 4 + a];
        bv[a + 4] = Bs[buf][kk][64 + tx * 4 + a];
      }
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] += av[a] * bv[b];
    }
    if (t + 1 < ntiles) store(buf ^ 1);
    __syncthreads();
  }
write_out:
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int64_t ii = i0 + (b < 4 ? tx * 4 + b : 64 + tx * 4 + (b - 4));
    if (ii >= n) continue;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int kk = k0 + (a < 4 ? ty * 4 + a : 64 + ty * 4 + (a - 4));
      if (kk < Kp) C[(size_t)ii * ldc + kk] = kk < Ka ? acc[a][b] : T(0);
    }
  }
}

template <typename T>
cudaError_t launch_gemm_tn(const T* A, int lda, int Ka, const T* B, int ldb,
                           int64_t n, int m, T* C, int ldc, int Kp, cudaStream_t st) {
  if (n <= 0 || Kp <= 0) return cudaSuccess;
  const int64_t gx = (n + GB_N - 1) / GB_N;
  if (gx > 0x7fffffff) return cudaErrorInvalidValue;
  dim3 grid((unsigned)gx, (Kp + GB_M - 1) / GB_M);
  gemm_tn_kernel<T><<<grid, 256, 0, st>>>(A, lda, Ka, B, ldb, n, m, C, ldc, Kp);
  return cudaGetLastError();
}

// Mirror the upper triangle into the lower one (Matrix::fillSymmetric after
// syrk), add the ridge to the first K diagonal entries, zero the padding.
template <typename T>
__global__ void symmetrize_kernel(T* G, int K, int Kp, T ridge) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)Kp * Kp) return;
  const int r = (int)(idx % Kp), c = (int)(idx / Kp);
  if (r >= K || c >= K) { G[idx] = 0; return; }
  if (r > c) G[idx] = G[(size_t)r * Kp + c];  // (r,c) <- (c,r), c < r: upper
  else if (r == c && ridge != T(0)) G[idx] += ridge;
}

template <typename T>
cudaError_t launch_symmetrize(T* G, int K, int Kp, T ridge, cudaStream_t st) {
  const int64_t tot = (int64_t)Kp * Kp;
  symmetrize_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(G, K, Kp, ridge);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gram(const T* D, int m, int K, int Kp, T ridge, T* G, cudaStream_t st) {
  cudaError_t e = launch_gemm_tn<T>(D, m, K, D, m, K, m, G, Kp, Kp, st);
  if (e != cudaSuccess) return e;
  // columns K..Kp-1 were not written by the GEMM
  const int64_t tot = (int64_t)Kp * Kp;
  symmetrize_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(G, K, Kp, ridge);
  return cudaGetLastError();
}

template <typename T>
__global__ void colnorms_kernel(const T* X, int m, int64_t n, T* norms) {
  const int64_t col = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (col >= n) return;
  const T* x = X + (size_t)col * m;
  T s = 0;
  for (int r = lane; r < m; r += 32) s += x[r] * x[r];
  s = warp_sum(s);
  if (lane == 0) norms[col] = s;
}

template <typename T>
cudaError_t launch_colnorms(const T* X, int m, int64_t n, T* norms, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  colnorms_kernel<T><<<(unsigned)((n + 7) / 8), 256, 0, st>>>(X, m, n, norms);
  return cudaGetLastError();
}

template <typename T>
__global__ void pad_rows_kernel(const T* src, int K, int64_t ldsrc, int64_t n, T* dst, int Kp) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)Kp * n) return;
  const int r = (int)(idx % Kp);
  const int64_t c = idx / Kp;
  dst[idx] = r < K ? src[(size_t)c * ldsrc + r] : T(0);
}

template <typename T>
cudaError_t launch_pad_rows(const T* src, int K, int64_t ldsrc, int64_t n, T* dst, int Kp,
                            cudaStream_t st) {
  const int64_t tot = (int64_t)Kp * n;
  if (tot <= 0) return cudaSuccess;
  pad_rows_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(src, K, ldsrc, n, dst, Kp);
  return cudaGetLastError();
}

template cudaError_t launch_gemm_tn<float>(const float*, int, int, const float*, int, int64_t, int, float*, int, int, cudaStream_t);
template cudaError_t launch_gemm_tn<double>(const double*, int, int, const double*, int, int64_t, int, double*, int, int, cudaStream_t);
template cudaError_t launch_gram<float>(const float*, int, int, int, float, float*, cudaStream_t);
template cudaError_t launch_symmetrize<float>(float*, int, int, float, cudaStream_t);
template cudaError_t launch_gram<double>(const double*, int, int, int, double, double*, cudaStream_t);
template cudaError_t launch_colnorms<float>(const float*, int, int64_t, float*, cudaStream_t);
template cudaError_t launch_colnorms<double>(const double*, int, int64_t, double*, cudaStream_t);
template cudaError_t launch_pad_rows<float>(const float*, int, int64_t, int64_t, float*, int, cudaStream_t);
template cudaError_t launch_pad_rows<double>(const double*, int, int64_t, int64_t, double*, int, cudaStream_t);

}  // namespace sc
