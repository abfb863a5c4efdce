// CSC assembly: the GPU form of SpMatrix::convert (linalg/linalg.h:4840-4861).
// The coding kernels leave, per signal, its active-set size and its (atom,
// coefficient) pairs already sorted by atom index in an n x L slab; here the
// sizes are scanned into column pointers and the pairs are gathered into the
// contiguous row / value arrays, one warp per column.
//
// Also here: the longest-first order of a persistent launch over signals with
// per-signal step caps L_i (a counting sort by descending L_i), so that the
// signals with the most steps start first and the shortest ones fill the tail.
#include "common.cuh"
#include "kernels.h"

namespace sc {

constexpr int SCAN_BLOCK = 1024;  // elements per block (one per thread)

__global__ void block_sums_kernel(const int* cnt, int64_t n, int64_t* sums) {
  __shared__ int64_t red[32];
  const int64_t i = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
  int64_t v = i < n ? cnt[i] : 0;
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t w = red[threadIdx.x];
    w = warp_sum(w);
    if (threadIdx.x == 0) sums[blockIdx.x] = w;
  }
}

// Exclusive scan of nb block sums in place, one block of 1024 threads.
__global__ void scan_sums_kernel(int64_t* sums, int64_t nb) {
  __shared__ int64_t wsum[32];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nb; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < nb ? sums[i] : 0;
    int64_t x = v;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      int64_t w = wsum[threadIdx.x];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += y;
      }
      wsum[threadIdx.x] = w;
    }
    __syncthreads();
    const int64_t incl = x + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0);
    if (i < nb) sums[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
}

__global__ void scan_final_kernel(const int* cnt, int64_t n, const int64_t* sums,
                                  int64_t* colptr, const int64_t* base) {
  __shared__ int64_t wsum[32];
  const int64_t i = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int64_t v = i < n ? cnt[i] : 0;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t w = wsum[threadIdx.x];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += y;
    }
    wsum[threadIdx.x] = w;
  }
  __syncthreads();
  const int64_t incl = x + ((threadIdx.x >> 5) ? wsum[(threadIdx.x >> 5) - 1] : 0);
  const int64_t off = sums[blockIdx.x] + (base ? *base : 0);
  if (i < n) colptr[i + 1] = off + incl;
  if (i == 0 && !base) colptr[0] = 0;
}

int64_t scan_scratch_len(int64_t n) { return (n + SCAN_BLOCK - 1) / SCAN_BLOCK + 1; }

cudaError_t launch_scan_counts(const int* cnt, int64_t n, int64_t* colptr, const int64_t* base,
                               int64_t* scratch, int64_t scratch_len, cudaStream_t st) {
  if (n <= 0) {
    if (!base) return cudaMemsetAsync(colptr, 0, sizeof(int64_t), st);
    return cudaSuccess;
  }
  const int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  if (scratch_len < nb) return cudaErrorInvalidValue;
  block_sums_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, st>>>(cnt, n, scratch);
  scan_sums_kernel<<<1, 1024, 0, st>>>(scratch, nb);
  scan_final_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, st>>>(cnt, n, scratch, colptr, base);
  return cudaGetLastError();
}

template <typename T>
__global__ void csc_gather_kernel(const int* slab_ind, const T* slab_val, int L,
                                  const int* cnt, const int64_t* colptr, int64_t n,
                                  const int64_t* sub, int64_t cap, int* capflag,
                                  int32_t* rows, T* vals) {
  const int64_t col = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (col >= n) return;
  const int c = cnt[col];
  const int64_t dst = colptr[col] - (sub ? *sub : 0);
  if (dst < 0 || dst + c > cap) {  // caller's arrays too small: record, write nothing
    if (lane == 0 && c > 0) atomicExch(capflag, 1);
    return;
  }
  const int* si = slab_ind + (size_t)col * L;
  const T* sv = slab_val + (size_t)col * L;
  for (int j = lane; j < c; j += 32) {
    rows[dst + j] = si[j];
    vals[dst + j] = sv[j];
  }
}

template <typename T>
cudaError_t launch_csc_gather(const int* slab_ind, const T* slab_val, int L, const int* cnt,
                              const int64_t* colptr, int64_t n, const int64_t* sub, int64_t cap,
                              int* capflag, int32_t* rows, T* vals, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  csc_gather_kernel<T><<<(unsigned)((n + 7) / 8), 256, 0, st>>>(
      slab_ind, slab_val, L, cnt, colptr, n, sub, cap, capflag, rows, vals);
  return cudaGetLastError();
}

// ---- longest-first order: bin k holds the signals with min(L_i, Lmax) = Lmax - k
__device__ __forceinline__ int order_bin(const int* vL, int64_t i, int Lmax) {
  const int l = vL[i];
  return Lmax - (l < 0 ? 0 : (l > Lmax ? Lmax : l));
}

__global__ void order_hist_kernel(const int* vL, int64_t n, int Lmax, int* hist) {
  extern __shared__ int sh[];
  const int nb = Lmax + 1;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) sh[b] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&sh[order_bin(vL, i, Lmax)], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// Exclusive scan of the nb bin counts in place (one block).
__global__ void order_scan_kernel(int* hist, int nb) {
  if (threadIdx.x != 0) return;
  int run = 0;
  for (int b = 0; b < nb; ++b) {
    const int v = hist[b];
    hist[b] = run;
    run += v;
  }
}

// Tiles of blockDim signals: each tile reserves its range of every bin with
// one global atomic per bin, then places its signals in it.
__global__ void order_scatter_kernel(const int* vL, int64_t n, int Lmax, int* offs,
                                     int64_t* list) {
  extern __shared__ int sh[];
  const int nb = Lmax + 1;
  int* scnt = sh;
  int* sbase = sh + nb;
  for (int64_t t0 = (int64_t)blockIdx.x * blockDim.x; t0 < n; t0 += (int64_t)gridDim.x * blockDim.x) {
    for (int b = threadIdx.x; b < nb; b += blockDim.x) scnt[b] = 0;
    __syncthreads();
    const int64_t i = t0 + threadIdx.x;
    const int b = i < n ? order_bin(vL, i, Lmax) : 0;
    const int local = i < n ? atomicAdd(&scnt[b], 1) : 0;
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
      if (scnt[k]) sbase[k] = atomicAdd(&offs[k], scnt[k]);
    __syncthreads();
    if (i < n) list[sbase[b] + local] = i;
    __syncthreads();
  }
}

cudaError_t launch_order_by_L_desc(const int* vL, int64_t n, int Lmax, int* scratch,
                                   int64_t* list, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (Lmax < 0 || Lmax > kOrderMaxL) return cudaErrorInvalidValue;
  const int nb = Lmax + 1;
  cudaError_t e = cudaMemsetAsync(scratch, 0, (size_t)nb * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (n + 255) / 256;
  const unsigned blocks = (unsigned)(tiles < 148 * 8 ? tiles : 148 * 8);
  order_hist_kernel<<<blocks, 256, (size_t)nb * sizeof(int), st>>>(vL, n, Lmax, scratch);
  order_scan_kernel<<<1, 32, 0, st>>>(scratch, nb);
  order_scatter_kernel<<<blocks, 256, (size_t)2 * nb * sizeof(int), st>>>(vL, n, Lmax, scratch,
                                                                          list);
  return cudaGetLastError();
}

template cudaError_t launch_csc_gather<float>(const int*, const float*, int, const int*,
                                              const int64_t*, int64_t, const int64_t*, int64_t,
                                              int*, int32_t*, float*, cudaStream_t);
template cudaError_t launch_csc_gather<double>(const int*, const double*, int, const int*,
                                               const int64_t*, int64_t, const int64_t*, int64_t,
                                               int*, int32_t*, double*, cudaStream_t);

}  // namespace sc
