// OMP for large dictionaries: one CTA of W warps per signal.
//
// The same Cholesky-form OMP as the warp-per-signal kernel (omp.cu; coreORMP,
// decomp/decomp.h:538-640) with the K rows of the residual correlations and
// atom norms split over W warps (warp w owns rows w*512 + 128 v + 4 lane + e).
// The inverse Cholesky factor and the selection bookkeeping sit once per CTA
// and are updated by warp 0; every warp updates its rows with the new
// orthogonal direction and proposes its best atom; a W-entry exchange picks
// the first index of the largest score.  Used for Kp = 512 .. 4096 and 6144,
// 8192, 12288, 16384 (W = Kp / 512: 1..8, 12, 16, 24, 32 warps).
#include "common.cuh"
#include "kernels.h"
#include "refactor.cuh"
#include "masked.cuh"

namespace sc {

// Small state: Un (Lc x ldu), RUn / vec / g (Lc each), ind (Lc).
__host__ __device__ inline size_t omp_cta_state(int Lc, size_t esz) {
  return align16(esz * ((size_t)Lc * state_ld(Lc) + 3 * (size_t)Lc) + 4 * (size_t)Lc);
}
// Shared memory: residual correlations and norms (2 Kp), exchange slots, the
// small state unless it lives in a global slab.
__host__ __device__ inline size_t omp_cta_smem(int Kp, int Lc, size_t esz, int W, bool gstate) {
  return align16(esz * (2 * (size_t)Kp + W) + 4 * ((size_t)W + 4)) +
         (gstate ? 0 : omp_cta_state(Lc, esz));
}

template <typename T, int W, bool MASKED>
__device__ __forceinline__ void omp_cta_body(const OmpArgs<T> a) {
  constexpr int NV = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int gw = threadIdx.x >> 5;
  const int Lc = a.Lcap;
  const int ldu = state_ld(Lc);
  T* sRdn = reinterpret_cast<T*>(smem_raw);
  T* sNorm = sRdn + a.Kp;
  T* exK = sNorm + a.Kp;
  int* exI = reinterpret_cast<int*>(exK + W);
  int* sIScal = exI + W;  // [0] job
  unsigned char* st_base =
      a.gstate ? reinterpret_cast<unsigned char*>(a.gstate) +
                     (size_t)blockIdx.x * omp_cta_state(Lc, sizeof(T))
               : smem_raw + align16(sizeof(T) * (2 * (size_t)a.Kp + W) + 4 * ((size_t)W + 4));
  T* sUn = reinterpret_cast<T*>(st_base);  // row-major: Un(r, c) at r * ldu + c
  T* sRUn = sUn + (size_t)Lc * ldu;
  T* sVec = sRUn + Lc;
  T* sGg = sVec + Lc;
  int* sInd = reinterpret_cast<int*>(sGg + Lc);

  const int K = a.K, Kp = a.Kp;
  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;
  const int rbase = gw * NV * 128;
  auto own_w = [](int r) { return r / (NV * 128); };
  auto own_l = [](int r) { return (r & 127) >> 2; };
  auto own_b = [](int r) { return (((r % (NV * 128)) >> 7) << 2) | (r & 3); };

  for (;;) {
    if (threadIdx.x == 0) sIScal[0] = (int)atomicAdd(a.work_counter, 1u);
    __syncthreads();
    const int job = sIScal[0];
    if (job >= n_jobs) break;
    const int64_t sig = a.sig_list ? a.sig_list[job] : (int64_t)job;

    const T eps = fabs(a.vEps ? a.vEps[sig] : a.eps);
    const int Ls = a.vL ? a.vL[sig] : a.Lsig;
    const int L = Ls < a.L ? Ls : a.L;
    const T lambda = a.vLambda ? a.vLambda[sig] : a.lambda;
    T normX = a.norms[sig];
    T* path = (a.path && sig == 0) ? a.path : nullptr;
    // masked variant: no row observed -> empty code; some -> the masked Gram
    const int mflag = MASKED ? (int)a.mk.flag[sig] : 2;
    const bool partial = MASKED && mflag == 1;
    const uint8_t* mrow = MASKED ? a.mk.mask + (size_t)sig * a.mk.m : nullptr;
    T* mw = MASKED ? a.mk.work + (size_t)blockIdx.x * a.mk.mpad : nullptr;

    // ---- load D^T x; norm = 1; first choice = first max |D^T x|
    const T* dtx = a.DtX + (size_t)sig * Kp;
    T bkey = -1;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = rbase + v * 128 + lane * 4;
      const Vec4<T> d = ldg4(dtx + r0);
      st4(sRdn + r0, d);
      st4(sNorm + r0, Vec4<T>{{T(1), T(1), T(1), T(1)}});
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = r0 + e;
        if (r < K) {
          T key = fabs(d.v[e]);
          if (key != key) key = -1;
          if (key > bkey || (key == bkey && r < bidx)) { bkey = key; bidx = r; }
        }
      }
    }
    auto exchange_max = [&](T key, int idx) {
      const int wi = warp_argmax_first(key, idx);
      const unsigned who = __ballot_sync(kFull, idx == wi);
      const T wk = __shfl_sync(kFull, key, who ? __ffs(who) - 1 : 0);
      if (lane == 0) { exK[gw] = wk; exI[gw] = wi; }
      __syncthreads();
      T bk = exK[0];
      int bi = exI[0];
      for (int w = 1; w < W; ++w)
        if (exK[w] > bk || (exK[w] == bk && exI[w] < bi)) { bk = exK[w]; bi = exI[w]; }
      return bi;
    };
    int c = exchange_max(bkey, bidx);

    int j = 0;
    bool overflow = false;
    uint32_t act = 0;
    const bool started = !(normX <= eps || L <= 0 || mflag == 0);
    if (started) {
      for (j = 0; j < L; ++j) {
        if (j >= Lc) { overflow = true; break; }
        const T nc = sNorm[c];
        if (nc < 1e-8) break;
        const T invNorm = T(1) / sqrt(nc);
        T RU = sRdn[c] * invNorm;
        // a small pivot (the atom's residual norm) loses digits in the
        // single-precision factor: warp 0 rebuilds Un, RUn and ||r||^2 in FP64
        // (the decision is the same in every warp: nc comes from shared memory)
        bool refactored = false;
        if (sizeof(T) == 4 && a.refactor && j < a.rf_cap && (int)blockIdx.x < a.rf_units &&
            !partial && (a.refactor == 2 || !(nc > T(kRefactorPivot)))) {
          if (gw == 0) {
            if (lane == 0) sInd[j] = c;
            __syncwarp();
            const double nx = refactor_un<T>(a.G, Kp, sInd, j + 1, a.DtX + (size_t)sig * Kp,
                                             a.norms[sig], sUn, ldu, sRUn,
                                             a.rf_scratch + (size_t)blockIdx.x * a.rf_cap * a.rf_cap);
            if (lane == 0) exK[0] = (T)nx;
          }
          __syncthreads();
          const T nx = exK[0];
          __syncthreads();  // exK is reused by the next exchange
          if (nx == nx) {
            refactored = true;
            RU = sRUn[j];
            normX = nx + RU * RU;  // the delta of this atom comes off below
          }
        }
        const T delta = RU * RU;
        if (delta < 2 * lambda) break;
        normX -= delta;
        if (gw == own_w(c) && lane == own_l(c)) act |= 1u << own_b(c);
        if (gw == 0 && refactored) {
          if (lane == 0) { sRUn[j] = RU; sInd[j] = c; }
          __syncwarp();
        } else if (gw == 0) {
          if (lane == 0) { sRUn[j] = RU; sInd[j] = c; }
          if (partial) {
            for (int l = 0; l < j; ++l) {
              const T g = masked_gram(a.mk, mrow, sInd[l], c);
              if (lane == 0) sGg[l] = g;
            }
          } else {
            const T* gcol = a.G + (size_t)c * Kp;
            for (int l = lane; l < j; l += 32) sGg[l] = gcol[sInd[l]];
          }
          __syncwarp();
          for (int k = lane; k < j; k += 32) {
            T s = 0;
            for (int l = 0; l <= k; ++l) s += sGg[l] * sUn[(size_t)l * ldu + k];
            sVec[k] = s;
          }
          __syncwarp();
          for (int r = lane; r < j; r += 32) {
            T s = 0;
            const T* row = sUn + (size_t)r * ldu;
            for (int k = r; k < j; ++k) s += row[k] * sVec[k];
            sUn[(size_t)r * ldu + j] = s * (-invNorm);
          }
          if (lane == 0) sUn[(size_t)j * ldu + j] = T(-1) * (-invNorm);
          __syncwarp();
        }
        __syncthreads();
        if (j == L - 1 || normX <= eps) { ++j; break; }
        if (path && gw == 0) {
          for (int r = lane; r <= j; r += 32) {
            T s = 0;
            for (int k = r; k <= j; ++k) s += sUn[(size_t)r * ldu + k] * sRUn[k];
            path[(size_t)j * K + sInd[r]] = s;
          }
        }
        // ---- Undn(:, j) on the own rows, residual / norm update, scores
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        if (partial) {
          masked_gram_times_cta<T, NV, W>(a.mk, mrow, mw, Kp, rbase, sInd, sUn + j, ldu, j + 1, A);
        } else {
#pragma unroll 4
          for (int l = 0; l <= j; ++l) {
            const T ul = sUn[(size_t)l * ldu + j];
            const T* gc = a.G + (size_t)sInd[l] * Kp + rbase + lane * 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) axpy4(A[v], ldg4(gc + v * 128), ul);
          }
        }
        const T mRU = -sRUn[j];
        T ck[4];
        int cix[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) { ck[e] = -1; cix[e] = 0x7fffffff; }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = rbase + v * 128 + lane * 4;
          Vec4<T> rd = ld4(sRdn + r0);
          Vec4<T> nm = ld4(sNorm + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const T u = A[v][e];
            rd.v[e] += u * mRU;
            nm.v[e] -= u * u;
            const int r = r0 + e;
            if (r < K) {
              T sc = (rd.v[e] * rd.v[e]) / nm.v[e];
              if ((act >> (v * 4 + e)) & 1u) sc = 0;
              T key = fabs(sc);
              if (key != key) key = -1;
              if (key > ck[e]) { ck[e] = key; cix[e] = r; }
            }
          }
          st4(sRdn + r0, rd);
          st4(sNorm + r0, nm);
        }
#pragma unroll
        for (int h = 1; h < 4; h <<= 1)
#pragma unroll
          for (int e = 0; e + h < 4; e += 2 * h)
            if (ck[e + h] > ck[e] || (ck[e + h] == ck[e] && cix[e + h] < cix[e])) {
              ck[e] = ck[e + h];
              cix[e] = cix[e + h];
            }
        c = exchange_max(ck[0], cix[0]);
      }
    }
    __syncthreads();

    if (threadIdx.x == 0 && a.steps && !overflow) atomicAdd(a.steps, (unsigned long long)j);
    if (overflow) {
      if (threadIdx.x == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig;
        a.out_cnt[sig] = 0;
      }
    } else if (gw == 0) {
      const int cnt = j;
      for (int r = lane; r < cnt; r += 32) {
        T s = 0;
        for (int k = r; k < cnt; ++k) s += sUn[(size_t)r * ldu + k] * sRUn[k];
        sVec[r] = s;
      }
      __syncwarp();
      int* oind = a.out_ind + (size_t)sig * a.L;
      T* oval = a.out_val + (size_t)sig * a.L;
      for (int r = lane; r < cnt; r += 32) {
        const int me = sInd[r];
        int rank = 0;
        for (int k = 0; k < cnt; ++k) rank += sInd[k] < me;
        oind[rank] = me;
        oval[rank] = sVec[r];
      }
      if (lane == 0) a.out_cnt[sig] = cnt;
      if (path && started) {
        for (int r = lane; r < L; r += 32) path[(size_t)(L - 1) * K + r] = 0;
        __syncwarp();
        for (int r = lane; r < cnt; r += 32) path[(size_t)(cnt - 1) * K + sInd[r]] = sVec[r];
      }
    }
    __syncthreads();
  }
}

template <typename T, int W, bool MASKED = false>
__global__ void __launch_bounds__(W * 32) omp_cta_kernel(const OmpArgs<T> a) {
  omp_cta_body<T, W, MASKED>(a);
}
// The same kernel built with at most 64 registers, so that up to 32 warps per
// SM can be resident (the per-step Gram-column reads from L2 need the
// parallelism).  The launcher takes it only where it raises residency, i.e.
// where shared memory is not the limit (small active-set capacity): 1.86 ->
// 1.40 ms per 20k signals of 18-step OMP on 1024 atoms, 5.87 -> 5.15 on 4096;
// with an 80-atom state it fits no more CTAs and its spills cost 5%.
template <typename T, int W, bool MASKED = false>
__global__ void __launch_bounds__(W * 32, 32 / W) omp_cta_kernel_lb(const OmpArgs<T> a) {
  omp_cta_body<T, W, MASKED>(a);
}

template <typename T, int W, bool MASKED>
static auto pick_omp_cta(size_t smem) {
  auto k = omp_cta_kernel<T, W, MASKED>;
  if constexpr (sizeof(T) == 4)
    k = more_resident(k, omp_cta_kernel_lb<T, W, MASKED>, W * 32, smem);
  return k;
}

template <typename T, int W>
static cudaError_t launch_w(const OmpArgs<T>& a, int grid, size_t smem, cudaStream_t st) {
  auto k = a.mk.mask ? pick_omp_cta<T, W, true>(smem) : pick_omp_cta<T, W, false>(smem);
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  e = fill_grid(k, W * 32, smem, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T, int W>
static int grid_w(size_t smem) {
  auto k = omp_cta_kernel<T, W>;
  if constexpr (sizeof(T) == 4) k = more_resident(k, omp_cta_kernel_lb<T, W>, W * 32, smem);
  int grid = 0;
  if (allow_smem(k, smem) != cudaSuccess || fill_grid(k, W * 32, smem, &grid) != cudaSuccess)
    return 0;
  return grid;
}

template <typename T>
int omp_cta_grid(int Kp, int Lc, bool gstate) {
  const size_t smem = omp_cta_smem(Kp, Lc, sizeof(T), Kp / 512, gstate);
  switch (Kp / 512) {
    case 1: return grid_w<T, 1>(smem);
    case 2: return grid_w<T, 2>(smem);
    case 3: return grid_w<T, 3>(smem);
    case 4: return grid_w<T, 4>(smem);
    case 5: return grid_w<T, 5>(smem);
    case 6: return grid_w<T, 6>(smem);
    case 7: return grid_w<T, 7>(smem);
    case 8: return grid_w<T, 8>(smem);
    case 12: return grid_w<T, 12>(smem);
    case 16: return grid_w<T, 16>(smem);
    case 24: return grid_w<T, 24>(smem);
    case 32: return grid_w<T, 32>(smem);
    default: return 0;
  }
}

template <typename T>
size_t omp_cta_smem_bytes(int Kp, int Lc, bool gstate) {
  return omp_cta_smem(Kp, Lc, sizeof(T), Kp / 512, gstate);
}
template <typename T>
size_t omp_cta_gstate_bytes(int Lc, int grid) {
  return (size_t)grid * omp_cta_state(Lc, sizeof(T));
}

template <typename T>
cudaError_t launch_omp_cta(const OmpArgs<T>& a, int grid, cudaStream_t st) {
  if (a.Kp % 512 != 0) return cudaErrorInvalidValue;
  const size_t smem = omp_cta_smem_bytes<T>(a.Kp, a.Lcap, a.gstate != nullptr);
  switch (a.Kp / 512) {
    case 1: return launch_w<T, 1>(a, grid, smem, st);
    case 2: return launch_w<T, 2>(a, grid, smem, st);
    case 3: return launch_w<T, 3>(a, grid, smem, st);
    case 4: return launch_w<T, 4>(a, grid, smem, st);
    case 5: return launch_w<T, 5>(a, grid, smem, st);
    case 6: return launch_w<T, 6>(a, grid, smem, st);
    case 7: return launch_w<T, 7>(a, grid, smem, st);
    case 8: return launch_w<T, 8>(a, grid, smem, st);
    case 12: return launch_w<T, 12>(a, grid, smem, st);
    case 16: return launch_w<T, 16>(a, grid, smem, st);
    case 24: return launch_w<T, 24>(a, grid, smem, st);
    case 32: return launch_w<T, 32>(a, grid, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template size_t omp_cta_smem_bytes<float>(int, int, bool);
template size_t omp_cta_smem_bytes<double>(int, int, bool);
template int omp_cta_grid<float>(int, int, bool);
template int omp_cta_grid<double>(int, int, bool);
template size_t omp_cta_gstate_bytes<float>(int, int);
template size_t omp_cta_gstate_bytes<double>(int, int);
template cudaError_t launch_omp_cta<float>(const OmpArgs<float>&, int, cudaStream_t);
template cudaError_t launch_omp_cta<double>(const OmpArgs<double>&, int, cudaStream_t);

}  // namespace sc
