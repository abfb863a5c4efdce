// Orthogonal Matching Pursuit (Cholesky / ORMP form) for every signal of a
// batch: one warp per signal, persistent grid fed by a device work counter.
//
// Restates coreORMP (decomp/decomp.h:538-640):
//   - atom choice: first index of the largest |score| (BLAS i?amax,
//     linalg/cblas_alt_template.h:787-797); scores start as D^T x, then
//     Rdn^2 / norm with the selected atoms zeroed (:624-629)
//   - stops: norm < 1e-8 (:566-569), RU^2 < 2 lambda (:570-575),
//     j == L-1 or normX <= eps (:600-603)
//   - new inverse-Cholesky column Un[:,j] = invNorm [-Un_j Undn(c,0:j); 1]
//     (:595-598).  The row Undn(c, 0:j) is not stored: it equals
//     g^T Un(0:j,0:j) with g_l = G(c, ind_l), which costs j^2/2 flops
//     instead of a K x L slab per signal.
//   - Undn(:,j) = G(:, ind(0:j)) Un(0:j, j) (:616-620), residual / norm update
//   - final coefficients Un RUn (:632-633)
//
// Lane `l` owns rows r = 128 v + 4 l + e as in the LARS kernel.
#include "common.cuh"
#include "kernels.h"
#include "masked.cuh"
#include "refactor.cuh"

namespace sc {

template <typename T, int NV, bool MASKED = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2)
omp_kernel(const OmpArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int Lc = a.Lcap;
  const int ldu = state_ld(Lc);
  const size_t per_warp = omp_state_bytes(a.Kp, Lc, sizeof(T));
  unsigned char* base =
      a.gstate ? reinterpret_cast<unsigned char*>(a.gstate) +
                     (size_t)(blockIdx.x * wpb + wib) * per_warp
               : smem_raw + (size_t)wib * per_warp;
  T* sRdn = reinterpret_cast<T*>(base);
  T* sNorm = sRdn + a.Kp;
  T* sUn = sNorm + a.Kp;  // row-major: Un(r, c) at r * ldu + c
  T* sRUn = sUn + (size_t)Lc * ldu;
  T* sVec = sRUn + Lc;
  T* sGg = sVec + Lc;
  int* sInd = reinterpret_cast<int*>(sGg + Lc);

  const int K = a.K, Kp = a.Kp;

  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;
  for (;;) {
    int job = 0;
    if (lane == 0) job = (int)atomicAdd(a.work_counter, 1u);
    job = __shfl_sync(kFull, job, 0);
    if (job >= n_jobs) break;
    const int64_t sig = a.sig_list ? a.sig_list[job] : (int64_t)job;

    const T eps = fabs(a.vEps ? a.vEps[sig] : a.eps);
    const int Ls = a.vL ? a.vL[sig] : a.Lsig;
    const int L = Ls < a.L ? Ls : a.L;  // MIN(*pL, Gs.n())
    const T lambda = a.vLambda ? a.vLambda[sig] : a.lambda;
    T normX = a.norms[sig];
    T* path = (a.path && sig == 0) ? a.path : nullptr;
    // masked variant: no row observed -> empty code; some -> the masked Gram
    const int mflag = MASKED ? (int)a.mk.flag[sig] : 2;
    const bool partial = MASKED && mflag == 1;
    const uint8_t* mrow = MASKED ? a.mk.mask + (size_t)sig * a.mk.m : nullptr;
    T* mw = MASKED ? a.mk.work + (size_t)(blockIdx.x * wpb + wib) * a.mk.mpad : nullptr;

    // ---- load D^T x; norm = 1; first choice = first max |D^T x|
    const T* dtx = a.DtX + (size_t)sig * Kp;
    T bkey = -1;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = v * 128 + lane * 4;
      const Vec4<T> d = ldg4(dtx + r0);
      st4(sRdn + r0, d);
      st4(sNorm + r0, Vec4<T>{{T(1), T(1), T(1), T(1)}});
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = r0 + e;
        if (r < K) {
          T key = fabs(d.v[e]);
          if (key != key) key = -1;  // NaN never wins
          if (key > bkey || (key == bkey && r < bidx)) { bkey = key; bidx = r; }
        }
      }
    }
    int c = warp_argmax_first(bkey, bidx);
    __syncwarp();

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
        // single-precision factor: rebuild Un, RUn and ||r||^2 in FP64
        bool refactored = false;
        const int unit = blockIdx.x * wpb + wib;
        if (sizeof(T) == 4 && a.refactor && j < a.rf_cap && unit < a.rf_units && !partial &&
            (a.refactor == 2 || !(nc > T(kRefactorPivot)))) {
          if (lane == 0) sInd[j] = c;
          __syncwarp();
          const double nx = refactor_un<T>(a.G, Kp, sInd, j + 1, a.DtX + (size_t)sig * Kp,
                                           a.norms[sig], sUn, ldu, sRUn,
                                           a.rf_scratch + (size_t)unit * a.rf_cap * a.rf_cap);
          if (nx == nx) {
            refactored = true;
            RU = sRUn[j];
            normX = (T)nx + RU * RU;  // the delta of this atom comes off below
          }
        }
        const T delta = RU * RU;
        if (delta < 2 * lambda) break;
        normX -= delta;
        if (lane == 0) { sRUn[j] = RU; sInd[j] = c; }
        if (lane == ((c & 127) >> 2)) act |= 1u << (((c >> 7) << 2) | (c & 3));
        if (refactored) {
          __syncwarp();
        } else {
        // g_l = G(c, ind_l), l < j
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
        // Undn(c, k) = sum_{l<=k} g_l Un(l, k), k < j
        for (int k = lane; k < j; k += 32) {
          T s = 0;
          for (int l = 0; l <= k; ++l) s += sGg[l] * sUn[(size_t)l * ldu + k];
          sVec[k] = s;
        }
        __syncwarp();
        // Un(0:j, j) = -invNorm * Un_j Undn(c, 0:j)^T ;  Un(j, j) = invNorm
        for (int r = lane; r < j; r += 32) {
          T s = 0;
          const T* row = sUn + (size_t)r * ldu;
          for (int k = r; k < j; ++k) s += row[k] * sVec[k];
          sUn[(size_t)r * ldu + j] = s * (-invNorm);
        }
        if (lane == 0) sUn[(size_t)j * ldu + j] = T(-1) * (-invNorm);
        __syncwarp();
        }
        if (j == L - 1 || normX <= eps) { ++j; break; }
        if (path) {
          // path(:, j) = Un_{j+1} RUn(0:j+1) scattered to the selected atoms
          for (int r = lane; r <= j; r += 32) {
            T s = 0;
            for (int k = r; k <= j; ++k) s += sUn[(size_t)r * ldu + k] * sRUn[k];
            path[(size_t)j * K + sInd[r]] = s;
          }
        }
        // ---- Undn(:, j) = G(:, ind(0:j)) Un(0:j, j)
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        if (partial) {
          masked_gram_times<T, NV>(a.mk, mrow, mw, Kp, sInd, sUn + j, ldu, j + 1, A);
        } else {
#pragma unroll 4
          for (int l = 0; l <= j; ++l) {
            const T ul = sUn[(size_t)l * ldu + j];
            const T* gc = a.G + (size_t)sInd[l] * Kp + lane * 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              const Vec4<T> g = ldg4(gc + v * 128);
#pragma unroll
              for (int e = 0; e < 4; ++e) A[v][e] += g.v[e] * ul;
            }
          }
        }
        // ---- residual correlations, norms, scores; next choice (first index
        // of the largest |score|, four independent chains merged at the end)
        const T mRU = -sRUn[j];
        T ck[4];
        int cix[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) { ck[e] = -1; cix[e] = 0x7fffffff; }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = v * 128 + lane * 4;
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
              if (key != key) key = -1;  // NaN never wins
              if (key > ck[e]) { ck[e] = key; cix[e] = r; }  // rows ascend per chain
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
        bkey = ck[0];
        bidx = cix[0];
        c = warp_argmax_first(bkey, bidx);
        __syncwarp();
      }
    }
    __syncwarp();

    if (a.steps && lane == 0 && !overflow) atomicAdd(a.steps, (unsigned long long)j);
    if (overflow) {
      if (lane == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig;
        a.out_cnt[sig] = 0;
      }
    } else {
      // coefficients = Un_j RUn(0:j), then sorted by atom index
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
    __syncwarp();
  }
}

template <typename T, int NV>
static cudaError_t launch_nv(const OmpArgs<T>& a, int grid, int wpb, size_t smem, cudaStream_t st) {
  auto k = a.mk.mask ? omp_kernel<T, NV, true> : omp_kernel<T, NV, false>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, wpb * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_omp(const OmpArgs<T>& a, int grid, int wpb, cudaStream_t st) {
  const size_t smem = a.gstate ? 0 : (size_t)wpb * omp_state_bytes(a.Kp, a.Lcap, sizeof(T));
  switch (a.Kp / 128) {
    case 1: return launch_nv<T, 1>(a, grid, wpb, smem, st);
    case 2: return launch_nv<T, 2>(a, grid, wpb, smem, st);
    case 3: return launch_nv<T, 3>(a, grid, wpb, smem, st);
    case 4: return launch_nv<T, 4>(a, grid, wpb, smem, st);
    case 5: return launch_nv<T, 5>(a, grid, wpb, smem, st);
    case 6: return launch_nv<T, 6>(a, grid, wpb, smem, st);
    case 7: return launch_nv<T, 7>(a, grid, wpb, smem, st);
    case 8: return launch_nv<T, 8>(a, grid, wpb, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T>
int omp_max_warps_per_sm(int Kp) {
  const void* fn = nullptr;
  switch (Kp / 128) {
    case 1: fn = (const void*)omp_kernel<T, 1>; break;
    case 2: fn = (const void*)omp_kernel<T, 2>; break;
    case 3: fn = (const void*)omp_kernel<T, 3>; break;
    case 4: fn = (const void*)omp_kernel<T, 4>; break;
    case 5: fn = (const void*)omp_kernel<T, 5>; break;
    case 6: fn = (const void*)omp_kernel<T, 6>; break;
    case 7: fn = (const void*)omp_kernel<T, 7>; break;
    case 8: fn = (const void*)omp_kernel<T, 8>; break;
    default: return 0;
  }
  cudaFuncAttributes attr;
  if (cudaFuncGetAttributes(&attr, fn) != cudaSuccess) return 0;
  const int regs = attr.numRegs > 0 ? attr.numRegs : 64;
  return 65536 / (regs * 32);
}

template cudaError_t launch_omp<float>(const OmpArgs<float>&, int, int, cudaStream_t);
template cudaError_t launch_omp<double>(const OmpArgs<double>&, int, int, cudaStream_t);
template int omp_max_warps_per_sm<float>(int);
template int omp_max_warps_per_sm<double>(int);

}  // namespace sc
