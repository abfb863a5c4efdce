// LARS-Lasso for large dictionaries: one CTA of W warps per signal.
//
// The same homotopy as the warp-per-signal kernel (lars.cu; coreLARS2,
// decomp/decomp.h:1706-1915) with the K rows split over W warps: warp w owns
// rows w*512 + 128 v + 4 lane + e (v < 4, e < 4).  The per-signal small
// matrices (inverse Gram, direction, active set) sit once in the CTA's shared
// memory and are updated by warp 0; the row work (A = G_A u, the joining-step
// candidates, the correlation update) runs on all warps; cross-warp
// arg-minima go through a W-entry exchange.  Every thread derives the step
// and the control flow from the same shared values, so they agree bitwise.
// Used for Kp = 512 .. 4096 and 6144, 8192, 12288, 16384 (W = Kp / 512: 1..8,
// 12, 16, 24, 32 warps) and active-set capacities up to L.
#include "common.cuh"
#include "kernels.h"
#include "refactor.cuh"
#include "masked.cuh"
#include "lars_screen.cuh"

namespace sc {

namespace {

template <typename T> __device__ __forceinline__ T mn_ref(T a, T b) { return a > b ? b : a; }

template <typename T>
__device__ __forceinline__ T dot_row_c(const T* __restrict__ row, const T* __restrict__ x, int n) {
  T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int c = 0;
  for (; c + 4 <= n; c += 4) {
    s0 += row[c] * x[c];
    s1 += row[c + 1] * x[c + 1];
    s2 += row[c + 2] * x[c + 2];
    s3 += row[c + 3] * x[c + 3];
  }
  for (; c < n; ++c) s0 += row[c] * x[c];
  return (s0 + s1) + (s2 + s3);
}

}  // namespace

// Per-signal small state: the inverse Gram (Lc x ldi), u / coef / sign / cA /
// w / g (Lc each), ind (Lc).  In shared memory after the correlations, or in a
// global slab per CTA for the overflow pass.
__host__ __device__ inline size_t lars_cta_state(int Lc, size_t esz) {
  return align16(esz * ((size_t)Lc * state_ld(Lc) + 6 * (size_t)Lc) + 4 * (size_t)Lc);
}
// Shared memory of one CTA: Kp correlations, W exchange slots, the small
// state unless it lives in global memory.
__host__ __device__ inline size_t lars_cta_smem(int Kp, int Lc, size_t esz, int W, bool gstate) {
  return align16(esz * ((size_t)Kp + 2 * W + 4) + 4 * ((size_t)W + 4)) +
         (gstate ? 0 : lars_cta_state(Lc, esz));
}

template <typename T, int W, bool MASKED>
__device__ __forceinline__ void lars_cta_body(const LarsArgs<T> a) {
  constexpr int NV = 4;  // 128-row chunks per warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int gw = threadIdx.x >> 5;
  const int Lc = a.Lcap;
  const int ldi = state_ld(Lc);
  T* sDtR = reinterpret_cast<T*>(smem_raw);
  T* exK = sDtR + a.Kp;    // W keys
  T* exV = exK + W;        // W carried values
  T* sScal = exV + W;      // [0] step_max
  int* exI = reinterpret_cast<int*>(sScal + 4);  // W indices
  int* sIScal = exI + W;   // [0] first_zero, [1] job
  unsigned char* st_base =
      a.gstate ? reinterpret_cast<unsigned char*>(a.gstate) +
                     (size_t)blockIdx.x * lars_cta_state(Lc, sizeof(T))
               : smem_raw + align16(sizeof(T) * ((size_t)a.Kp + 2 * W + 4) + 4 * ((size_t)W + 4));
  T* sInv = reinterpret_cast<T*>(st_base);
  T* sU = sInv + (size_t)Lc * ldi;
  T* sCoef = sU + Lc;
  T* sS = sCoef + Lc;
  T* sCA = sS + Lc;
  T* sW = sCA + Lc;
  T* sG = sW + Lc;
  int* sInd = reinterpret_cast<int*>(sG + Lc);

  const int K = a.K, Kp = a.Kp;
  const T INF = inf<T>();
  const int L = a.L < K ? a.L : K;
  const int length_path = a.length_path <= 1 ? 4 * L : a.length_path;
  const int mode = a.mode;
  const bool pos = a.pos != 0;
  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;
  const int rbase = gw * NV * 128;

  uint32_t pad_act = 0;
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (rbase + v * 128 + lane * 4 + e >= K) pad_act |= 1u << (v * 4 + e);
  // owner (warp, lane, bit) of row r
  auto own_w = [](int r) { return r / (NV * 128); };
  auto own_l = [](int r) { return (r & 127) >> 2; };
  auto own_b = [](int r) { return (((r % (NV * 128)) >> 7) << 2) | (r & 3); };

  for (;;) {
    if (threadIdx.x == 0) sIScal[1] = (int)atomicAdd(a.work_counter, 1u);
    __syncthreads();
    const int job = sIScal[1];
    if (job >= n_jobs) break;
    const int64_t sig = a.sig_list ? a.sig_list[job] : (int64_t)job;
    const T constraint = a.vConstraint ? a.vConstraint[sig] : a.constraint;
    T* path = (a.path && sig == 0) ? a.path : nullptr;
    // masked variant: no row observed -> empty code; some -> the masked Gram
    const int mflag = MASKED ? (int)a.mk.flag[sig] : 2;
    const bool partial = MASKED && mflag == 1;
    const uint8_t* mrow = MASKED ? a.mk.mask + (size_t)sig * a.mk.m : nullptr;
    T* mw = MASKED ? a.mk.work + (size_t)blockIdx.x * a.mk.mpad : nullptr;

    // ---- load D^T x (own rows) and find the first atom
    const T* dtx = a.DtX + (size_t)sig * Kp;
    T bkey = -INF;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = rbase + v * 128 + lane * 4;
      const Vec4<T> d = ldg4(dtx + r0);
      st4(sDtR + r0, d);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = r0 + e;
        if (r < K) {
          T key = pos ? d.v[e] : fabs(d.v[e]);
          if (key != key) key = -INF;
          if (key > bkey || (key == bkey && r < bidx)) { bkey = key; bidx = r; }
        }
      }
    }
    {
      const int wi = warp_argmax_first(bkey, bidx);
      T wk = __shfl_sync(kFull, bkey, 0);
      // the key of the warp's winner: the lane holding it
      const unsigned who = __ballot_sync(kFull, bidx == wi);
      wk = __shfl_sync(kFull, bkey, who ? __ffs(who) - 1 : 0);
      if (lane == 0) { exK[gw] = wk; exI[gw] = wi; }
    }
    for (int j = threadIdx.x; j < Lc; j += W * 32) sCoef[j] = 0;
    __syncthreads();
    int cur;
    {
      T bk = exK[0];
      int bi = exI[0];
      for (int w = 1; w < W; ++w)
        if (exK[w] > bk || (exK[w] == bk && exI[w] < bi)) { bk = exK[w]; bi = exI[w]; }
      cur = bi;
    }
    T normX = a.norms[sig];

    int cnt = 0;
    bool overflow = false;
    bool skip = L <= 0 || mflag == 0;
    if (!skip) {
      const T dc = sDtR[cur];
      if (mode == 2 && fabs(dc) < constraint) skip = true;
      if (mode == 1 && normX < constraint) skip = true;
    }

    uint32_t act = pad_act;
    int iter = 0;
    T c_end = 0;
    bool at_lambda = false;
    if (!skip) {
      bool newAtom = true;
      T thrs = 0;
      for (int i = 0; i < L; ++i) {
        ++iter;
        if (newAtom) {
          if (i >= Lc) { overflow = true; break; }
          ++cnt;
          if (gw == own_w(cur) && lane == own_l(cur)) act |= 1u << own_b(cur);
          if (gw == 0) {
            if (lane == 0) sInd[i] = cur;
            __syncwarp();
            if (partial) {
              for (int j = 0; j <= i; ++j) {
                const T g = masked_gram(a.mk, mrow, sInd[j], cur);
                if (lane == 0) sG[j] = g;
              }
            } else {
              const T* gcol = a.G + (size_t)cur * Kp;
              for (int j = lane; j <= i; j += 32) sG[j] = gcol[sInd[j]];
            }
            __syncwarp();
            if (i == 0) {
              if (lane == 0) sInv[0] = T(1) / sG[0];
            } else {
              for (int r = lane; r < i; r += 32) sW[r] = dot_row_c(sInv + (size_t)r * ldi, sG, i);
              __syncwarp();
              T part = 0;
              for (int r = lane; r < i; r += 32) part += sW[r] * sG[r];
              const T dot = warp_sum(part);
              const T piv = sG[i] - dot;
              // a small pivot loses digits in the update: rebuild the inverse in FP64
              bool refactored = false;
              if (sizeof(T) == 4 && a.refactor && i < a.rf_cap && (int)blockIdx.x < a.rf_units &&
                  !partial && (a.refactor == 2 || !(piv > T(kRefactorPivot) * sG[i]))) {
                double* rs = a.rf_scratch + (size_t)blockIdx.x * a.rf_cap * a.rf_cap;
                refactored = refactor_inverse<T>(a.G, Kp, sInd, i + 1, sInv, ldi, rs);
              }
              const T schur = T(1) / piv;
              if (!refactored) for (int r = lane; r < i; r += 32) {
                T* row = sInv + (size_t)r * ldi;
                const T wr = sW[r];
                for (int c = 0; c < i; ++c) {
                  const T whi = c > r ? sW[c] : wr;
                  const T wlo = c > r ? wr : sW[c];
                  row[c] += (schur * whi) * wlo;
                }
                const T off = (-schur) * wr;
                row[i] = off;
                sInv[(size_t)i * ldi + r] = off;
              }
              if (lane == 0 && !refactored) sInv[(size_t)i * ldi + i] = schur;
            }
            __syncwarp();
          }
        }
        // ---- direction u = invGs sign(DtR_A), zero crossings (warp 0)
        if (gw == 0) {
          for (int j = lane; j <= i; j += 32) {
            const T d = sDtR[sInd[j]];
            sCA[j] = d;
            sS[j] = d > 0 ? T(1) : T(-1);
          }
          __syncwarp();
          T zkey = INF;
          int zidx = -1;
          for (int r = lane; r <= i; r += 32) {
            const T s = dot_row_c(sInv + (size_t)r * ldi, sS, i + 1);
            sU[r] = s;
            const T ratio = -sCoef[r] / s;
            if (ratio > 0 && ratio <= zkey) { zkey = ratio; zidx = r; }
          }
          const ArgRes<T> zr = warp_argmin_last_u(zkey, zidx);
          if (lane == 0) { sScal[0] = zr.val; sIScal[0] = zr.idx; }
        }
        __syncthreads();
        const T step_max = sScal[0];
        const int first_zero = sIScal[0];
        const T C = fabs(sCA[0]);
        c_end = C;

        // ---- A = Ga u on the own rows
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        if (partial) {
          masked_gram_times_cta<T, NV, W>(a.mk, mrow, mw, Kp, rbase, sInd, sU, 1, i + 1, A);
        } else {
#pragma unroll 4
          for (int j = 0; j <= i; ++j) {
            const T uj = sU[j];
            const T* gc = a.G + (size_t)sInd[j] * Kp + rbase + lane * 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) axpy4(A[v], ldg4(gc + v * 128), uj);
          }
        }
        // ---- joining candidates of the own rows (lars_screen.cuh)
        {
          const ScreenBest<T> sb =
              lars_screen<NV>(A, sDtR + rbase + lane * 4, rbase + lane * 4, act, C, pos, K);
          const ArgRes<T> mr = warp_argmin_first(sb.key, sb.idx, sb.val);
          if (lane == 0) { exK[gw] = fabs(mr.val) < INF ? fabs(mr.val) : INF; exV[gw] = mr.val; exI[gw] = mr.idx; }
        }
        __syncthreads();
        T step;
        {
          T bk = exK[0], bv = exV[0];
          int bi = exI[0];
          for (int w = 1; w < W; ++w)
            if (exK[w] < bk || (exK[w] == bk && exI[w] < bi)) { bk = exK[w]; bi = exI[w]; bv = exV[w]; }
          step = bv;
          cur = join_atom(bi, K);
        }
        // ---- polynomial of normX along the step (every warp, same result)
        T p1 = 0, p2 = 0;
        for (int j = lane; j <= i; j += 32) {
          const T uj = sU[j];
          p1 += sCA[j] > 0 ? uj : -uj;
          p2 += sCA[j] * uj;
        }
        const T coeff1 = warp_sum(p1);
        const T coeff2 = warp_sum(p2);
        const T coeff3 = normX - constraint;
        T step_max2;
        if (mode == 2) {
          step_max2 = C - constraint;
        } else if (mode == 1) {
          const T delta = coeff2 * coeff2 - coeff1 * coeff3;
          step_max2 = delta < 0 ? INF : (coeff2 - sqrt(delta)) / coeff1;
          step_max2 = mn_ref(C, step_max2);
        } else {
          step_max2 = coeff1 < 0 ? INF : (constraint - thrs) / coeff1;
          step_max2 = mn_ref(C, step_max2);
        }
        step = mn_ref(mn_ref(step, step_max2), step_max);
        if (step == INF) break;

        // ---- updates
        if (gw == 0)
          for (int j = lane; j <= i; j += 32) {
            T c = sCoef[j] + step * sU[j];
            if (pos && c < 0) c = 0;
            sCoef[j] = c;
          }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = rbase + v * 128 + lane * 4;
          Vec4<T> d = ld4(sDtR + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) d.v[e] += (-step) * A[v][e];
          st4(sDtR + r0, d);
        }
        normX += coeff1 * step * step - 2 * coeff2 * step;
        thrs += mul_rn(step, coeff1);
        c_end = C - step;
        at_lambda = step == step_max2;
        if (gw == 0) {
          __syncwarp();
          if (path)
            for (int k = lane; k <= i; k += 32) path[(size_t)iter * K + sInd[k]] = sCoef[k];
        }

        if (step == step_max) {
          // ---- drop atom first_zero, downdate invGs (warp 0)
          const int fz = first_zero;
          const int rd = sInd[fz];
          if (gw == own_w(rd) && lane == own_l(rd)) act &= ~(1u << own_b(rd));
          --cnt;
          __syncthreads();  // every warp has read sInd[fz] before warp 0 shifts it
          if (gw == 0) {
            const T schur = sInv[(size_t)fz * ldi + fz];
            for (int r = lane; r < i; r += 32)
              sW[r] = sInv[(size_t)(r < fz ? r : r + 1) * ldi + fz];
            for (int j0 = fz; j0 < i; j0 += 32) {
              const int j = j0 + lane;
              int ti = 0;
              T tc = 0;
              if (j < i) { ti = sInd[j + 1]; tc = sCoef[j + 1]; }
              __syncwarp();
              if (j < i) { sInd[j] = ti; sCoef[j] = tc; }
              __syncwarp();
            }
            if (lane == 0) { sInd[i] = -1; sCoef[i] = 0; }
            __syncwarp();
            const T alpha = T(-1) / schur;
            for (int r = 0; r < i; ++r) {
              const T* src = sInv + (size_t)(r < fz ? r : r + 1) * ldi;
              T* dst = sInv + (size_t)r * ldi;
              const T wr = sW[r];
              for (int c0 = 0; c0 < i; c0 += 32) {
                const int c = c0 + lane;
                T val = 0;
                if (c < i) {
                  const T wc = sW[c];
                  const T whi = c > r ? wc : wr;
                  const T wlo = c > r ? wr : wc;
                  val = src[c < fz ? c : c + 1] + (alpha * whi) * wlo;
                }
                __syncwarp();
                if (c < i) dst[c] = val;
                __syncwarp();
              }
            }
          }
          newAtom = false;
          i -= 2;
        } else {
          newAtom = true;
        }
        __syncthreads();  // correlation updates and warp 0's state visible to all
        if ((iter >= length_path - 1) || fabs(step) < 1e-15 || step == step_max2 ||
            (normX < 1e-15) || (i == (L - 1)) ||
            (mode == 1 && normX - constraint < 1e-15) ||
            (mode == 0 && (constraint - thrs < 1e-15)))
          break;
      }
    }
    __syncthreads();

    if (threadIdx.x == 0 && a.steps && !overflow) atomicAdd(a.steps, (unsigned long long)iter);
    if (overflow) {
      if (threadIdx.x == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig;
        a.out_cnt[sig] = 0;
      }
    } else if (gw == 0) {
      int* oind = a.out_ind + (size_t)sig * a.L;
      T* oval = a.out_val + (size_t)sig * a.L;
      for (int j = lane; j < cnt; j += 32) {
        const int me = sInd[j];
        int rank = 0;
        for (int k = 0; k < cnt; ++k) rank += sInd[k] < me;
        oind[rank] = me;
        oval[rank] = sCoef[j];
      }
      if (lane == 0) {
        a.out_cnt[sig] = cnt;
        if (a.out_level) a.out_level[sig] = (mode == 2 && at_lambda) ? constraint : c_end;
      }
    }
    __syncthreads();
  }
}

template <typename T, int W, bool MASKED = false>
__global__ void __launch_bounds__(W * 32) lars_cta_kernel(const LarsArgs<T> a) {
  lars_cta_body<T, W, MASKED>(a);
}
// The same kernel built with at most 64 registers, taken only where it keeps
// more CTAs resident (2.57 -> 2.34 ms per 20k signals on 4096 atoms); where
// shared memory limits residency its spills only cost time.
template <typename T, int W, bool MASKED = false>
__global__ void __launch_bounds__(W * 32, 32 / W) lars_cta_kernel_lb(const LarsArgs<T> a) {
  lars_cta_body<T, W, MASKED>(a);
}

// The build a launch uses: register-bounded where that keeps more CTAs
// resident (the grid helper below makes the same choice, so a persistent grid
// matches the residency of the kernel it runs).  Unlike the warp kernel, this
// one has no constraint-mode specialisation: a PENALTY-only build ran slower
// (1.22 -> 1.47 ms per 1024-signal minibatch on 1024 atoms).
template <typename T, int W, bool MASKED = false>
static auto pick_kernel(size_t smem) {
  auto k = lars_cta_kernel<T, W, MASKED>;
  if constexpr (sizeof(T) == 4)
    k = more_resident(k, lars_cta_kernel_lb<T, W, MASKED>, W * 32, smem);
  return k;
}

template <typename T, int W>
static cudaError_t launch_w(const LarsArgs<T>& a, int grid, size_t smem, cudaStream_t st) {
  auto k = a.mk.mask ? pick_kernel<T, W, true>(smem) : pick_kernel<T, W, false>(smem);
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  e = fill_grid(k, W * 32, smem, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
size_t lars_cta_smem_bytes(int Kp, int Lc, bool gstate) {
  return lars_cta_smem(Kp, Lc, sizeof(T), Kp / 512, gstate);
}
template <typename T>
size_t lars_cta_gstate_bytes(int Lc, int grid) {
  return (size_t)grid * lars_cta_state(Lc, sizeof(T));
}

template <typename T, int W>
static int grid_w(size_t smem) {
  auto k = pick_kernel<T, W>(smem);
  int grid = 0;
  if (allow_smem(k, smem) != cudaSuccess || fill_grid(k, W * 32, smem, &grid) != cudaSuccess)
    return 0;
  return grid;
}

template <typename T>
int lars_cta_grid(int Kp, int Lc, bool gstate) {
  const size_t smem = lars_cta_smem_bytes<T>(Kp, Lc, gstate);
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
cudaError_t launch_lars_cta(const LarsArgs<T>& a, int grid, cudaStream_t st) {
  if (a.Kp % 512 != 0) return cudaErrorInvalidValue;
  const size_t smem = lars_cta_smem_bytes<T>(a.Kp, a.Lcap, a.gstate != nullptr);
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

template size_t lars_cta_smem_bytes<float>(int, int, bool);
template size_t lars_cta_smem_bytes<double>(int, int, bool);
template size_t lars_cta_gstate_bytes<float>(int, int);
template size_t lars_cta_gstate_bytes<double>(int, int);
template int lars_cta_grid<float>(int, int, bool);
template int lars_cta_grid<double>(int, int, bool);
template cudaError_t launch_lars_cta<float>(const LarsArgs<float>&, int, cudaStream_t);
template cudaError_t launch_lars_cta<double>(const LarsArgs<double>&, int, cudaStream_t);

}  // namespace sc
