// LARS-Lasso homotopy for every signal of a batch: one warp per signal,
// persistent grid fed by a device work counter.
//
// Restates coreLARS2 (decomp/decomp.h:1706-1915) step for step:
//   - add atom: inverse-Gram Schur update of invGs (symv / dot / syr, :1749-1771)
//   - direction u = invGs sign(DtR_A) (:1774-1777)
//   - zero-crossing step, last index among equal ratios ("<=", :1780-1788)
//   - A = Ga u over the active Gram columns (:1792-1795)
//   - joining steps over inactive atoms, first minimum of the 2K magnitudes
//     (the reference's own cblas_iamin, linalg/cblas_alt_template.h:1094-1105)
//   - mode bound step_max2 (:1826-1847), MIN macro of linalg/utils.h:46
//   - coefficient / correlation / normX / thrs updates (:1848-1866)
//   - drop + inverse downdate (:1875-1903), stopping rules (:1907-1913)
//
// Layout: G is Kp x Kp column-major (ld Kp, ridge on the diagonal, zero rows /
// columns beyond K); DtX is Kp x n column-major.  Lane `l` of a warp owns the
// rows r = 128 v + 4 l + e (v < NV, e < 4), so every Gram-column read is one
// 512-byte coalesced vector load per v.  The per-signal state (correlations,
// inverse Gram, active set) sits in shared memory, or, for the overflow pass
// that reruns signals whose active set outgrew the shared-memory capacity, in
// a global scratch slab per warp.
#include "common.cuh"
#include "kernels.h"
#include "refactor.cuh"
#include "masked.cuh"
#include "lars_screen.cuh"

namespace sc {

__device__ __forceinline__ int own_lane(int r) { return (r & 127) >> 2; }
__device__ __forceinline__ int own_bit(int r) { return ((r >> 7) << 2) | (r & 3); }

// MIN macro of linalg/utils.h:46.
template <typename T> __device__ __forceinline__ T ref_min(T a, T b) { return a > b ? b : a; }

// Screening division: approximate in single precision (a few ulp), exact in
// double precision.
__device__ __forceinline__ float fast_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fast_div(double a, double b) { return a / b; }

// Dot product of a shared-memory row with a vector, four accumulators.
template <typename T>
__device__ __forceinline__ T dot_row(const T* __restrict__ row, const T* __restrict__ x, int n) {
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

// Drop of active entry fz (rare: a coefficient crossed zero): shift the
// active set down and downdate the inverse Gram (decomp/decomp.h:1875-1903).
// Kept out of line so that the per-step path stays compact in the
// instruction cache (2.49 -> 2.42 ms on the 100k-signal lasso workload).
template <typename T>
__device__ __noinline__ void lars_drop_downdate(T* sInv, int ldi, T* sW, int* sInd, T* sCoef, int i,
                                                int fz) {
  const int lane = threadIdx.x & 31;
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

// Regularisation path entry of this step (signal 0 only), out of line.
template <typename T>
__device__ __noinline__ void lars_write_path(T* path, int iter, int K, const int* sInd,
                                             const T* sCoef, int i) {
  for (int k = (int)(threadIdx.x & 31); k <= i; k += 32) path[(size_t)iter * K + sInd[k]] = sCoef[k];
}

// j = lane, lane + 32, ... < n: a single guarded pass when the active-set
// capacity is at most 32 (SMALL).
template <bool SMALL, typename F>
__device__ __forceinline__ void lane_loop(int n, F&& f) {
  const int lane = threadIdx.x & 31;
  if constexpr (SMALL) {
    if (lane < n) f(lane);
  } else {
    for (int j = lane; j < n; j += 32) f(j);
  }
}

// Single precision: three 8-warp blocks per SM (80 registers); double
// precision keeps two so that its wider row state stays in registers.
// MODE >= 0 fixes the constraint mode at compile time (PENALTY without pos,
// the common case, prunes the other modes' code from the per-step path:
// 2.42 -> 2.22 ms on the 100k-signal lasso workload); -1 reads it from a.
// SMALL (active-set capacity at most 32) turns the loops over the active set
// into one guarded pass per lane (2.19 -> 2.03 ms on the same workload).
// GSTATE = false: the state is known to live in shared memory (the main pass
// with a small active-set capacity), so every state access compiles to a
// 32-bit shared-space load or store instead of a generic one.
template <typename T, int NV, bool MASKED = false, int MODE = -1, bool SMALL = false,
          bool GSTATE = true>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2)
lars_kernel(const LarsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int Lc = a.Lcap;
  const int ldi = state_ld(Lc);
  const size_t per_warp = lars_state_bytes(a.Kp, Lc, sizeof(T));
  unsigned char* base =
      (GSTATE && a.gstate) ? reinterpret_cast<unsigned char*>(a.gstate) +
                                 (size_t)(blockIdx.x * wpb + wib) * per_warp
                           : smem_raw + (size_t)wib * per_warp;
  T* sDtR = reinterpret_cast<T*>(base);
  T* sInv = sDtR + a.Kp;
  T* sU = sInv + (size_t)Lc * ldi;
  T* sCoef = sU + Lc;
  T* sS = sCoef + Lc;
  T* sCA = sS + Lc;
  T* sW = sCA + Lc;
  T* sG = sW + Lc;
  int* sInd = reinterpret_cast<int*>(sG + Lc);

  const int K = a.K, Kp = a.Kp;
  const T INF = inf<T>();
  const int L = a.L < K ? a.L : K;  // L = MIN(LL, K)
  const int length_path = a.length_path <= 1 ? 4 * L : a.length_path;
  const int mode = MODE >= 0 ? MODE : a.mode;
  const bool pos = MODE >= 0 ? false : a.pos != 0;

  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;
  // rows r >= K (padding up to Kp) never join: mark them active once
  uint32_t pad_act = 0;
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (v * 128 + lane * 4 + e >= K) pad_act |= 1u << (v * 4 + e);
  for (;;) {
    int job = 0;
    if (lane == 0) job = (int)atomicAdd(a.work_counter, 1u);
    job = __shfl_sync(kFull, job, 0);
    if (job >= n_jobs) break;
    const int64_t sig = a.sig_list ? a.sig_list[job] : (int64_t)job;
    const T constraint = a.vConstraint ? a.vConstraint[sig] : a.constraint;
    T* path = (a.path && sig == 0) ? a.path : nullptr;
    // masked variant: no row observed -> empty code; some -> the masked Gram
    const int mflag = MASKED ? (int)a.mk.flag[sig] : 2;
    const bool partial = MASKED && mflag == 1;
    const uint8_t* mrow = MASKED ? a.mk.mask + (size_t)sig * a.mk.m : nullptr;
    T* mw = MASKED ? a.mk.work + (size_t)(blockIdx.x * wpb + wib) * a.mk.mpad : nullptr;

    // ---- load D^T x and find the first atom
    const T* dtx = a.DtX + (size_t)sig * Kp;
    T bkey = -INF;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = v * 128 + lane * 4;
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
    int cur = warp_argmax_first(bkey, bidx);
    T normX = a.norms[sig];
    for (int j = lane; j < Lc; j += 32) sCoef[j] = 0;  // coeffs.setZeros()
    __syncwarp();

    int cnt = 0;
    bool overflow = false;
    bool skip = L <= 0 || mflag == 0;
    if (!skip) {
      const T dc = sDtR[cur];
      if (mode == 2 && fabs(dc) < constraint) skip = true;
      if (mode == 1 && normX < constraint) skip = true;
    }

    uint32_t act = pad_act;  // active flags of this lane's rows (+ padding rows)
    int iter = 0;
    T c_end = 0;        // correlation level of the active set at exit
    bool at_lambda = false;
    if (!skip) {
      bool newAtom = true;
      T thrs = 0;
      T g_next = 0;  // (SMALL) this lane's entry of the next atom's Gram column
      for (int i = 0; i < L; ++i) {
        ++iter;
        if (newAtom) {
          if (i >= Lc) { overflow = true; break; }
          if (lane == 0) sInd[i] = cur;
          if (lane == own_lane(cur)) act |= 1u << own_bit(cur);
          ++cnt;
          __syncwarp();
          if (partial) {
            for (int j = 0; j <= i; ++j) {
              const T g = masked_gram(a.mk, mrow, sInd[j], cur);
              if (lane == 0) sG[j] = g;
            }
          } else if (SMALL && i > 0) {
            if (lane <= i) sG[lane] = g_next;  // loaded by the previous step's screen
          } else {
            const T* gcol = a.G + (size_t)cur * Kp;
            lane_loop<SMALL>(i + 1, [&](int j) { sG[j] = gcol[sInd[j]]; });
          }
          __syncwarp();
          if (i == 0) {
            if (lane == 0) sInv[0] = T(1) / sG[0];
          } else {
            // w = invGs(0:i,0:i) g(0:i)
            lane_loop<SMALL>(i, [&](int r) { sW[r] = dot_row(sInv + (size_t)r * ldi, sG, i); });
            __syncwarp();
            T part = 0;
            lane_loop<SMALL>(i, [&](int r) { part += sW[r] * sG[r]; });
            const T dot = warp_sum(part);
            const T piv = sG[i] - dot;
            // a small pivot loses digits in the update: rebuild the inverse in FP64
            bool refactored = false;
            const int unit = blockIdx.x * wpb + wib;
            if (sizeof(T) == 4 && a.refactor && i < a.rf_cap && unit < a.rf_units && !partial &&
                (a.refactor == 2 || !(piv > T(kRefactorPivot) * sG[i]))) {
              double* rs = a.rf_scratch + (size_t)unit * a.rf_cap * a.rf_cap;
              refactored = refactor_inverse<T>(a.G, Kp, sInd, i + 1, sInv, ldi, rs);
            }
            const T schur = T(1) / piv;
            if (!refactored) lane_loop<SMALL>(i, [&](int r) {
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
            });
            if (lane == 0 && !refactored) sInv[(size_t)i * ldi + i] = schur;
          }
          __syncwarp();
        }

        // ---- direction u = invGs sign(DtR_A)
        lane_loop<SMALL>(i + 1, [&](int j) {
          const T d = sDtR[sInd[j]];
          sCA[j] = d;
          sS[j] = d > 0 ? T(1) : T(-1);
        });
        __syncwarp();
        T zkey = INF;
        int zidx = -1;
        lane_loop<SMALL>(i + 1, [&](int r) {
          const T s = dot_row(sInv + (size_t)r * ldi, sS, i + 1);
          sU[r] = s;
          const T ratio = -sCoef[r] / s;
          if (ratio > 0 && ratio <= zkey) { zkey = ratio; zidx = r; }
        });
        const ArgRes<T> zr = warp_argmin_last_u(zkey, zidx);  // warp-uniform
        const T step_max = zr.val;
        const int first_zero = zr.idx;
        __syncwarp();
        const T C = fabs(sCA[0]);
        c_end = C;

        // ---- A = Ga u
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        if (partial) {
          masked_gram_times<T, NV>(a.mk, mrow, mw, Kp, sInd, sU, 1, i + 1, A);
        } else {
#pragma unroll 4
          for (int j = 0; j <= i; ++j) {
            const T uj = sU[j];
            const T* gc = a.G + (size_t)sInd[j] * Kp + lane * 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) axpy4(A[v], ldg4(gc + v * 128), uj);
          }
        }

        // ---- joining steps: first minimum magnitude over the 2K candidates
        // (lars_screen.cuh); infinite candidates (active or padding atoms,
        // |A_j| beyond the bounds) never decide a step (the step is then
        // step_max or step_max2)
        const ScreenBest<T> sb = lars_screen<NV>(A, sDtR + lane * 4, lane * 4, act, C, pos, K);
        const ArgRes<T> mr = warp_argmin_first(sb.key, sb.idx, sb.val);  // warp-uniform
        T step = mr.val;
        cur = join_atom(mr.idx, K);
        // the joining atom's Gram entries against the active set and its
        // diagonal, loaded now so that their L2 latency overlaps the updates
        // (1.71 -> 1.67 ms of coding on the 100k-signal lasso workload)
        if constexpr (SMALL) {
          if (!partial && lane <= i + 1)
            g_next = a.G[(size_t)cur * Kp + (lane <= i ? sInd[lane] : cur)];
        }

        // ---- polynomial of normX along the step
        T p1 = 0, p2 = 0;
        lane_loop<SMALL>(i + 1, [&](int j) {
          const T uj = sU[j];
          p1 += sCA[j] > 0 ? uj : -uj;
          p2 += sCA[j] * uj;
        });
        const T coeff1 = warp_sum(p1);
        const T coeff2 = warp_sum(p2);
        const T coeff3 = normX - constraint;
        T step_max2;
        if (mode == 2) {
          step_max2 = C - constraint;
        } else if (mode == 1) {
          const T delta = coeff2 * coeff2 - coeff1 * coeff3;
          step_max2 = delta < 0 ? INF : (coeff2 - sqrt(delta)) / coeff1;
          step_max2 = ref_min(C, step_max2);
        } else {
          step_max2 = coeff1 < 0 ? INF : (constraint - thrs) / coeff1;
          step_max2 = ref_min(C, step_max2);
        }
        step = ref_min(ref_min(step, step_max2), step_max);
        if (step == INF) break;

        // ---- updates
        lane_loop<SMALL>(i + 1, [&](int j) {
          T c = sCoef[j] + step * sU[j];
          if (pos && c < 0) c = 0;
          sCoef[j] = c;
        });
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = v * 128 + lane * 4;
          Vec4<T> d = ld4(sDtR + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) d.v[e] += (-step) * A[v][e];
          st4(sDtR + r0, d);
        }
        normX += coeff1 * step * step - 2 * coeff2 * step;
        thrs += mul_rn(step, coeff1);
        c_end = C - step;
        at_lambda = step == step_max2;
        __syncwarp();
        if (path) lars_write_path<T>(path, iter, K, sInd, sCoef, i);

        if (step == step_max) {
          // ---- drop atom first_zero, downdate invGs
          const int fz = first_zero;
          const int rd = sInd[fz];
          if (lane == own_lane(rd)) act &= ~(1u << own_bit(rd));
          --cnt;
          lars_drop_downdate<T>(sInv, ldi, sW, sInd, sCoef, i, fz);
          newAtom = false;
          i -= 2;
        } else {
          newAtom = true;
        }
        if ((iter >= length_path - 1) || fabs(step) < 1e-15 || step == step_max2 ||
            (normX < 1e-15) || (i == (L - 1)) ||
            (mode == 1 && normX - constraint < 1e-15) ||
            (mode == 0 && (constraint - thrs < 1e-15)))
          break;
      }
    }
    __syncwarp();

    if (a.steps && lane == 0 && !overflow) atomicAdd(a.steps, (unsigned long long)iter);
    // ---- output: active set sorted by atom index
    if (overflow) {
      if (lane == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig;
        a.out_cnt[sig] = 0;
      }
    } else {
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
        // the level the final coefficients satisfy G_AA a = c_A - level s_A
        if (a.out_level) a.out_level[sig] = (mode == 2 && at_lambda) ? constraint : c_end;
      }
    }
    __syncwarp();
  }
}

template <typename T>
size_t lars_smem_per_warp(int Kp, int Lcap) { return lars_state_bytes(Kp, Lcap, sizeof(T)); }

template <typename T, int NV>
static cudaError_t launch_nv(const LarsArgs<T>& a, int grid, int warps_per_block,
                             size_t smem, cudaStream_t st) {
  const bool penalty = a.mode == 2 && !a.pos;
  auto k = a.mk.mask                          ? lars_kernel<T, NV, true>
           : penalty && a.Lcap <= 32 && !a.gstate ? lars_kernel<T, NV, false, 2, true, false>
           : penalty                           ? lars_kernel<T, NV, false, 2>
                                               : lars_kernel<T, NV, false>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, warps_per_block * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_lars(const LarsArgs<T>& a, int grid, int warps_per_block, cudaStream_t st) {
  const size_t smem = a.gstate ? 0 : (size_t)warps_per_block * lars_state_bytes(a.Kp, a.Lcap, sizeof(T));
  switch (a.Kp / 128) {
    case 1: return launch_nv<T, 1>(a, grid, warps_per_block, smem, st);
    case 2: return launch_nv<T, 2>(a, grid, warps_per_block, smem, st);
    case 3: return launch_nv<T, 3>(a, grid, warps_per_block, smem, st);
    case 4: return launch_nv<T, 4>(a, grid, warps_per_block, smem, st);
    case 5: return launch_nv<T, 5>(a, grid, warps_per_block, smem, st);
    case 6: return launch_nv<T, 6>(a, grid, warps_per_block, smem, st);
    case 7: return launch_nv<T, 7>(a, grid, warps_per_block, smem, st);
    case 8: return launch_nv<T, 8>(a, grid, warps_per_block, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T>
int lars_max_warps_per_sm(int Kp) {
  const void* fn = nullptr;
  switch (Kp / 128) {
    case 1: fn = (const void*)lars_kernel<T, 1>; break;
    case 2: fn = (const void*)lars_kernel<T, 2>; break;
    case 3: fn = (const void*)lars_kernel<T, 3>; break;
    case 4: fn = (const void*)lars_kernel<T, 4>; break;
    case 5: fn = (const void*)lars_kernel<T, 5>; break;
    case 6: fn = (const void*)lars_kernel<T, 6>; break;
    case 7: fn = (const void*)lars_kernel<T, 7>; break;
    case 8: fn = (const void*)lars_kernel<T, 8>; break;
    default: return 0;
  }
  cudaFuncAttributes attr;
  if (cudaFuncGetAttributes(&attr, fn) != cudaSuccess) return 0;
  const int regs = attr.numRegs > 0 ? attr.numRegs : 64;
  return 65536 / (regs * 32);
}

template cudaError_t launch_lars<float>(const LarsArgs<float>&, int, int, cudaStream_t);
template cudaError_t launch_lars<double>(const LarsArgs<double>&, int, int, cudaStream_t);
template int lars_max_warps_per_sm<float>(int);
template int lars_max_warps_per_sm<double>(int);

}  // namespace sc
