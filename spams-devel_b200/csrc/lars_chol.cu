// The Cholesky implementation of the Lasso homotopy, one warp per signal:
// the GPU form of coreLARS + downDateLasso (decomp/decomp.h:844-1093,
// 1096-1203), reached through lasso<T> (:735-842) when the caller asks for
// `cholesky` or `ols`.  It follows the reference's own arithmetic, which
// differs from coreLARS2 (lars.cu) in ways that change results:
//   - the active set's inverse Cholesky factor Un (upper, Un^T G_AA Un = I
//     with the atoms' signs folded into G_AA) is extended column by column;
//     an atom whose residual norm2 falls below 1e-15 ends the path
//   - the equiangular direction u = a Un Un^T 1, a = 1 / ||Un^T 1||
//   - joining candidates (Cmax -/+ c)/(a -/+ A) interleaved as 2r, 2r+1
//     (a non-positive denominator gives INF), the PENALTY bound
//     (Cmax - lambda)/a, zero crossings -coef/u (coef == 0 or <= 0 -> INF)
//   - ||r||^2 tracked as normX += g^2 - 2 g <Rdn_A, u>, leaving the path
//     (and dropping the last atom) when that increment is > 0, NaN or inf
//   - ols: the final coefficients are the least-squares fit Un RUn on the
//     support, with ||r||^2 from the projections RUn
//   - drops rebuild Un by the reference's rotation (R, its inverse, R^-T)
//   - the reference's stopping rules (thrs = |Rdn_ind0| in PENALTY, thrs =
//     ||a||_1 in L1COEFFS, normX in L2ERROR, iter >= length_path)
//
// Layout as in lars.cu: lane l owns rows r = 128 v + 4 l + e; the signed
// Gram columns Gs(:, k) = s_k G(:, ind_k) (rows of active atoms times their
// own sign) are never stored, A = Gs u is summed from G with the signs.
// Small state per warp: Un, Gsa (the signed G_AA) and R (downdate scratch),
// Lcap x ld each, column-major; vectors u, w, sig, coef, RUn, av; ind.
// Beyond 1024 atoms (or when the CTA family is asked for) the same steps run
// with one CTA per signal (lars_chol_cta_kernel below).
#include "common.cuh"
#include "kernels.h"

namespace sc {

__host__ __device__ inline size_t chol_state_bytes(int Kp, int Lc, size_t esz) {
  return align16(esz * ((size_t)Kp + 3 * (size_t)Lc * state_ld(Lc) + 6 * (size_t)Lc) +
                 4 * (size_t)Lc);
}

template <typename T>
__device__ __forceinline__ T sign_of(T v) { return v < T(0) ? T(-1) : T(1); }  // SIGN, utils.h
template <typename T>
__device__ __forceinline__ T min_ref(T a, T b) { return a > b ? b : a; }  // MIN, utils.h

// The reference's downDateLasso (decomp/decomp.h:1096-1203) for the warp's
// state: drop position mb of the active set 0..j (j > 0 entries after it).
// Unds, which coreLARS never reads back, is not kept.
template <typename T>
__device__ __noinline__ void chol_downdate(int j, int mb, bool pos, bool ols, T* Un, T* Gsa, T* R,
                                           int ld, T* sig, T* av, T* coef, T* RUn, int* ind,
                                           const T* dtx, T* normX_io, T* sRdn) {
  const int lane = threadIdx.x & 31;
  const int indB = ind[mb];
  if (!pos && sig[mb] < T(0) && lane == 0) sRdn[indB] = -sRdn[indB];
  const int num = j - mb;
  // Update Un: columns k > mb lose their component along column mb
  const T unn = Un[(size_t)mb * ld + mb];
  for (int k = mb + 1 + lane; k <= j; k += 32) av[k - mb - 1] = -Un[(size_t)k * ld + mb] / unn;
  __syncwarp();
  for (int k = mb + 1; k <= j; ++k) {
    const T ak = av[k - mb - 1];
    for (int r = lane; r < mb; r += 32) Un[(size_t)k * ld + r] += ak * Un[(size_t)mb * ld + r];
  }
  __syncwarp();
  // shift columns k -> k - 1 (rows < mb as they are, rows > mb up by one)
  for (int k = mb + 1; k <= j; ++k) {
    for (int r = lane; r < mb; r += 32) Un[(size_t)(k - 1) * ld + r] = Un[(size_t)k * ld + r];
    __syncwarp();
    for (int r = lane; r < num; r += 32) Un[(size_t)(k - 1) * ld + mb + r] = Un[(size_t)k * ld + mb + 1 + r];
    __syncwarp();
  }
  if (num > 0) {
    // R: lower triangular num x num (ld num in the reference; here ld `ld`)
    if (lane == 0) {
      T alpha = T(1);
      for (int k = 0; k < num; ++k) {
        for (int r = 0; r < num; ++r) R[(size_t)k * ld + r] = r == k ? T(1) : T(0);
      }
      for (int k = 0; k < num; ++k) {
        const T alphab = alpha + av[k] * av[k];
        const T rkk = sqrt(alphab / alpha);
        R[(size_t)k * ld + k] = rkk;
        const T gamma = av[k] * rkk / alphab;
        alpha = alphab;
        for (int r = k + 1; r < num; ++r) R[(size_t)k * ld + r] = gamma * av[r];
      }
      // R <- R^-1 (lower, non-unit), column by column
      for (int k = 0; k < num; ++k) {
        R[(size_t)k * ld + k] = T(1) / R[(size_t)k * ld + k];
        for (int r = k + 1; r < num; ++r) {
          T s = 0;
          for (int q = k; q < r; ++q) s += R[(size_t)q * ld + r] * R[(size_t)k * ld + q];
          R[(size_t)k * ld + r] = -s / R[(size_t)r * ld + r];
        }
      }
    }
    __syncwarp();
    // Un(0:j, mb:mb+num) <- Un(0:j, mb:mb+num) R^T   (trmm Right Lower Trans)
    for (int r = lane; r < j; r += 32) {
      // new(r, mb + c) = sum_{q <= c} old(r, mb + q) R(c, q); c descending keeps old values
      for (int c = num - 1; c >= 0; --c) {
        T s = 0;
        for (int q = 0; q <= c; ++q) s += Un[(size_t)(mb + q) * ld + r] * R[(size_t)q * ld + c];
        Un[(size_t)(mb + c) * ld + r] = s;
      }
    }
    __syncwarp();
  }
  // Update Gsa: remove row and column mb
  for (int k = mb + 1; k <= j; ++k) {
    for (int r = lane; r < mb; r += 32) Gsa[(size_t)(k - 1) * ld + r] = Gsa[(size_t)k * ld + r];
    __syncwarp();
    for (int r = lane; r < j - mb; r += 32) Gsa[(size_t)(k - 1) * ld + mb + r] = Gsa[(size_t)k * ld + mb + 1 + r];
    __syncwarp();
  }
  for (int k = 0; k < mb; ++k) {
    for (int l = mb + 1; l <= j; ++l) {
      if (lane == 0) Gsa[(size_t)k * ld + l - 1] = Gsa[(size_t)k * ld + l];
      __syncwarp();
    }
  }
  // sig, ind, coef shift down
  if (lane == 0) {
    for (int k = mb + 1; k <= j && !pos; ++k) sig[k - 1] = sig[k];
    for (int k = mb + 1; k <= j; ++k) ind[k - 1] = ind[k];
    ind[j] = -1;
    for (int k = mb + 1; k <= j; ++k) coef[k - 1] = coef[k];
    coef[j] = T(0);
  }
  __syncwarp();
  if (ols && lane == 0) {
    T normX = *normX_io;
    for (int k = mb; k <= j; ++k) normX += RUn[k] * RUn[k];
    for (int k = mb; k < j; ++k) {
      T s = 0;
      for (int l = 0; l <= k; ++l) s += sig[l] * dtx[ind[l]] * Un[(size_t)k * ld + l];
      RUn[k] = s;
      normX -= s * s;
    }
    *normX_io = normX;
  }
  __syncwarp();
}

template <typename T, int NV>
__global__ void __launch_bounds__(128) lars_chol_kernel(const LarsArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int Lc = a.Lcap;
  const int ld = state_ld(Lc);
  const size_t per_warp = chol_state_bytes(a.Kp, Lc, sizeof(T));
  unsigned char* base = a.gstate ? reinterpret_cast<unsigned char*>(a.gstate) +
                                       (size_t)(blockIdx.x * wpb + wib) * per_warp
                                 : smem_raw + (size_t)wib * per_warp;
  T* sRdn = reinterpret_cast<T*>(base);
  T* sUn = sRdn + a.Kp;
  T* sGsa = sUn + (size_t)Lc * ld;
  T* sR = sGsa + (size_t)Lc * ld;
  T* su = sR + (size_t)Lc * ld;
  T* sw = su + Lc;
  T* ssig = sw + Lc;
  T* scoef = ssig + Lc;
  T* sRUn = scoef + Lc;
  T* sav = sRUn + Lc;
  int* sInd = reinterpret_cast<int*>(sav + Lc);

  const int K = a.K, Kp = a.Kp;
  const T INF = inf<T>();
  const int L = a.L < K ? a.L : K;  // MIN(LL, K)
  const int length_path = a.length_path <= 1 ? 4 * L : a.length_path;
  const int mode = a.mode;
  const bool pos = a.pos != 0;
  const bool ols = a.ols != 0;
  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;

  uint32_t pad = 0;  // padding rows (r >= K): never candidates
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (v * 128 + lane * 4 + e >= K) pad |= 1u << (v * 4 + e);

  for (;;) {
    int job = 0;
    if (lane == 0) job = (int)atomicAdd(a.work_counter, 1u);
    job = __shfl_sync(kFull, job, 0);
    if (job >= n_jobs) break;
    const int64_t sig_i = a.sig_list ? a.sig_list[job] : (int64_t)job;
    const T constraint = a.vConstraint ? a.vConstraint[sig_i] : a.constraint;
    T* path = (a.path && sig_i == 0) ? a.path : nullptr;
    const T* dtx = a.DtX + (size_t)sig_i * Kp;
    T normX = a.norms[sig_i];

    // Rdn = D^T x; first atom: Vector::max (pos) or fmax (first index)
    T bkey = -INF;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = v * 128 + lane * 4;
      const Vec4<T> d = ldg4(dtx + r0);
      st4(sRdn + r0, d);
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
    for (int k = lane; k < Lc; k += 32) { scoef[k] = T(0); sInd[k] = -1; }
    __syncwarp();

    uint32_t act = pad;   // active rows (and padding)
    uint32_t neg = 0;     // active rows whose sign is negative
    int j = 0;
    int nact = 0;         // output entries: the active positions before the first -1
    int iters = 0;
    bool overflow = false;
    if (!(mode == 1 && normX < constraint) && L > 0) {
      bool newAtom = true;
      T Cmax = 0;
      int iter = 1;
      T thrs = 0;
      for (j = 0; j < L; ++j) {
        if (!newAtom && j < 0) break;  // the only atom was dropped
        if (newAtom) {
          if (j >= Lc) { overflow = true; break; }
          const T rc = sRdn[cur];
          const T sj = pos ? T(1) : sign_of(rc);
          Cmax = pos ? rc : fabs(rc);
          __syncwarp();
          if (lane == 0) {
            sInd[j] = cur;
            ssig[j] = sj;
            if (sj < T(0)) sRdn[cur] = -rc;
          }
          if (lane == ((cur & 127) >> 2)) {
            act |= 1u << (((cur >> 7) << 2) | (cur & 3));
            if (sj < T(0)) neg |= 1u << (((cur >> 7) << 2) | (cur & 3));
          }
          __syncwarp();
          // Gsa(:, j): s_k s_j G(c, ind_k), k < j; G(c, c) on the diagonal
          // (row c of the columns ind_k, as the reference reads a caller's Q)
          for (int k = lane; k <= j; k += 32) {
            const T g = a.G[(size_t)sInd[k] * Kp + cur];
            const T v = k == j ? g : ssig[k] * sj * g;
            sGsa[(size_t)j * ld + k] = v;
            sGsa[(size_t)k * ld + j] = v;
          }
          __syncwarp();
          // y_k = (Un^T Gsa(0:j, j))_k, k < j; norm2 = Gsa(j, j) - sum y_k^2
          for (int k = lane; k < j; k += 32) {
            T s = 0;
            for (int l = 0; l <= k; ++l) s += sUn[(size_t)k * ld + l] * sGsa[(size_t)j * ld + l];
            sw[k] = s;
          }
          __syncwarp();
          T norm2 = sGsa[(size_t)j * ld + j];
          for (int k = 0; k < j; ++k) norm2 -= sw[k] * sw[k];
          if (norm2 < T(1e-15)) {  // "bad exit": ind[j] = -1, the atom is not kept
            for (int r = lane; r < Lc; r += 32) sUn[(size_t)j * ld + r] = T(0);
            if (lane == 0) sRUn[j] = T(0);
            nact = j;
            __syncwarp();
            break;
          }
          nact = j + 1;
          // Un(0:j, j) = -invNorm Un_j y ; Un(j, j) = invNorm
          const T invNorm = T(1) / sqrt(norm2);
          for (int r = lane; r < j; r += 32) {
            T s = 0;
            for (int k = r; k < j; ++k) s += sUn[(size_t)k * ld + r] * sw[k];
            sUn[(size_t)j * ld + r] = s * (-invNorm);
          }
          for (int r = j + 1 + lane; r < Lc; r += 32) sUn[(size_t)j * ld + r] = T(0);
          if (lane == 0) sUn[(size_t)j * ld + j] = T(-1) * (-invNorm);
          __syncwarp();
        }

        // ---- direction: w = Un^T 1, a = 1/||w||, u = a Un w
        for (int k = lane; k <= j; k += 32) {
          T s = 0;
          for (int l = 0; l <= k; ++l) s += sUn[(size_t)k * ld + l];
          sw[k] = s;
        }
        __syncwarp();
        T nrm = 0;  // summed in the reference's order
        for (int k = 0; k <= j; ++k) nrm += sw[k] * sw[k];
        const T aa = T(1) / sqrt(nrm);
        for (int r = lane; r <= j; r += 32) {
          T s = 0;
          for (int k = r; k <= j; ++k) s += sUn[(size_t)k * ld + r] * sw[k];
          su[r] = aa * s;
        }
        __syncwarp();

        // ---- A = Gs u: sum_k G(:, ind_k) s_k u_k, active rows times their sign
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        for (int k = 0; k <= j; ++k) {
          const T uk = ssig[k] * su[k];
          const T* g = a.G + (size_t)sInd[k] * Kp + lane * 4;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const Vec4<T> gv = ldg4(g + v * 128);
#pragma unroll
            for (int e = 0; e < 4; ++e) A[v][e] += gv.v[e] * uk;
          }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if ((neg >> (v * 4 + e)) & 1u) A[v][e] = -A[v][e];

        T potentNorm = 0;
        if (!ols)
          for (int k = 0; k <= j; ++k) potentNorm += sRdn[sInd[k]] * su[k];

        // ---- joining candidates: first index of the smallest |work|
        T bk = INF, bv = INF;
        int bi = 0x7fffffff;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = v * 128 + lane * 4;
          const Vec4<T> d = ld4(sRdn + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if ((act >> (v * 4 + e)) & 1u) continue;
            const int r = r0 + e;
            const T Ar = A[v][e], c = d.v[e];
            if (pos) {
              const T diff = aa - Ar;
              T w = diff <= T(0) ? INF : (Cmax - c) / diff;
              if (w <= T(0)) w = INF;
              const T k = fabs(w);
              if (k < bk || (k == bk && r < bi)) { bk = k; bv = w; bi = r; }
            } else {
              const T d1 = aa - Ar;
              const T w1 = d1 <= T(0) ? INF : (Cmax - c) / d1;
              const T k1 = fabs(w1);
              if (k1 < bk || (k1 == bk && 2 * r < bi)) { bk = k1; bv = w1; bi = 2 * r; }
              const T d2 = aa + Ar;
              const T w2 = d2 <= T(0) ? INF : (Cmax + c) / d2;
              const T k2 = fabs(w2);
              if (k2 < bk || (k2 == bk && 2 * r + 1 < bi)) { bk = k2; bv = w2; bi = 2 * r + 1; }
            }
          }
        }
        if (!(bk < INF)) { bk = INF; bv = INF; }
        if (bk == INF && bi == 0x7fffffff) bi = 0;  // nothing finite: iamin returns index 0
        const ArgRes<T> mr = warp_argmin_first(bk, bi, bv);
        T gamma = mr.val;
        int nextInd = mr.idx;
        if (mode == 2) gamma = min_ref(gamma, (Cmax - constraint) / aa);
        // zero crossings
        T zk = INF, zv = INF;
        int zi = 0x7fffffff;
        for (int k = lane; k <= j; k += 32) {
          T w = -(scoef[k] / su[k]);
          if (scoef[k] == T(0) || w <= T(0)) w = INF;
          const T key = fabs(w);
          if (key < zk || (key == zk && k < zi)) { zk = key; zv = w; zi = k; }
        }
        if (zi == 0x7fffffff) zi = 0;
        const ArgRes<T> zr = warp_argmin_first(zk, zi, zv);
        const int minBasis = zr.idx;
        const T gammaMin = zr.val;
        if (gammaMin < gamma) gamma = gammaMin;
        if (mode == 0) {
          T tu = 0;
          for (int k = 0; k <= j; ++k) tu += su[k];
          if (tu > T(10e-10)) gamma = min_ref(gamma, (constraint - thrs) / tu);  // EPSILON
          thrs += mul_rn(gamma, tu);
        }
        if (!ols) {
          const T t = gamma * gamma - 2 * gamma * potentNorm;
          if (t > T(0) || t != t || isinf(t)) {  // ind[j] = -1: the last position is not kept
            nact = j;
            break;
          }
          normX += t;
        } else if (newAtom) {
          // RUn[j] = sum_k Xdn[ind_k] Un(k, j), Xdn the signed D^T x
          T s = 0;
          for (int k = 0; k <= j; ++k) s += ssig[k] * dtx[sInd[k]] * sUn[(size_t)j * ld + k];
          __syncwarp();
          if (lane == 0) sRUn[j] = s;
          __syncwarp();
          normX -= s * s;
        }
        // ---- updates
        for (int k = lane; k <= j; k += 32) {
          T c = scoef[k] + gamma * su[k];
          if (pos && c < T(0)) c = T(0);
          scoef[k] = c;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = v * 128 + lane * 4;
          Vec4<T> d = ld4(sRdn + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) d.v[e] += (-gamma) * A[v][e];
          st4(sRdn + r0, d);
        }
        __syncwarp();
        if (!pos) nextInd /= 2;
        if (path)
          for (int k = lane; k <= j; k += 32) path[(size_t)iter * K + sInd[k]] = scoef[k] * ssig[k];
        __syncwarp();
        if (gamma == gammaMin) {
          const int rd = sInd[minBasis];
          if (lane == ((rd & 127) >> 2)) {
            act &= ~(1u << (((rd >> 7) << 2) | (rd & 3)));
            neg &= ~(1u << (((rd >> 7) << 2) | (rd & 3)));
          }
          chol_downdate<T>(j, minBasis, pos, ols, sUn, sGsa, sR, ld, ssig, sav, scoef, sRUn, sInd,
                           dtx, &normX, sRdn);
          normX = __shfl_sync(kFull, normX, 0);
          nact = j;
          newAtom = false;
          Cmax = sInd[0] >= 0 ? fabs(sRdn[sInd[0]]) : T(0);  // (the path ends when j < 0)
          j -= 2;
        } else {
          newAtom = true;
          cur = nextInd;
        }
        ++iter;
        if (mode == 2 && j >= 0) thrs = fabs(sRdn[sInd[0]]);
        if ((j == L - 1) || (mode == 2 && (thrs - constraint < T(1e-15))) ||
            (mode == 0 && (thrs - constraint > T(-1e-15))) ||
            (newAtom && mode == 1 && (normX - constraint < T(1e-15))) || (normX < T(1e-15)) ||
            (iter >= length_path))
          break;
      }
      iters = iter - 1;
      if (!overflow) {
        if (j >= L) j = L - 1;  // (the loop leaves through a stop rule first)
        // the reference's final transform covers positions 0..j, which after
        // a drop is one position short of the active set
        const int tn = j + 1 < 0 ? 0 : j + 1;
        if (ols) {
          // coef(0:j) = Un RUn (the least-squares fit on the support)
          for (int r = lane; r < tn; r += 32) {
            T s = 0;
            for (int k = r; k < tn; ++k) s += sUn[(size_t)k * ld + r] * sRUn[k];
            sw[r] = s;
          }
          __syncwarp();
          for (int r = lane; r < tn; r += 32) scoef[r] = sw[r];
          __syncwarp();
        }
        for (int r = lane; r < tn; r += 32) scoef[r] *= ssig[r];  // vMul(j + 1, coef, sig)
        __syncwarp();
      }
    }
    __syncwarp();

    if (a.steps && lane == 0 && !overflow) atomicAdd(a.steps, (unsigned long long)iters);
    if (overflow) {
      if (lane == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig_i;
        a.out_cnt[sig_i] = 0;
      }
    } else {
      int* oind = a.out_ind + (size_t)sig_i * a.L;
      T* oval = a.out_val + (size_t)sig_i * a.L;
      for (int q = lane; q < nact; q += 32) {
        const int me = sInd[q];
        int rank = 0;
        for (int k = 0; k < nact; ++k) rank += sInd[k] < me;
        oind[rank] = me;
        oval[rank] = scoef[q];
      }
      if (lane == 0) a.out_cnt[sig_i] = nact;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// CTA form for dictionaries beyond 1024 atoms: one CTA of W warps per signal,
// warp w owning rows w*512 + 128 v + 4 lane + e (v < 4).  The small state
// (Un, Gsa, R and the vectors) sits once per CTA and is updated by warp 0;
// the row work (first atom, A = Gs u, the joining candidates, the Rdn
// update) runs on every warp, and the two row-wise reductions go through a
// W-entry exchange.  The scalar bookkeeping is computed by every thread from
// the shared state, in the warp kernel's order, so both forms give the same
// bits.
__host__ __device__ inline size_t chol_cta_small_bytes(int Lc, size_t esz) {
  return align16(esz * (3 * (size_t)Lc * state_ld(Lc) + 6 * (size_t)Lc) + 4 * (size_t)Lc);
}
__host__ __device__ inline size_t chol_cta_head_bytes(int Kp, int W, size_t esz) {
  return align16(esz * ((size_t)Kp + 2 * (size_t)W + 4) + 4 * ((size_t)W + 4));
}

template <typename T, int W>
__global__ void __launch_bounds__(W * 32) lars_chol_cta_kernel(const LarsArgs<T> a) {
  constexpr int NV = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int gw = threadIdx.x >> 5;
  const int Lc = a.Lcap;
  const int ld = state_ld(Lc);
  T* sRdn = reinterpret_cast<T*>(smem_raw);
  T* exK = sRdn + a.Kp;   // W keys
  T* exV = exK + W;       // W values
  T* sScal = exV + W;     // [0] normX after a drop
  int* exI = reinterpret_cast<int*>(sScal + 4);  // W indices
  int* sIScal = exI + W;  // [0] job
  unsigned char* base =
      a.gstate ? reinterpret_cast<unsigned char*>(a.gstate) +
                     (size_t)blockIdx.x * chol_cta_small_bytes(Lc, sizeof(T))
               : smem_raw + chol_cta_head_bytes(a.Kp, W, sizeof(T));
  T* sUn = reinterpret_cast<T*>(base);
  T* sGsa = sUn + (size_t)Lc * ld;
  T* sR = sGsa + (size_t)Lc * ld;
  T* su = sR + (size_t)Lc * ld;
  T* sw = su + Lc;
  T* ssig = sw + Lc;
  T* scoef = ssig + Lc;
  T* sRUn = scoef + Lc;
  T* sav = sRUn + Lc;
  int* sInd = reinterpret_cast<int*>(sav + Lc);

  const int K = a.K, Kp = a.Kp;
  const T INF = inf<T>();
  const int L = a.L < K ? a.L : K;  // MIN(LL, K)
  const int length_path = a.length_path <= 1 ? 4 * L : a.length_path;
  const int mode = a.mode;
  const bool pos = a.pos != 0;
  const bool ols = a.ols != 0;
  const int n_jobs = a.n_jobs_dev ? *a.n_jobs_dev : a.n_jobs;
  const int rbase = gw * NV * 128;
  const bool w0 = gw == 0;
  // owner (warp, lane, bit) of row r
  auto own_w = [](int r) { return r / (NV * 128); };
  auto own_l = [](int r) { return (r & 127) >> 2; };
  auto own_b = [](int r) { return (((r % (NV * 128)) >> 7) << 2) | (r & 3); };

  uint32_t pad = 0;  // padding rows (r >= K): never candidates
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (rbase + v * 128 + lane * 4 + e >= K) pad |= 1u << (v * 4 + e);

  for (;;) {
    if (threadIdx.x == 0) sIScal[0] = (int)atomicAdd(a.work_counter, 1u);
    __syncthreads();
    const int job = sIScal[0];
    if (job >= n_jobs) break;
    const int64_t sig_i = a.sig_list ? a.sig_list[job] : (int64_t)job;
    const T constraint = a.vConstraint ? a.vConstraint[sig_i] : a.constraint;
    T* path = (a.path && sig_i == 0) ? a.path : nullptr;
    const T* dtx = a.DtX + (size_t)sig_i * Kp;
    T normX = a.norms[sig_i];

    // Rdn = D^T x; first atom: Vector::max (pos) or fmax (first index)
    T bkey = -INF;
    int bidx = 0x7fffffff;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int r0 = rbase + v * 128 + lane * 4;
      const Vec4<T> d = ldg4(dtx + r0);
      st4(sRdn + r0, d);
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
      const unsigned who = __ballot_sync(kFull, bidx == wi);
      const T wk = __shfl_sync(kFull, bkey, who ? __ffs(who) - 1 : 0);
      if (lane == 0) { exK[gw] = wk; exI[gw] = wi; }
    }
    for (int k = threadIdx.x; k < Lc; k += W * 32) { scoef[k] = T(0); sInd[k] = -1; }
    __syncthreads();
    int cur;
    {
      T bk = exK[0];
      int bi = exI[0];
      for (int w = 1; w < W; ++w)
        if (exK[w] > bk || (exK[w] == bk && exI[w] < bi)) { bk = exK[w]; bi = exI[w]; }
      cur = bi;
    }

    uint32_t act = pad;   // active rows (and padding)
    uint32_t neg = 0;     // active rows whose sign is negative
    int j = 0;
    int nact = 0;         // output entries: the active positions before the first -1
    int iters = 0;
    bool overflow = false;
    if (!(mode == 1 && normX < constraint) && L > 0) {
      bool newAtom = true;
      T Cmax = 0;
      int iter = 1;
      T thrs = 0;
      for (j = 0; j < L; ++j) {
        if (!newAtom && j < 0) break;  // the only atom was dropped
        if (newAtom) {
          if (j >= Lc) { overflow = true; break; }
          const T rc = sRdn[cur];
          const T sj = pos ? T(1) : sign_of(rc);
          Cmax = pos ? rc : fabs(rc);
          if (gw == own_w(cur) && lane == own_l(cur)) {
            act |= 1u << own_b(cur);
            if (sj < T(0)) neg |= 1u << own_b(cur);
          }
          __syncthreads();  // every thread has read Rdn[cur]
          if (w0) {
            if (lane == 0) {
              sInd[j] = cur;
              ssig[j] = sj;
              if (sj < T(0)) sRdn[cur] = -rc;
            }
            __syncwarp();
            // Gsa(:, j): s_k s_j G(c, ind_k), k < j; G(c, c) on the diagonal
            for (int k = lane; k <= j; k += 32) {
              const T g = a.G[(size_t)sInd[k] * Kp + cur];
              const T v = k == j ? g : ssig[k] * sj * g;
              sGsa[(size_t)j * ld + k] = v;
              sGsa[(size_t)k * ld + j] = v;
            }
            __syncwarp();
            // y_k = (Un^T Gsa(0:j, j))_k, k < j
            for (int k = lane; k < j; k += 32) {
              T s = 0;
              for (int l = 0; l <= k; ++l) s += sUn[(size_t)k * ld + l] * sGsa[(size_t)j * ld + l];
              sw[k] = s;
            }
          }
          __syncthreads();
          T norm2 = sGsa[(size_t)j * ld + j];
          for (int k = 0; k < j; ++k) norm2 -= sw[k] * sw[k];
          if (norm2 < T(1e-15)) {  // "bad exit": ind[j] = -1, the atom is not kept
            if (w0) {
              for (int r = lane; r < Lc; r += 32) sUn[(size_t)j * ld + r] = T(0);
              if (lane == 0) sRUn[j] = T(0);
            }
            nact = j;
            __syncthreads();
            break;
          }
          nact = j + 1;
          // Un(0:j, j) = -invNorm Un_j y ; Un(j, j) = invNorm
          const T invNorm = T(1) / sqrt(norm2);
          if (w0) {
            for (int r = lane; r < j; r += 32) {
              T s = 0;
              for (int k = r; k < j; ++k) s += sUn[(size_t)k * ld + r] * sw[k];
              sUn[(size_t)j * ld + r] = s * (-invNorm);
            }
            for (int r = j + 1 + lane; r < Lc; r += 32) sUn[(size_t)j * ld + r] = T(0);
            if (lane == 0) sUn[(size_t)j * ld + j] = T(-1) * (-invNorm);
          }
          __syncthreads();
        }

        // ---- direction: w = Un^T 1, a = 1/||w||, u = a Un w
        if (w0)
          for (int k = lane; k <= j; k += 32) {
            T s = 0;
            for (int l = 0; l <= k; ++l) s += sUn[(size_t)k * ld + l];
            sw[k] = s;
          }
        __syncthreads();
        T nrm = 0;  // summed in the reference's order
        for (int k = 0; k <= j; ++k) nrm += sw[k] * sw[k];
        const T aa = T(1) / sqrt(nrm);
        if (w0)
          for (int r = lane; r <= j; r += 32) {
            T s = 0;
            for (int k = r; k <= j; ++k) s += sUn[(size_t)k * ld + r] * sw[k];
            su[r] = aa * s;
          }
        __syncthreads();

        // ---- A = Gs u on the own rows: sum_k G(:, ind_k) s_k u_k, active rows times their sign
        T A[NV][4];
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e) A[v][e] = 0;
        for (int k = 0; k <= j; ++k) {
          const T uk = ssig[k] * su[k];
          const T* g = a.G + (size_t)sInd[k] * Kp + rbase + lane * 4;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const Vec4<T> gv = ldg4(g + v * 128);
#pragma unroll
            for (int e = 0; e < 4; ++e) A[v][e] += gv.v[e] * uk;
          }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if ((neg >> (v * 4 + e)) & 1u) A[v][e] = -A[v][e];

        T potentNorm = 0;
        if (!ols)
          for (int k = 0; k <= j; ++k) potentNorm += sRdn[sInd[k]] * su[k];

        // ---- joining candidates of the own rows: first index of the smallest |work|
        {
          T bk = INF, bv = INF;
          int bi = 0x7fffffff;
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const int r0 = rbase + v * 128 + lane * 4;
            const Vec4<T> d = ld4(sRdn + r0);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              if ((act >> (v * 4 + e)) & 1u) continue;
              const int r = r0 + e;
              const T Ar = A[v][e], c = d.v[e];
              if (pos) {
                const T diff = aa - Ar;
                T w = diff <= T(0) ? INF : (Cmax - c) / diff;
                if (w <= T(0)) w = INF;
                const T k = fabs(w);
                if (k < bk || (k == bk && r < bi)) { bk = k; bv = w; bi = r; }
              } else {
                const T d1 = aa - Ar;
                const T w1 = d1 <= T(0) ? INF : (Cmax - c) / d1;
                const T k1 = fabs(w1);
                if (k1 < bk || (k1 == bk && 2 * r < bi)) { bk = k1; bv = w1; bi = 2 * r; }
                const T d2 = aa + Ar;
                const T w2 = d2 <= T(0) ? INF : (Cmax + c) / d2;
                const T k2 = fabs(w2);
                if (k2 < bk || (k2 == bk && 2 * r + 1 < bi)) { bk = k2; bv = w2; bi = 2 * r + 1; }
              }
            }
          }
          if (!(bk < INF)) { bk = INF; bv = INF; }
          if (bk == INF && bi == 0x7fffffff) bi = 0;  // nothing finite: iamin returns index 0
          const ArgRes<T> mr = warp_argmin_first(bk, bi, bv);
          // the warp's minimum: key |val| (the keys are the values' magnitudes)
          if (lane == 0) { exK[gw] = fabs(mr.val); exV[gw] = mr.val; exI[gw] = mr.idx; }
        }
        // zero crossings (every warp, from the shared state, before warp 0
        // updates coef)
        T zk = INF, zv = INF;
        int zi = 0x7fffffff;
        for (int k = lane; k <= j; k += 32) {
          T w = -(scoef[k] / su[k]);
          if (scoef[k] == T(0) || w <= T(0)) w = INF;
          const T key = fabs(w);
          if (key < zk || (key == zk && k < zi)) { zk = key; zv = w; zi = k; }
        }
        if (zi == 0x7fffffff) zi = 0;
        const ArgRes<T> zr = warp_argmin_first(zk, zi, zv);
        __syncthreads();
        T gamma;
        int nextInd;
        {
          T bk = exK[0], bv = exV[0];
          int bi = exI[0];
          for (int w = 1; w < W; ++w)
            if (exK[w] < bk || (exK[w] == bk && exI[w] < bi)) { bk = exK[w]; bv = exV[w]; bi = exI[w]; }
          gamma = bv;
          nextInd = bi;
        }
        if (mode == 2) gamma = min_ref(gamma, (Cmax - constraint) / aa);
        const int minBasis = zr.idx;
        const T gammaMin = zr.val;
        if (gammaMin < gamma) gamma = gammaMin;
        if (mode == 0) {
          T tu = 0;
          for (int k = 0; k <= j; ++k) tu += su[k];
          if (tu > T(10e-10)) gamma = min_ref(gamma, (constraint - thrs) / tu);  // EPSILON
          thrs += mul_rn(gamma, tu);
        }
        if (!ols) {
          const T t = gamma * gamma - 2 * gamma * potentNorm;
          if (t > T(0) || t != t || isinf(t)) {  // ind[j] = -1: the last position is not kept
            nact = j;
            break;
          }
          normX += t;
        } else if (newAtom) {
          // RUn[j] = sum_k Xdn[ind_k] Un(k, j), Xdn the signed D^T x
          T s = 0;
          for (int k = 0; k <= j; ++k) s += ssig[k] * dtx[sInd[k]] * sUn[(size_t)j * ld + k];
          if (threadIdx.x == 0) sRUn[j] = s;
          normX -= s * s;
        }
        // ---- updates
        if (w0)
          for (int k = lane; k <= j; k += 32) {
            T c = scoef[k] + gamma * su[k];
            if (pos && c < T(0)) c = T(0);
            scoef[k] = c;
          }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const int r0 = rbase + v * 128 + lane * 4;
          Vec4<T> d = ld4(sRdn + r0);
#pragma unroll
          for (int e = 0; e < 4; ++e) d.v[e] += (-gamma) * A[v][e];
          st4(sRdn + r0, d);
        }
        __syncthreads();
        if (!pos) nextInd /= 2;
        if (path && w0)
          for (int k = lane; k <= j; k += 32) path[(size_t)iter * K + sInd[k]] = scoef[k] * ssig[k];
        __syncthreads();
        if (gamma == gammaMin) {
          const int rd = sInd[minBasis];
          if (gw == own_w(rd) && lane == own_l(rd)) {
            act &= ~(1u << own_b(rd));
            neg &= ~(1u << own_b(rd));
          }
          __syncthreads();  // every thread has read ind before the downdate shifts it
          if (w0) {
            chol_downdate<T>(j, minBasis, pos, ols, sUn, sGsa, sR, ld, ssig, sav, scoef, sRUn,
                             sInd, dtx, &normX, sRdn);
            if (lane == 0) sScal[0] = normX;
          }
          __syncthreads();
          normX = sScal[0];
          nact = j;
          newAtom = false;
          Cmax = sInd[0] >= 0 ? fabs(sRdn[sInd[0]]) : T(0);  // (the path ends when j < 0)
          j -= 2;
        } else {
          newAtom = true;
          cur = nextInd;
        }
        ++iter;
        if (mode == 2 && j >= 0) thrs = fabs(sRdn[sInd[0]]);
        if ((j == L - 1) || (mode == 2 && (thrs - constraint < T(1e-15))) ||
            (mode == 0 && (thrs - constraint > T(-1e-15))) ||
            (newAtom && mode == 1 && (normX - constraint < T(1e-15))) || (normX < T(1e-15)) ||
            (iter >= length_path))
          break;
        __syncthreads();  // the state the next step's warp 0 rewrites has been read
      }
      iters = iter - 1;
      __syncthreads();
      if (!overflow) {
        if (j >= L) j = L - 1;  // (the loop leaves through a stop rule first)
        // the reference's final transform covers positions 0..j, which after
        // a drop is one position short of the active set
        const int tn = j + 1 < 0 ? 0 : j + 1;
        if (w0) {
          if (ols) {
            // coef(0:j) = Un RUn (the least-squares fit on the support)
            for (int r = lane; r < tn; r += 32) {
              T s = 0;
              for (int k = r; k < tn; ++k) s += sUn[(size_t)k * ld + r] * sRUn[k];
              sw[r] = s;
            }
            __syncwarp();
            for (int r = lane; r < tn; r += 32) scoef[r] = sw[r];
            __syncwarp();
          }
          for (int r = lane; r < tn; r += 32) scoef[r] *= ssig[r];  // vMul(j + 1, coef, sig)
        }
      }
    }
    __syncthreads();

    if (a.steps && threadIdx.x == 0 && !overflow) atomicAdd(a.steps, (unsigned long long)iters);
    if (overflow) {
      if (threadIdx.x == 0) {
        const int slot = atomicAdd(a.overflow_count, 1);
        a.overflow_list[slot] = sig_i;
        a.out_cnt[sig_i] = 0;
      }
    } else if (w0) {
      int* oind = a.out_ind + (size_t)sig_i * a.L;
      T* oval = a.out_val + (size_t)sig_i * a.L;
      for (int q = lane; q < nact; q += 32) {
        const int me = sInd[q];
        int rank = 0;
        for (int k = 0; k < nact; ++k) rank += sInd[k] < me;
        oind[rank] = me;
        oval[rank] = scoef[q];
      }
      if (lane == 0) a.out_cnt[sig_i] = nact;
    }
    __syncthreads();
  }
}

size_t lars_chol_state_bytes(int Kp, int Lc, size_t esz) { return chol_state_bytes(Kp, Lc, esz); }

template <typename T, int NV>
static cudaError_t launch_chol_nv(const LarsArgs<T>& a, int grid, int wpb, size_t smem,
                                  cudaStream_t st) {
  auto k = lars_chol_kernel<T, NV>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  e = fill_grid(k, wpb * 32, smem, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, wpb * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_lars_chol(const LarsArgs<T>& a, int grid, int wpb, cudaStream_t st) {
  const size_t smem = a.gstate ? 0 : (size_t)wpb * chol_state_bytes(a.Kp, a.Lcap, sizeof(T));
  switch (a.Kp / 128) {
    case 1: return launch_chol_nv<T, 1>(a, grid, wpb, smem, st);
    case 2: return launch_chol_nv<T, 2>(a, grid, wpb, smem, st);
    case 3: return launch_chol_nv<T, 3>(a, grid, wpb, smem, st);
    case 4: return launch_chol_nv<T, 4>(a, grid, wpb, smem, st);
    case 5: return launch_chol_nv<T, 5>(a, grid, wpb, smem, st);
    case 6: return launch_chol_nv<T, 6>(a, grid, wpb, smem, st);
    case 7: return launch_chol_nv<T, 7>(a, grid, wpb, smem, st);
    case 8: return launch_chol_nv<T, 8>(a, grid, wpb, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_lars_chol<float>(const LarsArgs<float>&, int, int, cudaStream_t);
template cudaError_t launch_lars_chol<double>(const LarsArgs<double>&, int, int, cudaStream_t);

size_t lars_chol_cta_smem_bytes(int Kp, int Lc, size_t esz, bool gstate) {
  const int W = Kp / 512;
  return chol_cta_head_bytes(Kp, W, esz) + (gstate ? 0 : chol_cta_small_bytes(Lc, esz));
}
size_t lars_chol_cta_gstate_bytes(int Lc, size_t esz) { return chol_cta_small_bytes(Lc, esz); }

template <typename T, int W>
static cudaError_t launch_chol_w(const LarsArgs<T>& a, int grid, size_t smem, cudaStream_t st) {
  auto k = lars_chol_cta_kernel<T, W>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess) return e;
  e = fill_grid(k, W * 32, smem, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_lars_chol_cta(const LarsArgs<T>& a, int grid, cudaStream_t st) {
  if (a.Kp % 512 != 0) return cudaErrorInvalidValue;
  const size_t smem = lars_chol_cta_smem_bytes(a.Kp, a.Lcap, sizeof(T), a.gstate != nullptr);
  switch (a.Kp / 512) {
    case 1: return launch_chol_w<T, 1>(a, grid, smem, st);
    case 2: return launch_chol_w<T, 2>(a, grid, smem, st);
    case 3: return launch_chol_w<T, 3>(a, grid, smem, st);
    case 4: return launch_chol_w<T, 4>(a, grid, smem, st);
    case 5: return launch_chol_w<T, 5>(a, grid, smem, st);
    case 6: return launch_chol_w<T, 6>(a, grid, smem, st);
    case 7: return launch_chol_w<T, 7>(a, grid, smem, st);
    case 8: return launch_chol_w<T, 8>(a, grid, smem, st);
    case 12: return launch_chol_w<T, 12>(a, grid, smem, st);
    case 16: return launch_chol_w<T, 16>(a, grid, smem, st);
    case 24: return launch_chol_w<T, 24>(a, grid, smem, st);
    case 32: return launch_chol_w<T, 32>(a, grid, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_lars_chol_cta<float>(const LarsArgs<float>&, int, cudaStream_t);
template cudaError_t launch_lars_chol_cta<double>(const LarsArgs<double>&, int, cudaStream_t);

}  // namespace sc
