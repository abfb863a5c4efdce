// Kernel argument blocks and launch entry points shared by the engine.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sc {

// Leading dimension of the small per-signal square matrices (inverse Gram,
// inverse Cholesky factor): odd, so that lanes walking a column hit distinct
// shared-memory banks.
__host__ __device__ inline int state_ld(int Lc) { return (Lc & 1) ? Lc : Lc + 1; }

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// Per-warp LARS state: DtR[Kp], invGs[Lc x ld], u/coef/sign/cA/w/g[Lc], ind[Lc].
__host__ __device__ inline size_t lars_state_bytes(int Kp, int Lc, size_t esz) {
  return align16(esz * ((size_t)Kp + (size_t)Lc * state_ld(Lc) + 6 * (size_t)Lc) +
                 4 * (size_t)Lc);
}

// Per-warp OMP state: Rdn[Kp], norm[Kp], Un[Lc x ld], RUn/vec/g[Lc], ind[Lc].
__host__ __device__ inline size_t omp_state_bytes(int Kp, int Lc, size_t esz) {
  return align16(esz * (2 * (size_t)Kp + (size_t)Lc * state_ld(Lc) + 3 * (size_t)Lc) +
                 4 * (size_t)Lc);
}

// Row masks of the masked variants (lasso_mask / omp_mask, decomp/decomp.h:
// 406-519, 1466-1561): a signal whose rows are all observed is coded as
// usual; one with some observed rows is coded against the Gram of its
// observed rows (D_mᵀ D_m + ridge I), whose entries the kernel forms on the
// fly: G_m(a, b) as a masked dot product of two atoms, and G_m(:, A) u as
// Dᵀ (mask ∘ (D_A u)).  Its correlations and ||x||^2 come from the masked
// signal (rows outside the mask set to zero).
template <typename T>
struct MaskArgs {
  const uint8_t* mask = nullptr;  // m x n chunk, column-major, nonzero = observed row
  const int8_t* flag = nullptr;   // n: 0 no row observed (empty code), 1 some, 2 all
  const T* D = nullptr;           // m x K column-major
  const T* Dt = nullptr;          // Kp x m column-major: Dᵀ with zero rows past K
  int m = 0, mpad = 0;
  T ridge = 0;                    // ridge of the masked Grams
  T* work = nullptr;              // one mpad-vector per warp of the launch (global)
};

template <typename T>
struct LarsArgs {
  const T* G;          // Kp x Kp, ld Kp, ridge included, zero padded
  const T* DtX;        // Kp x n, ld Kp (zero rows beyond K)
  const T* norms;      // n: ||x_i||^2
  int K, Kp;           // atoms, padded to a multiple of 128
  int L;               // driver L (clamped by the facade): slab stride, path cap
  int Lcap;            // active-set capacity of the per-warp state
  int mode;            // 0 L1COEFFS, 1 L2ERROR, 2 PENALTY
  T constraint;        // lambda1
  const T* vConstraint;  // per-signal lambda1 (device) or NULL
  int pos;
  int length_path;
  int n_jobs;          // signals in this launch
  const int* n_jobs_dev;    // if set, the job count is read from device memory
  const int64_t* sig_list;  // job -> signal index, or NULL for identity
  unsigned* work_counter;   // queue head, zero at launch
  int* out_ind;        // n x L slabs: sorted atom indices
  T* out_val;          // n x L slabs: coefficients
  int* out_cnt;        // n: active-set size (0 for overflowed signals)
  int64_t* overflow_list;   // signals whose active set outgrew Lcap
  int* overflow_count;
  T* gstate;           // NULL: state in shared memory; else per-warp global slabs
  T* path;             // K x length_path for signal 0, or NULL
  unsigned long long* steps;  // if set: total homotopy steps are added here
  T* out_level;        // if set: n correlation levels of the final active sets
  MaskArgs<T> mk;      // masked variant (mk.mask set), warp kernels only
  // FP64 refactor of the single-precision inverse Gram (refactor.cuh):
  // 0 never, 1 when an added atom's relative pivot falls below
  // kRefactorPivot, 2 on every added atom; rf_scratch: rf_units units of
  // rf_cap x rf_cap doubles, one per warp (warp kernels) or per CTA (CTA
  // kernels) of the launch; active sets of up to rf_cap atoms are refactored
  int refactor;
  double* rf_scratch;
  int rf_cap, rf_units;
  int ols;             // Cholesky kernel only: final least-squares fit on the support
};

template <typename T>
struct OmpArgs {
  const T* G;          // Kp x Kp, ld Kp, no ridge, zero padded
  const T* DtX;        // Kp x n
  const T* norms;      // n
  int K, Kp;
  int L;               // driver L: min(m, L, K); slab stride
  int Lcap;
  T eps, lambda;       // scalar stopping values
  int Lsig;            // scalar per-signal L (before the min with L)
  const int* vL;       // per-signal L (device) or NULL
  const T* vEps;       // per-signal eps or NULL
  const T* vLambda;    // per-signal lambda or NULL
  int n_jobs;
  const int* n_jobs_dev;
  const int64_t* sig_list;
  unsigned* work_counter;
  int* out_ind;
  T* out_val;
  int* out_cnt;
  int64_t* overflow_list;
  int* overflow_count;
  T* gstate;
  T* path;             // K x L for signal 0, or NULL
  unsigned long long* steps;  // if set: total OMP steps are added here
  MaskArgs<T> mk;      // masked variant (mk.mask set), warp kernels only
  // FP64 refactor of the single-precision inverse Cholesky factor when the
  // selected atom's residual norm (its pivot) falls below kRefactorPivot (1)
  // or on every selected atom (2); scratch as in LarsArgs
  int refactor;
  double* rf_scratch;
  int rf_cap, rf_units;
};

template <typename T>
cudaError_t launch_lars(const LarsArgs<T>& a, int grid, int warps_per_block, cudaStream_t st);
template <typename T>
int lars_max_warps_per_sm(int Kp);

// One CTA of Kp / 512 warps per signal (Kp a multiple of 512: 512..4096, 6144,
// 8192, 12288 or 16384);
// a.gstate set: per-CTA small state in global slabs (lars_cta_gstate_bytes).
// grid <= 0: as many persistent blocks as fit on the device.
template <typename T>
cudaError_t launch_lars_cta(const LarsArgs<T>& a, int grid, cudaStream_t st);
template <typename T>
size_t lars_cta_smem_bytes(int Kp, int Lc, bool gstate);
template <typename T>
size_t lars_cta_gstate_bytes(int Lc, int grid);
// The persistent grid the CTA launcher fills the device with (0 on error).
template <typename T>
int lars_cta_grid(int Kp, int Lc, bool gstate);

// The Cholesky implementation of the homotopy (coreLARS + downDateLasso),
// one warp per signal, Kp <= 1024 (lars_chol.cu); a.gstate set: per-warp
// state in global slabs of lars_chol_state_bytes(Kp, a.Lcap, sizeof(T)).
// grid <= 0: as many persistent blocks as fit on the device.
template <typename T>
cudaError_t launch_lars_chol(const LarsArgs<T>& a, int grid, int warps_per_block, cudaStream_t st);
size_t lars_chol_state_bytes(int Kp, int Lc, size_t esz);
// Its CTA form: one CTA of Kp / 512 warps per signal (Kp as for
// launch_lars_cta); a.gstate set: per-CTA small state in global slabs of
// lars_chol_cta_gstate_bytes(a.Lcap, sizeof(T)).
template <typename T>
cudaError_t launch_lars_chol_cta(const LarsArgs<T>& a, int grid, cudaStream_t st);
size_t lars_chol_cta_smem_bytes(int Kp, int Lc, size_t esz, bool gstate);
size_t lars_chol_cta_gstate_bytes(int Lc, size_t esz);

template <typename T>
cudaError_t launch_omp(const OmpArgs<T>& a, int grid, int warps_per_block, cudaStream_t st);
template <typename T>
cudaError_t launch_omp_cta(const OmpArgs<T>& a, int grid, cudaStream_t st);
template <typename T>
size_t omp_cta_smem_bytes(int Kp, int Lc, bool gstate);
template <typename T>
size_t omp_cta_gstate_bytes(int Lc, int grid);
// The persistent grid the OMP CTA launcher fills the device with (0 on error).
template <typename T>
int omp_cta_grid(int Kp, int Lc, bool gstate);
template <typename T>
int omp_max_warps_per_sm(int Kp);

// ---- masked variants
template <typename T>
cudaError_t launch_transpose_pad(const T* D, int m, int K, int Kp, T* Dt, cudaStream_t st);
// X (in place): unobserved rows zeroed; flag: 0 / 1 / 2 = none / some / all
// rows observed; out = value * count / m when some rows are and `scale`,
// value otherwise (value = vbase[j], or base when vbase is NULL).
template <typename T>
cudaError_t launch_mask_prep(T* X, int m, int64_t n, const uint8_t* mask, int8_t* flag,
                             const T* vbase, T base, int scale, T* out, cudaStream_t st);

// ---- dense products ------------------------------------------------------
// C (Kp x n, ld ldc) = A^T B with A m x Ka (ld lda), B m x n (ld ldb),
// column-major; rows Ka..Kp-1 of C are written as zero.
template <typename T>
cudaError_t launch_gemm_tn(const T* A, int lda, int Ka, const T* B, int ldb,
                           int64_t n, int m, T* C, int ldc, int Kp, cudaStream_t st);
// G (Kp x Kp) = D^T D + ridge I on the first K diagonal entries, symmetric,
// zero beyond K.
template <typename T>
cudaError_t launch_gram(const T* D, int m, int K, int Kp, T ridge, T* G, cudaStream_t st);
// Mirror G's upper triangle into the lower one, add the ridge to the first K
// diagonal entries, zero rows / columns K..Kp-1.
template <typename T>
cudaError_t launch_symmetrize(T* G, int K, int Kp, T ridge, cudaStream_t st);
// norms[i] = ||x_i||^2
template <typename T>
cudaError_t launch_colnorms(const T* X, int m, int64_t n, T* norms, cudaStream_t st);
// Copy a K x n block (ld ldsrc) into a Kp x n block (ld Kp), zero padding.
template <typename T>
cudaError_t launch_pad_rows(const T* src, int K, int64_t ldsrc, int64_t n, T* dst,
                            int Kp, cudaStream_t st);

// ---- double-precision solves on the final active sets ---------------------
// For every signal with a non-empty active set A (sorted atom indices and
// coefficients in the slabs):
//     a_A = G_AA^{-1} (D_A^T x - level * sign(a_A))   (level != NULL: lasso refinement)
//     a_A = G_AA^{-1}  D_A^T x                        (level == NULL: OMP refinement, ols)
// in double precision.  D_A^T x comes from D and X, or from Q (the caller's
// D^T X, ld ldq) when Q is given.  Active sets of more than 32 atoms go to a
// second pass (big_grid blocks of 4 warps, each warp a slab of
// L (L + 1) + L doubles in `scratch`, refine_scratch_bytes).
template <typename T>
cudaError_t launch_refine(const T* D, int m, const T* X, const T* Q, int ldq, const T* G, int Kp,
                          const int* slab_ind, T* slab_val, int L, const int* cnt, const T* level,
                          int64_t n, int64_t* big_list, int* big_count, unsigned* counter,
                          double* scratch, int big_grid, cudaStream_t st);
size_t refine_scratch_bytes(int L, int grid);

// ---- CSC assembly ----------------------------------------------------------
// colptr[i+1] = base + cnt[0] + ... + cnt[i]; with base == NULL the base is 0
// and colptr[0] is written as 0, otherwise colptr[0] is left alone (it is
// *base, written by the previous chunk).
cudaError_t launch_scan_counts(const int* cnt, int64_t n, int64_t* colptr, const int64_t* base,
                               int64_t* scratch, int64_t scratch_len, cudaStream_t st);
int64_t scan_scratch_len(int64_t n);
// rows/vals[colptr[i] - *sub + j] = slab pairs of column i (sub NULL: 0).
// A column that would not fit in `cap` entries is skipped and *capflag set.
template <typename T>
cudaError_t launch_csc_gather(const int* slab_ind, const T* slab_val, int L,
                              const int* cnt, const int64_t* colptr, int64_t n,
                              const int64_t* sub, int64_t cap, int* capflag,
                              int32_t* rows, T* vals, cudaStream_t st);

// list[0..n) = 0..n-1 ordered by descending min(vL[i], Lmax) (ties in no
// particular order): the longest-first schedule of a persistent launch.
// scratch: Lmax + 1 ints; Lmax <= kOrderMaxL.  Four launches (a memset and
// three kernels).
constexpr int kOrderMaxL = 4096;
cudaError_t launch_order_by_L_desc(const int* vL, int64_t n, int Lmax, int* scratch,
                                   int64_t* list, cudaStream_t st);

// ---- BF16 hi/lo split tensor-core products (sm_100a tcgen05) --------------
bool tc_gemm_available();
// rows of the bf16 split operands: m rounded up to the 64-element k-block
int tc_pad_m(int m);
// x (rows x cols fp32, ld ldx) -> hi / lo bf16 (rows_pad x cols), zero padded
// With lo3 set, also the third piece lo3 = bf16(x - hi - lo) (hi + lo + lo3
// carries FP32's 24 significant bits).
cudaError_t launch_bf16_split(const float* x, int rows, int64_t ldx, int64_t cols, int rows_pad,
                              void* hi, void* lo, cudaStream_t st, void* lo3 = nullptr);
// C = sum over the first `nterms` of (Dhi,Xhi), (Dhi,Xlo), (Dlo,Xhi) of
// D^T X on tcgen05: rows 0..rows_out-1 (rows_out <= K rounded up to 128;
// rows beyond K come out zero) of each of the n columns (ld ldc).  *err is
// set when a bounded wait gave up.
cudaError_t launch_tc_corr(const void* Dhi, const void* Dlo, int K, const void* Xhi,
                           const void* Xlo, int64_t n, int m_pad, int nterms, float* C, int ldc,
                           int rows_out, int* err, cudaStream_t st);
// The same product for fp32 X (m x n, ld ldx >= m) with the split of X done
// inside the kernel (persistent, one CTA per SM, two TMEM accumulators).
cudaError_t launch_tc_corr_fused(const void* Dhi, const void* Dlo, int K, const float* X,
                                 int64_t ldx, int m, int64_t n, int m_pad, float* C, int ldc,
                                 int rows_out, int* err, cudaStream_t st);
// The X-stationary form: D given as np bf16 pieces (2: hi, lo with three
// products; 3: hi, mid, lo with six, FP32-grade), X fp32 split in the
// kernel once per signal tile.  cudaErrorNotSupported where a signal tile's
// pieces do not fit in shared memory (large m); the caller then takes
// launch_tc_corr_fused.
cudaError_t launch_tc_corr_xs(const void* const* Dpieces, int np, int K, const float* X,
                              int64_t ldx, int m, int64_t n, int m_pad, float* C, int ldc,
                              int rows_out, int* err, cudaStream_t st);
// G (Kp x Kp) = D^T D + ridge I from the three-piece BF16 split of D
// (hi, mid = the lo half of the two-piece split, lo3; m_pad x K each) and D
// itself (fp32, m x K): six tensor-core products, FP32-grade, symmetrised,
// zero beyond K (the FP32 CUDA-core product where the tensor-core form does
// not apply).
cudaError_t launch_gram_tc(const void* Dhi, const void* Dmid, const void* Dlo3, const float* D,
                           int m, int m_pad, int K, int Kp, float ridge, float* G, int* err,
                           cudaStream_t st);

}  // namespace sc
