// Dictionary-learning inner loop: the minibatch step of Trainer::train
// (dictLearn/dicts.h:526-603) on the device.
//
// One step, all on one stream and without host synchronisation (so that it
// can be captured in a CUDA graph and replayed per minibatch):
//   1. G = DᵀD + max(lambda2, 1e-10) I                         (dicts.h:528-532)
//   2. the minibatch x_j = X[:, perm[(j + it * batch) % M]], j < batch, with
//      `it` read from a device counter                          (dicts.h:548)
//   3. its codes: coreLARS2 in modes L1COEFFS / L2ERROR / PENALTY, coreORMPB in
//      SPARSITY (L = lambda), L2ERROR2 (eps = lambda) and PENALTY2
//      (lambda = lambda)                                        (dicts.h:569-588)
//   4. A <- beta A + gamma sum_j a_j a_jᵀ and B <- beta B + gamma sum_j x_j a_jᵀ,
//      the rank-1 accumulations of AT / BT (dicts.h:597-598)
//   5. it <- it + 1
// The codes go through the same coding pipeline as the C ABI calls.  The
// accumulations are deterministic: the codes are regrouped by atom (counting
// sort, then each atom's signals in increasing order) and column k of A and B
// sums its signals in that order, like the reference's sequential loop.
#include <algorithm>

#include "common.cuh"
#include "engine.h"
#include "kernels.h"

namespace sc {

namespace {

__global__ void dl_gather_kernel(const float* __restrict__ X, int m, int64_t M,
                                 const int32_t* __restrict__ perm, const int64_t* __restrict__ it,
                                 int batch, float* __restrict__ Xb) {
  const int j = blockIdx.x;
  if (j >= batch) return;
  const int64_t pos = ((int64_t)j + *it * (int64_t)batch) % M;
  const int64_t src = perm ? (int64_t)perm[pos] : pos;
  const float* x = X + (size_t)src * m;
  float* y = Xb + (size_t)j * m;
  for (int r = threadIdx.x; r < m; r += blockDim.x) y[r] = x[r];
}

// per-atom counts of the codes
__global__ void dl_count_kernel(const int64_t* __restrict__ colptr, const int32_t* __restrict__ rows,
                                int n, int* __restrict__ cntK) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= n) return;
  for (int64_t e = colptr[j] + (threadIdx.x & 31); e < colptr[j + 1]; e += 32)
    atomicAdd(&cntK[rows[e]], 1);
}

// codes regrouped by atom (signal order fixed by the sort below)
__global__ void dl_fill_kernel(const int64_t* __restrict__ colptr, const int32_t* __restrict__ rows,
                               const float* __restrict__ vals, int n,
                               const int64_t* __restrict__ ptrK, int* __restrict__ fillK,
                               int* __restrict__ sigK, float* __restrict__ valK) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= n) return;
  for (int64_t e = colptr[j] + (threadIdx.x & 31); e < colptr[j + 1]; e += 32) {
    const int k = rows[e];
    const int64_t p = ptrK[k] + atomicAdd(&fillK[k], 1);
    sigK[p] = j;
    valK[p] = vals[e];
  }
}

// each atom's list in increasing signal order (one warp per atom, rank sort
// through a scratch copy; signal indices are distinct within an atom)
__global__ void dl_sort_kernel(const int64_t* __restrict__ ptrK, int K, int* __restrict__ sigK,
                               float* __restrict__ valK, int* __restrict__ sigT,
                               float* __restrict__ valT) {
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= K) return;
  const int64_t p0 = ptrK[k], c = ptrK[k + 1] - p0;
  if (c <= 1) return;
  for (int64_t a = lane; a < c; a += 32) {
    sigT[p0 + a] = sigK[p0 + a];
    valT[p0 + a] = valK[p0 + a];
  }
  __syncwarp();
  for (int64_t a = lane; a < c; a += 32) {
    const int me = sigT[p0 + a];
    int64_t rank = 0;
    for (int64_t b = 0; b < c; ++b) rank += sigT[p0 + b] < me;
    sigK[p0 + rank] = me;
    valK[p0 + rank] = valT[p0 + a];
  }
}

// column k of A and B: beta * old + gamma * (sum over the atom's signals, in
// increasing signal order)
__global__ void __launch_bounds__(256)
dl_accumulate_kernel(const int64_t* __restrict__ colptr, const int32_t* __restrict__ rows,
                     const float* __restrict__ vals, const float* __restrict__ Xb, int m, int K,
                     const int64_t* __restrict__ ptrK, const int* __restrict__ sigK,
                     const float* __restrict__ valK, float* __restrict__ A,
                     float* __restrict__ B, float beta, float gamma) {
  extern __shared__ float acc[];  // K
  const int k = blockIdx.x;
  const int64_t p0 = ptrK[k], p1 = ptrK[k + 1];
  if (A) {
    for (int r = threadIdx.x; r < K; r += blockDim.x) acc[r] = 0.f;
    __syncthreads();
    for (int64_t p = p0; p < p1; ++p) {
      const int j = sigK[p];
      const float v = valK[p];
      // the rows of one signal are distinct: no two threads share an entry
      for (int64_t e = colptr[j] + threadIdx.x; e < colptr[j + 1]; e += blockDim.x)
        acc[rows[e]] += v * vals[e];
      __syncthreads();
    }
    float* a = A + (size_t)k * K;
    for (int r = threadIdx.x; r < K; r += blockDim.x)
      a[r] = (beta == 0.f ? 0.f : beta * a[r]) + gamma * acc[r];
  }
  if (B) {
    float* b = B + (size_t)k * m;
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      float s = 0.f;
      for (int64_t p = p0; p < p1; ++p) s += valK[p] * Xb[(size_t)sigK[p] * m + r];
      b[r] = (beta == 0.f ? 0.f : beta * b[r]) + gamma * s;
    }
  }
}

__global__ void dl_advance_kernel(int64_t* it) { *it += 1; }

}  // namespace
}  // namespace sc

using namespace sc;

struct sc_dl {
  int device = 0;
  int m = 0, K = 0, Kp = 0, batch = 0;
  int mode = 2;
  float lambda1 = 0, lambda2 = 0;
  int pos = 0, precision = 0;
  int L = 0;
  bool profile = false;
  DeviceCtx* ctx = nullptr;
  Buf G, Xb, split, colptr, rows, vals, cntK, ptrK, fillK, sigK, valK, sigT, valT, scan, tcerr;
};

extern "C" {

sc_status sc_dl_create(int device, int m, int K, int batch, int mode, float lambda1,
                       float lambda2, int posAlpha, int precision, sc_dl** out) {
  if (!out) return fail(SC_ERR_INVALID_ARG, "dictionary learning: null output");
  *out = nullptr;
  if (m <= 0 || K <= 0 || batch <= 0)
    return fail(SC_ERR_INVALID_ARG, "dictionary learning: bad dimensions");
  if (mode < 0 || mode > 5)
    return fail(SC_ERR_UNSUPPORTED, "dictionary learning: mode %d not supported", mode);
  if (mode == 2 && lambda1 == 0.f && lambda2 > 0.f && !posAlpha)
    return fail(SC_ERR_UNSUPPORTED,
                "dictionary learning: the ridge-only conjugate-gradient case is not implemented");
  if (precision != SC_PREC_FP32 && precision != SC_PREC_BF16X3)
    return fail(SC_ERR_INVALID_ARG, "unknown precision mode %d", precision);
  if (precision == SC_PREC_BF16X3 && !tc_gemm_available())
    return fail(SC_ERR_UNSUPPORTED, "BF16x3 products need the CUDA driver's tensor-map encoder");
  SC_TRY(check_atoms(K));
  DeviceCtx* c = nullptr;
  SC_TRY(create_ctx(device, &c));
  sc_dl* s = new sc_dl();
  s->device = device;
  s->m = m;
  s->K = K;
  s->Kp = pad_atoms(K);
  s->batch = batch;
  s->mode = mode;
  s->lambda1 = lambda1;
  s->lambda2 = lambda2;
  s->pos = posAlpha != 0;
  s->precision = precision;
  s->ctx = c;
  // dicts.h:386-387: L = lambda in SPARSITY mode, min(m, K) otherwise
  s->L = mode == 3 ? std::min((int)lambda1, std::min(m, K)) : std::min(m, K);
  if (s->L < 1) {
    sc_dl_destroy(s);
    return fail(SC_ERR_INVALID_ARG, "dictionary learning: L = %d", s->L);
  }
  *out = s;
  return SC_OK;
}

sc_status sc_dl_destroy(sc_dl* s) {
  if (!s) return SC_OK;
  cudaSetDevice(s->device);
  if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
  for (Buf* b : {&s->G, &s->Xb, &s->split, &s->colptr, &s->rows, &s->vals, &s->cntK, &s->ptrK,
                 &s->fillK, &s->sigK, &s->valK, &s->sigT, &s->valT, &s->scan, &s->tcerr})
    b->release();
  destroy_ctx(s->ctx);
  delete s;
  return SC_OK;
}

sc_status sc_dl_step_f32(sc_dl* s, const float* dD, const float* dX, int64_t M,
                         const int32_t* dperm, int64_t* d_iter, float* dA, float* dB, float beta,
                         float gamma, void* stream) {
  if (!s || !dD || !dX || !d_iter || M <= 0)
    return fail(SC_ERR_INVALID_ARG, "dictionary learning: null argument or empty X");
  SC_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int m = s->m, K = s->K, Kp = s->Kp, n = s->batch, L = s->L;
  // workspaces (grown on the first step; a captured step must not grow them)
  SC_TRY(s->G.reserve((size_t)Kp * Kp * 4));
  SC_TRY(s->Xb.reserve((size_t)m * n * 4));
  SC_TRY(s->colptr.reserve((size_t)(n + 1) * 8));
  SC_TRY(s->rows.reserve((size_t)n * L * 4));
  SC_TRY(s->vals.reserve((size_t)n * L * 4));
  SC_TRY(s->cntK.reserve((size_t)K * 4));
  SC_TRY(s->fillK.reserve((size_t)K * 4));
  SC_TRY(s->ptrK.reserve((size_t)(K + 1) * 8));
  for (Buf* b : {&s->sigK, &s->sigT}) SC_TRY(b->reserve((size_t)n * L * 4));
  for (Buf* b : {&s->valK, &s->valT}) SC_TRY(b->reserve((size_t)n * L * 4));
  const int64_t slen = scan_scratch_len(K);
  SC_TRY(s->scan.reserve((size_t)slen * 8));
  const bool tc = s->precision == SC_PREC_BF16X3;
  const int mp = tc_pad_m(m);
  if (tc) SC_TRY(s->split.reserve((size_t)mp * K * 6));  // hi, lo, lo3 pieces of D
  if (tc) SC_TRY(s->tcerr.reserve(256));

  // the thread's sc_profile describes this step: its launches always, its
  // coding stages' times when profiling is on
  profile_reset();
  int own_launches = 0;
  // 1. Gram with the ridge: FP32, or in the BF16x3 form from the three-piece
  // split of the updated D on the tensor cores (FP32-grade)
  float* G = reinterpret_cast<float*>(s->G.ptr);
  const float ridge = std::max(s->lambda2, 1e-10f);
  if (tc) {
    char* sp = static_cast<char*>(s->split.ptr);
    const size_t piece = (size_t)mp * K * 2;
    SC_CUDA(launch_bf16_split(dD, m, m, K, mp, sp, sp + piece, st, sp + 2 * piece));
    SC_CUDA(launch_gram_tc(sp, sp + piece, sp + 2 * piece, dD, m, mp, K, Kp, ridge, G,
                           reinterpret_cast<int*>(s->tcerr.ptr), st));
    own_launches += 3;
  } else {
    SC_CUDA(launch_gram<float>(dD, m, K, Kp, ridge, G, st));
    own_launches += 2;
  }
  // 2. the minibatch
  float* Xb = reinterpret_cast<float*>(s->Xb.ptr);
  dl_gather_kernel<<<n, 128, 0, st>>>(dX, m, M, dperm, d_iter, n, Xb);
  SC_CUDA(cudaGetLastError());
  own_launches += 1;
  // 3. its codes
  BatchDesc b;
  b.lars = s->mode <= 2;
  b.dX = Xb;
  b.m = m;
  b.n = n;
  b.dD = dD;
  b.G = G;
  b.dDsplit = tc ? s->split.ptr : nullptr;
  b.K = K;
  b.Kp = Kp;
  b.L = L;
  b.tc = tc;
  if (b.lars) {
    b.mode = s->mode;
    b.pos = s->pos;
    b.lambda1 = s->lambda1;
    b.length_path = 4 * L;  // coreLARS2's default path length (decomp/decomp.h:1722)
  } else {
    b.Lsig = L;
    b.eps = s->mode == 4 ? s->lambda1 : 0.f;
    b.lambda = s->mode == 5 ? s->lambda1 : 0.f;
  }
  int64_t* colptr = reinterpret_cast<int64_t*>(s->colptr.ptr);
  int32_t* rows = reinterpret_cast<int32_t*>(s->rows.ptr);
  float* vals = reinterpret_cast<float*>(s->vals.ptr);
  b.d_colptr = colptr;
  b.d_rows = rows;
  b.d_vals = vals;
  b.cap = (int64_t)n * L;
  b.stream = st;
  b.profile = s->profile;
  SC_TRY(code_batch_f32(*s->ctx, b));
  // 4. A and B
  if (dA || dB) {
    int* cntK = reinterpret_cast<int*>(s->cntK.ptr);
    int* fillK = reinterpret_cast<int*>(s->fillK.ptr);
    int64_t* ptrK = reinterpret_cast<int64_t*>(s->ptrK.ptr);
    int* sigK = reinterpret_cast<int*>(s->sigK.ptr);
    float* valK = reinterpret_cast<float*>(s->valK.ptr);
    SC_CUDA(cudaMemsetAsync(cntK, 0, (size_t)K * 4, st));
    SC_CUDA(cudaMemsetAsync(fillK, 0, (size_t)K * 4, st));
    const int wblocks = (n + 7) / 8;
    dl_count_kernel<<<wblocks, 256, 0, st>>>(colptr, rows, n, cntK);
    SC_CUDA(cudaGetLastError());
    SC_CUDA(launch_scan_counts(cntK, K, ptrK, nullptr, reinterpret_cast<int64_t*>(s->scan.ptr),
                               slen, st));
    dl_fill_kernel<<<wblocks, 256, 0, st>>>(colptr, rows, vals, n, ptrK, fillK, sigK, valK);
    SC_CUDA(cudaGetLastError());
    dl_sort_kernel<<<(K + 7) / 8, 256, 0, st>>>(ptrK, K, sigK, valK,
                                                reinterpret_cast<int*>(s->sigT.ptr),
                                                reinterpret_cast<float*>(s->valT.ptr));
    SC_CUDA(cudaGetLastError());
    const size_t smem = dA ? (size_t)K * 4 : 0;
    if (smem > 48 * 1024)
      SC_CUDA(cudaFuncSetAttribute(dl_accumulate_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dl_accumulate_kernel<<<K, 256, smem, st>>>(colptr, rows, vals, Xb, m, K, ptrK, sigK, valK, dA,
                                               dB, beta, gamma);
    SC_CUDA(cudaGetLastError());
    own_launches += 7;  // count, the three scan kernels, fill, sort, accumulate
  }
  // 5. next minibatch
  dl_advance_kernel<<<1, 1, 0, st>>>(d_iter);
  SC_CUDA(cudaGetLastError());
  profile_add_launches(own_launches + 1);
  return SC_OK;
}

sc_status sc_dl_profile(sc_dl* s, int on) {
  if (!s) return fail(SC_ERR_INVALID_ARG, "dictionary learning: null argument");
  s->profile = on != 0;
  return SC_OK;
}

sc_status sc_dl_codes(sc_dl* s, const int64_t** colptr, const int32_t** rows, const float** vals) {
  if (!s || !colptr || !rows || !vals) return fail(SC_ERR_INVALID_ARG, "dictionary learning: null argument");
  *colptr = reinterpret_cast<const int64_t*>(s->colptr.ptr);
  *rows = reinterpret_cast<const int32_t*>(s->rows.ptr);
  *vals = reinterpret_cast<const float*>(s->vals.ptr);
  return SC_OK;
}

}  // extern "C"
