/* spams_b200.h - C ABI of the B200 batched sparse-coding engine.
 *
 * The engine codes every column x_i of a signal matrix X (m x n, column-major)
 * against a dictionary D (m x K, column-major, unit-norm columns for OMP) with
 * Orthogonal Matching Pursuit or LARS-Lasso, on one GPU, and returns the codes
 * as a K x n CSC matrix with row indices sorted inside each column.
 *
 * These entry points are what the SPAMS facade calls would bind to; each one
 * names the reference interface it replaces.  Semantics (argument meaning,
 * clamps of L, stopping rules, first-index tie-breaks, error strings) follow
 * the reference; numThreads is accepted and ignored (the work runs on the GPU).
 *
 * Host vs device pointers:
 *   sc_omp_* / sc_lasso_* / sc_lasso_gram_* take HOST arrays and return a CSC
 *   matrix in host arrays owned by the library (page-locked blocks from a
 *   reused pool where possible, else malloc'd; free them with sc_csc_free,
 *   never with free()).  They copy the inputs to the device, run, and copy
 *   the result back (blocking).
 *   sc_*_dev variants take DEVICE arrays, write the CSC into caller-provided
 *   device arrays and run asynchronously on the given CUDA stream.
 *
 * Every entry point returns an sc_status; sc_last_error() gives a message.
 * There is no CPU fallback: without a usable CUDA device the calls return
 * SC_ERR_NO_DEVICE.
 */
#ifndef SPAMS_B200_H
#define SPAMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SC_OK = 0,
  SC_ERR_INVALID_ARG = 1,    /* null pointer / negative size / bad option */
  SC_ERR_DIMENSIONS = 2,     /* "incompatible matrix dimensions" (facade throw) */
  SC_ERR_NO_CRITERION = 3,   /* omp: "You should either provide L, eps or lambda" */
  SC_ERR_CUDA = 4,           /* a CUDA runtime call failed */
  SC_ERR_OUT_OF_MEMORY = 5,  /* device or host allocation failed */
  SC_ERR_NO_DEVICE = 6,      /* no CUDA device / driver: no CPU fallback exists */
  SC_ERR_CAPACITY = 7,       /* device CSC output arrays too small (nnz reported) */
  SC_ERR_TIMEOUT = 8,        /* a bounded device-side wait gave up */
  SC_ERR_UNSUPPORTED = 9     /* option combination not implemented */
} sc_status;

/* Lasso constraint modes: enum constraint_type, decomp/decomp.h:95. */
enum { SC_L1COEFFS = 0, SC_L2ERROR = 1, SC_PENALTY = 2 };

/* Numerical form of the correlation / Gram products.
 *   SC_PREC_FP32: plain FP32 products (CUDA cores), FP32 iterations.
 *   SC_PREC_BF16X3: tcgen05 tensor-core products from a BF16 hi/lo split
 *                   (hi*hi + hi*lo + lo*hi, FP32 accumulate), FP32 iterations;
 *                   with sc_options.refine, FP64 refinement of the final
 *                   active-set coefficients.
 * Double-precision entry points always compute in FP64. */
enum { SC_PREC_FP32 = 0, SC_PREC_BF16X3 = 1 };

/* CSC result in host memory (reference SpMatrix<T>, linalg/linalg.h:775-935):
 * colptr has n+1 entries (pB; pE = pB+1), rows/vals have nnz entries. */
typedef struct {
  int64_t m, n, nnz;
  int64_t* colptr;
  int32_t* rows;
  float* vals;
} sc_csc_f32;

typedef struct {
  int64_t m, n, nnz;
  int64_t* colptr;
  int32_t* rows;
  double* vals;
} sc_csc_f64;

/* Per-call engine options; zero-initialise for defaults. */
typedef struct {
  int precision;  /* SC_PREC_* (single precision calls only); default FP32 */
  int device;     /* CUDA device ordinal; default 0 */
  int profile;    /* nonzero: time each stage with CUDA events and count the
                     coding steps (the call then synchronises its stream) */
  int refine;     /* > 0: refine the final single-precision coefficients in
                     FP64 on their active sets (from D, X and the Gram);
                     default off */
  int kernel;     /* SC_KERNEL_*: which coding kernels may run; default
                     SC_KERNEL_AUTO (timed once per shape, then cached).
                     Every choice gives the same results. */
  int refactor;   /* single-precision calls: 0 (default) rebuilds the active
                     set's state in FP64 when an added atom's pivot falls
                     below 1e-3 of its diagonal (Lasso: the inverse Gram;
                     OMP: the inverse Cholesky factor, the projections RUn and
                     the residual norm), for active sets up to 96 atoms;
                     > 0 on every added atom; < 0 never */
  int reserved[2];
} sc_options;

/* Coding kernels: one warp per signal (up to 1024 atoms) or one CTA of
 * Kp / 512 warps per signal (Kp, the padded atom count, a multiple of 512).
 * SC_KERNEL_AUTO lets the engine time the admissible ones on the first call
 * of each shape (set SC_AUTOTUNE=0 in the environment for the static rule:
 * warp up to 1024 atoms, CTA beyond). */
enum { SC_KERNEL_AUTO = 0, SC_KERNEL_WARP = 1, SC_KERNEL_CTA = 2 };

/* What the calling thread's last coding call did on the device.  Stage times
 * are filled only when that call ran with sc_options.profile set. */
typedef struct {
  double ms_gram;      /* Gram matrix D^T D (+ ridge) */
  double ms_norms;     /* ||x_i||^2 */
  double ms_corr;      /* correlations D^T X */
  double ms_code;      /* OMP / LARS kernels, overflow rerun included */
  double ms_refine;    /* FP64 refinement of the final coefficients (BF16X3) */
  double ms_csc;       /* CSC scan and gather */
  double ms_total;     /* first to last stage event */
  int64_t launches;    /* engine kernels launched by the call */
  int64_t signals;     /* signals coded */
  int64_t steps;       /* OMP / LARS steps summed over the signals (profile) */
  int64_t overflowed;  /* signals rerun with global-memory state (profile) */
  int32_t kernel;      /* coding kernel family of the last chunk: SC_KERNEL_WARP or
                          SC_KERNEL_CTA */
  int32_t lcap;        /* its active-set capacity in shared memory (atoms) */
} sc_profile;

/* ---- library / status ------------------------------------------------- */
const char* sc_version(void);
const char* sc_last_error(void);          /* thread-local message of the last failure */
sc_status sc_device_count(int* count);    /* number of usable CUDA devices */
void sc_csc_free_f32(sc_csc_f32* a);      /* frees colptr/rows/vals, zeroes the struct */
void sc_csc_free_f64(sc_csc_f64* a);
/* Releases the engine's cached device workspaces and streams on all devices,
 * returns the free blocks of the stream-ordered memory pool the workspaces
 * grow from to the device, and frees the unused page-locked result blocks. */
void sc_release_all(void);
/* Copies the calling thread's last-call profile (see sc_profile). */
sc_status sc_last_profile(sc_profile* out);

/* ---- OMP ----------------------------------------------------------------
 * Replaces _omp<T> (cpp_library/spams.h:250-293) -> omp<T>
 * (decomp/decomp.h:322-404) -> coreORMP (decomp/decomp.h:538-640).
 *   L, eps, lambda: arrays of 1 (scalar) or n (per signal) entries; an array
 *   with count 0 means "not given" (defaults L=min(m,K), eps=0, lambda=0; at
 *   least one must be given).  path (optional): K x min(m,K) column-major,
 *   receives the regularisation path of the first signal. */
sc_status sc_omp_f32(const float* X, int m, int64_t n, const float* D, int K,
                     const int* L, int64_t nL, const float* eps, int64_t nEps,
                     const float* lambda, int64_t nLambda, int numThreads,
                     float* path, const sc_options* opt, sc_csc_f32* out);
sc_status sc_omp_f64(const double* X, int m, int64_t n, const double* D, int K,
                     const int* L, int64_t nL, const double* eps, int64_t nEps,
                     const double* lambda, int64_t nLambda, int numThreads,
                     double* path, const sc_options* opt, sc_csc_f64* out);

/* ---- LARS-Lasso ---------------------------------------------------------
 * Replaces _lassoD<T> (cpp_library/spams.h:107-143) -> lasso2<T>
 * (decomp/decomp.h:1563-1571, 1574-1646) -> coreLARS2 (:1706-1915).
 *   L < 0: K; max_length_path < 0: 4L; clamps as the facade.
 *   mode: SC_L1COEFFS / SC_L2ERROR / SC_PENALTY; pos: non-negative codes.
 *   path (optional): K x max_length_path, path of the first signal.
 *   ols / cholesky select the reference's Cholesky implementation (lasso<T>
 *   -> coreLARS + downDateLasso, decomp/decomp.h:735-1203; ols implies it, as
 *   in _lassoD): its own stopping rules in all three modes, and with ols the
 *   final least-squares fit on the support.  Dictionaries as the coding
 *   kernels (one warp per signal up to 1024 atoms, one CTA beyond). */
sc_status sc_lasso_f32(const float* X, int m, int64_t n, const float* D, int K,
                       int L, float lambda1, float lambda2, int mode, int pos,
                       int ols, int numThreads, int max_length_path,
                       int cholesky, float* path, const sc_options* opt,
                       sc_csc_f32* out);
sc_status sc_lasso_f64(const double* X, int m, int64_t n, const double* D, int K,
                       int L, double lambda1, double lambda2, int mode, int pos,
                       int ols, int numThreads, int max_length_path,
                       int cholesky, double* path, const sc_options* opt,
                       sc_csc_f64* out);

/* Precomputed products: replaces _lassoQq<T> (cpp_library/spams.h:145-188)
 * -> lasso2<T>(Data X, G, DtX) (decomp/decomp.h:1574-1646).
 *   Q = G (K x K, used as given: no ridge added), q = D^T X (K x n);
 *   X only supplies ||x_i||^2 and the signal length m.  lambda2 only enters
 *   the facade's clamp of L, as in the reference. */
sc_status sc_lasso_gram_f32(const float* X, int m, int64_t n, const float* Q,
                            int K, const float* q, int L, float lambda1,
                            float lambda2, int mode, int pos, int numThreads,
                            int max_length_path, float* path,
                            const sc_options* opt, sc_csc_f32* out);
sc_status sc_lasso_gram_f64(const double* X, int m, int64_t n, const double* Q,
                            int K, const double* q, int L, double lambda1,
                            double lambda2, int mode, int pos, int numThreads,
                            int max_length_path, double* path,
                            const sc_options* opt, sc_csc_f64* out);

/* The same with _lassoQq's ols / cholevsky arguments (cpp_library/spams.h:
 * 145-188; ols sets cholevsky, :182-183): the Cholesky implementation
 * lasso<T>(Data X, G, DtX, ..., ols, ...) (decomp/decomp.h:746-842 ->
 * coreLARS) on the given products, as for sc_lasso_f32 with cholesky / ols;
 * with both zero it is sc_lasso_gram_*. */
sc_status sc_lasso_gram_chol_f32(const float* X, int m, int64_t n, const float* Q, int K,
                                 const float* q, int L, float lambda1, float lambda2, int mode,
                                 int pos, int ols, int cholesky, int numThreads,
                                 int max_length_path, float* path, const sc_options* opt,
                                 sc_csc_f32* out);
sc_status sc_lasso_gram_chol_f64(const double* X, int m, int64_t n, const double* Q, int K,
                                 const double* q, int L, double lambda1, double lambda2, int mode,
                                 int pos, int ols, int cholesky, int numThreads,
                                 int max_length_path, double* path, const sc_options* opt,
                                 sc_csc_f64* out);

/* ---- device-resident variants -------------------------------------------
 * Same computations with X and D in DEVICE memory.  The facade defaults are
 * resolved by the caller: scalar L / eps / lambda are passed by value, and
 * d_L / d_eps / d_lambda (DEVICE arrays of n entries, or NULL) override them
 * per signal.  The CSC goes to caller-provided device arrays: d_colptr (n+1
 * int64), d_rows / d_vals with capacity `cap` entries (n * L_clamped always
 * fits).  The call enqueues its work on `stream` (a cudaStream_t; NULL = the
 * legacy default stream); *nnz_out (host) is written after a stream
 * synchronisation when nnz_out is non-NULL, otherwise the call returns as
 * soon as the work is enqueued. */
sc_status sc_omp_f32_dev(const float* dX, int m, int64_t n, const float* dD,
                         int K, int L, float eps, float lambda, const int* d_L,
                         const float* d_eps, const float* d_lambda,
                         int64_t* d_colptr, int32_t* d_rows, float* d_vals,
                         int64_t cap, int64_t* nnz_out, void* stream,
                         const sc_options* opt);
sc_status sc_lasso_f32_dev(const float* dX, int m, int64_t n, const float* dD,
                           int K, int L, float lambda1, float lambda2, int mode,
                           int pos, int max_length_path, int64_t* d_colptr,
                           int32_t* d_rows, float* d_vals, int64_t cap,
                           int64_t* nnz_out, void* stream,
                           const sc_options* opt);

/* ---- products -----------------------------------------------------------
 * Correlations C = D^T X (K x n, column-major, ld ldc >= K) of device arrays,
 * in the numerical form `precision` (SC_PREC_FP32 or SC_PREC_BF16X3): the
 * product the coding calls compute first.  Replaces ProdMatrix<T>'s D^T X
 * (linalg/linalg.h:1021-1067, 5101-5190; Matrix::mult with transA).
 * Asynchronous on `stream`. */
sc_status sc_corr_f32_dev(const float* dD, int m, int K, const float* dX, int64_t n,
                          float* dC, int ldc, int precision, void* stream);

/* The same BF16 hi/lo tensor-core product (SC_PREC_BF16X3) for callers that
 * cannot allocate device memory: those that run with a device-memory budget
 * fixed in advance (a serving process whose own pool already holds the free
 * memory, where cudaMalloc fails or fragments it) and those that must avoid
 * the implicit device synchronisation of cudaMalloc / cudaFree.  No counterpart
 * in the reference (SPAMS allocates its workspaces with new[] on the host).
 *   The caller passes inputs and output as for sc_corr_f32_dev; the hi / lo
 *   halves of D and X are staged in a fixed 16 MiB array compiled into the
 *   library (held on every GPU that loads the library until exit), so
 *   256 + 2 * r(2 * m64 * K) + 2 * r(2 * m64 * n) bytes must fit in 16 MiB,
 *   m64 = m rounded up to a multiple of 64 and r(b) = b rounded up to a
 *   multiple of 256 (larger calls return SC_ERR_CAPACITY; split X by columns).
 *   The first call on a device looks up the array's address there
 *   (cudaGetSymbolAddress).  All calls share the array: calls that
 *   overlap on the GPU race and must be serialised.  Every call synchronises
 *   its stream (it reads back the pipeline's timeout flag) and returns after
 *   the stream has finished the product.  No cudaMalloc / cudaFree or other
 *   allocating routine is called. */
sc_status sc_corr_bf16x3_noalloc_f32(const float* dD, int m, int K, const float* dX, int64_t n,
                                     float* dC, int ldc, void* stream);

/* ---- Masked variants ---------------------------------------------------
 * Each signal x_i comes with a row mask (column i of `mask`, m x n bytes,
 * column-major, nonzero = observed row): the code of x_i is computed from its
 * observed rows only, i.e. against the rows of D that the mask keeps.
 *   sc_omp_mask_*    replaces _ompMask<T>   (cpp_library/spams.h:296-343;
 *                    omp_mask, decomp/decomp.h:406-481): a mask with no
 *                    observed row gives an empty column, a full mask the plain
 *                    OMP code; otherwise the masked Gram gets a 1e-10 ridge and
 *                    eps scales by the observed fraction.  path as sc_omp_*.
 *   sc_lasso_mask_*  replaces _lassoMask<T> (cpp_library/spams.h:191-214;
 *                    lasso_mask, decomp/decomp.h:1466-1561): ridge
 *                    max(lambda2, 1e-10); PENALTY and L2ERROR constraints scale
 *                    by the observed fraction; L clamped as in _lassoD; no path.
 * Dictionaries as the coding kernels (one warp per signal up to 1024 atoms,
 * one CTA beyond). */
sc_status sc_omp_mask_f32(const float* X, int m, int64_t n, const float* D, int K,
                          const uint8_t* mask, const int* L, int64_t nL, const float* eps,
                          int64_t nEps, const float* lambda, int64_t nLambda, int numThreads,
                          float* path, const sc_options* opt, sc_csc_f32* out);
sc_status sc_omp_mask_f64(const double* X, int m, int64_t n, const double* D, int K,
                          const uint8_t* mask, const int* L, int64_t nL, const double* eps,
                          int64_t nEps, const double* lambda, int64_t nLambda, int numThreads,
                          double* path, const sc_options* opt, sc_csc_f64* out);
sc_status sc_lasso_mask_f32(const float* X, int m, int64_t n, const float* D, int K,
                            const uint8_t* mask, int L, float lambda1, float lambda2, int mode,
                            int pos, int numThreads, const sc_options* opt, sc_csc_f32* out);
sc_status sc_lasso_mask_f64(const double* X, int m, int64_t n, const double* D, int K,
                            const uint8_t* mask, int L, double lambda1, double lambda2, int mode,
                            int pos, int numThreads, const sc_options* opt, sc_csc_f64* out);

/* ---- Serving: a request loop over resident dictionaries -----------------
 * No counterpart in the reference (each SPAMS call is synchronous and brings
 * its own dictionary).  A server keeps dictionaries resident on one GPU (D,
 * its Gram matrices and BF16 split, keyed by a caller-chosen id) and codes the
 * requests submitted to it, float32 only.  `slots` worker threads each own a
 * CUDA stream and workspaces; a free slot takes the oldest pending request and
 * merges every pending request with the same dictionary and options
 * (algorithm; Lasso mode, pos and L; precision; refine) into one launch of at
 * most max_batch_signals signals, with per-signal L / eps / lambda.  A launch
 * is admitted when the resident dictionaries plus every slot's workspaces stay
 * within hbm_budget_bytes; a request that cannot fit even alone fails with
 * SC_ERR_OUT_OF_MEMORY.  Each signal is coded exactly as sc_omp_f32 /
 * sc_lasso_f32 code it (L, eps, lambda1, mode, pos with their facade
 * defaults), whichever requests share its launch. */
typedef struct sc_server sc_server;

enum { SC_REQ_OMP = 0, SC_REQ_LASSO = 1 };
/* sc_request.flags: the server frees the result itself (replays, load tests). */
enum { SC_REQ_DISCARD = 1 };

typedef struct {
  int64_t dict_id;
  int algo;          /* SC_REQ_OMP or SC_REQ_LASSO */
  const float* X;    /* host, m x n column-major; valid until the request completes */
  int64_t n;
  int L;             /* OMP: <= 0 means not given (min(m, K)); Lasso: as _lassoD (-1: K) */
  float eps;         /* OMP: residual target (0: not given) */
  float lambda1;     /* OMP: lambda (0: not given); Lasso: lambda1 */
  int mode;          /* Lasso: SC_L1COEFFS / SC_L2ERROR / SC_PENALTY */
  int pos;           /* Lasso: non-negative codes */
  int precision;     /* SC_PREC_FP32 or SC_PREC_BF16X3 */
  int refine;        /* FP64 refinement of the final coefficients */
  int flags;         /* SC_REQ_DISCARD */
} sc_request;

typedef struct {
  int64_t completed, signals, batches, rejected, pending;
  double lat_p50_ms, lat_p99_ms, lat_mean_ms, lat_max_ms; /* arrival to result on the host */
  double busy_s;                /* wall time with at least one launch in flight */
  int64_t peak_device_bytes;    /* high-water mark of the admission count */
  double mean_batch_requests;   /* requests merged per launch */
  char last_error[256];         /* message of the last failed request ("" if none) */
} sc_server_stats;

sc_status sc_server_create(int device, int64_t hbm_budget_bytes, int slots,
                           int64_t max_batch_signals, sc_server** out);
/* Codes the requests still pending, then frees everything. */
sc_status sc_server_destroy(sc_server* s);
/* Uploads D (host, m x K column-major) and forms its Grams (blocking).  Also
 * grows the device's stream-ordered memory pool, from which the slots'
 * workspaces are drawn, to slots x the workspace of a max_batch_signals batch
 * on the largest dictionary added so far (within the budget), so that no
 * slot grows the pool while requests run. */
sc_status sc_server_add_dictionary_f32(sc_server* s, int64_t dict_id, const float* D, int m,
                                       int K);
/* Fails while requests against the dictionary are pending or in flight. */
sc_status sc_server_remove_dictionary(sc_server* s, int64_t dict_id);
sc_status sc_server_submit(sc_server* s, const sc_request* r, int64_t* ticket);
/* Blocks until the request is done (or timeout_s passes: SC_ERR_TIMEOUT, the
 * ticket stays valid); returns its K x n CSC (free with sc_csc_free_f32) and
 * its latency from submission. */
sc_status sc_server_wait(sc_server* s, int64_t ticket, double timeout_s, sc_csc_f32* out,
                         double* latency_ms);
/* Open-loop load: submits reqs[i] at arrival_s[i] seconds after the call
 * starts (results discarded; latency counted from the scheduled arrival) and
 * returns when all have completed. */
sc_status sc_server_replay(sc_server* s, const sc_request* reqs, const double* arrival_s,
                           int64_t count);
/* Counters and latency percentiles since the last reset. */
sc_status sc_server_stats_get(sc_server* s, int reset, sc_server_stats* out);

/* ---- Dictionary-learning inner loop -------------------------------------
 * The minibatch step of Trainer::train (dictLearn/dicts.h:526-603) on device
 * arrays, float32: G = DᵀD + max(lambda2, 1e-10) I; the minibatch
 * x_j = X[:, perm[(j + it * batch) % M]] (perm NULL: identity) with `it` read
 * from the device counter *d_iter; its codes (mode as constraint_type:
 * L1COEFFS / L2ERROR / PENALTY run coreLARS2 with constraint lambda1 and
 * posAlpha; SPARSITY / L2ERROR2 / PENALTY2 run coreORMPB with L = lambda1,
 * eps = lambda1 or lambda = lambda1; L = min(m, K) otherwise); then
 * A <- beta A + gamma sum_j a_j a_jᵀ (K x K) and B <- beta B + gamma sum_j x_j a_jᵀ
 * (m x K), column-major (either may be NULL: skipped); finally *d_iter += 1.
 * Everything is enqueued on `stream` without host synchronisation, so a step
 * can be captured in a CUDA graph once a first step has sized the workspaces.
 * The ridge-only conjugate-gradient case of the reference (PENALTY with
 * lambda1 = 0, lambda2 > 0) returns SC_ERR_UNSUPPORTED.  No counterpart in
 * the reference's C API (Trainer runs this loop inside train()). */
typedef struct sc_dl sc_dl;

sc_status sc_dl_create(int device, int m, int K, int batch, int mode, float lambda1,
                       float lambda2, int posAlpha, int precision, sc_dl** out);
sc_status sc_dl_destroy(sc_dl* s);
sc_status sc_dl_step_f32(sc_dl* s, const float* dD, const float* dX, int64_t M,
                         const int32_t* dperm, int64_t* d_iter, float* dA, float* dB, float beta,
                         float gamma, void* stream);
/* on != 0: later steps record the coding stages' device times, read with
 * sc_last_profile on the calling thread (this synchronises the stream: not
 * inside a graph capture). */
sc_status sc_dl_profile(sc_dl* s, int on);
/* Device CSC (batch + 1 column pointers, rows, values) of the last step's codes. */
sc_status sc_dl_codes(sc_dl* s, const int64_t** colptr, const int32_t** rows, const float** vals);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* SPAMS_B200_H */
