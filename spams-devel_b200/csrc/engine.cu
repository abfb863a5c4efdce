// Host engine behind the C ABI (include/spams_b200.h): argument checks and
// the reference facade's clamps, per-device workspaces and streams, and the
// chunked coding pipeline
//     ||x||^2, D^T X  ->  per-signal OMP / LARS  ->  overflow rerun  ->  CSC
// All arithmetic runs on the GPU; there is no CPU fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/spams_b200.h"
#include "engine.h"
#include "kernels.h"
#include "shape_plan.h"
#include "refactor.cuh"

namespace sc {

// ---------------------------------------------------------------------------
// errors
static thread_local char g_err[512] = "";

sc_status fail(sc_status st, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return st;
}
const char* last_error() { return g_err; }


// ---------------------------------------------------------------------------
// device buffers (grow-only, cached per device)
static thread_local cudaStream_t t_alloc_stream = nullptr;

// Gives the stream-ordered pool's free blocks of `device` back to the system
// (after its streams' work: the caller has synchronised).
void trim_pool(int device) {
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
}
AllocStream::AllocStream(cudaStream_t st) : prev(t_alloc_stream) { t_alloc_stream = st; }
AllocStream::~AllocStream() { t_alloc_stream = prev; }

sc_status Buf::reserve(size_t b) {
  if (b <= bytes) return SC_OK;
  const size_t want = std::max(b, (size_t)256);
  const cudaStream_t st = t_alloc_stream;
  if (st) {
    // stream-ordered: the old block goes back to the pool after the work
    // already on `st`, the new one comes from the pool (no device-wide sync)
    if (ptr) {
      if (pooled) cudaFreeAsync(ptr, st);
      else cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
    pooled = false;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, want, st);
    if (e == cudaErrorMemoryAllocation) {
      // the pool's free blocks may be what is missing: return them, retry once
      cudaGetLastError();
      int dev = 0;
      cudaStreamSynchronize(st);
      if (cudaGetDevice(&dev) == cudaSuccess) trim_pool(dev);
      p = nullptr;
      e = cudaMallocAsync(&p, want, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // usable on every stream
    if (e == cudaSuccess) {
      ptr = p;
      bytes = want;
      pooled = true;
      return SC_OK;
    }
    if (p) cudaFreeAsync(p, st);
    cudaGetLastError();  // fall back to cudaMalloc below
  }
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  pooled = false;
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    return fail(SC_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu bytes) failed: %s", want,
                cudaGetErrorString(e));
  }
  bytes = want;
  return SC_OK;
}
void Buf::release() {
  if (ptr) cudaFree(ptr);  // (also for stream-ordered blocks: synchronises)
  ptr = nullptr;
  bytes = 0;
  pooled = false;
}

sc_status DeviceCtx::pinned_cols(size_t bytes) {
  if (bytes <= pinned_col_bytes) return SC_OK;
  if (pinned_col) cudaFreeHost(pinned_col);
  pinned_col = nullptr;
  pinned_col_bytes = 0;
  cudaError_t e = cudaHostAlloc(&pinned_col, bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    pinned_col = nullptr;
    cudaGetLastError();
    return fail(SC_ERR_OUT_OF_MEMORY, "cudaHostAlloc(%zu bytes) failed: %s", bytes,
                cudaGetErrorString(e));
  }
  pinned_col_bytes = bytes;
  return SC_OK;
}

static std::mutex g_ctx_mu;
static std::vector<DeviceCtx*> g_ctx;

static sc_status count_devices(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return fail(SC_ERR_NO_DEVICE, "no CUDA device available (%s); the engine has no CPU path",
                e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
  }
  if (device < 0 || device >= count)
    return fail(SC_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, count);
  return SC_OK;
}

sc_status create_ctx(int device, DeviceCtx** out) {
  SC_TRY(count_devices(device));
  SC_CUDA(cudaSetDevice(device));
  DeviceCtx* c = new DeviceCtx();
  c->device = device;
  auto init = [&]() -> sc_status {
    SC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    SC_CUDA(cudaEventCreateWithFlags(&c->last_use, cudaEventDisableTiming));
    SC_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    SC_CUDA(cudaDeviceGetAttribute(&c->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    SC_CUDA(cudaDeviceGetAttribute(&c->smem_per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    SC_CUDA(cudaHostAlloc(&c->pinned_small, 4096, cudaHostAllocDefault));
    // the stream-ordered allocator keeps freed workspace blocks for reuse
    // rather than unmapping them at every synchronisation (AllocStream)
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    SC_CUDA(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
    SC_CUDA(cudaStreamCreateWithFlags(&c->d2h_stream, cudaStreamNonBlocking));
    SC_CUDA(cudaStreamCreateWithFlags(&c->lane[1].stream, cudaStreamNonBlocking));
    SC_CUDA(cudaEventCreateWithFlags(&c->lane[1].done, cudaEventDisableTiming));
    SC_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
      SC_CUDA(cudaEventCreateWithFlags(&c->ev_h2d[i], cudaEventDisableTiming));
      SC_CUDA(cudaEventCreateWithFlags(&c->ev_xfree[i], cudaEventDisableTiming));
      SC_CUDA(cudaEventCreateWithFlags(&c->ev_out[i], cudaEventDisableTiming));
      SC_CUDA(cudaEventCreateWithFlags(&c->ev_d2h[i], cudaEventDisableTiming));
    }
    return SC_OK;
  };
  const sc_status st = init();
  if (st != SC_OK) {
    destroy_ctx(c);
    return st;
  }
  *out = c;
  return SC_OK;
}

void destroy_ctx(DeviceCtx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (cudaStream_t s : {c->h2d_stream, c->d2h_stream, c->lane[1].stream})
    if (s) cudaStreamSynchronize(s);
  for (Buf* b : c->all_bufs()) b->release();
  for (cudaStream_t s : {c->stream, c->h2d_stream, c->d2h_stream, c->lane[1].stream})
    if (s) cudaStreamDestroy(s);
  if (c->last_use) cudaEventDestroy(c->last_use);
  if (c->lane[1].done) cudaEventDestroy(c->lane[1].done);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  for (int i = 0; i < 2; ++i)
    for (cudaEvent_t e : {c->ev_h2d[i], c->ev_xfree[i], c->ev_out[i], c->ev_d2h[i]})
      if (e) cudaEventDestroy(e);
  if (c->pinned_small) cudaFreeHost(c->pinned_small);
  if (c->pinned_col) cudaFreeHost(c->pinned_col);
  delete c;
}

sc_status get_ctx(int device, DeviceCtx** out) {
  SC_TRY(count_devices(device));
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  int count = 0;
  cudaGetDeviceCount(&count);
  if ((int)g_ctx.size() < count) g_ctx.resize(count, nullptr);
  SC_CUDA(cudaSetDevice(device));
  if (!g_ctx[device]) SC_TRY(create_ctx(device, &g_ctx[device]));
  *out = g_ctx[device];
  return SC_OK;
}

void release_all() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  for (size_t dev = 0; dev < g_ctx.size(); ++dev) {
    if (!g_ctx[dev]) continue;
    destroy_ctx(g_ctx[dev]);
    g_ctx[dev] = nullptr;
    trim_pool((int)dev);
  }
}

// ---------------------------------------------------------------------------
// Byte offsets inside the per-device 256-byte `misc` buffer.  The first 64
// bytes (queue heads, overflow count) are cleared before every chunk.
enum : size_t {
  MISC_COUNTERS = 0,     // unsigned[2]: work-queue heads (main pass, overflow pass)
  MISC_OVF_COUNT = 16,   // int: signals sent to the overflow pass
  MISC_RF_COUNT = 64,    // int: active sets queued to the large-set refinement pass
  MISC_RF_CTR = 68,      // unsigned: its work-queue head
  MISC_CAPFLAG = 128,    // int: device CSC arrays too small
  MISC_TC_ERR = 192,     // int: tensor-core pipeline wait gave up
  MISC_STEPS = 224,      // unsigned long long: coding steps (profile)
  MISC_BYTES = 256
};
template <typename P> static inline P* misc_at(const Buf& b, size_t off) {
  return reinterpret_cast<P*>(static_cast<char*>(b.ptr) + off);
}

// ---------------------------------------------------------------------------
// per-call profile (stage events when requested, launch counts always)
static thread_local sc_profile g_prof;

enum { ST_GRAM = 0, ST_NORMS, ST_CORR, ST_CODE, ST_REFINE, ST_CSC, ST_OTHER, ST_N };

struct Prof {
  bool on = false;
  cudaStream_t st = nullptr;
  std::vector<cudaEvent_t> evs;
  std::vector<int> stage;  // stage that starts at evs[i]
  void mark(int s) {
    if (!on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, st);
    evs.push_back(e);
    stage.push_back(s);
  }
  void launches(int k) { g_prof.launches += k; }
  void finish() {
    if (!on || evs.empty()) return;
    cudaEventSynchronize(evs.back());
    double acc[ST_N] = {0};
    for (size_t i = 0; i + 1 < evs.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, evs[i], evs[i + 1]);
      acc[stage[i]] += ms;
    }
    float tot = 0;
    cudaEventElapsedTime(&tot, evs.front(), evs.back());
    g_prof.ms_gram += acc[ST_GRAM];
    g_prof.ms_norms += acc[ST_NORMS];
    g_prof.ms_corr += acc[ST_CORR];
    g_prof.ms_code += acc[ST_CODE];
    g_prof.ms_refine += acc[ST_REFINE];
    g_prof.ms_csc += acc[ST_CSC];
    g_prof.ms_total += tot;
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    evs.clear();
    stage.clear();
  }
  ~Prof() { for (cudaEvent_t e : evs) cudaEventDestroy(e); }
};

static void prof_reset() { memset(&g_prof, 0, sizeof(g_prof)); }
void profile_reset() { prof_reset(); }
void profile_add_launches(int k) { g_prof.launches += k; }

// Blocks of the refinement pass for active sets beyond 32 atoms.
constexpr int kRefineBigGrid = 32;
// ---------------------------------------------------------------------------
// launch shapes and their autotuner
//
// The candidate shapes (shape_plan.h; kWarpMaxKp / kCtaMaxKp there are the
// largest padded atom counts of the warp- and CTA-per-signal kernels) for
// this device and the kernels' state sizes.  The first call of each
// (algorithm, precision, Kp, L class, batch-size class) times every candidate
// on its first chunk and keeps the fastest (pick_fastest); SC_AUTOTUNE=0 in
// the environment selects the static rule instead (warp kernel up to 1024
// atoms).
template <typename T>
static std::vector<Shape> candidates_for(const DeviceCtx& c, bool lars, int Kp, int L,
                                         int kernel) {
  DeviceLimits d;
  d.num_sms = c.num_sms;
  d.smem_per_block = (size_t)c.smem_per_block;
  d.smem_per_sm = (size_t)c.smem_per_sm;
  auto state = [&](int lc) {
    return lars ? lars_state_bytes(Kp, lc, sizeof(T)) : omp_state_bytes(Kp, lc, sizeof(T));
  };
  auto bytes = [&](int lc) {
    return lars ? lars_cta_smem_bytes<T>(Kp, lc, false) : omp_cta_smem_bytes<T>(Kp, lc, false);
  };
  const int regw = Kp > kWarpMaxKp ? 0
                   : (lars ? lars_max_warps_per_sm<T>(Kp) : omp_max_warps_per_sm<T>(Kp));
  return shape_candidates(d, Kp, L, kernel, state, regw, bytes);
}
// The Cholesky implementation's shape: the warp kernel (4 warps per block, a
// 32-atom state) up to kWarpMaxKp atoms unless the CTA family is asked for,
// else the CTA kernel with the capacity cta_shape gives its shared memory.
template <typename T>
static Shape chol_shape(const DeviceCtx& c, int Kp, int L, int kernel) {
  if (Kp <= kWarpMaxKp && kernel != SC_KERNEL_CTA) return Shape{false, std::min(L, 32), 4, 0};
  DeviceLimits d;
  d.num_sms = c.num_sms;
  d.smem_per_block = (size_t)c.smem_per_block;
  d.smem_per_sm = (size_t)c.smem_per_sm;
  return cta_shape(d, Kp, L, [&](int lc) { return lars_chol_cta_smem_bytes(Kp, lc, sizeof(T), false); });
}

struct TuneKey {
  int lars, dbl, Kp, lclass, nclass, kernel, masked;
  bool operator<(const TuneKey& o) const {
    return std::tie(lars, dbl, Kp, lclass, nclass, kernel, masked) <
           std::tie(o.lars, o.dbl, o.Kp, o.lclass, o.nclass, o.kernel, o.masked);
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, int> g_tune;  // key -> index into shape_candidates, or kTuning
constexpr int kTuning = -1;            // a call is timing the key's candidates

static bool autotune_enabled() {
  static const bool on = [] {
    const char* e = getenv("SC_AUTOTUNE");
    return !(e && e[0] == '0');
  }();
  return on;
}

// ---------------------------------------------------------------------------
// the coding pipeline
template <typename T>
struct Problem {
  bool lars = true;
  const T* dX = nullptr;          // device X (m x n)
  const T* hX = nullptr;          // host X, staged chunk by chunk
  const T* dDtX = nullptr;        // device D^T X given by the caller (K x n)
  const T* dD = nullptr;          // device D (m x K)
  int m = 0;
  int64_t n = 0;
  int K = 0, Kp = 0;
  int L = 0;                      // clamped driver L (slab stride)
  int mode = 2; T lambda1 = 0; int pos = 0; int length_path = 0;
  int Lsig = 0; T eps = 0, lambda = 0;
  const int* dLv = nullptr; const T* dEps = nullptr; const T* dLam = nullptr;
  const T* dLam1 = nullptr;       // per-signal lambda1 of the Lasso, or nullptr
  // device CSC output (device entry points); unused with a host sink
  int64_t* d_colptr = nullptr; int32_t* d_rows = nullptr; T* d_vals = nullptr;
  int64_t cap = 0;
  T* d_path = nullptr;            // device path of signal 0 (zeroed), or nullptr
  // BF16 hi/lo tensor-core correlations + FP64 refinement (float only)
  bool tc = false;
  bool refine = false;            // FP64 refinement of the final coefficients
  bool ols = false;               // least-squares fit on the final support (lasso ols)
  bool chol = false;              // the Cholesky implementation (coreLARS, lars_chol.cu)
  int kernel = SC_KERNEL_AUTO;    // SC_KERNEL_*: kernel family (AUTO: tuned)
  int refactor = 1;               // FP64 refactor: 0 never, 1 small pivots, 2 always
  // masked variants (lasso_mask / omp_mask): host row mask m x n, the ridge of
  // the masked Grams, and whether the Lasso constraint is scaled by the
  // observed fraction (PENALTY / L2ERROR; OMP always scales eps)
  const uint8_t* hmask = nullptr;
  T mask_ridge = 0;
  int mask_scale = 0;
  const void* dDsplit = nullptr;  // Dhi, Dlo, Dlo3 (mp x K bf16 each), consecutive
  int mp = 0;                     // m rounded up to the 64-element k-block
  int* d_tc_err = nullptr;
};

// Host result arrays: page-locked blocks from a process-wide pool, so that
// the read-back of each chunk's CSC is a DMA straight into the result at
// full link speed, runs asynchronously, and touches no fresh pages (a
// malloc'd result is pageable: its copies are staged and synchronous, and its
// first touch faults every page in).  Blocks go back to the pool when the
// caller frees the result (sc_csc_free_*); past kResultPoolBytes of pinned
// memory, or when page-locking fails, results fall back to malloc.
constexpr size_t kResultPoolBytes = (size_t)1 << 30;
struct ResultPool {
  std::mutex mu;
  std::map<void*, std::pair<size_t, bool>> blocks;  // base -> (bytes, in use)
  size_t total = 0;
};
static ResultPool& result_pool() {
  static ResultPool* p = new ResultPool();  // outlives every caller's result
  return *p;
}
// A block of at least `bytes` (pinned when possible), or NULL.
static void* result_alloc(size_t bytes) {
  if (bytes == 0) bytes = 1;
  ResultPool& rp = result_pool();
  {
    std::lock_guard<std::mutex> lk(rp.mu);
    void* best = nullptr;
    size_t best_size = 0;
    for (auto& kv : rp.blocks)  // smallest free block that fits, at most 4x too large
      if (!kv.second.second && kv.second.first >= bytes && kv.second.first <= 4 * bytes &&
          (!best || kv.second.first < best_size)) {
        best = kv.first;
        best_size = kv.second.first;
      }
    if (best) {
      rp.blocks[best].second = true;
      return best;
    }
  }
  size_t sz = 4096;
  while (sz < bytes) sz <<= 1;  // power-of-two sizes, so that blocks are reused
  void* p = nullptr;
  {
    std::lock_guard<std::mutex> lk(rp.mu);
    if (rp.total + sz <= kResultPoolBytes &&
        cudaHostAlloc(&p, sz, cudaHostAllocPortable) == cudaSuccess) {
      rp.blocks[p] = {sz, true};
      rp.total += sz;
      return p;
    }
  }
  (void)cudaGetLastError();  // a refused page-lock is not a sticky error
  return malloc(bytes);
}
// Frees a result array from result_alloc (or malloc).
static void result_free(void* p) {
  if (!p) return;
  ResultPool& rp = result_pool();
  {
    std::lock_guard<std::mutex> lk(rp.mu);
    auto it = rp.blocks.find(p);
    if (it != rp.blocks.end()) {
      it->second.second = false;
      return;
    }
  }
  free(p);
}
// Returns the pool's free blocks to the system (sc_release_all).
static void result_pool_trim() {
  ResultPool& rp = result_pool();
  std::lock_guard<std::mutex> lk(rp.mu);
  for (auto it = rp.blocks.begin(); it != rp.blocks.end();) {
    if (!it->second.second) {
      cudaFreeHost(it->first);
      rp.total -= it->second.first;
      it = rp.blocks.erase(it);
    } else {
      ++it;
    }
  }
}

// CSC result assembled on the host in result_alloc blocks, whose ownership
// moves to the caller's sc_csc_* (freed by sc_csc_free_*).
template <typename T>
struct HostSink {
  int64_t* colptr = nullptr;
  int32_t* rows = nullptr;
  T* vals = nullptr;
  size_t cap = 0, nnz = 0;
  HostSink() = default;
  HostSink(const HostSink&) = delete;
  HostSink& operator=(const HostSink&) = delete;
  ~HostSink() { result_free(colptr); result_free(rows); result_free(vals); }
  sc_status init(int64_t n) {
    colptr = (int64_t*)result_alloc(((size_t)n + 1) * sizeof(int64_t));
    if (!colptr) return fail(SC_ERR_OUT_OF_MEMORY, "host allocation failed");
    memset(colptr, 0, ((size_t)n + 1) * sizeof(int64_t));
    return SC_OK;
  }
  // Moves the first nnz entries into blocks of `want` entries; false (and no
  // change) when an allocation fails.  No copy into the old blocks may be in
  // flight.
  bool resize(size_t want) {
    int32_t* r = (int32_t*)result_alloc(want * sizeof(int32_t));
    T* v = (T*)result_alloc(want * sizeof(T));
    if (!r || !v) {
      result_free(r);
      result_free(v);
      return false;
    }
    if (nnz) {
      memcpy(r, rows, nnz * sizeof(int32_t));
      memcpy(v, vals, nnz * sizeof(T));
    }
    result_free(rows);
    result_free(vals);
    rows = r;
    vals = v;
    cap = want;
    return true;
  }
  // Best-effort capacity for `want` entries (a failed allocation is left to
  // grow()).
  void hint(size_t want) {
    if (want > cap) (void)resize(want);
  }
  sc_status grow(size_t need) {
    if (need <= cap) return SC_OK;
    if (!resize(std::max(need, cap + cap / 2)))
      return fail(SC_ERR_OUT_OF_MEMORY, "host allocation failed");
    return SC_OK;
  }
};

// Host-array calls code their signals in chunks (chunk_signals / plan_chunks,
// shape_plan.h).  The result arrays are sized after the first chunk from its
// entries per signal (one allocation instead of a growing series of
// reallocations and copies).

template <typename T>
static sc_status run_pipeline(DeviceCtx& c, cudaStream_t st, Problem<T>& p, const T* dG,
                              HostSink<T>* sink, int* d_capflag, Prof& pr) {
  const int Kp = p.Kp;
  // the Cholesky implementation has one shape per layout: up to 1024 atoms
  // warps of 4 per block with a 32-atom state in shared memory, beyond (or
  // with the CTA family asked for) one CTA per signal; the overflow pass
  // with capacity L
  std::vector<Shape> cands =
      p.chol ? std::vector<Shape>{chol_shape<T>(c, Kp, p.L, p.kernel)}
             : candidates_for<T>(c, p.lars, Kp, p.L, p.kernel);
  // FP64 refactor of the single-precision state (refactor.cuh): one scratch
  // unit per warp (warp kernels) or CTA (CTA kernels, whose grid is then fixed
  // here)
  const bool refac = sizeof(T) == 4 && p.refactor != 0 && !p.chol;
  if (refac || p.hmask)  // per-CTA scratch (refactor, masked products): a fixed grid
    for (Shape& sh : cands)
      if (sh.cta)
        sh.grid = p.lars ? lars_cta_grid<T>(Kp, sh.Lcap, false) : omp_cta_grid<T>(Kp, sh.Lcap, false);
  const bool piped = sink && p.hX && !p.hmask;
  const int nbuf = piped ? 2 : 1;
  // chunk size: bound D^T X + slabs (+ staged X) to about 2 GiB
  const size_t per_sig = (size_t)Kp * sizeof(T) + (size_t)p.L * (sizeof(T) + 4) + 64 +
                         (p.hX ? (size_t)nbuf * p.m * sizeof(T) : 0) +
                         (sink ? (size_t)nbuf * (p.L * (sizeof(T) + 4) + 8) : 0);
  const int64_t nc = chunk_signals(p.n, per_sig, piped);
  // chunk i covers signals [chunk_start(i), chunk_start(i) + chunk_len(i));
  // with more than one chunk of host signals, chunks alternate between the
  // two coding lanes (not while profiling, whose stage events need one stream)
  const ChunkPlan plan = plan_chunks(p.n, nc, piped);
  const int64_t nchunks = plan.count;
  const bool dual = piped && !pr.on && nchunks > 1;
  const int nlanes = dual ? 2 : 1;

  SC_TRY(c.misc.reserve(MISC_BYTES));
  const int64_t scan_len = scan_scratch_len(nc);
  const size_t xslot = align16((size_t)nc * p.m * sizeof(T));
  if (p.hX) SC_TRY(c.xstage.reserve(xslot * nbuf));
  // OMP with per-signal step caps: each launch takes its signals longest first
  const bool ordered = !p.lars && p.dLv && p.L <= kOrderMaxL;
  for (int li = 0; li < nlanes; ++li) {
    Lane& W = c.lane[li];
    SC_TRY(W.dtx.reserve((size_t)Kp * nc * sizeof(T)));
    SC_TRY(W.norms.reserve((size_t)nc * sizeof(T)));
    SC_TRY(W.slab_ind.reserve((size_t)nc * p.L * 4));
    SC_TRY(W.slab_val.reserve((size_t)nc * p.L * sizeof(T)));
    SC_TRY(W.cnt.reserve((size_t)nc * 4));
    SC_TRY(W.ovf_list.reserve((size_t)nc * 8));
    SC_TRY(W.misc.reserve(MISC_BYTES));
    SC_TRY(W.scan.reserve((size_t)scan_len * 8));
    if (p.ols || p.refine) {
      SC_TRY(W.rlist.reserve((size_t)nc * 8));
      if (p.L > 32) SC_TRY(W.rscratch.reserve(refine_scratch_bytes(p.L, kRefineBigGrid)));
    }
    SC_TRY(W.level.reserve((size_t)nc * sizeof(T)));
    if (ordered) {
      SC_TRY(W.order.reserve((size_t)nc * 8));
      SC_TRY(W.ordscr.reserve((size_t)(p.L + 1) * 4));
    }
  }
  const size_t col_slot = align16((size_t)(nc + 1) * 8);
  const size_t ent_slot = (size_t)nc * p.L;
  if (sink) {
    SC_TRY(c.ccolptr.reserve(col_slot * nbuf));
    SC_TRY(c.crows.reserve(align16(ent_slot * 4) * nbuf));
    SC_TRY(c.cvals.reserve(align16(ent_slot * sizeof(T)) * nbuf));
    SC_TRY(c.pinned_cols(col_slot * nbuf));
    SC_TRY(sink->init(p.n));
  }
  // overflow pass: state in global slabs with capacity L (per warp, or per
  // CTA for the CTA-per-signal kernels), at most 256 MiB
  struct Ovf { int wpb, grid; size_t bytes; };
  auto ovf_plan = [&](const Shape& sh) {
    Ovf o;
    o.wpb = sh.cta ? 1 : 4;
    const size_t per =
        p.chol ? (sh.cta ? lars_chol_cta_gstate_bytes(p.L, sizeof(T))
                         : lars_chol_state_bytes(Kp, p.L, sizeof(T)))
        : sh.cta ? (p.lars ? lars_cta_gstate_bytes<T>(p.L, 1) : omp_cta_gstate_bytes<T>(p.L, 1))
                 : (p.lars ? lars_state_bytes(Kp, p.L, sizeof(T)) : omp_state_bytes(Kp, p.L, sizeof(T)));
    o.grid = sh.cta ? 2 * c.num_sms : c.num_sms;
    while (o.grid > 1 && (size_t)o.grid * o.wpb * per > ((size_t)256 << 20)) o.grid >>= 1;
    o.bytes = (size_t)o.grid * o.wpb * per;
    return o;
  };
  for (const Shape& sh : cands)
    if (sh.Lcap < p.L)
      for (int li = 0; li < nlanes; ++li) SC_TRY(c.lane[li].gstate.reserve(ovf_plan(sh).bytes));
  // refactor scratch: the largest launch's units, each for the largest
  // refactored active set of any launch
  int rf_units = 0;
  if (refac) {
    size_t units = 0;
    int cap = refactor_cap(p.L);
    for (const Shape& sh : cands) {
      units = std::max(units, (size_t)sh.grid * (sh.cta ? 1 : sh.wpb));
      const Ovf ov = ovf_plan(sh);
      units = std::max(units, (size_t)ov.grid * ov.wpb);
      cap = std::max(cap, refactor_cap(sh.Lcap));
    }
    for (int li = 0; li < nlanes; ++li)
      SC_TRY(c.lane[li].rfscr.reserve(units * (size_t)cap * cap * sizeof(double)));
    rf_units = (int)units;
  }
  // masked variants: Dᵀ, the chunk's mask / classes / scaled parameters, and
  // one m-vector of scratch per warp (warp kernels) or CTA (CTA kernels) of
  // the largest launch
  MaskArgs<T> mk{};
  if (p.hmask) {
    mk.m = p.m;
    mk.mpad = (p.m + 31) / 32 * 32;
    mk.ridge = p.mask_ridge;
    mk.D = p.dD;
    SC_TRY(c.Dt.reserve((size_t)Kp * p.m * sizeof(T)));
    SC_CUDA(launch_transpose_pad<T>(p.dD, p.m, p.K, Kp, reinterpret_cast<T*>(c.Dt.ptr), st));
    mk.Dt = reinterpret_cast<const T*>(c.Dt.ptr);
    SC_TRY(c.mask.reserve((size_t)nc * p.m));
    SC_TRY(c.mflag.reserve((size_t)nc));
    SC_TRY(c.mvec.reserve((size_t)nc * sizeof(T)));
    size_t warps = 0;
    for (const Shape& sh : cands) {
      warps = std::max(warps, (size_t)sh.grid * (sh.cta ? 1 : sh.wpb));
      const Ovf ov = ovf_plan(sh);
      warps = std::max(warps, (size_t)ov.grid * ov.wpb);
    }
    SC_TRY(c.mwork.reserve(warps * mk.mpad * sizeof(T)));
    mk.mask = reinterpret_cast<const uint8_t*>(c.mask.ptr);
    mk.flag = reinterpret_cast<const int8_t*>(c.mflag.ptr);
    mk.work = reinterpret_cast<T*>(c.mwork.ptr);
  }

  unsigned long long* d_steps =
      pr.on ? misc_at<unsigned long long>(c.lane[0].misc, MISC_STEPS) : nullptr;
  if (d_steps) SC_CUDA(cudaMemsetAsync(d_steps, 0, 8, st));
  g_prof.signals += p.n;

  auto chunk_start = [&](int64_t i) { return plan.start(i); };
  auto chunk_len = [&](int64_t i) { return plan.len(i); };
  auto xslot_ptr = [&](int64_t i) {
    return reinterpret_cast<T*>(static_cast<char*>(c.xstage.ptr) + (i & 1) * (piped ? xslot : 0));
  };
  // copy of chunk i's signals into its staging slot, once the chunk that used
  // the slot before has finished reading it
  auto issue_h2d = [&](int64_t i) -> sc_status {
    cudaStream_t cs = piped ? c.h2d_stream : st;
    if (piped) SC_CUDA(cudaStreamWaitEvent(cs, c.ev_xfree[i & 1], 0));
    SC_CUDA(cudaMemcpyAsync(xslot_ptr(i), p.hX + (size_t)chunk_start(i) * p.m,
                            (size_t)chunk_len(i) * p.m * sizeof(T), cudaMemcpyHostToDevice, cs));
    if (piped) SC_CUDA(cudaEventRecord(c.ev_h2d[i & 1], cs));
    return SC_OK;
  };
  // chunk i's CSC: its column pointers were read back into pinned memory on
  // the coding stream; the entries are copied straight into the result
  int64_t nnz_total = 0;
  bool d2h_pending[2] = {false, false};  // an entry read-back per slot still in flight
  struct D2hDrain {  // no read-back outlives the call, whatever its exit
    DeviceCtx& c;
    bool* pending;
    ~D2hDrain() {
      for (int k = 0; k < 2; ++k)
        if (pending[k]) cudaEventSynchronize(c.ev_d2h[k]);
    }
  } d2h_guard{c, d2h_pending};
  auto finalize = [&](int64_t i) -> sc_status {
    const int64_t cn = chunk_len(i);
    const int slot = piped ? (int)(i & 1) : 0;
    SC_CUDA(cudaEventSynchronize(c.ev_out[slot]));
    const int64_t* hcol =
        reinterpret_cast<const int64_t*>(static_cast<char*>(c.pinned_col) + slot * col_slot);
    const int64_t cnnz = hcol[cn];
    // entry copies still in flight must land before the result blocks move
    // (a resize), and before the device slot they read is refilled (the
    // chunk after next waits on the host for this finalize)
    auto drain = [&]() -> sc_status {
      for (int k = 0; k < 2; ++k)
        if (d2h_pending[k]) {
          SC_CUDA(cudaEventSynchronize(c.ev_d2h[k]));
          d2h_pending[k] = false;
        }
      return SC_OK;
    };
    const size_t need = (size_t)(nnz_total + cnnz);
    if (i == 0 && p.n > cn) {  // the whole result at the first chunk's density, +15%
      SC_TRY(drain());
      sink->hint((size_t)((double)cnnz * (double)p.n / (double)cn * 1.15) + 1024);
    }
    if (need > sink->cap) SC_TRY(drain());
    SC_TRY(sink->grow(need));
    if (d2h_pending[slot]) {
      SC_CUDA(cudaEventSynchronize(c.ev_d2h[slot]));
      d2h_pending[slot] = false;
    }
    if (cnnz > 0) {
      cudaStream_t cs = piped ? c.d2h_stream : st;
      SC_CUDA(cudaMemcpyAsync(sink->rows + nnz_total,
                              static_cast<char*>(c.crows.ptr) + slot * align16(ent_slot * 4),
                              (size_t)cnnz * 4, cudaMemcpyDeviceToHost, cs));
      SC_CUDA(cudaMemcpyAsync(sink->vals + nnz_total,
                              static_cast<char*>(c.cvals.ptr) + slot * align16(ent_slot * sizeof(T)),
                              (size_t)cnnz * sizeof(T), cudaMemcpyDeviceToHost, cs));
      SC_CUDA(cudaEventRecord(c.ev_d2h[slot], cs));
      d2h_pending[slot] = true;
      if (!piped || i + 1 == nchunks) SC_TRY(drain());
    }
    int64_t* dst = sink->colptr + chunk_start(i);
    for (int64_t k = 0; k <= cn; ++k) dst[k] = nnz_total + hcol[k];
    nnz_total += cnnz;
    sink->nnz = (size_t)nnz_total;
    return SC_OK;
  };

  // kernel family: a single candidate, the cached choice of an earlier call,
  // the static rule, or timed on the first chunk (tune)
  int chosen = cands.size() == 1 ? 0 : -1;
  TuneKey key{p.lars ? 1 : 0, sizeof(T) == 8 ? 1 : 0, Kp, tune_lclass(p.L), 0, p.kernel,
              p.hmask ? 1 : 0};
  key.nclass = tune_nclass(std::min<int64_t>(nc, p.n));
  if (chosen < 0 && !autotune_enabled()) chosen = 0;
  bool claimed = false;  // this call times the candidates for `key`
  if (chosen < 0) {
    // one call per key times the candidates (kTuning marks the claim);
    // calls that meet a claim meanwhile (other threads, serving slots) take
    // the static rule's shape rather than time candidates concurrently
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it == g_tune.end()) {
      g_tune[key] = kTuning;
      claimed = true;
    } else {
      chosen = it->second >= 0 && it->second < (int)cands.size() ? it->second : 0;
    }
  }
  struct TuneClaim {  // an unfinished claim is withdrawn, whatever the exit
    bool& on;
    TuneKey k;
    ~TuneClaim() {
      if (!on) return;
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(k);
      if (it != g_tune.end() && it->second == kTuning) g_tune.erase(it);
    }
  } tune_claim{claimed, key};
  auto tune = [&](int64_t cn, auto& code, int& out) -> sc_status {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    SC_CUDA(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) {  // no timing inside a graph capture
      out = 0;
      return SC_OK;  // (the claim is withdrawn: a later call times the key)
    }
    const int64_t sample = std::min<int64_t>(cn, 16384);
    cudaEvent_t e0, e1;
    SC_CUDA(cudaEventCreate(&e0));
    SC_CUDA(cudaEventCreate(&e1));
    // two interleaved rounds, the faster time of each candidate
    std::vector<float> t(cands.size(), 0.f);
    sc_status stt = SC_OK;
    for (int round = 0; round < 2 && stt == SC_OK; ++round)
      for (size_t i = 0; i < cands.size() && stt == SC_OK; ++i) {
        if (round == 0) {
          stt = code(cands[i], std::min<int64_t>(sample, 64), false);  // module load, attributes
          if (stt != SC_OK) break;
        }
        cudaEventRecord(e0, st);
        stt = code(cands[i], sample, false);
        cudaEventRecord(e1, st);
        if (stt != SC_OK) break;
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (round == 0 || ms < t[i]) t[i] = ms;
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stt != SC_OK) return stt;
    const int best = pick_fastest(t);  // the static rule's shape unless clearly beaten
    out = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = best;
    claimed = false;
    return SC_OK;
  };

  if (piped && nchunks > 0) {
    SC_CUDA(cudaStreamWaitEvent(c.h2d_stream, c.last_use, 0));
    SC_TRY(issue_h2d(0));
  }
  if (dual) {  // lane 1 starts after the call's earlier work on st (the Gram, the split of D)
    SC_CUDA(cudaEventRecord(c.ev_fork, st));
    SC_CUDA(cudaStreamWaitEvent(c.lane[1].stream, c.ev_fork, 0));
  }
  const cudaStream_t st0 = st;
  for (int64_t ci = 0; ci < nchunks; ++ci) {
    const int64_t start = chunk_start(ci);
    const int64_t cn = chunk_len(ci);
    const int li = dual ? (int)(ci & 1) : 0;
    Lane& W = c.lane[li];
    const cudaStream_t st = li ? W.stream : st0;  // this chunk's stream
    unsigned* d_counter = misc_at<unsigned>(W.misc, MISC_COUNTERS);
    int* d_ovf_count = misc_at<int>(W.misc, MISC_OVF_COUNT);
    T* dtx = reinterpret_cast<T*>(W.dtx.ptr);
    T* norms = reinterpret_cast<T*>(W.norms.ptr);
    // ---- inputs: ||x||^2 and D^T x
    const T* xchunk = nullptr;
    pr.mark(ST_OTHER);
    if (p.hX) {
      if (piped) {
        if (ci + 1 < nchunks) SC_TRY(issue_h2d(ci + 1));
        SC_CUDA(cudaStreamWaitEvent(st, c.ev_h2d[ci & 1], 0));
      } else {
        SC_TRY(issue_h2d(ci));
      }
      xchunk = xslot_ptr(ci);
    } else {
      xchunk = p.dX + (size_t)start * p.m;
    }
    T* mvec = nullptr;
    if (p.hmask) {
      // masked signal, observation classes, parameters scaled by the observed fraction
      SC_CUDA(cudaMemcpyAsync(c.mask.ptr, p.hmask + (size_t)start * p.m, (size_t)cn * p.m,
                              cudaMemcpyHostToDevice, st));
      mvec = reinterpret_cast<T*>(c.mvec.ptr);
      if (p.lars)
        SC_CUDA(launch_mask_prep<T>(const_cast<T*>(xchunk), p.m, cn,
                                    reinterpret_cast<const uint8_t*>(c.mask.ptr),
                                    reinterpret_cast<int8_t*>(c.mflag.ptr), nullptr, p.lambda1,
                                    p.mask_scale, mvec, st));
      else
        SC_CUDA(launch_mask_prep<T>(const_cast<T*>(xchunk), p.m, cn,
                                    reinterpret_cast<const uint8_t*>(c.mask.ptr),
                                    reinterpret_cast<int8_t*>(c.mflag.ptr),
                                    p.dEps ? p.dEps + start : nullptr, p.eps, 1, mvec, st));
    }
    pr.mark(ST_NORMS);
    SC_CUDA(launch_colnorms<T>(xchunk, p.m, cn, norms, st));
    pr.mark(ST_CORR);
    if (p.dDtX) {
      SC_CUDA(launch_pad_rows<T>(p.dDtX + (size_t)start * p.K, p.K, p.K, cn, dtx, Kp, st));
      pr.launches(2);
    } else if (p.tc) {
      if constexpr (std::is_same<T, float>::value) {
        // BF16 split products with the split of X done inside the kernel.
        // OMP reads its selections and eps stops off the correlations, so it
        // takes the three-piece form (six products, FP32-grade); the LARS
        // path keeps the hi / lo form (three products).
        const char* ds = reinterpret_cast<const char*>(p.dDsplit);
        const size_t piece = (size_t)p.mp * p.K * 2;
        const void* dp[3] = {ds, ds + piece, ds + 2 * piece};
        cudaError_t e = launch_tc_corr_xs(dp, p.lars ? 2 : 3, p.K, xchunk, p.m, p.m, cn, p.mp,
                                          dtx, Kp, Kp, p.d_tc_err, st);
        if (e == cudaErrorNotSupported)  // large m: the streaming hi / lo form
          e = launch_tc_corr_fused(ds, ds + piece, p.K, xchunk, p.m, p.m, cn, p.mp, dtx, Kp,
                                   Kp, p.d_tc_err, st);
        SC_CUDA(e);
        pr.launches(1);
      }
    } else {
      SC_CUDA(launch_gemm_tn<T>(p.dD, p.m, p.K, xchunk, p.m, cn, p.m, dtx, Kp, Kp, st));
      pr.launches(2);
    }
    // ---- coding (+ rerun of the signals whose active set outgrew Lcap)
    const int64_t* order = nullptr;
    if (ordered) {
      SC_CUDA(launch_order_by_L_desc(p.dLv + start, cn, p.L, reinterpret_cast<int*>(W.ordscr.ptr),
                                     reinterpret_cast<int64_t*>(W.order.ptr), st));
      pr.launches(3);
      order = reinterpret_cast<const int64_t*>(W.order.ptr);
    }
    int* cnt = reinterpret_cast<int*>(W.cnt.ptr);
    int* sind = reinterpret_cast<int*>(W.slab_ind.ptr);
    T* sval = reinterpret_cast<T*>(W.slab_val.ptr);
    int64_t* ovf_list = reinterpret_cast<int64_t*>(W.ovf_list.ptr);
    T* path = start == 0 ? p.d_path : nullptr;
    auto code = [&](const Shape& shp, int64_t jobs, bool final_run) -> sc_status {
      SC_CUDA(cudaMemsetAsync(W.misc.ptr, 0, 64, st));
      const bool may_overflow = shp.Lcap < p.L;
      const Ovf ov = ovf_plan(shp);
      if (p.lars) {
        LarsArgs<T> a{};
        a.G = dG; a.DtX = dtx; a.norms = norms; a.K = p.K; a.Kp = Kp; a.L = p.L;
        a.Lcap = shp.Lcap; a.mode = p.mode; a.constraint = p.lambda1; a.pos = p.pos;
        a.vConstraint = mvec ? mvec : (p.dLam1 ? p.dLam1 + start : nullptr);
        a.mk = mk;
        a.length_path = p.length_path; a.n_jobs = (int)jobs; a.n_jobs_dev = nullptr;
        a.sig_list = nullptr; a.work_counter = d_counter; a.out_ind = sind; a.out_val = sval;
        a.out_cnt = cnt; a.overflow_list = ovf_list; a.overflow_count = d_ovf_count;
        a.gstate = nullptr; a.path = final_run ? path : nullptr;
        a.steps = final_run ? d_steps : nullptr;
        a.out_level = (p.refine && !p.ols) ? reinterpret_cast<T*>(W.level.ptr) : nullptr;
        a.refactor = refac ? p.refactor : 0;
        a.rf_scratch = refac ? reinterpret_cast<double*>(W.rfscr.ptr) : nullptr;
        a.rf_cap = refactor_cap(shp.Lcap);
        a.rf_units = refac ? rf_units : 0;
        a.ols = p.ols ? 1 : 0;
        if (p.chol && shp.cta) SC_CUDA(launch_lars_chol_cta<T>(a, shp.grid, st));
        else if (p.chol) SC_CUDA(launch_lars_chol<T>(a, shp.grid, shp.wpb, st));
        else if (shp.cta) SC_CUDA(launch_lars_cta<T>(a, shp.grid, st));
        else SC_CUDA(launch_lars<T>(a, shp.grid, shp.wpb, st));
        if (final_run) pr.launches(1);
        if (may_overflow) {
          if (final_run) pr.launches(1);
          a.Lcap = p.L; a.n_jobs = 0; a.n_jobs_dev = d_ovf_count; a.sig_list = ovf_list;
          a.work_counter = d_counter + 1; a.overflow_list = nullptr; a.overflow_count = nullptr;
          a.gstate = reinterpret_cast<T*>(W.gstate.ptr);
          a.rf_cap = refactor_cap(p.L);
          if (p.chol && shp.cta) SC_CUDA(launch_lars_chol_cta<T>(a, ov.grid, st));
          else if (p.chol) SC_CUDA(launch_lars_chol<T>(a, ov.grid, ov.wpb, st));
          else if (shp.cta) SC_CUDA(launch_lars_cta<T>(a, ov.grid, st));
          else SC_CUDA(launch_lars<T>(a, ov.grid, ov.wpb, st));
        }
      } else {
        OmpArgs<T> a{};
        a.G = dG; a.DtX = dtx; a.norms = norms; a.K = p.K; a.Kp = Kp; a.L = p.L;
        a.Lcap = shp.Lcap; a.eps = p.eps; a.lambda = p.lambda; a.Lsig = p.Lsig;
        a.vL = p.dLv ? p.dLv + start : nullptr;
        a.vEps = mvec ? mvec : (p.dEps ? p.dEps + start : nullptr);
        a.vLambda = p.dLam ? p.dLam + start : nullptr;
        a.mk = mk;
        a.n_jobs = (int)jobs; a.n_jobs_dev = nullptr; a.sig_list = order;
        a.work_counter = d_counter; a.out_ind = sind; a.out_val = sval; a.out_cnt = cnt;
        a.overflow_list = ovf_list; a.overflow_count = d_ovf_count; a.gstate = nullptr;
        a.path = final_run ? path : nullptr;
        a.steps = final_run ? d_steps : nullptr;
        a.refactor = refac ? p.refactor : 0;
        a.rf_scratch = refac ? reinterpret_cast<double*>(W.rfscr.ptr) : nullptr;
        a.rf_cap = refactor_cap(shp.Lcap);
        a.rf_units = refac ? rf_units : 0;
        if (shp.cta) SC_CUDA(launch_omp_cta<T>(a, shp.grid, st));
        else SC_CUDA(launch_omp<T>(a, shp.grid, shp.wpb, st));
        if (final_run) pr.launches(1);
        if (may_overflow) {
          if (final_run) pr.launches(1);
          a.Lcap = p.L; a.n_jobs = 0; a.n_jobs_dev = d_ovf_count; a.sig_list = ovf_list;
          a.work_counter = d_counter + 1; a.overflow_list = nullptr; a.overflow_count = nullptr;
          a.gstate = reinterpret_cast<T*>(W.gstate.ptr);
          a.rf_cap = refactor_cap(p.L);
          if (shp.cta) SC_CUDA(launch_omp_cta<T>(a, ov.grid, st));
          else SC_CUDA(launch_omp<T>(a, ov.grid, ov.wpb, st));
        }
      }
      return SC_OK;
    };
    if (chosen < 0 && claimed) SC_TRY(tune(cn, code, chosen));
    if (chosen < 0) chosen = 0;
    const Shape& shp = cands[(size_t)chosen];
    const bool may_overflow = shp.Lcap < p.L;
    g_prof.kernel = shp.cta ? SC_KERNEL_CTA : SC_KERNEL_WARP;
    g_prof.lcap = shp.Lcap;
    pr.mark(ST_CODE);
    SC_TRY(code(shp, cn, true));
    // ---- double-precision solves on the final active sets: the ols
    // projection, or the refinement of single-precision codes
    if ((p.ols && !p.chol) || (p.refine && !p.chol && (p.dD || p.dDtX))) {
      pr.mark(ST_REFINE);
      const bool with_level = p.lars && !p.ols;
      const T* q = p.dDtX ? p.dDtX + (size_t)start * p.K : nullptr;
      SC_CUDA(launch_refine<T>(q ? nullptr : p.dD, p.m, q ? nullptr : xchunk, q, p.K, dG, Kp, sind,
                               sval, p.L, cnt,
                               with_level ? reinterpret_cast<const T*>(W.level.ptr) : nullptr, cn,
                               reinterpret_cast<int64_t*>(W.rlist.ptr),
                               misc_at<int>(W.misc, MISC_RF_COUNT),
                               misc_at<unsigned>(W.misc, MISC_RF_CTR),
                               reinterpret_cast<double*>(W.rscratch.ptr), kRefineBigGrid, st));
      pr.launches(2);
    }
    if (piped) SC_CUDA(cudaEventRecord(c.ev_xfree[ci & 1], st));  // staging slot free again
    if (pr.on && may_overflow) {
      SC_CUDA(cudaMemcpyAsync(c.pinned_small, d_ovf_count, 4, cudaMemcpyDeviceToHost, st));
      SC_CUDA(cudaStreamSynchronize(st));
      g_prof.overflowed += *reinterpret_cast<int*>(c.pinned_small);
    }
    // ---- CSC
    pr.mark(ST_CSC);
    pr.launches(4);
    int64_t* scratch = reinterpret_cast<int64_t*>(W.scan.ptr);
    if (sink) {
      const int slot = piped ? (int)(ci & 1) : 0;
      // the column pointers of the chunk that used these slots before were
      // read on the host (finalize); its entries' read-back is waited for
      // on the device below
      int64_t* ccol = reinterpret_cast<int64_t*>(static_cast<char*>(c.ccolptr.ptr) + slot * col_slot);
      int32_t* crow = reinterpret_cast<int32_t*>(static_cast<char*>(c.crows.ptr) +
                                                 slot * align16(ent_slot * 4));
      T* cval = reinterpret_cast<T*>(static_cast<char*>(c.cvals.ptr) +
                                     slot * align16(ent_slot * sizeof(T)));
      // the read-back of the chunk that last used this slot's entries ends first
      if (d2h_pending[slot]) SC_CUDA(cudaStreamWaitEvent(st, c.ev_d2h[slot], 0));
      SC_CUDA(launch_scan_counts(cnt, cn, ccol, nullptr, scratch, scan_len, st));
      SC_CUDA(launch_csc_gather<T>(sind, sval, p.L, cnt, ccol, cn, nullptr, cn * (int64_t)p.L,
                                   d_capflag, crow, cval, st));
      SC_CUDA(cudaMemcpyAsync(static_cast<char*>(c.pinned_col) + slot * col_slot, ccol,
                              (size_t)(cn + 1) * 8, cudaMemcpyDeviceToHost, st));
      SC_CUDA(cudaEventRecord(c.ev_out[slot], st));
      if (!piped) SC_TRY(finalize(ci));
      else if (ci >= 1) SC_TRY(finalize(ci - 1));
    } else {
      int64_t* col = p.d_colptr + start;
      SC_CUDA(launch_scan_counts(cnt, cn, col, start == 0 ? nullptr : col, scratch, scan_len, st));
      SC_CUDA(launch_csc_gather<T>(sind, sval, p.L, cnt, col, cn, nullptr, p.cap, d_capflag,
                                   p.d_rows, p.d_vals, st));
    }
  }
  if (dual) {  // the call's stream waits for lane 1's last chunk
    SC_CUDA(cudaEventRecord(c.lane[1].done, c.lane[1].stream));
    SC_CUDA(cudaStreamWaitEvent(st, c.lane[1].done, 0));
  }
  if (piped && nchunks > 0) SC_TRY(finalize(nchunks - 1));
  pr.mark(ST_OTHER);
  if (d_steps) {
    SC_CUDA(cudaMemcpyAsync(c.pinned_small, d_steps, 8, cudaMemcpyDeviceToHost, st));
    SC_CUDA(cudaStreamSynchronize(st));
    g_prof.steps += (int64_t)*reinterpret_cast<unsigned long long*>(c.pinned_small);
  }
  pr.finish();
  return SC_OK;
}

// ---------------------------------------------------------------------------
// result helpers
template <typename T> struct CscOf;
template <> struct CscOf<float> { using type = sc_csc_f32; };
template <> struct CscOf<double> { using type = sc_csc_f64; };

template <typename T>
static sc_status emit_empty(int64_t m, int64_t n, typename CscOf<T>::type* out) {
  out->m = m;
  out->n = n;
  out->nnz = 0;
  out->colptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  out->rows = (int32_t*)malloc(sizeof(int32_t));
  out->vals = (T*)malloc(sizeof(T));
  if (!out->colptr || !out->rows || !out->vals) return fail(SC_ERR_OUT_OF_MEMORY, "host malloc failed");
  return SC_OK;
}

template <typename T>
static sc_status emit_sink(int64_t m, int64_t n, HostSink<T>& s, typename CscOf<T>::type* out) {
  if (!s.colptr) SC_TRY(s.init(n));
  if (!s.rows) SC_TRY(s.grow(1));
  out->m = m;
  out->n = n;
  out->nnz = (int64_t)s.nnz;
  out->colptr = s.colptr;
  out->rows = s.rows;
  out->vals = s.vals;
  s.colptr = nullptr;
  s.rows = nullptr;
  s.vals = nullptr;
  return SC_OK;
}

static inline int pad128(int K) { return ((K + 127) / 128) * 128; }
// Padded atom count: a multiple of 128 up to 1024 atoms (one warp per signal),
// beyond that the CTA kernels' layout (one CTA of Kp / 512 warps per signal).
int pad_atoms(int K) {
  const int p = pad128(K);
  return p <= kWarpMaxKp ? p : cta_pad_atoms(K);
}
// The layout for a forced kernel family: the CTA kernels' own.
static int pad_atoms_for(int K, const sc_options* opt) {
  return opt && opt->kernel == SC_KERNEL_CTA ? cta_pad_atoms(K) : pad_atoms(K);
}
static sc_status check_kernel(int K, const sc_options* opt) {
  if (opt && opt->kernel == SC_KERNEL_WARP && pad128(K) > kWarpMaxKp)
    return fail(SC_ERR_UNSUPPORTED, "the warp-per-signal kernels take at most %d atoms (K=%d)",
                kWarpMaxKp, K);
  return SC_OK;
}

// Per-call device guard: serialises calls on one device and orders this
// call's stream after the previous user of the shared workspaces.
// Orders the calls on one device's shared workspaces: a call waits for the
// previous call's device work and marks its own end.  A call made while its
// stream is being captured into a CUDA graph does neither (the graph's own
// order applies; replays of a graph that uses these workspaces must not
// overlap other calls on the device).
struct CallGuard {
  DeviceCtx* c;
  cudaStream_t st;
  std::lock_guard<std::mutex> lk;
  bool capturing = false;
  // workspace growth ordered on the call's stream after the previous call
  // (none while capturing: growth there fails as before)
  AllocStream alloc;
  CallGuard(DeviceCtx* ctx, cudaStream_t s)
      : c(ctx), st(s), lk(ctx->mu), capturing(is_capturing(s)), alloc(capturing ? nullptr : s) {
    if (!capturing) cudaStreamWaitEvent(st, c->last_use, 0);
  }
  static bool is_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
  }
  ~CallGuard() {
    if (!capturing) {
      cudaEventRecord(c->last_use, st);
      // no copy-in of a caller's host buffer outlives the call, whatever its
      // exit (on success every copy has long been consumed)
      if (c->h2d_stream) cudaStreamSynchronize(c->h2d_stream);
    }
  }
};

// Single-precision calls take SC_PREC_FP32 or SC_PREC_BF16X3; double
// precision calls always compute in FP64 and ignore the field.
template <typename T>
static sc_status check_opts(const sc_options* opt) {
  if (opt && (opt->kernel < SC_KERNEL_AUTO || opt->kernel > SC_KERNEL_CTA))
    return fail(SC_ERR_INVALID_ARG, "unknown kernel choice %d", opt->kernel);
  if (!opt || !std::is_same<T, float>::value) return SC_OK;
  if (opt->precision != SC_PREC_FP32 && opt->precision != SC_PREC_BF16X3)
    return fail(SC_ERR_INVALID_ARG, "unknown precision mode %d", opt->precision);
  if (opt->precision == SC_PREC_BF16X3 && !tc_gemm_available())
    return fail(SC_ERR_UNSUPPORTED, "BF16x3 products need the CUDA driver's tensor-map encoder");
  return SC_OK;
}

static bool want_tc(const sc_options* opt) { return opt && opt->precision == SC_PREC_BF16X3; }
static bool want_refine(const sc_options* opt) { return opt && opt->refine > 0; }

// Splits D into its BF16 hi / lo halves for the tensor-core products.  With
// G set, also a third piece lo3 = bf16(d - hi - lo), from which the Gram
// D^T D + ridge I is formed on the tensor cores to FP32 grade (the BF16x3
// form computes both products that way).
template <typename T>
static sc_status prepare_tc(DeviceCtx& c, cudaStream_t st, Problem<T>& p, Prof& pr,
                            T* G = nullptr, T ridge = T(0)) {
  if constexpr (std::is_same<T, float>::value) {
    p.tc = true;
    p.mp = tc_pad_m(p.m);
    SC_TRY(c.dsplit.reserve((size_t)p.mp * p.K * (G ? 6 : 4)));
    SC_TRY(c.misc.reserve(MISC_BYTES));
    p.d_tc_err = misc_at<int>(c.misc, MISC_TC_ERR);
    SC_CUDA(cudaMemsetAsync(p.d_tc_err, 0, 4, st));
    char* ds = reinterpret_cast<char*>(c.dsplit.ptr);
    pr.mark(ST_GRAM);
    const size_t piece = (size_t)p.mp * p.K * 2;
    SC_CUDA(launch_bf16_split(p.dD, p.m, p.m, p.K, p.mp, ds, ds + piece, st,
                              G ? ds + 2 * piece : nullptr));
    pr.launches(1);
    p.dDsplit = ds;
    if (G) {
      SC_CUDA(launch_gram_tc(ds, ds + piece, ds + 2 * piece, p.dD, p.m, p.mp, p.K, p.Kp, ridge,
                             G, p.d_tc_err, st));
      pr.launches(2);
    }
  } else {
    (void)c; (void)st; (void)p; (void)pr; (void)G; (void)ridge;
  }
  return SC_OK;
}
// Whether a call forms its products on the tensor cores (BF16x3, float).
template <typename T>
static bool tc_form(const sc_options* opt) {
  return opt && opt->precision == SC_PREC_BF16X3 && std::is_same<T, float>::value;
}

// After the stream has drained: a tensor-core pipeline wait that gave up.
template <typename T>
static sc_status check_tc(DeviceCtx& c, cudaStream_t st, const Problem<T>& p) {
  if (!p.tc) return SC_OK;
  int* h = reinterpret_cast<int*>(c.pinned_small) + 16;
  SC_CUDA(cudaMemcpyAsync(h, p.d_tc_err, 4, cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaStreamSynchronize(st));
  if (*h) return fail(SC_ERR_TIMEOUT, "tensor-core correlation pipeline: a bounded wait gave up");
  return SC_OK;
}

sc_status check_atoms(int K) {
  if (pad_atoms(K) > kCtaMaxKp)
    return fail(SC_ERR_UNSUPPORTED, "dictionaries with more than %d atoms are not supported (K=%d)",
                kCtaMaxKp, K);
  return SC_OK;
}
// OMP keeps two K-vectors per signal in shared memory (residual correlations
// and atom norms): in double precision that is 256 KB at 16384 atoms, past
// the 227 KB a block may use, so double-precision OMP stops at 12288.
template <typename T>
static sc_status check_omp_atoms(int K) {
  SC_TRY(check_atoms(K));
  constexpr int kOmpF64MaxKp = 12288;
  if (sizeof(T) == 8 && pad_atoms(K) > kOmpF64MaxKp)
    return fail(SC_ERR_UNSUPPORTED,
                "double-precision omp takes at most %d atoms (K=%d; single precision: %d)",
                kOmpF64MaxKp, K, kCtaMaxKp);
  return SC_OK;
}

// ---------------------------------------------------------------------------
// OMP (host arrays)
template <typename T>
static sc_status omp_host(const T* X, int m, int64_t n, const T* D, int K, const int* Lv,
                          int64_t nL, const T* eps, int64_t nEps, const T* lam, int64_t nLam,
                          T* path, const sc_options* opt, typename CscOf<T>::type* out,
                          const uint8_t* mask = nullptr) {
  if (!out) return fail(SC_ERR_INVALID_ARG, "omp : null output");
  memset(out, 0, sizeof(*out));
  if (m < 0 || n < 0 || K < 0) return fail(SC_ERR_INVALID_ARG, "omp : negative dimension");
  if ((n > 0 && m > 0 && !X) || (K > 0 && m > 0 && !D))
    return fail(SC_ERR_INVALID_ARG, "omp : null input matrix");
  if (nL == 0 && nEps == 0 && nLam == 0)
    return fail(SC_ERR_NO_CRITERION, "omp : You should either provide L, eps or lambda");
  auto bad_count = [&](int64_t c) { return c < 0 || (c > 1 && c != n); };
  if (bad_count(nL) || bad_count(nEps) || bad_count(nLam))
    return fail(SC_ERR_INVALID_ARG, "omp : L/eps/lambda must hold 1 or n entries");
  if ((nL > 0 && !Lv) || (nEps > 0 && !eps) || (nLam > 0 && !lam))
    return fail(SC_ERR_INVALID_ARG, "omp : null L/eps/lambda array");
  const int scalar_L = std::min(m, K);
  const bool vecL = nL > 1, vecE = nEps > 1, vecLa = nLam > 1;
  const int Lsig = nL == 0 ? scalar_L : Lv[0];
  const T eps0 = nEps == 0 ? T(0) : eps[0];
  const T lam0 = nLam == 0 ? T(0) : lam[0];
  if (path) memset(path, 0, sizeof(T) * (size_t)K * scalar_L);
  int L = Lsig;
  if (vecL) {
    L = Lv[0];
    for (int64_t i = 1; i < n; ++i) L = std::max(L, Lv[i]);
  }
  if (L <= 0) return emit_empty<T>(0, 0, out);  // spalpha.clear(); return
  L = std::min(m, std::min(L, K));
  if (n == 0 || L <= 0) return emit_empty<T>(K, n, out);
  SC_TRY(check_omp_atoms<T>(K));

  SC_TRY(check_opts<T>(opt));
  SC_TRY(check_kernel(K, opt));
  DeviceCtx* c = nullptr;
  SC_TRY(get_ctx(opt ? opt->device : 0, &c));
  CallGuard g(c, c->stream);
  cudaStream_t st = c->stream;
  Prof pr;
  pr.on = opt && opt->profile;
  pr.st = st;
  const int Kp = pad_atoms_for(K, opt);
  SC_TRY(c->D.reserve((size_t)m * K * sizeof(T)));
  SC_TRY(c->G.reserve((size_t)Kp * Kp * sizeof(T)));
  SC_CUDA(cudaMemcpyAsync(c->D.ptr, D, (size_t)m * K * sizeof(T), cudaMemcpyHostToDevice, st));
  if (!tc_form<T>(opt)) {  // (the BF16x3 form computes it with the split below)
    pr.mark(ST_GRAM);
    SC_CUDA(launch_gram<T>((const T*)c->D.ptr, m, K, Kp, T(0), (T*)c->G.ptr, st));
    pr.launches(2);
  }
  // per-signal vectors
  const size_t vbytes = (vecL ? 4 * (size_t)n : 0) + (vecE ? sizeof(T) * (size_t)n : 0) +
                        (vecLa ? sizeof(T) * (size_t)n : 0) + 64;
  SC_TRY(c->vecs.reserve(vbytes));
  char* vp = (char*)c->vecs.ptr;
  Problem<T> p;
  p.lars = false;
  if (vecE) {
    p.dEps = (const T*)vp;
    SC_CUDA(cudaMemcpyAsync(vp, eps, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    vp += align16(sizeof(T) * n);
  }
  if (vecLa) {
    p.dLam = (const T*)vp;
    SC_CUDA(cudaMemcpyAsync(vp, lam, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    vp += align16(sizeof(T) * n);
  }
  if (vecL) {
    p.dLv = (const int*)vp;
    SC_CUDA(cudaMemcpyAsync(vp, Lv, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
  }
  p.hX = X; p.dD = (const T*)c->D.ptr; p.m = m; p.n = n; p.K = K; p.Kp = Kp; p.L = L;
  p.Lsig = Lsig; p.eps = eps0; p.lambda = lam0;
  if (path) {
    SC_TRY(c->path.reserve(sizeof(T) * (size_t)K * scalar_L));
    SC_CUDA(cudaMemsetAsync(c->path.ptr, 0, sizeof(T) * (size_t)K * scalar_L, st));
    p.d_path = (T*)c->path.ptr;
  }
  SC_TRY(c->misc.reserve(MISC_BYTES));
  int* d_capflag = misc_at<int>(c->misc, MISC_CAPFLAG);
  HostSink<T> sink;
  if (want_tc(opt) && p.dD) SC_TRY(prepare_tc<T>(*c, st, p, pr, (T*)c->G.ptr, T(0)));
  p.refine = want_refine(opt) && std::is_same<T, float>::value;
  p.kernel = opt ? opt->kernel : SC_KERNEL_AUTO;
  p.refactor = !opt || opt->refactor == 0 ? 1 : (opt->refactor > 0 ? 2 : 0);
  if (mask) {  // omp_mask: masked Grams get a 1e-10 ridge, eps scales (decomp/decomp.h:477-481)
    p.hmask = mask;
    p.mask_ridge = T(1e-10);
    // the warp kernel unless a family is asked for (beyond 1024 atoms the CTA kernel)
    if (p.kernel == SC_KERNEL_AUTO) p.kernel = SC_KERNEL_WARP;
    p.refine = false;
  }
  SC_TRY(run_pipeline<T>(*c, st, p, (const T*)c->G.ptr, &sink, d_capflag, pr));
  SC_TRY(check_tc<T>(*c, st, p));
  if (path)
    SC_CUDA(cudaMemcpyAsync(path, c->path.ptr, sizeof(T) * (size_t)K * scalar_L,
                            cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaStreamSynchronize(st));
  return emit_sink<T>(K, n, sink, out);
}

// ---------------------------------------------------------------------------
// LARS-Lasso (host arrays)
template <typename T>
static int lasso_clamp(int m, int K, int L, T lambda1, T lambda2, int mode, int pos,
                       int* max_length_path) {
  // _lassoD / _lassoQq, cpp_library/spams.h:116-130
  if (L < 0) L = K;
  if (*max_length_path < 0) *max_length_path = 4 * L;
  const bool keep = mode == SC_PENALTY && std::fabs((double)lambda1) < 1e-99 && !pos && lambda2 > 0;
  if (L > m && !keep) L = m;
  if (L > K) L = K;
  return L;
}

template <typename T>
static sc_status lasso_host(const T* X, int m, int64_t n, const T* D, const T* Q, const T* q,
                            int K, int L, T lambda1, T lambda2, int mode, int pos, int ols,
                            int max_length_path, int cholesky, T* path, const sc_options* opt,
                            typename CscOf<T>::type* out, const uint8_t* mask = nullptr) {
  if (!out) return fail(SC_ERR_INVALID_ARG, "lasso : null output");
  memset(out, 0, sizeof(*out));
  if (m < 0 || n < 0 || K < 0) return fail(SC_ERR_INVALID_ARG, "lasso : negative dimension");
  if (n > 0 && m > 0 && !X) return fail(SC_ERR_INVALID_ARG, "lasso : null X");
  if (Q) {
    if (K > 0 && !Q) return fail(SC_ERR_INVALID_ARG, "lasso : null Q");
    if (K > 0 && n > 0 && !q) return fail(SC_ERR_INVALID_ARG, "lasso : null q");
  } else if (K > 0 && m > 0 && !D) {
    return fail(SC_ERR_INVALID_ARG, "lasso : null D");
  }
  if (mode < 0 || mode > 2)
    return fail(SC_ERR_UNSUPPORTED, "lasso : mode %d not supported by the coding path", mode);
  L = lasso_clamp<T>(m, K, L, lambda1, lambda2, mode, pos, &max_length_path);
  // ols or cholesky select the Cholesky implementation (lasso<T> / coreLARS,
  // decomp/decomp.h:735-1093; _lassoD sets cholesky when ols is set)
  const bool chol = ols || cholesky;
  if (path) memset(path, 0, sizeof(T) * (size_t)K * std::max(0, max_length_path));
  if (L <= 0) return emit_empty<T>(0, 0, out);
  if (n == 0) return emit_empty<T>(K, 0, out);
  SC_TRY(check_atoms(K));

  SC_TRY(check_opts<T>(opt));
  SC_TRY(check_kernel(K, opt));
  DeviceCtx* c = nullptr;
  SC_TRY(get_ctx(opt ? opt->device : 0, &c));
  CallGuard g(c, c->stream);
  cudaStream_t st = c->stream;
  Prof pr;
  pr.on = opt && opt->profile;
  pr.st = st;
  const int Kp = pad_atoms_for(K, opt);
  SC_TRY(c->G.reserve((size_t)Kp * Kp * sizeof(T)));
  Problem<T> p;
  p.lars = true;
  if (Q) {
    // use Q as given (no ridge), zero padded
    SC_TRY(c->D.reserve((size_t)K * K * sizeof(T) + (size_t)K * n * sizeof(T)));
    SC_CUDA(cudaMemcpyAsync(c->D.ptr, Q, (size_t)K * K * sizeof(T), cudaMemcpyHostToDevice, st));
    SC_CUDA(launch_pad_rows<T>((const T*)c->D.ptr, K, K, K, (T*)c->G.ptr, Kp, st));
    if (Kp > K)
      SC_CUDA(cudaMemsetAsync((T*)c->G.ptr + (size_t)Kp * K, 0, sizeof(T) * (size_t)Kp * (Kp - K), st));
    T* dq = (T*)c->D.ptr + (size_t)K * K;
    SC_CUDA(cudaMemcpyAsync(dq, q, (size_t)K * n * sizeof(T), cudaMemcpyHostToDevice, st));
    p.dDtX = dq;
  } else {
    SC_TRY(c->D.reserve((size_t)m * K * sizeof(T)));
    SC_CUDA(cudaMemcpyAsync(c->D.ptr, D, (size_t)m * K * sizeof(T), cudaMemcpyHostToDevice, st));
    const T ridge = lambda2 > T(1e-10) ? lambda2 : T(1e-10);  // MAX(lambda2, 1e-10)
    if (!tc_form<T>(opt)) {  // (the BF16x3 form computes it with the split below)
      pr.mark(ST_GRAM);
      SC_CUDA(launch_gram<T>((const T*)c->D.ptr, m, K, Kp, ridge, (T*)c->G.ptr, st));
      pr.launches(2);
    }
    p.dD = (const T*)c->D.ptr;
  }
  p.hX = X; p.m = m; p.n = n; p.K = K; p.Kp = Kp; p.L = L;
  p.mode = mode; p.lambda1 = lambda1; p.pos = pos; p.length_path = max_length_path;
  p.ols = ols != 0;
  p.chol = chol;
  // coreLARS2 replaces a path length <= 1 by 4L (decomp/decomp.h:1722) and
  // writes that many columns; the device buffer covers them, only the
  // caller's max_length_path columns are returned.
  const int dev_cols = max_length_path <= 1 ? 4 * std::min(L, K) : max_length_path;
  if (path && max_length_path > 0) {
    SC_TRY(c->path.reserve(sizeof(T) * (size_t)K * dev_cols));
    SC_CUDA(cudaMemsetAsync(c->path.ptr, 0, sizeof(T) * (size_t)K * dev_cols, st));
    p.d_path = (T*)c->path.ptr;
  }
  SC_TRY(c->misc.reserve(MISC_BYTES));
  int* d_capflag = misc_at<int>(c->misc, MISC_CAPFLAG);
  HostSink<T> sink;
  if (want_tc(opt) && p.dD)
    SC_TRY(prepare_tc<T>(*c, st, p, pr, (T*)c->G.ptr, lambda2 > T(1e-10) ? lambda2 : T(1e-10)));
  p.refine = want_refine(opt) && std::is_same<T, float>::value && !chol;
  p.kernel = opt ? opt->kernel : SC_KERNEL_AUTO;
  p.refactor = !opt || opt->refactor == 0 ? 1 : (opt->refactor > 0 ? 2 : 0);
  if (mask) {
    // lasso_mask: ridge max(lambda2, 1e-10) on the masked Grams, PENALTY and
    // L2ERROR constraints scaled by the observed fraction, coreLARS2's default
    // path length 4 L (decomp/decomp.h:1520-1545)
    p.hmask = mask;
    p.mask_ridge = lambda2 > T(1e-10) ? lambda2 : T(1e-10);
    p.mask_scale = (mode == SC_PENALTY || mode == SC_L2ERROR) ? 1 : 0;
    p.length_path = 4 * L;
    // the warp kernel unless a family is asked for (beyond 1024 atoms the CTA kernel)
    if (p.kernel == SC_KERNEL_AUTO) p.kernel = SC_KERNEL_WARP;
    p.refine = false;
    p.ols = false;
  }
  SC_TRY(run_pipeline<T>(*c, st, p, (const T*)c->G.ptr, &sink, d_capflag, pr));
  SC_TRY(check_tc<T>(*c, st, p));
  if (p.d_path)
    SC_CUDA(cudaMemcpyAsync(path, c->path.ptr, sizeof(T) * (size_t)K * max_length_path,
                            cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaStreamSynchronize(st));
  return emit_sink<T>(K, n, sink, out);
}

// ---------------------------------------------------------------------------
// device-resident entry points
template <typename T>
static sc_status finish_dev(DeviceCtx* c, cudaStream_t st, int64_t* d_colptr, int64_t n,
                            int* d_capflag, int64_t* nnz_out) {
  if (!nnz_out) return SC_OK;
  int64_t* h = reinterpret_cast<int64_t*>(c->pinned_small);
  SC_CUDA(cudaMemcpyAsync(h, d_colptr + n, 8, cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaMemcpyAsync(h + 1, d_capflag, 4, cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaStreamSynchronize(st));
  *nnz_out = h[0];
  if (*reinterpret_cast<int*>(h + 1))
    return fail(SC_ERR_CAPACITY, "output capacity too small: nnz = %lld",
                (long long)h[0]);
  return SC_OK;
}

template <typename T>
static sc_status lasso_dev(const T* dX, int m, int64_t n, const T* dD, int K, int L, T lambda1,
                           T lambda2, int mode, int pos, int max_length_path,
                           int64_t* d_colptr, int32_t* d_rows, T* d_vals, int64_t cap,
                           int64_t* nnz_out, void* stream, const sc_options* opt) {
  if (m <= 0 || n < 0 || K <= 0) return fail(SC_ERR_INVALID_ARG, "lasso : bad dimensions");
  if (!dX || !dD || !d_colptr || (cap > 0 && (!d_rows || !d_vals)))
    return fail(SC_ERR_INVALID_ARG, "lasso : null device pointer");
  if (mode < 0 || mode > 2) return fail(SC_ERR_UNSUPPORTED, "lasso : mode %d", mode);
  L = lasso_clamp<T>(m, K, L, lambda1, lambda2, mode, pos, &max_length_path);
  SC_TRY(check_atoms(K));
  SC_TRY(check_opts<T>(opt));
  SC_TRY(check_kernel(K, opt));
  DeviceCtx* c = nullptr;
  SC_TRY(get_ctx(opt ? opt->device : 0, &c));
  cudaStream_t st = (cudaStream_t)stream;
  CallGuard g(c, st);
  Prof pr;
  pr.on = opt && opt->profile;
  pr.st = st;
  SC_TRY(c->misc.reserve(MISC_BYTES));
  int* d_capflag = misc_at<int>(c->misc, MISC_CAPFLAG);
  SC_CUDA(cudaMemsetAsync(d_capflag, 0, 4, st));
  if (n == 0 || L <= 0) {
    SC_CUDA(cudaMemsetAsync(d_colptr, 0, sizeof(int64_t) * (size_t)(n + 1), st));
    return finish_dev<T>(c, st, d_colptr, n, d_capflag, nnz_out);
  }
  const int Kp = pad_atoms_for(K, opt);
  SC_TRY(c->G.reserve((size_t)Kp * Kp * sizeof(T)));
  const T ridge = lambda2 > T(1e-10) ? lambda2 : T(1e-10);
  if (!tc_form<T>(opt)) {  // (the BF16x3 form computes it with the split below)
    pr.mark(ST_GRAM);
    SC_CUDA(launch_gram<T>(dD, m, K, Kp, ridge, (T*)c->G.ptr, st));
    pr.launches(2);
  }
  Problem<T> p;
  p.lars = true; p.dX = dX; p.dD = dD; p.m = m; p.n = n; p.K = K; p.Kp = Kp; p.L = L;
  p.mode = mode; p.lambda1 = lambda1; p.pos = pos; p.length_path = max_length_path;
  p.d_colptr = d_colptr; p.d_rows = d_rows; p.d_vals = d_vals; p.cap = cap;
  if (want_tc(opt)) SC_TRY(prepare_tc<T>(*c, st, p, pr, (T*)c->G.ptr, ridge));
  p.refine = want_refine(opt) && std::is_same<T, float>::value;
  p.kernel = opt ? opt->kernel : SC_KERNEL_AUTO;
  p.refactor = !opt || opt->refactor == 0 ? 1 : (opt->refactor > 0 ? 2 : 0);
  SC_TRY(run_pipeline<T>(*c, st, p, (const T*)c->G.ptr, nullptr, d_capflag, pr));
  if (nnz_out) SC_TRY(check_tc<T>(*c, st, p));
  return finish_dev<T>(c, st, d_colptr, n, d_capflag, nnz_out);
}

template <typename T>
static sc_status omp_dev(const T* dX, int m, int64_t n, const T* dD, int K, int Lsig, T eps,
                         T lambda, const int* d_L, const T* d_eps, const T* d_lambda,
                         int64_t* d_colptr, int32_t* d_rows, T* d_vals, int64_t cap,
                         int64_t* nnz_out, void* stream, const sc_options* opt) {
  if (m <= 0 || n < 0 || K <= 0) return fail(SC_ERR_INVALID_ARG, "omp : bad dimensions");
  if (!dX || !dD || !d_colptr || (cap > 0 && (!d_rows || !d_vals)))
    return fail(SC_ERR_INVALID_ARG, "omp : null device pointer");
  SC_TRY(check_omp_atoms<T>(K));
  SC_TRY(check_opts<T>(opt));
  SC_TRY(check_kernel(K, opt));
  DeviceCtx* c = nullptr;
  SC_TRY(get_ctx(opt ? opt->device : 0, &c));
  cudaStream_t st = (cudaStream_t)stream;
  CallGuard g(c, st);
  Prof pr;
  pr.on = opt && opt->profile;
  pr.st = st;
  SC_TRY(c->misc.reserve(MISC_BYTES));
  int* d_capflag = misc_at<int>(c->misc, MISC_CAPFLAG);
  SC_CUDA(cudaMemsetAsync(d_capflag, 0, 4, st));
  // the driver L: with per-signal L the caller passes their maximum as Lsig
  int L = std::min(m, std::min(Lsig, K));
  if (n == 0 || L <= 0) {
    SC_CUDA(cudaMemsetAsync(d_colptr, 0, sizeof(int64_t) * (size_t)(n + 1), st));
    return finish_dev<T>(c, st, d_colptr, n, d_capflag, nnz_out);
  }
  const int Kp = pad_atoms_for(K, opt);
  SC_TRY(c->G.reserve((size_t)Kp * Kp * sizeof(T)));
  pr.mark(ST_GRAM);
  if (!tc_form<T>(opt)) {  // (the BF16x3 form computes it with the split below)
    SC_CUDA(launch_gram<T>(dD, m, K, Kp, T(0), (T*)c->G.ptr, st));
    pr.launches(2);
  }
  Problem<T> p;
  p.lars = false; p.dX = dX; p.dD = dD; p.m = m; p.n = n; p.K = K; p.Kp = Kp; p.L = L;
  p.Lsig = Lsig; p.eps = eps; p.lambda = lambda; p.dLv = d_L; p.dEps = d_eps; p.dLam = d_lambda;
  p.d_colptr = d_colptr; p.d_rows = d_rows; p.d_vals = d_vals; p.cap = cap;
  if (want_tc(opt)) SC_TRY(prepare_tc<T>(*c, st, p, pr, (T*)c->G.ptr, T(0)));
  p.refine = want_refine(opt) && std::is_same<T, float>::value;
  p.kernel = opt ? opt->kernel : SC_KERNEL_AUTO;
  p.refactor = !opt || opt->refactor == 0 ? 1 : (opt->refactor > 0 ? 2 : 0);
  SC_TRY(run_pipeline<T>(*c, st, p, (const T*)c->G.ptr, nullptr, d_capflag, pr));
  if (nnz_out) SC_TRY(check_tc<T>(*c, st, p));
  return finish_dev<T>(c, st, d_colptr, n, d_capflag, nnz_out);
}

// ---------------------------------------------------------------------------
// batches of device-resident signals (the serving slots)
sc_status code_batch_f32(DeviceCtx& c, const BatchDesc& b) {
  cudaStream_t st = b.stream;
  SC_TRY(c.misc.reserve(MISC_BYTES));
  int* d_capflag = misc_at<int>(c.misc, MISC_CAPFLAG);
  SC_CUDA(cudaMemsetAsync(d_capflag, 0, 4, st));
  Problem<float> p;
  p.lars = b.lars; p.dX = b.dX; p.dD = b.dD; p.m = b.m; p.n = b.n; p.K = b.K; p.Kp = b.Kp;
  p.L = b.L; p.mode = b.mode; p.lambda1 = b.lambda1; p.pos = b.pos;
  p.length_path = b.length_path; p.dLam1 = b.dLam1;
  p.Lsig = b.Lsig; p.eps = b.eps; p.lambda = b.lambda;
  p.dLv = b.dLv; p.dEps = b.dEps; p.dLam = b.dLam;
  p.d_colptr = b.d_colptr; p.d_rows = b.d_rows; p.d_vals = b.d_vals; p.cap = b.cap;
  p.refine = b.refine;
  p.kernel = b.kernel;
  if (b.tc) {
    if (!b.dDsplit) return fail(SC_ERR_INVALID_ARG, "batch: BF16 products without the split dictionary");
    p.tc = true;
    p.mp = tc_pad_m(b.m);
    p.dDsplit = b.dDsplit;
    p.d_tc_err = misc_at<int>(c.misc, MISC_TC_ERR);
    SC_CUDA(cudaMemsetAsync(p.d_tc_err, 0, 4, st));
  }
  if (b.n == 0) {
    SC_CUDA(cudaMemsetAsync(b.d_colptr, 0, 8, st));
    return SC_OK;
  }
  Prof pr;
  pr.st = st;
  pr.on = b.profile;
  return run_pipeline<float>(c, st, p, b.G, nullptr, d_capflag, pr);
}

sc_status finish_batch(DeviceCtx& c, const BatchDesc& b, int64_t* nnz) {
  cudaStream_t st = b.stream;
  int64_t* h = reinterpret_cast<int64_t*>(c.pinned_small);
  SC_CUDA(cudaMemcpyAsync(h, b.d_colptr + b.n, 8, cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaMemcpyAsync(h + 1, misc_at<int>(c.misc, MISC_CAPFLAG), 4, cudaMemcpyDeviceToHost,
                          st));
  int* herr = reinterpret_cast<int*>(h + 2);
  *herr = 0;
  if (b.tc)
    SC_CUDA(cudaMemcpyAsync(herr, misc_at<int>(c.misc, MISC_TC_ERR), 4, cudaMemcpyDeviceToHost,
                            st));
  SC_CUDA(cudaStreamSynchronize(st));
  *nnz = h[0];
  if (*reinterpret_cast<int*>(h + 1))
    return fail(SC_ERR_CAPACITY, "batch output capacity too small: nnz = %lld", (long long)h[0]);
  if (*herr) return fail(SC_ERR_TIMEOUT, "tensor-core correlation pipeline: a bounded wait gave up");
  return SC_OK;
}

}  // namespace sc

// ---------------------------------------------------------------------------
// C ABI
using namespace sc;

extern "C" {

const char* sc_version(void) { return "spams_b200 0.1"; }
const char* sc_last_error(void) { return sc::last_error(); }

sc_status sc_device_count(int* count) {
  if (!count) return fail(SC_ERR_INVALID_ARG, "null count");
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return fail(SC_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  return SC_OK;
}

void sc_csc_free_f32(sc_csc_f32* a) {
  if (!a) return;
  sc::result_free(a->colptr); sc::result_free(a->rows); sc::result_free(a->vals);
  memset(a, 0, sizeof(*a));
}
void sc_csc_free_f64(sc_csc_f64* a) {
  if (!a) return;
  sc::result_free(a->colptr); sc::result_free(a->rows); sc::result_free(a->vals);
  memset(a, 0, sizeof(*a));
}
void sc_release_all(void) {
  sc::release_all();
  sc::result_pool_trim();
}

sc_status sc_last_profile(sc_profile* out) {
  if (!out) return fail(SC_ERR_INVALID_ARG, "null profile");
  *out = sc::g_prof;
  return SC_OK;
}

sc_status sc_omp_f32(const float* X, int m, int64_t n, const float* D, int K, const int* L,
                     int64_t nL, const float* eps, int64_t nEps, const float* lambda,
                     int64_t nLambda, int numThreads, float* path, const sc_options* opt,
                     sc_csc_f32* out) {
  (void)numThreads;
  prof_reset();
  return omp_host<float>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda, path, opt, out);
}
sc_status sc_omp_f64(const double* X, int m, int64_t n, const double* D, int K, const int* L,
                     int64_t nL, const double* eps, int64_t nEps, const double* lambda,
                     int64_t nLambda, int numThreads, double* path, const sc_options* opt,
                     sc_csc_f64* out) {
  (void)numThreads;
  prof_reset();
  return omp_host<double>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda, path, opt, out);
}

sc_status sc_lasso_f32(const float* X, int m, int64_t n, const float* D, int K, int L,
                       float lambda1, float lambda2, int mode, int pos, int ols, int numThreads,
                       int max_length_path, int cholesky, float* path, const sc_options* opt,
                       sc_csc_f32* out) {
  (void)numThreads;
  prof_reset();
  return lasso_host<float>(X, m, n, D, nullptr, nullptr, K, L, lambda1, lambda2, mode, pos, ols,
                           max_length_path, cholesky, path, opt, out);
}
sc_status sc_lasso_f64(const double* X, int m, int64_t n, const double* D, int K, int L,
                       double lambda1, double lambda2, int mode, int pos, int ols,
                       int numThreads, int max_length_path, int cholesky, double* path,
                       const sc_options* opt, sc_csc_f64* out) {
  (void)numThreads;
  prof_reset();
  return lasso_host<double>(X, m, n, D, nullptr, nullptr, K, L, lambda1, lambda2, mode, pos,
                            ols, max_length_path, cholesky, path, opt, out);
}

sc_status sc_omp_mask_f32(const float* X, int m, int64_t n, const float* D, int K,
                          const uint8_t* mask, const int* L, int64_t nL, const float* eps,
                          int64_t nEps, const float* lambda, int64_t nLambda, int numThreads,
                          float* path, const sc_options* opt, sc_csc_f32* out) {
  (void)numThreads;
  prof_reset();
  if (!mask && n > 0 && m > 0) return fail(SC_ERR_INVALID_ARG, "ompMask : null mask");
  static const uint8_t none = 1;
  return omp_host<float>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda, path, opt, out,
                         mask ? mask : &none);
}
sc_status sc_omp_mask_f64(const double* X, int m, int64_t n, const double* D, int K,
                          const uint8_t* mask, const int* L, int64_t nL, const double* eps,
                          int64_t nEps, const double* lambda, int64_t nLambda, int numThreads,
                          double* path, const sc_options* opt, sc_csc_f64* out) {
  (void)numThreads;
  prof_reset();
  if (!mask && n > 0 && m > 0) return fail(SC_ERR_INVALID_ARG, "ompMask : null mask");
  static const uint8_t none = 1;
  return omp_host<double>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda, path, opt, out,
                          mask ? mask : &none);
}
sc_status sc_lasso_mask_f32(const float* X, int m, int64_t n, const float* D, int K,
                            const uint8_t* mask, int L, float lambda1, float lambda2, int mode,
                            int pos, int numThreads, const sc_options* opt, sc_csc_f32* out) {
  (void)numThreads;
  prof_reset();
  if (!mask && n > 0 && m > 0) return fail(SC_ERR_INVALID_ARG, "lassoMask : null mask");
  static const uint8_t none = 1;
  return lasso_host<float>(X, m, n, D, nullptr, nullptr, K, L, lambda1, lambda2, mode, pos, 0, -1,
                           0, nullptr, opt, out, mask ? mask : &none);
}
sc_status sc_lasso_mask_f64(const double* X, int m, int64_t n, const double* D, int K,
                            const uint8_t* mask, int L, double lambda1, double lambda2, int mode,
                            int pos, int numThreads, const sc_options* opt, sc_csc_f64* out) {
  (void)numThreads;
  prof_reset();
  if (!mask && n > 0 && m > 0) return fail(SC_ERR_INVALID_ARG, "lassoMask : null mask");
  static const uint8_t none = 1;
  return lasso_host<double>(X, m, n, D, nullptr, nullptr, K, L, lambda1, lambda2, mode, pos, 0,
                            -1, 0, nullptr, opt, out, mask ? mask : &none);
}

sc_status sc_lasso_gram_f32(const float* X, int m, int64_t n, const float* Q, int K,
                            const float* q, int L, float lambda1, float lambda2, int mode,
                            int pos, int numThreads, int max_length_path, float* path,
                            const sc_options* opt, sc_csc_f32* out) {
  (void)numThreads;
  if (!Q && K > 0) return fail(SC_ERR_INVALID_ARG, "lasso : null Q");
  static const float dummy = 0;
  prof_reset();
  return lasso_host<float>(X, m, n, nullptr, Q ? Q : &dummy, q, K, L, lambda1, lambda2, mode,
                           pos, 0, max_length_path, 0, path, opt, out);
}
sc_status sc_lasso_gram_f64(const double* X, int m, int64_t n, const double* Q, int K,
                            const double* q, int L, double lambda1, double lambda2, int mode,
                            int pos, int numThreads, int max_length_path, double* path,
                            const sc_options* opt, sc_csc_f64* out) {
  (void)numThreads;
  if (!Q && K > 0) return fail(SC_ERR_INVALID_ARG, "lasso : null Q");
  static const double dummy = 0;
  prof_reset();
  return lasso_host<double>(X, m, n, nullptr, Q ? Q : &dummy, q, K, L, lambda1, lambda2, mode,
                            pos, 0, max_length_path, 0, path, opt, out);
}

sc_status sc_lasso_gram_chol_f32(const float* X, int m, int64_t n, const float* Q, int K,
                                 const float* q, int L, float lambda1, float lambda2, int mode,
                                 int pos, int ols, int cholesky, int numThreads,
                                 int max_length_path, float* path, const sc_options* opt,
                                 sc_csc_f32* out) {
  (void)numThreads;
  if (!Q && K > 0) return fail(SC_ERR_INVALID_ARG, "lasso : null Q");
  static const float dummy = 0;
  prof_reset();
  return lasso_host<float>(X, m, n, nullptr, Q ? Q : &dummy, q, K, L, lambda1, lambda2, mode,
                           pos, ols, max_length_path, cholesky, path, opt, out);
}
sc_status sc_lasso_gram_chol_f64(const double* X, int m, int64_t n, const double* Q, int K,
                                 const double* q, int L, double lambda1, double lambda2, int mode,
                                 int pos, int ols, int cholesky, int numThreads,
                                 int max_length_path, double* path, const sc_options* opt,
                                 sc_csc_f64* out) {
  (void)numThreads;
  if (!Q && K > 0) return fail(SC_ERR_INVALID_ARG, "lasso : null Q");
  static const double dummy = 0;
  prof_reset();
  return lasso_host<double>(X, m, n, nullptr, Q ? Q : &dummy, q, K, L, lambda1, lambda2, mode,
                            pos, ols, max_length_path, cholesky, path, opt, out);
}

sc_status sc_omp_f32_dev(const float* dX, int m, int64_t n, const float* dD, int K, int L,
                         float eps, float lambda, const int* d_L, const float* d_eps,
                         const float* d_lambda, int64_t* d_colptr, int32_t* d_rows,
                         float* d_vals, int64_t cap, int64_t* nnz_out, void* stream,
                         const sc_options* opt) {
  prof_reset();
  return omp_dev<float>(dX, m, n, dD, K, L, eps, lambda, d_L, d_eps, d_lambda, d_colptr, d_rows,
                        d_vals, cap, nnz_out, stream, opt);
}

sc_status sc_corr_f32_dev(const float* dD, int m, int K, const float* dX, int64_t n, float* dC,
                          int ldc, int precision, void* stream) {
  prof_reset();
  if (m <= 0 || K <= 0 || n < 0 || ldc < K || !dD || !dX || (n > 0 && !dC))
    return fail(SC_ERR_INVALID_ARG, "corr : bad arguments");
  DeviceCtx* c = nullptr;
  SC_TRY(get_ctx(0, &c));
  cudaStream_t st = (cudaStream_t)stream;
  CallGuard g(c, st);
  if (n == 0) return SC_OK;
  if (precision == SC_PREC_FP32) {
    SC_CUDA(launch_gemm_tn<float>(dD, m, K, dX, m, n, m, dC, ldc, K, st));
    return SC_OK;
  }
  if (precision != SC_PREC_BF16X3) return fail(SC_ERR_UNSUPPORTED, "corr : precision %d", precision);
  if (!tc_gemm_available()) return fail(SC_ERR_UNSUPPORTED, "corr : tensor-map encoder unavailable");
  const int mp = tc_pad_m(m);
  SC_TRY(c->D.reserve((size_t)mp * K * 4));  // hi + lo
  SC_TRY(c->misc.reserve(MISC_BYTES));
  int* d_err = misc_at<int>(c->misc, MISC_TC_ERR);
  char* dh = (char*)c->D.ptr;
  SC_CUDA(cudaMemsetAsync(d_err, 0, 4, st));
  SC_CUDA(launch_bf16_split(dD, m, m, K, mp, dh, dh + (size_t)mp * K * 2, st));
  const void* dp[2] = {dh, dh + (size_t)mp * K * 2};
  cudaError_t e = launch_tc_corr_xs(dp, 2, K, dX, m, m, n, mp, dC, ldc, K, d_err, st);
  if (e == cudaErrorNotSupported)  // large m: the streaming form
    e = launch_tc_corr_fused(dp[0], dp[1], K, dX, m, m, n, mp, dC, ldc, K, d_err, st);
  SC_CUDA(e);
  int* h = reinterpret_cast<int*>(c->pinned_small);
  SC_CUDA(cudaMemcpyAsync(h, d_err, 4, cudaMemcpyDeviceToHost, st));
  SC_CUDA(cudaStreamSynchronize(st));
  if (*h) return fail(SC_ERR_TIMEOUT, "corr : tensor-core pipeline wait timed out");
  return SC_OK;
}

sc_status sc_lasso_f32_dev(const float* dX, int m, int64_t n, const float* dD, int K, int L,
                           float lambda1, float lambda2, int mode, int pos, int max_length_path,
                           int64_t* d_colptr, int32_t* d_rows, float* d_vals, int64_t cap,
                           int64_t* nnz_out, void* stream, const sc_options* opt) {
  prof_reset();
  return lasso_dev<float>(dX, m, n, dD, K, L, lambda1, lambda2, mode, pos, max_length_path,
                          d_colptr, d_rows, d_vals, cap, nnz_out, stream, opt);
}

}  // extern "C"
