// Engine internals shared by the C ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "../../include/spams_b200.h"

namespace sc {

sc_status fail(sc_status st, const char* fmt, ...);
const char* last_error();

#define SC_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess)                                                         \
      return fail(_e == cudaErrorMemoryAllocation ? SC_ERR_OUT_OF_MEMORY          \
                                                  : SC_ERR_CUDA,                   \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                  __LINE__);                                                       \
  } while (0)

#define SC_TRY(expr)                    \
  do {                                  \
    sc_status _s = (expr);              \
    if (_s != SC_OK) return _s;         \
  } while (0)


// A grow-only device allocation cached between calls.
struct Buf {
  void* ptr = nullptr;
  size_t bytes = 0;
  bool pooled = false;  // from the stream-ordered allocator
  sc_status reserve(size_t b);
  void release();
};

// While one is in scope on a thread, Buf::reserve grows workspaces through
// the stream-ordered allocator on `st` (the old block freed, the new one
// allocated, then `st` alone waited for) instead of cudaFree / cudaMalloc,
// whose implicit device-wide synchronisation stalls every other stream, other
// serving slots' launches included, at each growth.  The scope's owner
// guarantees that every earlier use of the thread's workspaces is ordered
// before `st`'s current work (a call's guard after its wait on the previous
// call; a serving slot after its previous batch completed).
struct AllocStream {
  cudaStream_t prev;
  explicit AllocStream(cudaStream_t st);
  ~AllocStream();
};
// Returns the stream-ordered pool's free blocks of `device` to the system
// (the pool otherwise keeps them for reuse): sc_release_all, server teardown.
void trim_pool(int device);

// Per-chunk workspaces of a coding lane.  Host-array calls code consecutive
// chunks on two lanes (lane 1 on its own stream), so that one chunk's
// products and coding start while the previous chunk's persistent grid is
// still draining; every other call codes on lane 0 in its own stream.
struct Lane {
  Buf dtx, norms, slab_ind, slab_val, cnt, ovf_list, misc, scan, level, rlist, rscratch,
      gstate, rfscr, order, ordscr;
  cudaStream_t stream = nullptr;  // lane 1's stream
  cudaEvent_t done = nullptr;     // end of lane 1's part of a call
  std::vector<Buf*> bufs() {
    return {&dtx, &norms, &slab_ind, &slab_val, &cnt, &ovf_list, &misc, &scan, &level,
            &rlist, &rscratch, &gstate, &rfscr, &order, &ordscr};
  }
};

// Per-device state: one stream, cached workspaces.  Calls on one device are
// serialised by `mu`.
struct DeviceCtx {
  int device = 0;
  int num_sms = 0;
  int smem_per_sm = 0;
  int smem_per_block = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t last_use = nullptr;  // end of the previous call's device work
  std::mutex mu;
  void* pinned_small = nullptr;  // 4 KiB pinned scratch for small readbacks
  // chunk pipeline of the host-array calls: input copies and result
  // read-backs on their own streams, double-buffered slots
  cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
  cudaEvent_t ev_h2d[2] = {}, ev_xfree[2] = {}, ev_out[2] = {}, ev_d2h[2] = {};
  void* pinned_col = nullptr;  // pinned column pointers of the chunks being read back
  size_t pinned_col_bytes = 0;
  sc_status pinned_cols(size_t bytes);
  Buf X, D, G, misc;
  Buf ccolptr, crows, cvals, path, vecs, xstage, dsplit;
  Buf mask, mflag, mvec, Dt, mwork;  // masked variants
  Lane lane[2];
  cudaEvent_t ev_fork = nullptr;     // lane 1 starts after the call's earlier work
  std::vector<Buf*> all_bufs() {
    std::vector<Buf*> v = {&X, &D, &G, &misc, &ccolptr, &crows, &cvals, &path, &vecs, &xstage,
                           &dsplit, &mask, &mflag, &mvec, &Dt, &mwork};
    for (Lane& l : lane)
      for (Buf* b : l.bufs()) v.push_back(b);
    return v;
  }
};

sc_status get_ctx(int device, DeviceCtx** out);
void release_all();
// A private context (own streams and workspaces), not shared with the C ABI
// calls; the serving slots each own one.
sc_status create_ctx(int device, DeviceCtx** out);
void destroy_ctx(DeviceCtx* c);

// One coding launch over signals already on the device (float32), with
// per-signal parameters; the CSC goes to caller-owned device arrays.  Enqueued
// on b.stream; finish_batch waits for it and checks its status flags.
struct BatchDesc {
  bool lars = true;
  const float* dX = nullptr;   // m x n, column-major
  int m = 0;
  int64_t n = 0;
  const float* dD = nullptr;   // m x K
  const float* G = nullptr;    // Kp x Kp Gram (with the ridge for the Lasso)
  const void* dDsplit = nullptr;  // three BF16 pieces of D (hi, lo, lo3; tc), or NULL
  int K = 0, Kp = 0;
  int L = 0;                   // slab stride: the largest L of the batch
  // Lasso
  int mode = 2, pos = 0, length_path = -1;
  float lambda1 = 0;
  const float* dLam1 = nullptr;   // per-signal lambda1
  // OMP
  int Lsig = 0;
  float eps = 0, lambda = 0;
  const int* dLv = nullptr;
  const float* dEps = nullptr;
  const float* dLam = nullptr;
  bool tc = false, refine = false;
  int kernel = SC_KERNEL_AUTO;
  int64_t* d_colptr = nullptr;
  int32_t* d_rows = nullptr;
  float* d_vals = nullptr;
  int64_t cap = 0;
  cudaStream_t stream = nullptr;  // the stream to enqueue on (NULL: the legacy default stream)
  bool profile = false;  // per-stage device times into the thread's sc_profile (synchronises)
};
void profile_reset();
// Adds k engine kernel launches to the calling thread's sc_profile.
void profile_add_launches(int k);
sc_status code_batch_f32(DeviceCtx& c, const BatchDesc& b);
sc_status finish_batch(DeviceCtx& c, const BatchDesc& b, int64_t* nnz);
int pad_atoms(int K);
sc_status check_atoms(int K);

}  // namespace sc
