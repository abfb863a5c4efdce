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

// A grow-only device allocation cached between calls.
struct Buf {
  void* ptr = nullptr;
  size_t bytes = 0;
  sc_status reserve(size_t b);
  void release();
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
  Buf X, D, G, dtx, norms, slab_ind, slab_val, cnt, ovf_list, misc, scan, gstate;
  Buf ccolptr, crows, cvals, path, vecs, xstage, xsplit, dsplit, level, rlist, rscratch;
  std::vector<Buf*> all_bufs() {
    return {&X, &D, &G, &dtx, &norms, &slab_ind, &slab_val, &cnt, &ovf_list, &misc,
            &scan, &gstate, &ccolptr, &crows, &cvals, &path, &vecs, &xstage, &xsplit,
            &dsplit, &level, &rlist, &rscratch};
  }
};

sc_status get_ctx(int device, DeviceCtx** out);
void release_all();

}  // namespace sc
