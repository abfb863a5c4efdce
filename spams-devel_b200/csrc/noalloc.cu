// sc_corr_bf16x3_noalloc_f32: the BF16 hi/lo tensor-core correlation product
// D^T X for callers that cannot allocate device memory.
//
// Who needs it: code that runs with a device-memory budget fixed in advance
// (for instance a serving process that has handed all free memory to its own
// pool, where a cudaMalloc fails or fragments that pool) and code that must
// not make the implicit device synchronisations that cudaMalloc / cudaFree can
// make.  sc_corr_f32_dev needs workspace for the hi / lo halves of D and X and
// takes it from the engine's cached allocations; this entry point takes it
// from a fixed array compiled into the library instead, and calls no
// allocating routine.
//
// The scratch is the file-scope array below: kNoAllocScratchBytes (16 MiB) of
// device memory that every GPU which loads the library holds until the
// process exits.  Its device address is looked up once per device, on the
// first call made with that device current (cudaGetSymbolAddress).  All
// calls share the array and it
// keeps the last call's contents, so calls that overlap on the GPU (two
// streams, or two host threads) race: serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/spams_b200.h"
#include "engine.h"
#include "kernels.h"

namespace sc {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr size_t kNoAllocHeader = 256;  // timeout flag of the tensor-core pipeline

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_addr[64];

// Device address of the scratch array for the current device.
static sc_status noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SC_ERR_NO_DEVICE, "corr noalloc : no CUDA device (%s)", cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= 64) return fail(SC_ERR_INVALID_ARG, "corr noalloc : device %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(SC_ERR_CUDA, "corr noalloc : cudaGetSymbolAddress failed (%s)",
                  cudaGetErrorString(e));
    }
    g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_addr[dev];
  return SC_OK;
}

static inline size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace sc

using namespace sc;

extern "C" sc_status sc_corr_bf16x3_noalloc_f32(const float* dD, int m, int K, const float* dX,
                                                int64_t n, float* dC, int ldc, void* stream) {
  if (m <= 0 || K <= 0 || n < 0 || ldc < K || !dD || !dX || (n > 0 && !dC))
    return fail(SC_ERR_INVALID_ARG, "corr noalloc : bad arguments");
  if (!tc_gemm_available())
    return fail(SC_ERR_UNSUPPORTED, "corr noalloc : the CUDA driver's tensor-map encoder is unavailable");
  const int mp = tc_pad_m(m);
  const size_t dbytes = round256((size_t)mp * K * 2);  // one bf16 half of D
  const size_t xbytes = round256((size_t)mp * n * 2);  // one bf16 half of X
  const size_t need = kNoAllocHeader + 2 * dbytes + 2 * xbytes;
  if (need > kNoAllocScratchBytes)
    return fail(SC_ERR_CAPACITY,
                "corr noalloc : D (%d x %d) and X (%d x %lld) need %zu bytes of scratch, more "
                "than the fixed %zu; split X into smaller column blocks",
                m, K, m, (long long)n, need, kNoAllocScratchBytes);
  if (n == 0) return SC_OK;
  unsigned char* base = nullptr;
  sc_status s = noalloc_scratch(&base);
  if (s != SC_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  int* err = reinterpret_cast<int*>(base);
  unsigned char* dh = base + kNoAllocHeader;
  unsigned char* dl = dh + dbytes;
  unsigned char* xh = dl + dbytes;
  unsigned char* xl = xh + xbytes;
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);  // the flag must start at zero
  if (e == cudaSuccess) e = launch_bf16_split(dD, m, m, K, mp, dh, dl, st);
  if (e == cudaSuccess) e = launch_bf16_split(dX, m, m, n, mp, xh, xl, st);
  if (e == cudaSuccess) e = launch_tc_corr(dh, dl, K, xh, xl, n, mp, 3, dC, ldc, K, err, st);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SC_ERR_CUDA, "corr noalloc : %s", cudaGetErrorString(e));
  }
  if (h) return fail(SC_ERR_TIMEOUT, "corr noalloc : a bounded tensor-core pipeline wait gave up");
  return SC_OK;
}
