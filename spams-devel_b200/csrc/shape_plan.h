// Launch-shape planning for the coding kernels, the autotuner's choice rule
// and the host-array calls' chunking, as plain C++ (no CUDA calls) so that the
// arithmetic is unit-tested on the CPU (tests/cpp/shape_plan_test.cpp).  No
// counterpart in the reference, whose coding loops run one signal per OpenMP
// thread.
//
// A signal is coded either by one warp (Kp <= kWarpMaxKp; its correlations in
// that warp's registers) or by one CTA of Kp / 512 warps (Kp a multiple of
// 512: any of 1..8 warps, then 12, 16, 24 or 32, up to kCtaMaxKp atoms).  Both run the same arithmetic in the same order, so they give the same
// bits; they differ in speed: the warp kernel packs more signals per SM, the
// CTA kernel holds larger active sets in shared memory and codes each signal
// with more threads (lower latency when the batch is small or the active sets
// outgrow the warp's capacity and take the overflow rerun).
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "spams_b200.h"

namespace sc {

constexpr int kWarpMaxKp = 1024;
constexpr int kCtaMaxKp = 16384;

// Warps per signal the CTA kernels are built for.
inline bool cta_warps_ok(int w) { return (w >= 1 && w <= 8) || w == 12 || w == 16 || w == 24 || w == 32; }
// The CTA kernels' layout for K atoms: K rounded up to a multiple of 512
// whose warp count is built (beyond 4096 atoms: 6144, 8192, 12288, 16384);
// kCtaMaxKp + 512 past the largest.
inline int cta_pad_atoms(int K) {
  int w = (K + 511) / 512;
  if (w < 1) w = 1;
  while (w <= kCtaMaxKp / 512 && !cta_warps_ok(w)) ++w;
  return w <= kCtaMaxKp / 512 ? w * 512 : kCtaMaxKp + 512;
}

struct Shape {
  bool cta = false;  // one CTA per signal
  int Lcap = 0;      // active-set capacity in shared memory
  int wpb = 0;       // warps per block (warp kernels) / per signal (CTA kernels)
  int grid = 0;      // persistent blocks (0: filled by the CTA launcher)
};

// What the device offers a launch.
struct DeviceLimits {
  int num_sms = 0;
  size_t smem_per_block = 0;  // opt-in dynamic shared memory per block
  size_t smem_per_sm = 0;
};

// Warp kernel with an active-set capacity of at most `cap` atoms.
// state(lc): one warp's shared-memory state for capacity lc; regw: the warps
// per SM the kernel's registers allow.  Blocks of up to 8 warps (fewer when a
// block's state would not fit), as many blocks per SM as shared memory (1 KB
// reserved per block), registers and the 64-warp limit allow.
template <typename StateBytes>
inline Shape warp_shape(const DeviceLimits& d, int L, int cap, StateBytes state, int regw) {
  Shape s;
  s.cta = false;
  s.Lcap = std::max(1, std::min(L, cap));
  s.wpb = 8;
  const size_t per_warp = state(s.Lcap);
  while (s.wpb > 1 && (size_t)s.wpb * per_warp > d.smem_per_block) s.wpb >>= 1;
  const size_t per_block = (size_t)s.wpb * per_warp + 1024;
  int bps = (int)(d.smem_per_sm / per_block);
  bps = std::min(bps, std::max(1, regw / s.wpb));
  bps = std::max(1, std::min(bps, 64 / s.wpb));
  s.grid = d.num_sms * bps;
  return s;
}

// CTA kernel: the small state is per CTA, so it can hold more atoms (up to
// 80); the capacity shrinks in steps of 16 until two CTAs fit per SM, where
// two fit at all (beyond 8192 atoms the correlations alone fill most of an
// SM's shared memory: one CTA per SM keeps the full capacity).
// bytes(lc): one CTA's shared memory for capacity lc.
template <typename CtaBytes>
inline Shape cta_shape(const DeviceLimits& d, int Kp, int L, CtaBytes bytes) {
  Shape s;
  s.cta = true;
  s.wpb = Kp / 512;
  s.grid = 0;
  s.Lcap = std::max(1, std::min(L, 80));
  while (s.Lcap > 16 && bytes(s.Lcap) > d.smem_per_block) s.Lcap -= 16;
  if (2 * (bytes(std::min(s.Lcap, 16)) + 1024) <= d.smem_per_sm)
    while (s.Lcap > 16 && 2 * (bytes(s.Lcap) + 1024) > d.smem_per_sm) s.Lcap -= 16;
  return s;
}

// Every shape the layout Kp admits, the static rule's first (warp kernel up
// to kWarpMaxKp atoms with a 32-atom state, CTA kernel beyond): the warp
// kernel with a 32- and, when L > 32, a 64-atom state, and the CTA kernel;
// `kernel` (SC_KERNEL_*) keeps only one family.
template <typename WarpState, typename CtaBytes>
inline std::vector<Shape> shape_candidates(const DeviceLimits& d, int Kp, int L, int kernel,
                                           WarpState state, int regw, CtaBytes bytes) {
  std::vector<Shape> v;
  const bool warp_ok = Kp <= kWarpMaxKp, cta_ok = Kp % 512 == 0 && cta_warps_ok(Kp / 512);
  if (warp_ok && kernel != SC_KERNEL_CTA) {
    v.push_back(warp_shape(d, L, 32, state, regw));
    if (L > 32) v.push_back(warp_shape(d, L, 64, state, regw));
  }
  if (cta_ok && kernel != SC_KERNEL_WARP) v.push_back(cta_shape(d, Kp, L, bytes));
  if (v.empty())
    v.push_back(Kp > kWarpMaxKp ? cta_shape(d, Kp, L, bytes) : warp_shape(d, L, 32, state, regw));
  return v;
}

// The autotuner keys its choice by L only through this class: the candidate
// shapes differ at 32 and 64 atoms, and a serving stream's batches carry many
// different L.
inline int tune_lclass(int L) { return L <= 32 ? 0 : (L <= 64 ? 1 : 2); }

// ... and by the batch size (signals of the first chunk) through this class:
// latency-bound batches (a few persistent waves at most), mid-size and large
// ones.  A class per power of two made a serving stream, whose merged batches
// span 1 to ~10^5 signals, tune the same dictionary again for every size,
// each time on samples of up to 16384 signals per candidate.
inline int tune_nclass(int64_t n) { return n < 512 ? 0 : (n < 4096 ? 1 : (n < 32768 ? 2 : 3)); }

// A candidate replaces the one kept so far only below this fraction of its
// sample time.
constexpr float kTuneMargin = 0.95f;

// The autotuner's pick from the candidates' sample times (the static rule's
// shape first): another shape replaces the one kept so far only when clearly
// faster, since near-ties decided by timing noise made the choice, and so
// the full-batch speed, vary from run to run.
inline int pick_fastest(const std::vector<float>& t, float margin = kTuneMargin) {
  int best = 0;
  for (size_t i = 1; i < t.size(); ++i)
    if (t[i] < t[(size_t)best] * margin) best = (int)i;
  return best;
}

// Host-array calls code their signals in chunks of about n / kPipeChunks
// (at least kPipeMinChunk signals) after a first chunk half that size: while
// one chunk is coded, the next one is copied in on the H2D stream and the
// previous chunk's CSC is read back.  Measured on the 100k-signal lasso
// workload, with page-locked results (the H2D of its 102 MB alone takes
// 1.85 ms): 2.77 ms end to end; 2.83 with a quarter-size first chunk, 2.88
// with 8 chunks, 3.17 with 10 (more chunks, more persistent-grid tails).
constexpr int kPipeChunks = 5;
constexpr int64_t kPipeMinChunk = 16384;
constexpr int64_t kPipeFirstDiv = 2;

// Signals per chunk: one chunk's device buffers (per_sig bytes per signal)
// bounded to about 2 GiB, and, with the copy pipeline, about n / kPipeChunks.
inline int64_t chunk_signals(int64_t n, size_t per_sig, bool piped) {
  int64_t nc = (int64_t)std::max<size_t>(4096, ((size_t)2 << 30) / per_sig);
  nc = std::min<int64_t>(nc, std::max<int64_t>(n, 1));
  nc = std::min<int64_t>(nc, (int64_t)1 << 30);
  if (piped) {
    const int64_t k = std::max<int64_t>(1, std::min<int64_t>(kPipeChunks, n / kPipeMinChunk));
    nc = std::min<int64_t>(nc, (n + k - 1) / k);
  }
  return nc;
}

// Chunk i covers signals [start(i), start(i) + len(i)).  With the pipeline the
// first chunk is 1/kPipeFirstDiv of the others: its copy-in is the only one
// nothing overlaps.
struct ChunkPlan {
  int64_t n = 0, nc = 0, first = 0, count = 0;
  int64_t start(int64_t i) const { return i == 0 ? (int64_t)0 : first + (i - 1) * nc; }
  int64_t len(int64_t i) const { return std::min<int64_t>(i == 0 ? first : nc, n - start(i)); }
};
inline ChunkPlan plan_chunks(int64_t n, int64_t nc, bool piped) {
  ChunkPlan c;
  c.n = n;
  c.nc = nc;
  c.first = piped ? std::max<int64_t>(1, std::min<int64_t>(n, nc / kPipeFirstDiv)) : nc;
  c.count = n <= 0 ? 0 : (n <= c.first ? 1 : 1 + (n - c.first + nc - 1) / nc);
  return c;
}

}  // namespace sc
