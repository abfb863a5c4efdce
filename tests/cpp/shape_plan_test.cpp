// Unit checks of the coding kernels' launch-shape planning and the
// autotuner's choice rule (shape_plan.h), compiled and run by
// tests/test_shape_plan.py on the CPU.  Device limits are a B200's (148 SMs,
// 227 KB opt-in shared memory per block, 228 KB per SM); the warp kernels'
// state sizes are the engine's own (kernels.h).
#include <cstdio>
#include <vector>

#include "kernels.h"
#include "shape_plan.h"

using namespace sc;

static int failures = 0;
#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      ++failures;                                             \
    }                                                         \
  } while (0)

static DeviceLimits b200() {
  DeviceLimits d;
  d.num_sms = 148;
  d.smem_per_block = 232448;
  d.smem_per_sm = 233472;
  return d;
}

// Single-precision LARS warp state, and a CTA layout of the same kind
// (Kp correlations + the small state of capacity lc) for the CTA planner.
static auto lars_warp(int Kp) {
  return [Kp](int lc) { return lars_state_bytes(Kp, lc, 4); };
}
static auto cta_bytes(int Kp) {
  return [Kp](int lc) {
    return align16(4 * ((size_t)Kp + 20)) + align16(4 * ((size_t)lc * state_ld(lc) + 6 * (size_t)lc) +
                                                    4 * (size_t)lc);
  };
}

int main() {
  const DeviceLimits d = b200();

  // the 100k-signal lasso workload: Kp 512, L = min(m, K) = 256, warp family
  // forced, 80-register kernel (3 blocks of 8 warps per SM)
  {
    auto v = shape_candidates(d, 512, 256, SC_KERNEL_WARP, lars_warp(512), 24, cta_bytes(512));
    CHECK(v.size() == 2);
    CHECK(!v[0].cta && v[0].Lcap == 32 && v[0].wpb == 8 && v[0].grid == 444);
    CHECK(lars_state_bytes(512, 32, 4) * 8 == 57344);  // the 57.3 KB per block ncu reports
    CHECK(!v[1].cta && v[1].Lcap == 64 && v[1].wpb == 8 && v[1].grid == 148);
  }
  // automatic family on the same layout adds the CTA kernel (one warp per signal)
  {
    auto v = shape_candidates(d, 512, 256, SC_KERNEL_AUTO, lars_warp(512), 24, cta_bytes(512));
    CHECK(v.size() == 3);
    CHECK(v[2].cta && v[2].wpb == 1 && v[2].Lcap == 80 && v[2].grid == 0);
  }
  // dictionary learning: Kp 1024, L 144 -> warp 32 / 64 and the CTA kernel of 2 warps
  {
    auto v = shape_candidates(d, 1024, 144, SC_KERNEL_AUTO, lars_warp(1024), 24, cta_bytes(1024));
    CHECK(v.size() == 3);
    CHECK(v[0].Lcap == 32 && v[1].Lcap == 64 && v[2].cta && v[2].wpb == 2 && v[2].Lcap == 80);
  }
  // L at most 32: no 64-atom warp shape, and capacities follow L
  {
    auto v = shape_candidates(d, 512, 20, SC_KERNEL_AUTO, lars_warp(512), 24, cta_bytes(512));
    CHECK(v.size() == 2 && v[0].Lcap == 20 && v[1].cta && v[1].Lcap == 20);
  }
  // beyond the warp kernel's 1024 atoms only the CTA kernel, whatever is forced
  {
    auto v = shape_candidates(d, 2048, 68, SC_KERNEL_AUTO, lars_warp(1024), 0, cta_bytes(2048));
    CHECK(v.size() == 1 && v[0].cta && v[0].wpb == 4 && v[0].Lcap == 68);
    v = shape_candidates(d, 4096, 512, SC_KERNEL_WARP, lars_warp(1024), 0, cta_bytes(4096));
    CHECK(v.size() == 1 && v[0].cta && v[0].wpb == 8 && v[0].Lcap == 80);
  }
  // a layout the CTA kernel cannot take (Kp not a multiple of 512) falls back
  // to the warp kernel even when the CTA family is forced
  {
    auto v = shape_candidates(d, 384, 40, SC_KERNEL_CTA, lars_warp(384), 24, cta_bytes(384));
    CHECK(v.size() == 1 && !v[0].cta && v[0].Lcap == 32);
  }
  // the CTA capacity shrinks in steps of 16 until two CTAs fit per SM
  {
    DeviceLimits small = d;
    small.smem_per_sm = 2 * (cta_bytes(4096)(48) + 1024);
    Shape s = cta_shape(small, 4096, 200, cta_bytes(4096));
    CHECK(s.Lcap == 48);
  }
  // a small shared-memory budget halves the warps per block; registers cap the blocks
  {
    DeviceLimits small = d;
    small.smem_per_block = 49152;
    small.smem_per_sm = 102400;
    Shape s = warp_shape(small, 256, 64, lars_warp(512), 64);
    CHECK(s.wpb == 2);  // 8 or 4 warps of 20 KB state do not fit 48 KB
    CHECK(s.grid == 148 * 2);
    s = warp_shape(d, 256, 32, lars_warp(512), 8);
    CHECK(s.wpb == 8 && s.grid == 148);  // 8 register-limited warps per SM: one block
  }
  // the tuner's key classes and its margin rule
  CHECK(tune_lclass(1) == 0 && tune_lclass(32) == 0 && tune_lclass(33) == 1);
  CHECK(tune_lclass(64) == 1 && tune_lclass(65) == 2 && tune_lclass(512) == 2);
  CHECK(tune_nclass(1) == 0 && tune_nclass(511) == 0 && tune_nclass(512) == 1);
  CHECK(tune_nclass(4095) == 1 && tune_nclass(4096) == 2 && tune_nclass(32767) == 2);
  CHECK(tune_nclass(32768) == 3 && tune_nclass((int64_t)1 << 40) == 3);
  CHECK(pick_fastest({}) == 0);
  CHECK(pick_fastest({1.0f}) == 0);
  CHECK(pick_fastest({1.0f, 0.97f}) == 0);  // within the margin: the static rule's shape stays
  CHECK(pick_fastest({1.0f, 0.90f}) == 1);
  CHECK(pick_fastest({1.0f, 0.90f, 0.88f}) == 1);  // must beat the kept one by the margin
  CHECK(pick_fastest({1.0f, 0.90f, 0.85f}) == 2);
  CHECK(pick_fastest({1.0f, 2.0f, 0.5f}) == 2);

  // the CTA kernels' layouts: multiples of 512 up to 4096 atoms, then the
  // built warp counts 12, 16, 24, 32 (6144 .. 16384 atoms)
  CHECK(cta_pad_atoms(1025) == 1536 && cta_pad_atoms(4096) == 4096);
  CHECK(cta_pad_atoms(4097) == 6144 && cta_pad_atoms(6144) == 6144);
  CHECK(cta_pad_atoms(6145) == 8192 && cta_pad_atoms(8193) == 12288);
  CHECK(cta_pad_atoms(16384) == 16384 && cta_pad_atoms(16385) > kCtaMaxKp);
  for (int w = 1; w <= 40; ++w)
    CHECK(cta_warps_ok(w) == ((w <= 8) || w == 12 || w == 16 || w == 24 || w == 32));
  {
    // 16384 atoms: 64 KB of correlations per CTA; two CTAs never fit, so the
    // capacity is not cut for them
    DeviceLimits d{148, 227 * 1024, 228 * 1024};
    auto bytes = [](int lc) { return (size_t)16384 * 4 * 2 + (size_t)lc * (lc + 1) * 4 + 4096; };
    const Shape s = cta_shape(d, 16384, 200, bytes);
    CHECK(s.cta && s.wpb == 32 && s.Lcap == 80);
    // 2048 atoms: two CTAs fit once the capacity is cut to 64 or below
    auto small = [](int lc) { return (size_t)2048 * 4 * 2 + (size_t)lc * (lc + 1) * 4 * 30; };
    const Shape t = cta_shape(d, 2048, 200, small);
    CHECK(t.Lcap <= 64 && 2 * (small(t.Lcap) + 1024) <= d.smem_per_sm);
  }

  // host-array chunking: contiguous chunks covering [0, n), the first one half
  // the others with the copy pipeline
  auto covers = [](const ChunkPlan& c) {
    int64_t at = 0;
    for (int64_t i = 0; i < c.count; ++i) {
      if (c.start(i) != at || c.len(i) <= 0) return false;
      at += c.len(i);
    }
    return at == c.n;
  };
  {
    // the 100k-signal lasso workload's host call (Kp 512, L 256, m 256, BF16 split)
    const size_t per_sig = 512 * 4 + 256 * 8 + 64 + 2 * 256 * 4 + 256 * 4 + 2 * (256 * 8 + 8);
    const int64_t nc = chunk_signals(100000, per_sig, true);
    CHECK(nc == 20000);
    const ChunkPlan c = plan_chunks(100000, nc, true);
    CHECK(c.count == 6 && c.first == 10000 && covers(c));
    CHECK(c.len(1) == 20000 && c.len(4) == 20000 && c.len(5) == 10000);
  }
  {
    // without the pipeline: one chunk up to the ~2 GiB buffer bound
    const int64_t nc = chunk_signals(100000, 8192, false);
    CHECK(nc == 100000);
    ChunkPlan c = plan_chunks(100000, nc, false);
    CHECK(c.count == 1 && covers(c));
    const int64_t big = chunk_signals(1000000, 8192, false);
    CHECK(big == ((int64_t)2 << 30) / 8192);
    c = plan_chunks(1000000, big, false);
    CHECK(c.count == 4 && covers(c));
  }
  {
    // small host calls: one chunk of everything (fewer than 2 x 16384 signals)
    const int64_t nc = chunk_signals(20000, 4096, true);
    CHECK(nc == 20000);
    const ChunkPlan c = plan_chunks(20000, nc, true);
    CHECK(c.first == 10000 && c.count == 2 && covers(c));
    CHECK(plan_chunks(1, chunk_signals(1, 4096, true), true).count == 1);
    CHECK(plan_chunks(0, chunk_signals(0, 4096, true), true).count == 0);
  }
  for (int64_t n : {16384, 50000, 99999, 100001, 1000000, 3333333}) {
    const int64_t nc = chunk_signals(n, 4096, true);
    const ChunkPlan c = plan_chunks(n, nc, true);
    CHECK(covers(c) && c.first == std::max<int64_t>(1, nc / kPipeFirstDiv));
    // at most kPipeChunks full chunks unless the buffer bound (2 GiB / 4096 B)
    // makes them smaller
    if (nc < ((int64_t)2 << 30) / 4096) CHECK(c.count <= kPipeChunks + 1);
    else CHECK(nc == ((int64_t)2 << 30) / 4096);
  }

  if (failures) {
    std::printf("%d check(s) failed\n", failures);
    return 1;
  }
  std::printf("all checks passed\n");
  return 0;
}
