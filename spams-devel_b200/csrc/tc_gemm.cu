// Correlations C = D^T X on the 5th-generation tensor cores (sm_100a):
// BF16 hi/lo split operands, FP32 accumulation in tensor memory.
//
//   x = hi(x) + lo(x), hi = bf16(x), lo = bf16(x - hi)
//   C = Dhi^T Xhi + Dhi^T Xlo + Dlo^T Xhi        (the lo*lo term is dropped)
//
// The three products are one GEMM over a reduction dimension of 3 m_pad: the
// k-block loop walks the three (A, B) operand pairs in turn.  Operands are
// K-major (the signal dimension m is contiguous in both D and X), staged by
// TMA into 128-byte-swizzled shared-memory tiles, multiplied by tcgen05.mma
// (M = 128 atoms, N = 128 signals, K = 16) issued by one thread, accumulated
// in TMEM and read back by four warps with tcgen05.ld for a column-major
// store of C (atoms contiguous per signal, the layout the coding kernels
// read).  Every mbarrier wait is bounded: on timeout the CTA records an error,
// drains its own copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace sc {

constexpr int TC_BM = 128;          // atoms per tile (MMA M)
constexpr int TC_BN = 128;          // signals per tile (MMA N)
constexpr int TC_BK = 64;           // bf16 per 128-byte swizzled row
constexpr int TC_STAGES = 3;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;
constexpr int TC_B_BYTES = TC_BN * TC_BK * 2;
constexpr int TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr int TC_TMEM_COLS = 128;   // fp32 accumulator columns (= TC_BN)
constexpr size_t TC_SMEM = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr long long TC_TIMEOUT_CYCLES = 4000000000LL;  // ~2 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// Wait for the phase of the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > TC_TIMEOUT_CYCLES) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor: K-major operand in 128-byte swizzled rows,
// 8-row core-matrix groups 1024 bytes apart (tile base 1024-byte aligned).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1u << 16;                            // leading offset (unused for SW128 K-major)
  d |= (uint64_t)(1024u >> 4) << 32;                  // stride offset: 8 rows x 128 B
  d |= (uint64_t)1u << 46;                            // descriptor version (sm_100)
  d |= (uint64_t)2u << 61;                            // swizzle mode: 128 B
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, M = TC_BM, N = TC_BN.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((uint32_t)(TC_BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__global__ void __launch_bounds__(128, 1)
tc_corr_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
               const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB0,
               const __grid_constant__ CUtensorMap mB1, const __grid_constant__ CUtensorMap mB2,
               uint32_t term_code, float* __restrict__ C, int ldc, int rows_out, int64_t n,
               int m_pad, int nterms,
               int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TC_STAGES * TC_STAGE_BYTES);
  // bars[0..S) full, bars[S..2S) empty, bars[2S] accumulator ready
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * TC_STAGES + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * TC_BM;
  const int64_t n0 = (int64_t)blockIdx.y * TC_BN;
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (TC_STAGES + s); };
  const uint32_t acc_bar = bar0 + 8u * (2 * TC_STAGES);

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(acc_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int kb_per_term = m_pad / TC_BK;
  const int total_kb = nterms * kb_per_term;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    int issued = 0;
    for (int kb = 0; kb < total_kb; ++kb) {
      const int s = kb % TC_STAGES;
      const uint32_t round = kb / TC_STAGES;
      if (*abort_flag || !mbar_wait(empty_bar(s), (round & 1u) ^ 1u)) { *abort_flag = 1; break; }
      const int term = kb / kb_per_term;
      const int kx = (kb % kb_per_term) * TC_BK;
      // term t multiplies A piece (code >> 4t) & 3 by B piece (code >> 4t + 2) & 3
      const uint32_t ia = (term_code >> (4 * term)) & 3u, ib = (term_code >> (4 * term + 2)) & 3u;
      const CUtensorMap* ma = ia == 0 ? &mA0 : (ia == 1 ? &mA1 : &mA2);
      const CUtensorMap* mb = ib == 0 ? &mB0 : (ib == 1 ? &mB1 : &mB2);
      uint8_t* st = smem + (size_t)s * TC_STAGE_BYTES;
      mbar_expect_tx(full_bar(s), TC_STAGE_BYTES);
      tma_load_2d(smem_u32(st), ma, full_bar(s), kx, m0);
      tma_load_2d(smem_u32(st + TC_A_BYTES), mb, full_bar(s), kx, (int)n0);
      issued = kb + 1;
    }
    if (*abort_flag) {
      // drain: every issued stage whose completion was not observed by the
      // MMA thread lands before the CTA may exit
      for (int kb = issued - TC_STAGES < 0 ? 0 : issued - TC_STAGES; kb < issued; ++kb)
        mbar_wait(full_bar(kb % TC_STAGES), (uint32_t)(kb / TC_STAGES) & 1u);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int kb = 0; kb < total_kb; ++kb) {
      const int s = kb % TC_STAGES;
      const uint32_t round = kb / TC_STAGES;
      if (*abort_flag || !mbar_wait(full_bar(s), round & 1u)) { *abort_flag = 1; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_addr = smem_u32(smem + (size_t)s * TC_STAGE_BYTES);
      const uint32_t b_addr = a_addr + TC_A_BYTES;
#pragma unroll
      for (int k = 0; k < TC_BK / 16; ++k)
        umma_bf16(tmem, sw128_desc(a_addr + 32u * k), sw128_desc(b_addr + 32u * k),
                  (kb > 0 || k > 0) ? 1u : 0u);
      umma_commit(empty_bar(s));  // stage free once these MMAs have read it
    }
    umma_commit(acc_bar);  // accumulator complete (also after an abort)
  }
  __syncwarp();

  // ---- epilogue: TMEM -> registers -> C (column-major, atoms contiguous)
  const bool acc_ok = mbar_wait(acc_bar, 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (acc_ok && !*abort_flag) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < TC_BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
            "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
            "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
            "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < rows_out) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int64_t col = n0 + c0 + j;
          if (col < n) C[(size_t)col * ldc + row] = __uint_as_float(v[j]);
        }
      }
    }
  }
  if ((!acc_ok || *abort_flag) && threadIdx.x == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TC_TMEM_COLS)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Persistent form with the split of X fused in: C = D^T X for fp32 X.
//
// One CTA per SM loops over 128-atom x 128-signal output tiles (consecutive
// tiles of a CTA share their signals, so X is read from HBM once and from L2
// for the other atom tiles).  Per 64-deep k-block a stage holds Dhi and Dlo
// (TMA, 128-byte swizzle) and Xhi and Xlo, which four converter warps write
// from the fp32 signals in the same swizzled layout (the 16-byte chunk j of
// row r at chunk j ^ (r & 7) of the row's 128-byte line), so no split copy of
// X exists in memory.  The MMA thread issues the three products of the
// k-block (Dhi Xhi, Dhi Xlo, Dlo Xhi) into one of two TMEM accumulators;
// four epilogue warps read the other accumulator with tcgen05.ld and store
// its tile while the next one is multiplied.
//   warps 0-3  convert X          warps 4-7  epilogue (TMEM lanes 0-127)
//   warp 8     TMA of D           warp 9     MMA issue
// Every wait is bounded: on timeout the CTA records an error, stops issuing
// work, waits for what it issued and frees its TMEM.
constexpr int T2_STAGES = 3;
constexpr int T2_TILE_BYTES = TC_BM * TC_BK * 2;  // 16 KB: one 128 x 64 bf16 operand tile
constexpr int T2_STAGE_BYTES = 4 * T2_TILE_BYTES; // Dhi | Dlo | Xhi | Xlo
constexpr int T2_TMEM_COLS = 2 * TC_BN;           // two 128-column accumulators
constexpr int T2_THREADS = 320;
constexpr size_t T2_SMEM = (size_t)T2_STAGES * T2_STAGE_BYTES + 1024 + 256;

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

template <bool VEC>
__global__ void __launch_bounds__(T2_THREADS, 1)
tc_corr_fused_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                     const float* __restrict__ X, int64_t ldx, int m, int64_t n, int m_pad,
                     float* __restrict__ C, int ldc, int rows_out, int m_tiles, int64_t n_tiles,
                     int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + T2_STAGES * T2_STAGE_BYTES);
  // bars: full[S], empty[S], acc_full[2], acc_empty[2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * T2_STAGES + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar0 = smem_u32(bars);
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (T2_STAGES + s); };
  auto accf_bar = [&](int b) { return bar0 + 8u * (2 * T2_STAGES + b); };
  auto acce_bar = [&](int b) { return bar0 + 8u * (2 * T2_STAGES + 2 + b); };

  if (threadIdx.x == 0) {
    for (int s = 0; s < T2_STAGES; ++s) {
      mbar_init(full_bar(s), 5);   // four converter warps + the TMA thread (with its bytes)
      mbar_init(empty_bar(s), 1);  // tcgen05.commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);   // tcgen05.commit
      mbar_init(acce_bar(b), 4);   // four epilogue warps
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(T2_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int kblocks = m_pad / TC_BK;
  const int64_t tiles = (int64_t)m_tiles * n_tiles;

  if (warp < 4) {
    // ---- converter: Xhi / Xlo of every k-block of the tile's 128 signals
    int64_t kbg = 0;
    for (int64_t t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
      const int64_t n0 = (t / m_tiles) * TC_BN;
      for (int kb = 0; kb < kblocks; ++kb, ++kbg) {
        const int s = (int)(kbg % T2_STAGES);
        const uint32_t round = (uint32_t)(kbg / T2_STAGES);
        // every lane waits; the warp goes on only if all of them saw the phase
        if (!__all_sync(kFull, mbar_wait(empty_bar(s), (round & 1u) ^ 1u))) {
          *abort_flag = 1;
          break;
        }
        uint8_t* xh = smem + (size_t)s * T2_STAGE_BYTES + 2 * T2_TILE_BYTES;
        uint8_t* xl = xh + T2_TILE_BYTES;
        const int k0 = kb * TC_BK;
        // 128 rows x 8 chunks of 8 values: unit u = threadIdx.x + 128 q
        float v[8][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int u = threadIdx.x + 128 * q;
          const int row = u >> 3, ch = u & 7;
          const int64_t sig = n0 + row;
          const int k = k0 + ch * 8;
          if (VEC && sig < n && k + 8 <= m) {
            const float* src = X + (size_t)sig * ldx + k;
            const float4 a = __ldg(reinterpret_cast<const float4*>(src));
            const float4 b = __ldg(reinterpret_cast<const float4*>(src + 4));
            v[q][0] = a.x; v[q][1] = a.y; v[q][2] = a.z; v[q][3] = a.w;
            v[q][4] = b.x; v[q][5] = b.y; v[q][6] = b.z; v[q][7] = b.w;
          } else {
#pragma unroll
            for (int e = 0; e < 8; ++e)
              v[q][e] = (sig < n && k + e < m) ? X[(size_t)sig * ldx + k + e] : 0.f;
          }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int u = threadIdx.x + 128 * q;
          const int row = u >> 3, ch = u & 7;
          __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            h[e] = __float2bfloat16_rn(v[q][e]);
            l[e] = __float2bfloat16_rn(v[q][e] - __bfloat162float(h[e]));
          }
          const uint32_t off = (uint32_t)row * 128u + ((uint32_t)(ch ^ (row & 7)) << 4);
          *reinterpret_cast<uint4*>(xh + off) = *reinterpret_cast<const uint4*>(h);
          *reinterpret_cast<uint4*>(xl + off) = *reinterpret_cast<const uint4*>(l);
        }
        // make the generic-proxy writes visible to the tensor cores, then arrive
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(full_bar(s));
      }
    }
  } else if (warp < 8) {
    // ---- epilogue: TMEM -> registers -> C (column-major, atoms contiguous)
    int it = 0;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int b = it & 1;
      if (*abort_flag || !__all_sync(kFull, mbar_wait(accf_bar(b), (uint32_t)(it >> 1) & 1u))) {
        *abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int m0 = (int)(t % m_tiles) * TC_BM;
      const int64_t n0 = (t / m_tiles) * TC_BN;
      const int wl = warp & 3;  // TMEM lanes 32 wl .. 32 wl + 31
      const int row = m0 + wl * 32 + lane;
#pragma unroll 1
      for (int c0 = 0; c0 < TC_BN; c0 += 32) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(wl * 32) << 16) + (uint32_t)(b * TC_BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
              "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
              "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
              "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < rows_out) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int64_t col = n0 + c0 + j;
            if (col < n) C[(size_t)col * ldc + row] = __uint_as_float(v[j]);
          }
        }
      }
      // the accumulator may take the next tile
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(acce_bar(b));
    }
  } else if (warp == 8) {
    // ---- TMA producer of the D halves
    if (lane == 0) {
      int64_t kbg = 0, issued = 0;
      for (int64_t t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
        const int m0 = (int)(t % m_tiles) * TC_BM;
        for (int kb = 0; kb < kblocks; ++kb, ++kbg) {
          const int s = (int)(kbg % T2_STAGES);
          const uint32_t round = (uint32_t)(kbg / T2_STAGES);
          if (*abort_flag || !mbar_wait(empty_bar(s), (round & 1u) ^ 1u)) { *abort_flag = 1; break; }
          uint8_t* st = smem + (size_t)s * T2_STAGE_BYTES;
          mbar_expect_tx(full_bar(s), 2 * T2_TILE_BYTES);
          tma_load_2d(smem_u32(st), &mAh, full_bar(s), kb * TC_BK, m0);
          tma_load_2d(smem_u32(st + T2_TILE_BYTES), &mAl, full_bar(s), kb * TC_BK, m0);
          issued = kbg + 1;
        }
      }
      if (*abort_flag) {
        // the copies of the last stages must land before the CTA may exit
        for (int64_t k = issued - T2_STAGES < 0 ? 0 : issued - T2_STAGES; k < issued; ++k)
          mbar_wait(full_bar((int)(k % T2_STAGES)), (uint32_t)(k / T2_STAGES) & 1u);
      }
    }
  } else {
    // ---- MMA issuer
    if (lane == 0) {
      int64_t kbg = 0;
      int it = 0;
      bool any = false;
      for (int64_t t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x, ++it) {
        const int b = it & 1;
        if (!mbar_wait(acce_bar(b), ((uint32_t)(it >> 1) & 1u) ^ 1u)) { *abort_flag = 1; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(b * TC_BN);
        for (int kb = 0; kb < kblocks; ++kb, ++kbg) {
          const int s = (int)(kbg % T2_STAGES);
          const uint32_t round = (uint32_t)(kbg / T2_STAGES);
          if (*abort_flag || !mbar_wait(full_bar(s), round & 1u)) { *abort_flag = 1; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t dh = smem_u32(smem + (size_t)s * T2_STAGE_BYTES);
          const uint32_t dl = dh + T2_TILE_BYTES, xh = dh + 2 * T2_TILE_BYTES,
                         xl = dh + 3 * T2_TILE_BYTES;
#pragma unroll
          for (int k = 0; k < TC_BK / 16; ++k) {
            const uint32_t o = 32u * k;
            umma_bf16(acc, sw128_desc(dh + o), sw128_desc(xh + o), (kb > 0 || k > 0) ? 1u : 0u);
            umma_bf16(acc, sw128_desc(dh + o), sw128_desc(xl + o), 1u);
            umma_bf16(acc, sw128_desc(dl + o), sw128_desc(xh + o), 1u);
          }
          umma_commit(empty_bar(s));  // the stage is free once these have read it
          any = true;
        }
        if (*abort_flag) break;
        umma_commit(accf_bar(b));  // the tile's accumulator is complete
      }
      if (*abort_flag && any) {
        // every issued MMA has finished before TMEM is freed: a last commit
        // arrives on an accumulator barrier once all earlier ones are done
        umma_commit(accf_bar(it & 1));
        mbar_wait(accf_bar(it & 1), (uint32_t)(it >> 1) & 1u);
      }
    }
  }
  __syncwarp();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(T2_TMEM_COLS)
                 : "memory");
}

// ---------------------------------------------------------------------------
// X-stationary persistent form: C = D^T X for fp32 X, each signal tile's
// split formed once in shared memory and multiplied by every atom tile.
//
// A CTA takes units of BN signals x a group of 128-atom tiles.  For one unit
// the fp32 signals arrive by TMA, half a k-block (32 values per signal) at a
// time, in a ring of staging buffers; eight converter warps split them into
// NP bf16 pieces, written in the 128-byte-swizzled K-major layout the MMA
// reads (the 16-byte chunk j of row r at chunk j ^ (r & 7)), and the pieces
// of all k-blocks stay resident while the group's atom tiles are walked, the
// pieces of D streaming by TMA through a second ring.  A k-block's resident
// pieces go back to the converters for the next unit as soon as the group's
// last atom tile has read them; by then the staging ring already holds the
// next unit's signals.  The atom tiles form one group when there are signal
// tiles enough to fill the SMs, and are spread over several groups (each
// converting the signals again) when there are not.
//   NP = 2: x = hi + lo,        3 products  hi hi, hi lo, lo hi
//   NP = 3: x = hi + mid + lo,  6 products  + hi lo, lo hi, mid mid
// (NP = 3 carries FP32's 24 significant bits and drops only products below
// FP32 rounding; D comes split the same way, its pieces in global memory.)
// The MMA thread accumulates each tile into one of two TMEM buffers while
// eight epilogue warps drain the other with tcgen05.ld (two warps per lane
// quarter, half the columns each) and store it.  A buffer holds two
// accumulators: the leading product (hi hi) and the sum of the correction
// products, added in FP32 in the epilogue.  The tensor cores' FP32
// accumulation loses low bits on every MMA relative to the accumulator's
// magnitude; the corrections, 2^-8 of it and smaller, would otherwise lose
// about as much as they add (the six-product form then measured no better
// than three products against FP64).
//   warps 0-3  convert X      warps 4-11  epilogue
//   warp 12    TMA of D       warp 13     MMA issue      warp 14  TMA of X
// Every wait is bounded: on timeout the CTA records an error, stops issuing
// work, waits for what it issued and frees its TMEM.
constexpr int XS_THREADS = 480;  // 4 converter + 8 epilogue + 3 single-thread warps
constexpr int XS_CONV_THREADS = 128;
constexpr int XS_EPI_WARPS = 8;
constexpr int XS_CONV_WARPS = XS_CONV_THREADS / 32;
constexpr int XS_MAX_KB = 32;                   // m_pad <= 2048
constexpr int XS_D_TILE = TC_BM * TC_BK * 2;    // 16 KB: one 128 x 64 bf16 piece of D
constexpr int XS_MAX_S = 3;                     // stages of the D ring
constexpr int XS_MAX_NSTG = 4;                  // staging buffers of half a k-block
constexpr size_t XS_SMEM_LIMIT = 232448;        // 227 KB of dynamic shared memory

__host__ __device__ constexpr size_t xs_xres_bytes(int np, int bn, int kblocks) {
  return (size_t)kblocks * np * bn * 128;
}
__host__ __device__ constexpr size_t xs_smem_bytes(int np, int bn, int kblocks, int s, int nstg) {
  return xs_xres_bytes(np, bn, kblocks) + (size_t)s * np * XS_D_TILE + (size_t)nstg * bn * 128 +
         1024 + 1024;
}

template <int BN>
__device__ __forceinline__ void umma_bf16_n(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t accumulate) {
  constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                             ((uint32_t)(TC_BM >> 4) << 24);
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 16 columns of fp32 from TMEM (this warp's lane quarter).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int NP, int BN>
__global__ void __launch_bounds__(XS_THREADS, 1)
tc_corr_xs_kernel(const __grid_constant__ CUtensorMap mD0, const __grid_constant__ CUtensorMap mD1,
                  const __grid_constant__ CUtensorMap mD2, const __grid_constant__ CUtensorMap mX,
                  int64_t n, int m_pad, float* __restrict__ C, int ldc, int rows_out,
                  int m_tiles, int groups, int per_group, int64_t units, int S, int NSTG,
                  int* err) {
  constexpr int STAGE = NP * XS_D_TILE;
  constexpr int XPIECE = BN * 128;                 // one k-block of one piece of the signals
  constexpr int STG = BN * 128;                    // BN signals x 32 fp32
  constexpr uint32_t TMEM_COLS = 4 * BN < 32 ? 32 : 4 * BN;  // 2 buffers x (main, corrections)
  constexpr int UNITS = BN * 4;                    // 8-value chunks per staging buffer
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  const int kblocks = m_pad / TC_BK;
  const int halves = 2 * kblocks;
  uint8_t* xres = smem;                                         // [kb][piece] BN x 128 B
  uint8_t* dring = smem + xs_xres_bytes(NP, BN, kblocks);       // [stage] NP x 16 KB
  uint8_t* sring = dring + (size_t)S * STAGE;                   // [stage] BN x 128 B fp32
  uint64_t* bars = reinterpret_cast<uint64_t*>(sring + (size_t)NSTG * STG);
  // dfull[S] dempty[S] sfull[NSTG] sempty[NSTG] xfull[MAX_KB] xempty[MAX_KB] accf[2] acce[2]
  // (slots for the largest S and NSTG)
  uint32_t* tmem_slot =
      reinterpret_cast<uint32_t*>(bars + 2 * XS_MAX_S + 2 * XS_MAX_NSTG + 2 * XS_MAX_KB + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar0 = smem_u32(bars);
  constexpr int B_S = 2 * XS_MAX_S, B_X = B_S + 2 * XS_MAX_NSTG, B_A = B_X + 2 * XS_MAX_KB;
  auto dfull = [&](int s) { return bar0 + 8u * s; };
  auto dempty = [&](int s) { return bar0 + 8u * (XS_MAX_S + s); };
  auto sfull = [&](int s) { return bar0 + 8u * (B_S + s); };
  auto sempty = [&](int s) { return bar0 + 8u * (B_S + XS_MAX_NSTG + s); };
  auto xfull = [&](int k) { return bar0 + 8u * (B_X + k); };
  auto xempty = [&](int k) { return bar0 + 8u * (B_X + XS_MAX_KB + k); };
  auto accf = [&](int b) { return bar0 + 8u * (B_A + b); };
  auto acce = [&](int b) { return bar0 + 8u * (B_A + 2 + b); };

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(dfull(s), 1);   // the TMA thread's expect_tx arrival (and the bytes)
      mbar_init(dempty(s), 1);  // tcgen05.commit
    }
    for (int s = 0; s < NSTG; ++s) {
      mbar_init(sfull(s), 1);               // the X TMA thread (and the bytes)
      mbar_init(sempty(s), XS_CONV_WARPS);  // every converter warp has read it
    }
    for (int k = 0; k < kblocks; ++k) {
      mbar_init(xfull(k), XS_CONV_WARPS);  // every converter warp has written it
      mbar_init(xempty(k), 1);             // tcgen05.commit after the group's last atom tile
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf(b), 1);  // tcgen05.commit
      mbar_init(acce(b), XS_EPI_WARPS);  // every epilogue warp
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp < XS_CONV_WARPS) {
    // ---- converter: staging (fp32) -> the NP resident pieces
    int jt = 0;
    int64_t g = 0;  // staging buffers consumed
    bool ok = true;
    for (int64_t u0 = blockIdx.x; u0 < units && ok; u0 += gridDim.x, ++jt) {
      for (int h = 0; h < halves; ++h, ++g) {
        const int kb = h >> 1;
        const int s = (int)(g % NSTG);
        const uint32_t round = (uint32_t)(g / NSTG);
        // every lane waits; the warp goes on only if all of them saw the phase
        if (*abort_flag ||
            ((h & 1) == 0 &&
             !__all_sync(kFull, mbar_wait(xempty(kb), ((uint32_t)jt & 1u) ^ 1u))) ||
            !__all_sync(kFull, mbar_wait(sfull(s), round & 1u))) {
          ok = false;
          break;
        }
        const uint8_t* src = sring + (size_t)s * STG;
        uint8_t* xk = xres + (size_t)kb * NP * XPIECE;
        for (int u = threadIdx.x; u < UNITS; u += XS_CONV_THREADS) {
          const int row = u >> 2, c = u & 3;
          const float4 a = *reinterpret_cast<const float4*>(src + row * 128 + c * 32);
          const float4 b = *reinterpret_cast<const float4*>(src + row * 128 + c * 32 + 16);
          const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
          __align__(16) __nv_bfloat16 p[NP][8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            float r = v[e];
#pragma unroll
            for (int w = 0; w < NP; ++w) {
              p[w][e] = __float2bfloat16_rn(r);
              r -= __bfloat162float(p[w][e]);
            }
          }
          const int ch = (h & 1) * 4 + c;
          const uint32_t off = (uint32_t)row * 128u + ((uint32_t)(ch ^ (row & 7)) << 4);
#pragma unroll
          for (int w = 0; w < NP; ++w)
            *reinterpret_cast<uint4*>(xk + (size_t)w * XPIECE + off) =
                *reinterpret_cast<const uint4*>(p[w]);
        }
        // make the generic-proxy writes visible to the tensor cores, then
        // release the staging buffer (and, with its second half, the k-block)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(sempty(s));
          if (h & 1) mbar_arrive(xfull(kb));
        }
      }
    }
    if (!ok) *abort_flag = 1;
  } else if (warp < XS_CONV_WARPS + XS_EPI_WARPS) {
    // ---- epilogue: TMEM -> registers -> C (column-major, atoms contiguous)
    const int wl = warp & 3;  // TMEM lanes 32 wl .. 32 wl + 31
    // columns [c_lo, c_hi) of the tile: the two warps of a lane quarter split them
    constexpr int HALF = BN / 2 < 16 ? 16 : BN / 2;
    const int c_lo = ((warp - XS_CONV_WARPS) >> 2) * HALF;
    const int c_hi = c_lo + HALF < BN ? c_lo + HALF : BN;
    int it = 0;
    bool ok = true;
    for (int64_t u0 = blockIdx.x; u0 < units && ok; u0 += gridDim.x) {
      const int64_t n0 = (u0 / groups) * BN;
      const int mt0 = (int)(u0 % groups) * per_group;
      const int mt1 = min(m_tiles, mt0 + per_group);
      for (int mt = mt0; mt < mt1; ++mt, ++it) {
        const int b = it & 1;
        if (*abort_flag || !__all_sync(kFull, mbar_wait(accf(b), (uint32_t)(it >> 1) & 1u))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = mt * TC_BM + wl * 32 + lane;
        const uint32_t tl = tmem + ((uint32_t)(wl * 32) << 16) + (uint32_t)(b * 2 * BN);
#pragma unroll 1
        for (int c0 = c_lo; c0 < c_hi; c0 += 16) {
          uint32_t v[16], w[16];
          tmem_ld16(tl + (uint32_t)c0, v);
          tmem_ld16(tl + (uint32_t)(BN + c0), w);
          const int64_t col0 = n0 + c0;
          if (row < rows_out) {
            float* dst = C + (size_t)col0 * ldc + row;
            const int cmax = n - col0 < 16 ? (int)(n - col0) : 16;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              if (j < cmax) *dst = __uint_as_float(v[j]) + __uint_as_float(w[j]);
              dst += ldc;
            }
          }
        }
        // the accumulator may take the next tile
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(acce(b));
      }
    }
    if (!ok) *abort_flag = 1;
  } else if (warp == XS_CONV_WARPS + XS_EPI_WARPS) {
    // ---- TMA producer of the pieces of D
    if (lane == 0) {
      const CUtensorMap* maps[3] = {&mD0, &mD1, &mD2};
      int64_t g = 0, issued = 0;
      bool ok = true;
      for (int64_t u0 = blockIdx.x; u0 < units && ok; u0 += gridDim.x) {
        const int mt0 = (int)(u0 % groups) * per_group;
        const int mt1 = min(m_tiles, mt0 + per_group);
        for (int mt = mt0; mt < mt1 && ok; ++mt) {
          for (int kb = 0; kb < kblocks; ++kb, ++g) {
            const int s = (int)(g % S);
            const uint32_t round = (uint32_t)(g / S);
            if (*abort_flag || !mbar_wait(dempty(s), (round & 1u) ^ 1u)) { ok = false; break; }
            const uint32_t st = smem_u32(dring + (size_t)s * STAGE);
            mbar_expect_tx(dfull(s), STAGE);
#pragma unroll
            for (int w = 0; w < NP; ++w)
              tma_load_2d(st + w * XS_D_TILE, maps[w], dfull(s), kb * TC_BK, mt * TC_BM);
            issued = g + 1;
          }
        }
      }
      if (!ok) {
        *abort_flag = 1;
        // the copies of the last stages must land before the CTA may exit
        for (int64_t k = issued - S < 0 ? 0 : issued - S; k < issued; ++k)
          mbar_wait(dfull((int)(k % S)), (uint32_t)(k / S) & 1u);
      }
    }
  } else if (warp == XS_CONV_WARPS + XS_EPI_WARPS + 2) {
    // ---- TMA producer of the fp32 signals (half a k-block per buffer)
    if (lane == 0) {
      int64_t g = 0, issued = 0;
      bool ok = true;
      for (int64_t u0 = blockIdx.x; u0 < units && ok; u0 += gridDim.x) {
        const int y = (int)((u0 / groups) * BN);
        for (int h = 0; h < halves; ++h, ++g) {
          const int s = (int)(g % NSTG);
          const uint32_t round = (uint32_t)(g / NSTG);
          if (*abort_flag || !mbar_wait(sempty(s), (round & 1u) ^ 1u)) { ok = false; break; }
          mbar_expect_tx(sfull(s), STG);
          tma_load_2d(smem_u32(sring + (size_t)s * STG), &mX, sfull(s), h * 32, y);
          issued = g + 1;
        }
      }
      if (!ok) {
        *abort_flag = 1;
        for (int64_t k = issued - NSTG < 0 ? 0 : issued - NSTG; k < issued; ++k)
          mbar_wait(sfull((int)(k % NSTG)), (uint32_t)(k / NSTG) & 1u);
      }
    }
  } else {
    // ---- MMA issuer
    if (lane == 0) {
      int64_t g = 0;
      int it = 0, jt = 0;
      bool any = false, ok = true;
      for (int64_t u0 = blockIdx.x; u0 < units && ok; u0 += gridDim.x, ++jt) {
        const int mt0 = (int)(u0 % groups) * per_group;
        const int mt1 = min(m_tiles, mt0 + per_group);
        for (int mt = mt0; mt < mt1 && ok; ++mt, ++it) {
          const int b = it & 1;
          if (*abort_flag || !mbar_wait(acce(b), ((uint32_t)(it >> 1) & 1u) ^ 1u)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t acc = tmem + (uint32_t)(b * 2 * BN), acc2 = acc + BN;
          for (int kb = 0; kb < kblocks; ++kb, ++g) {
            const int s = (int)(g % S);
            const uint32_t round = (uint32_t)(g / S);
            if (*abort_flag || !mbar_wait(dfull(s), round & 1u) ||
                (mt == mt0 && !mbar_wait(xfull(kb), (uint32_t)jt & 1u))) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // descriptors of the pieces (the k-th 16-wide step adds 32 bytes,
            // 2 in the descriptor's 16-byte address field, which cannot carry
            // out of its 14 bits below 256 KB of shared memory)
            const uint64_t da = sw128_desc(smem_u32(dring + (size_t)s * STAGE));
            const uint64_t xa = sw128_desc(smem_u32(xres + (size_t)kb * NP * XPIECE));
            constexpr uint64_t DP = XS_D_TILE >> 4, XP = XPIECE >> 4;
            const uint32_t first = kb > 0 ? 1u : 0u;
#pragma unroll
            for (int k = 0; k < TC_BK / 16; ++k) {
              const uint64_t o = 2u * k;
              const uint32_t acc_in = k > 0 ? 1u : first;
              // (D piece, X piece): the leading product, then the corrections
              umma_bf16_n<BN>(acc, da + o, xa + o, acc_in);
              umma_bf16_n<BN>(acc2, da + o, xa + XP + o, acc_in);
              umma_bf16_n<BN>(acc2, da + DP + o, xa + o, 1u);
              if constexpr (NP == 3) {
                umma_bf16_n<BN>(acc2, da + o, xa + 2 * XP + o, 1u);
                umma_bf16_n<BN>(acc2, da + 2 * DP + o, xa + o, 1u);
                umma_bf16_n<BN>(acc2, da + DP + o, xa + XP + o, 1u);
              }
            }
            umma_commit(dempty(s));                      // the D stage is free once read
            if (mt == mt1 - 1) umma_commit(xempty(kb));  // and so is the k-block of X
            any = true;
          }
          if (!ok) break;
          umma_commit(accf(b));  // the tile's accumulator is complete
        }
      }
      if (!ok) {
        *abort_flag = 1;
        if (any) {
          // every issued MMA has finished before TMEM is freed: a last commit
          // arrives on an accumulator barrier once all earlier ones are done
          umma_commit(accf(it & 1));
          mbar_wait(accf(it & 1), (uint32_t)(it >> 1) & 1u);
        }
      }
    }
  }
  __syncwarp();
  if (*abort_flag && threadIdx.x == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
}

// x (rows x cols, ld ldx, fp32) -> hi, lo (rows_pad x cols, bf16), zero rows
// beyond `rows`.  One thread converts 8 consecutive rows of a column (two
// 16-byte loads when the column is 16-byte aligned, two 16-byte stores).
__global__ void bf16_split_kernel(const float* __restrict__ x, int rows, int64_t ldx, int64_t cols,
                                  int rows_pad, bool vec, __nv_bfloat16* __restrict__ hi,
                                  __nv_bfloat16* __restrict__ lo, __nv_bfloat16* __restrict__ lo3) {
  const int groups = rows_pad >> 3;
  const int64_t total = cols * groups;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total;
       gid += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = gid / groups;
    const int r0 = (int)(gid - c * groups) << 3;
    const float* src = x + (size_t)c * ldx + r0;
    float v[8];
    if (vec && r0 + 8 <= rows) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(src));
      const float4 b = __ldg(reinterpret_cast<const float4*>(src + 4));
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
      v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = r0 + k < rows ? src[k] : 0.f;
    }
    __align__(16) __nv_bfloat16 h[8], l[8], l3[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      h[k] = __float2bfloat16_rn(v[k]);
      const float r = v[k] - __bfloat162float(h[k]);
      l[k] = __float2bfloat16_rn(r);
      l3[k] = __float2bfloat16_rn(r - __bfloat162float(l[k]));
    }
    const size_t o = (size_t)c * rows_pad + r0;
    *reinterpret_cast<uint4*>(hi + o) = *reinterpret_cast<const uint4*>(h);
    *reinterpret_cast<uint4*>(lo + o) = *reinterpret_cast<const uint4*>(l);
    if (lo3) *reinterpret_cast<uint4*>(lo3 + o) = *reinterpret_cast<const uint4*>(l3);
  }
}

// ---------------------------------------------------------------------------
// host side
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static bool load_encode() {
  if (g_encode) return true;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return false;
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return true;
}

// 2-D bf16 tensor of `outer` rows of `inner` contiguous elements; box of
// 64 x box_rows with 128-byte swizzle, zero fill out of range.
static bool make_map(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer,
                     uint32_t box_rows) {
  if (((uintptr_t)base & 15u) != 0 || (inner * 2) % 16 != 0) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * 2};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tc_gemm_available() { return load_encode(); }

int tc_pad_m(int m) { return ((m + TC_BK - 1) / TC_BK) * TC_BK; }

cudaError_t launch_bf16_split(const float* x, int rows, int64_t ldx, int64_t cols, int rows_pad,
                              void* hi, void* lo, cudaStream_t st, void* lo3) {
  if (rows_pad % 8 != 0 || ((uintptr_t)hi & 15u) || ((uintptr_t)lo & 15u) ||
      ((uintptr_t)lo3 & 15u))
    return cudaErrorInvalidValue;
  const int64_t tot = (int64_t)(rows_pad / 8) * cols;
  if (tot <= 0) return cudaSuccess;
  const bool vec = (ldx % 4 == 0) && (((uintptr_t)x & 15u) == 0);
  const int64_t blocks = std::min<int64_t>((tot + 255) / 256, (int64_t)148 * 32);
  bf16_split_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, rows, ldx, cols, rows_pad, vec,
                                                      reinterpret_cast<__nv_bfloat16*>(hi),
                                                      reinterpret_cast<__nv_bfloat16*>(lo),
                                                      reinterpret_cast<__nv_bfloat16*>(lo3));
  return cudaGetLastError();
}

cudaError_t launch_tc_corr(const void* Dhi, const void* Dlo, int K, const void* Xhi,
                           const void* Xlo, int64_t n, int m_pad, int nterms, float* C, int ldc,
                           int rows_out, int* err, cudaStream_t st) {
  if (n <= 0 || K <= 0) return cudaSuccess;
  if (!load_encode()) return cudaErrorNotSupported;
  const int Kp = ((K + TC_BM - 1) / TC_BM) * TC_BM;
  if (m_pad % TC_BK != 0 || nterms < 1 || nterms > 3 || ldc < rows_out)
    return cudaErrorInvalidValue;
  if (rows_out > Kp) {  // rows past the last tile (a wider padding of K) are zero
    cudaError_t e = cudaMemset2DAsync(C + Kp, (size_t)ldc * sizeof(float), 0,
                                      (size_t)(rows_out - Kp) * sizeof(float), (size_t)n, st);
    if (e != cudaSuccess) return e;
    rows_out = Kp;
  }
  CUtensorMap mAh, mAl, mBh, mBl;
  if (!make_map(&mAh, Dhi, m_pad, K, TC_BM) || !make_map(&mAl, Dlo, m_pad, K, TC_BM) ||
      !make_map(&mBh, Xhi, m_pad, n, TC_BN) || !make_map(&mBl, Xlo, m_pad, n, TC_BN))
    return cudaErrorInvalidValue;
  const int64_t gy = (n + TC_BN - 1) / TC_BN;
  if (gy > 65535) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(tc_corr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)TC_SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid(Kp / TC_BM, (unsigned)gy);
  // terms (hi, hi), (hi, lo), (lo, hi): pieces (A, B) = (0, 0), (0, 1), (1, 0)
  const uint32_t code = 0u | (4u << 4) | (1u << 8);
  tc_corr_kernel<<<grid, 128, TC_SMEM, st>>>(mAh, mAl, mAl, mBh, mBl, mBl, code, C, ldc, rows_out,
                                              n, m_pad, nterms, err);
  return cudaGetLastError();
}

// G = D^T D (+ ridge on the diagonal) from the three-piece BF16 split of D
// (d = hi + mid + lo, 24 significant bits as in FP32): the X-stationary
// kernel with D itself as the signals (six products, the leading one in its
// own accumulator), then the upper triangle mirrored (as
// Matrix::fillSymmetric does after syrk) with the ridge added and the
// padding zeroed.  Where that kernel does not apply (m beyond its resident
// tile, or D not 16-byte aligned with m a multiple of 4) the Gram is the
// FP32 CUDA-core product.
cudaError_t launch_gram_tc(const void* Dhi, const void* Dmid, const void* Dlo3, const float* D,
                           int m, int m_pad, int K, int Kp, float ridge, float* G, int* err,
                           cudaStream_t st) {
  if (K <= 0) return cudaSuccess;
  const void* dp[3] = {Dhi, Dmid, Dlo3};
  cudaError_t e = launch_tc_corr_xs(dp, 3, K, D, m, m, K, m_pad, G, Kp, Kp, err, st);
  if (e == cudaErrorNotSupported) return launch_gram<float>(D, m, K, Kp, ridge, G, st);
  if (e != cudaSuccess) return e;
  return launch_symmetrize<float>(G, K, Kp, ridge, st);
}

cudaError_t launch_tc_corr_fused(const void* Dhi, const void* Dlo, int K, const float* X,
                                 int64_t ldx, int m, int64_t n, int m_pad, float* C, int ldc,
                                 int rows_out, int* err, cudaStream_t st) {
  if (n <= 0 || K <= 0) return cudaSuccess;
  if (!load_encode()) return cudaErrorNotSupported;
  const int Kp = ((K + TC_BM - 1) / TC_BM) * TC_BM;
  if (m <= 0 || m_pad % TC_BK != 0 || m > m_pad || ldx < m || ldc < rows_out || !X || !C)
    return cudaErrorInvalidValue;
  if (rows_out > Kp) {  // rows past the last tile (a wider padding of K) are zero
    cudaError_t e = cudaMemset2DAsync(C + Kp, (size_t)ldc * sizeof(float), 0,
                                      (size_t)(rows_out - Kp) * sizeof(float), (size_t)n, st);
    if (e != cudaSuccess) return e;
    rows_out = Kp;
  }
  CUtensorMap mAh, mAl;
  if (!make_map(&mAh, Dhi, m_pad, K, TC_BM) || !make_map(&mAl, Dlo, m_pad, K, TC_BM))
    return cudaErrorInvalidValue;
  const int m_tiles = Kp / TC_BM;
  const int64_t n_tiles = (n + TC_BN - 1) / TC_BN;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int64_t tiles = (int64_t)m_tiles * n_tiles;
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, sms > 0 ? sms : 1);
  const bool vec = (ldx % 4 == 0) && (((uintptr_t)X & 15u) == 0);
  auto k = vec ? tc_corr_fused_kernel<true> : tc_corr_fused_kernel<false>;
  e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T2_SMEM);
  if (e != cudaSuccess) return e;
  k<<<grid, T2_THREADS, T2_SMEM, st>>>(mAh, mAl, X, ldx, m, n, m_pad, C, ldc, rows_out, m_tiles,
                                         n_tiles, err);
  return cudaGetLastError();
}


// 2-D fp32 tensor of `outer` rows of `inner` elements (row stride ld
// elements); box of box_inner x box_rows, no swizzle, zero fill out of range.
static bool make_map_f32(CUtensorMap* mp, const float* base, uint64_t inner, uint64_t outer,
                         uint64_t ld, uint32_t box_inner, uint32_t box_rows) {
  if (((uintptr_t)base & 15u) != 0 || (ld * 4) % 16 != 0) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld * 4};
  cuuint32_t box[2] = {box_inner, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// A launch shape of the X-stationary kernel: signals per tile, stages of the
// D ring, staging buffers of half a k-block.
struct XsShape { int bn, s, nstg; };

// Wide signal tiles first (fewer passes over D per signal), each with the
// deepest rings that fit in shared memory.
static bool xs_pick(int np, int kblocks, XsShape* out) {
  static const XsShape prefs[] = {{128, 3, 4}, {128, 3, 2}, {128, 2, 2}, {64, 3, 4}, {64, 2, 2},
                                  {32, 3, 4},  {32, 2, 2},  {16, 3, 4},  {16, 2, 2}};
  if (kblocks > XS_MAX_KB) return false;
  for (const XsShape& p : prefs)
    if (xs_smem_bytes(np, p.bn, kblocks, p.s, p.nstg) <= XS_SMEM_LIMIT) {
      *out = p;
      return true;
    }
  return false;
}

template <int NP, int BN>
static cudaError_t xs_launch(const CUtensorMap (&maps)[3], const CUtensorMap& mx, int64_t n,
                             int m_pad, float* C, int ldc, int rows_out, int m_tiles, int s,
                             int nstg, int sms, int* err, cudaStream_t st) {
  const int kblocks = m_pad / TC_BK;
  const size_t smem = xs_smem_bytes(NP, BN, kblocks, s, nstg);
  const int64_t n_tiles = (n + BN - 1) / BN;
  // spread the atom tiles over groups while the signal tiles leave SMs idle
  int groups = (int)std::max<int64_t>(1, std::min<int64_t>(m_tiles, sms / n_tiles));
  const int per_group = (m_tiles + groups - 1) / groups;
  groups = (m_tiles + per_group - 1) / per_group;  // no empty group
  const int64_t units = n_tiles * groups;
  const unsigned grid = (unsigned)std::min<int64_t>(units, sms);
  auto k = tc_corr_xs_kernel<NP, BN>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, XS_THREADS, smem, st>>>(maps[0], maps[1], maps[2], mx, n, m_pad, C, ldc, rows_out,
                                     m_tiles, groups, per_group, units, s, nstg, err);
  return cudaGetLastError();
}

static cudaError_t launch_tc_corr_xs_shape(const void* const* Dpieces, int np, int K,
                                           const float* X, int64_t ldx, int m, int64_t n,
                                           int m_pad, float* C, int ldc, int rows_out, int* err,
                                           const XsShape& shp, cudaStream_t st) {
  const int Kp = ((K + TC_BM - 1) / TC_BM) * TC_BM;
  CUtensorMap maps[3], mx;
  for (int w = 0; w < np; ++w)
    if (!make_map(&maps[w], Dpieces[w], m_pad, K, TC_BM)) return cudaErrorInvalidValue;
  if (np == 2) maps[2] = maps[1];
  if (!make_map_f32(&mx, X, (uint64_t)m, (uint64_t)n, (uint64_t)ldx, 32, (uint32_t)shp.bn))
    return cudaErrorNotSupported;
  if (rows_out > Kp) {  // rows past the last tile (a wider padding of K) are zero
    cudaError_t e = cudaMemset2DAsync(C + Kp, (size_t)ldc * sizeof(float), 0,
                                      (size_t)(rows_out - Kp) * sizeof(float), (size_t)n, st);
    if (e != cudaSuccess) return e;
    rows_out = Kp;
  }
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (sms <= 0) sms = 1;
  const int m_tiles = Kp / TC_BM;
#define SC_XS(NP_, BN_)                                                                     \
  if (np == NP_ && shp.bn == BN_)                                                           \
    return xs_launch<NP_, BN_>(maps, mx, n, m_pad, C, ldc, rows_out, m_tiles, shp.s, shp.nstg, \
                               sms, err, st);
  SC_XS(2, 128) SC_XS(2, 64) SC_XS(2, 32) SC_XS(2, 16)
  SC_XS(3, 128) SC_XS(3, 64) SC_XS(3, 32) SC_XS(3, 16)
#undef SC_XS
  return cudaErrorInvalidValue;
}

// C = D^T X from the np pieces of D (np = 2: hi, lo; 3: hi, mid, lo) and
// fp32 X, split in the kernel; cudaErrorNotSupported when a signal tile's
// pieces do not fit in shared memory (m_pad * np * 2 * 16 bytes at the
// smallest tile) or X is not 16-byte aligned with a multiple-of-4 leading
// dimension, for the caller to take the streaming two-piece form.
cudaError_t launch_tc_corr_xs(const void* const* Dpieces, int np, int K, const float* X,
                              int64_t ldx, int m, int64_t n, int m_pad, float* C, int ldc,
                              int rows_out, int* err, cudaStream_t st) {
  if (n <= 0 || K <= 0) return cudaSuccess;
  if (np != 2 && np != 3) return cudaErrorInvalidValue;
  if (!load_encode()) return cudaErrorNotSupported;
  if (m <= 0 || m_pad % TC_BK != 0 || m > m_pad || ldx < m || ldc < rows_out || !X || !C)
    return cudaErrorInvalidValue;
  XsShape shp;
  if (!xs_pick(np, m_pad / TC_BK, &shp)) return cudaErrorNotSupported;
  return launch_tc_corr_xs_shape(Dpieces, np, K, X, ldx, m, n, m_pad, C, ldc, rows_out, err, shp,
                                 st);
}

}  // namespace sc
