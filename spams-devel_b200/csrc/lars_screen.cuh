// Joining-step screen of the LARS-Lasso homotopy, shared by the warp- and
// CTA-per-signal kernels (lars.cu, lars_cta.cu).
//
// coreLARS2 (decomp/decomp.h:1797-1823) fills, for every atom j not in the
// active set,
//   work[j]     = (A_j < INF && A_j > -1) ? (DtR_j + C) / (1 + A_j) : INF   (INF when pos)
//   work[j + K] = (A_j < INF && A_j <  1) ? (C - DtR_j) / (1 - A_j) : INF
// and takes index = cblas_iamin(2K, work): the FIRST index of the smallest
// magnitude of the rounded quotients (linalg/cblas_alt_template.h:1094-1105);
// the step is work[index] (signed) and the next atom index % K.
//
// A lane owns the rows row0 + 128 v + e (v < NV, e < 4) and returns its best
// candidate (|value|, index, value); the caller reduces lanes (and warps) by
// (|value|, first index), which the reference's order makes exact.
//
// Double precision evaluates every admissible quotient with IEEE division
// and keeps the first index among equal rounded magnitudes, so the decision
// is the reference's in all cases, exact ties included.  Single precision
// submits one candidate per row, the smaller side (c <= C a picks the plus
// side), compared by cross multiplication in four independent chains and
// divided exactly once per lane; it agrees with the reference except where
// two candidates of one lane lie within rounding of each other.
#pragma once
#include "common.cuh"

namespace sc {

template <typename T> struct ScreenBest { T key; T val; int idx; };

// The atom of a joining index in [0, 2K) (index % K without the division);
// any other index (no candidate at all) maps to atom 0.
__device__ __forceinline__ int join_atom(int idx, int K) {
  const unsigned u = (unsigned)idx;
  return u < (unsigned)K ? idx : (u < 2u * (unsigned)K ? idx - K : 0);
}

// Reference-exact screen (used in double precision).
template <int NV>
__device__ __forceinline__ ScreenBest<double> lars_screen(const double (&A)[NV][4],
                                                         const double* __restrict__ dtr_row0,
                                                         int row0, uint32_t act, double C,
                                                         bool pos, int K) {
  const double INF = inf<double>();
  double bkey = INF, bval = INF;
  int bidx = 0x7fffffff;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const Vec4<double> d = ld4(dtr_row0 + v * 128);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if ((act >> (v * 4 + e)) & 1u) continue;  // active atoms and padding rows
      const int r = row0 + v * 128 + e;
      const double a = A[v][e], c = d.v[e];
      if (!pos && a < INF && a > -1.0) {
        const double q = (c + C) / (1.0 + a);
        const double k = fabs(q);
        if (k < bkey || (k == bkey && r < bidx)) { bkey = k; bval = q; bidx = r; }
      }
      if (a < INF && a < 1.0) {
        const double q = (C - c) / (1.0 - a);
        const double k = fabs(q);
        if (k < bkey || (k == bkey && r + K < bidx)) { bkey = k; bval = q; bidx = r + K; }
      }
    }
  }
  if (!(bkey < INF)) { bkey = INF; bval = INF; }  // NaN never wins
  return ScreenBest<double>{bkey, bval, bidx};
}

// Fast screen (single precision).
template <int NV>
__device__ __forceinline__ ScreenBest<float> lars_screen(const float (&A)[NV][4],
                                                        const float* __restrict__ dtr_row0,
                                                        int row0, uint32_t act, float C, bool pos,
                                                        int K) {
  const float INF = inf<float>();
  float cn[4], cd[4];
  int ci[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) { cn[e] = INF; cd[e] = 1.f; ci[e] = 0x7fffffff; }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const Vec4<float> d = ld4(dtr_row0 + v * 128);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = row0 + v * 128 + e;
      const bool active = (act >> (v * 4 + e)) & 1u;  // padding rows are marked active
      const float aa = A[v][e], c = d.v[e];
      const bool okp = !pos && aa > -1.f && aa < INF;  // (C + c)/(1 + a) admissible
      const bool okm = aa < 1.f;                       // (C - c)/(1 - a) admissible
      const bool plus = okp && (!okm || c <= C * aa);
      const float num = plus ? C + c : C - c;
      const float den = plus ? 1.f + aa : 1.f - aa;
      const int idx = plus ? r : r + K;
      const float lhs = fabsf(num) * cd[e], rhs = fabsf(cn[e]) * den;
      const bool take = !active && (okp || okm) && (lhs < rhs || (lhs == rhs && idx < ci[e]));
      cn[e] = take ? num : cn[e];
      cd[e] = take ? den : cd[e];
      ci[e] = take ? idx : ci[e];
    }
  }
#pragma unroll
  for (int h = 1; h < 4; h <<= 1) {
#pragma unroll
    for (int e = 0; e + h < 4; e += 2 * h) {
      const float lhs = fabsf(cn[e + h]) * cd[e], rhs = fabsf(cn[e]) * cd[e + h];
      if (lhs < rhs || (lhs == rhs && ci[e + h] < ci[e])) {
        cn[e] = cn[e + h]; cd[e] = cd[e + h]; ci[e] = ci[e + h];
      }
    }
  }
  float val = cn[0] / cd[0];
  float key = fabsf(val);
  if (!(key < INF)) { key = INF; val = INF; }  // NaN never wins
  return ScreenBest<float>{key, val, ci[0]};
}

}  // namespace sc
