// Combining the exact level sums of a split product in FP64, and cutting
// values into balanced base-256 digits.
#pragma once

#include "ptx.cuh"

namespace ef {

// The S levels of one TMEM column, combined: Σ_l L_l 2^{-8(l+2)}, in groups
// of three summed exactly in int64 (|L_l| < 2^31, so three of them shifted
// by 8 bits fit in 2^48) and added from the smallest group up.
template <int S, int N>
__device__ __forceinline__ double combine_levels(const int32_t (&L)[S][N], int i) {
  double v = 0.0;
#pragma unroll
  for (int g = (S - 1) / 3; g >= 0; g--) {
    long long part = 0;
    const int l0 = 3 * g, l1 = (3 * g + 3 < S ? 3 * g + 3 : S);
#pragma unroll
    for (int l = l0; l < l1; l++) part = part * 256 + (long long)L[l][i];
    v += (double)part * ptx::pow2(-8 * (l1 + 1));
  }
  return v;
}

// The same for levels small enough that two of them, one shifted by 8 bits,
// fit in int32 (|L_l| < 2^23): pairs combined in int32, then converted.
template <int S, int N>
__device__ __forceinline__ double combine_levels_small(const int32_t (&L)[S][N], int i) {
  double v = (S & 1) ? (double)L[S - 1][i] * ptx::pow2(-8 * (S + 1)) : 0.0;
#pragma unroll
  for (int p = S / 2 - 1; p >= 0; p--)
    v = fma((double)(L[2 * p][i] * 256 + L[2 * p + 1][i]), ptx::pow2(-8 * (2 * p + 3)), v);
  return v;
}

// The exponent e with |x| < 2^(e-2) for the largest magnitude x of a row
// (0 for a row of zeros): digits of x / 2^e then start below 64.
__device__ __forceinline__ int slice_exponent(double largest) {
  int e = 0;
  if (largest > 0.0) {
    frexp(largest, &e);
    e += 2;
  }
  return e;
}

// Cuts X (|X| < 2^(8S-2), S <= 7) into S balanced base-256 digits, most
// significant first, packing digit s of value i into byte (i & 3) of
// word[s][i >> 2], in 32-bit arithmetic: the low 24 bits give the last three
// digits, and their carry joins the high part.
template <int S, int W>
__device__ __forceinline__ void cut_digits32(long long X, int i, uint32_t (&word)[S][W]) {
  int lo = (int)(X & 0xFFFFFF);
  int hi = (int)(X >> 24);
#pragma unroll
  for (int s = S - 1; s >= S - 3; s--) {
    const int d = ((lo + 128) & 255) - 128;
    word[s][i >> 2] |= ((uint32_t)(d & 255)) << (8 * (i & 3));
    lo = (lo - d) >> 8;
  }
  hi += lo;
#pragma unroll
  for (int s = S - 4; s >= 0; s--) {
    const int d = ((hi + 128) & 255) - 128;
    word[s][i >> 2] |= ((uint32_t)(d & 255)) << (8 * (i & 3));
    hi = (hi - d) >> 8;
  }
}

}  // namespace ef
