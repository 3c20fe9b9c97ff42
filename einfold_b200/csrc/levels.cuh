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

// x as a double, exactly, with an add on the FP64 pipe rather than a
// conversion: the double whose high word is 0x43300000 and low word
// x + 2^31 is 2^52 + 2^31 + x.
__device__ __forceinline__ double i2d(int x) {
  return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}

// The same for levels small enough that two of them, one shifted by 8 bits,
// fit in int32 (|L_l| < 2^23): pairs combined in int32, then converted.
template <int S, int N>
__device__ __forceinline__ double combine_levels_small(const int32_t (&L)[S][N], int i) {
  double v = (S & 1) ? i2d(L[S - 1][i]) * ptx::pow2(-8 * (S + 1)) : 0.0;
#pragma unroll
  for (int p = S / 2 - 1; p >= 0; p--) v = fma(i2d(L[2 * p][i] * 256 + L[2 * p + 1][i]), ptx::pow2(-8 * (2 * p + 3)), v);
  return v;
}

// The S digit planes of four values already scaled to integers-to-be
// (|x| < 2^(8S-2), S <= 6), four columns a word: x rounds to the nearest
// integer W (ties to even, as llrint) by adding 1.5·2^52, and W's balanced
// base-256 digits d_s in [-128, 127] are the bytes of W + 0x80…80 with
// their top bits flipped (byte s of W + Σ 128·256^s is d_s + 128). planes[s]
// holds digit s (most significant first) of the four values, byte c for
// value c: the bytes the split product's digit planes hold.
template <int S>
__device__ __forceinline__ void digit_planes4(const double (&x)[4], uint32_t (&planes)[S]) {
  static_assert(S <= 6, "six digits or fewer fit the 48-bit window");
  constexpr long long kBias = 0x4338000000000000ll - 0x808080808080ll;
  uint32_t lo[4], hi[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const long long u = __double_as_longlong(x[c] + 6755399441055744.0) - kBias;  // 1.5·2^52
    lo[c] = (uint32_t)u;
    hi[c] = (uint32_t)(u >> 32);
  }
#pragma unroll
  for (int s = 0; s < S; s++) {
    const int b = S - 1 - s;  // byte of W holding digit s
    const uint32_t* h = b < 4 ? lo : hi;
    const uint32_t sel = (uint32_t)((b & 3) | (((b & 3) + 4) << 4));
    const uint32_t t01 = __byte_perm(h[0], h[1], sel), t23 = __byte_perm(h[2], h[3], sel);
    planes[s] = __byte_perm(t01, t23, 0x5410) ^ 0x80808080u;
  }
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

}  // namespace ef
