// exp(x) in FP64 for the softmax weights, by Tang's table-driven method
// (P. T. P. Tang, "Table-driven implementation of the exponential function
// in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989), with a table of
// 64 entries: x = (64m + j)·ln2/64 + r, |r| <= ln2/128, and
// exp(x) = 2^m · 2^(j/64) · p(r), p the degree-5 Taylor polynomial of e^r
// (truncation below 4e-17 relative). The reduction splits ln2/64 into a
// 36-bit head, whose products with |64m + j| < 2^17 are exact, and a tail.
// Results are within 3 units in the last place of the exact value (2.17
// the largest error measured over 1.1e7 arguments on [-708, 709]);
// arguments below -708 (subnormal or zero results), above 709 and NaN go
// to the math library's exp.
#pragma once

#include <cstdint>

#include "ptx.cuh"

namespace ef {

constexpr double kLn2Over64Hi = 0x1.62e42fefa0000p-7;
constexpr double kLn2Over64Lo = 0x1.cf79abc9e3b3ap-46;
constexpr double k64OverLn2 = 92.33248261689366;

// The table 2^(j/64), j < 64, for the calling thread's device (computed in
// long double on the host and rounded once); kernels copy it to shared
// memory.
const double* exp_table(int device);

__device__ __forceinline__ double exp_tang(double x, const double* __restrict__ table) {
  if (!(x >= -708.0 && x <= 709.0)) return exp(x);
  // k = x·64/ln2 rounded to the nearest integer by adding 1.5·2^52 (one
  // rounding of the exact product), read from the sum's low word.
  const double t = fma(x, k64OverLn2, 6755399441055744.0);
  const double kf = t - 6755399441055744.0;
  const int k = __double2loint(t);
  double r = fma(-kf, kLn2Over64Hi, x);
  r = fma(-kf, kLn2Over64Lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return p * table[k & 63] * ptx::pow2(k >> 6);
}

// 2^shift · exp(x) for softmax weights (x <= 0 and 0 <= shift <= 64, or
// shift = 0), without the range test: x is clamped to [-708, 709], so the
// scaling stays a normal power of two. Below -708 the result (under 2^(shift-1021)) stands in for a weight
// that no digit of W = 2^shift · w keeps and that a sum of weights holding
// the row's heaviest one (2^shift) absorbs. A NaN argument gives a finite
// value, for callers that select another one for it.
__device__ __forceinline__ double exp_weight(double x, const double* __restrict__ table, int shift) {
  x = fmin(fmax(x, -708.0), 709.0);
  const double t = fma(x, k64OverLn2, 6755399441055744.0);
  const double kf = t - 6755399441055744.0;
  const int k = __double2loint(t);
  double r = fma(-kf, kLn2Over64Hi, x);
  r = fma(-kf, kLn2Over64Lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return p * table[k & 63] * ptx::pow2((k >> 6) + shift);
}

}  // namespace ef
