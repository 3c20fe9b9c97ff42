// Attention-shaped pipelines on the tensor cores: the mask of a pipeline's
// conditions, and the split forward pass over placed matrices.
#pragma once

#include <vector>

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace ef {

constexpr int kMaxMask = 8;

// The conditions between the one X and the one J dimension of a pipeline,
// each as `x <cmp> j + off`, and the positions per batch along X and J.
struct Mask {
  int n = 0;
  int cmp[kMaxMask] = {};
  int64_t off[kMaxMask] = {};
  int64_t lnx = 1, lnj = 0;
  // Ragged batches (arrays of one length per batch, null: every batch
  // full; device memory in kernels, host memory on the host): batch w's X
  // positions at or past xlen[w] join nothing, and its J positions at or
  // past jlen[w] are joined by none.
  const int64_t* xlen = nullptr;
  const int64_t* jlen = nullptr;
};

// allowed(x) (fused.rs:350-368): the half-open J interval that X position
// x may join, the intersection of each condition's, in 128-bit integers,
// clamped to x's batch (and to its lengths when ragged).
__host__ __device__ inline void allowed(const Mask& m, int64_t x, int64_t& lo_out, int64_t& hi_out) {
  const int64_t w = x / m.lnx;
  const int64_t group_start = w * m.lnj;
  const __int128 xx = x % m.lnx;
  __int128 n = m.lnj;
  if (m.jlen) n = m.jlen[w] < m.lnj ? m.jlen[w] : m.lnj;
  if (m.xlen && xx >= m.xlen[w]) n = 0;
  __int128 lo = 0, hi = n;
  for (int i = 0; i < m.n; i++) {
    const __int128 bound = xx - (__int128)m.off[i];
    switch (m.cmp[i]) {
      case 3: if (bound + 1 < hi) hi = bound + 1; break;  // x >= j + c
      case 2: if (bound < hi) hi = bound; break;          // x >  j + c
      case 1: if (bound > lo) lo = bound; break;          // x <= j + c
      default: if (bound + 1 > lo) lo = bound + 1; break; // x <  j + c
    }
  }
  const __int128 l = lo < 0 ? 0 : (lo > n ? n : lo);
  __int128 h = hi > lo ? hi : lo;
  h = h < 0 ? 0 : (h > n ? n : h);
  lo_out = group_start + (int64_t)l;
  hi_out = group_start + (int64_t)h;
}

// Per-query key ranges [lo, hi) (2·queries values, the same in every batch)
// as conditions: true when every range is [x + a, x + b) clamped to
// [0, keys) for constants a and b, as a pipeline's conditions give.
bool ranges_as_mask(const int64_t* ranges, int64_t queries, int64_t keys, Mask& m);

// Each row's largest and smallest nonzero value magnitude over its allowed
// keys (the bounds of Bounds::hold, fused.rs:1058-1086): block_extrema takes
// the extrema of blocks of 64 keys, row_value_bounds those of each row's
// allowed range.
__global__ void block_extrema(int64_t nj, const double* __restrict__ largest, const double* __restrict__ smallest,
                              double* __restrict__ bmax, double* __restrict__ bmin);
__global__ void row_value_bounds(int64_t nx, Mask m, const double* __restrict__ largest,
                                 const double* __restrict__ smallest, const double* __restrict__ bmax,
                                 const double* __restrict__ bmin, double* __restrict__ rl, double* __restrict__ rs);

// A softmax-weighted average over placed matrices, batch by batch:
// q [w][x][e], k [w][j][e], v [w][j][y] for w < batches, x < lnx, j < lnj,
// e < ne, y < ny; out [w·lnx + x][y] = Σ_j exp(s_xj − m_x) v_jy / z_x over the
// allowed j, with s_xj = scale(q_x · k_j), m_x the row's largest score and
// z_x its sum of weights; lse (if given) = m_x + ln z_x. `largest` and
// `smallest` hold each J position's largest and smallest nonzero magnitude
// of v (for the reference's underflow guard).
struct AttentionProblem {
  const double* q = nullptr;
  const double* k = nullptr;
  const double* v = nullptr;
  int64_t batches = 0, lnx = 0, lnj = 0, ne = 0, ny = 0;
  Mask mask;
  int scale_kind = 0;  // 0 one, 1 times c, 2 over c
  double scale_c = 1.0;
  const double* largest = nullptr;
  const double* smallest = nullptr;
  double* out = nullptr;
  double* lse = nullptr;
  // Ragged batches: host copies of the mask's lengths (empty: full).
  std::vector<int64_t> xlen_host, jlen_host;
};

enum AttentionOutcome { ATTENTION_DONE = 0, ATTENTION_INELIGIBLE = 1, ATTENTION_GUARDED = 2 };

// The split forward pass: q·k and w·v as int8 digit products on the tensor
// cores (S slices each, level sums exact in TMEM), the online softmax in
// FP64. INELIGIBLE when an operand isn't finite or the scores could
// overflow (nothing written); GUARDED when the reference's overflow or
// underflow guard fires on a row (the pipeline declines).
AttentionOutcome attention_split(Context& ctx, const AttentionProblem& p, int slices, cudaStream_t stream);

// The FP64 form on the FP64 tensor pipe (mma.sync f64): product scores, the
// online softmax and the weighted sums in FP64, with the reference's guards.
// INELIGIBLE (nothing written) when q or k isn't finite, a score could
// overflow, or d > 128; the caller's value statistics (largest, smallest)
// must be set and v finite.
AttentionOutcome attention_f64_mma(Context& ctx, const AttentionProblem& p, cudaStream_t stream);

// Whether EINFOLD_FP64_TILES=1 asks for the CUDA cores' FP64 tile kernels.
bool fp64_tiles_requested();

// The forward pass over placed matrices: the split form when `precision`
// is 0 and it applies, else the FP64 form on the FP64 tensor pipe where it
// applies, else the FP64 tile kernel (fused.rs's tile, in FP64 on the CUDA
// cores, for non-finite operands). Computes each J position's value
// statistics itself.
AttentionOutcome attention_forward(Context& ctx, AttentionProblem p, int precision, int slices, cudaStream_t stream);

// The gradients of the forward pass's out, from its saved lse:
// d_v = Pᵀ·d_out, d_k = scale·dSᵀ·q, d_q = scale·dS·k, with
// P = exp(s - lse) over the allowed pairs, dS = P∘(d_out·vᵀ - D),
// D = rowsum(d_out∘out).
struct AttentionGradients {
  AttentionProblem f;  // q, k, v, shapes, mask, scale
  const double* out = nullptr;
  const double* lse = nullptr;
  const double* d_out = nullptr;
  double* d_q = nullptr;
  double* d_k = nullptr;
  double* d_v = nullptr;
  // The caller's budget (null: none): the split backward asks it for the
  // export buffers, a smaller plan at each refusal, and gives them back at
  // the end of the call; with nothing granted it recomputes the scores.
  Budget* budget = nullptr;
};
// The FP64 backward on the FP64 tensor pipe (d, dv <= 64, scale one or times
// c; false, nothing written, otherwise): d_k and d_v from a kernel with keys
// as rows (`keys_mask` the transposed mask), d_q from one with queries as
// rows, scores recomputed from lse, D = rowsum(d_out∘out) given.
bool backward_f64_mma(Context& ctx, const AttentionGradients& g, const Mask& keys_mask, const double* dd,
                      cudaStream_t stream);
void attention_backward(Context& ctx, const AttentionGradients& g, int precision, cudaStream_t stream);

}  // namespace ef
