// The fused pipeline on the device (crates/einfold-kernels/src/fused.rs:151-1086).
//
// Host side: the reference's control logic, roles W/X/E/J/Y, the mask of
// conditions between the one X and the one J dimension, which columns the
// producer reads, the decline rules. Device side: keys and extents, the
// placement of each read column as a dense matrix with duplicate detection,
// each J position's value statistics, the tiles, and the output columns.
//
// Layout in HBM: each column q reads as q[x][e]; each column k reads as
// k[j][e] (e contiguous: the scores' K-major operands), the values v[j][y];
// the result out[x][y]. Batch keys W lead both X and J, so that a batch's
// positions are a contiguous range of each.
//
// The tile kernel computes, per 64-row X tile and 64-wide chunk of Y, what
// fused.rs:694-1019 computes per X tile: the J tiles of 64 between the
// first and last allowed J position of its rows, scores by a product or a
// row expression summed over E, weights by an online softmax shifted by
// the running maximum or by an expression of the score, the weighted sums,
// the normalisation, and every guard that sends the pipeline back to the
// host plan (overflows :1024-1028, Bounds::hold :1058-1086). A chunk of Y
// recomputes its tile's scores; each guard is a conjunction over outputs,
// so the chunks' flags OR to the whole row's.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <optional>

#include "attention.cuh"
#include "expr.cuh"
#include "fold.h"
#include "stage.cuh"

namespace ef {
namespace {

constexpr int XT = 64, JT = 64;  // fused.rs XT, JT: tiles visited count in these
constexpr int YC = 64;           // outputs per CTA along y
constexpr int kMaxSlots = 8;
constexpr int kThreads = 256;
constexpr int kNarrow = 8;       // value columns up to which a chunk sums by half-warp reductions

// The interpreter out of line, once per kind of call (a row expression
// over slots; a weight expression of the score).
template <int DEPTH>
__device__ __noinline__ double eval_slots(const ExprNode* __restrict__ nodes, int n, const double* slots) {
  return eval<DEPTH>(nodes, n, [slots](int k) { return slots[k]; });
}
template <int DEPTH>
__device__ __noinline__ double eval_score(const ExprNode* __restrict__ nodes, int n, double score) {
  return eval<DEPTH>(nodes, n, [score](int) { return score; });
}

enum : uint8_t { J_FINITE = 1, J_INFINITE = 2 };

// Expressions the tile kernel computes without the interpreter: the same
// operations in the same order, so the same bits.
enum ScoreShape : int {
  SCORE_INTERPRETED = 0,
  SCORE_NEG_SQUARED_DIFF = 1,  // -power(a - b, 2), a Gaussian kernel's exponent
};
enum WeightShape : int {
  WEIGHT_INTERPRETED = 0,
  WEIGHT_SIGMOID = 1,  // c1 / (c2 + exp(-s))
  WEIGHT_CAUCHY = 2,   // c1 / (c2 + s * s)
};

struct TileArgs {
  int64_t nx, ne, nj, ny;
  Mask mask;
  int weight_expr, scale_kind, shifted, normalizer;
  double scale_c;
  double wc1, wc2;  // the weight shape's constants
  const ExprNode* wnodes;
  int wn;
  int weight_shape;  // WeightShape: a weight expression computed without the interpreter
  int score_expr;
  int score_shape;   // ScoreShape, with the two slots it reads
  int shape_a, shape_b;
  const double* q;  // [x][e]
  const double* k;  // [j][e]
  const ExprNode* snodes;
  int sn, n_slots;
  const double* mats[kMaxSlots];
  int side[kMaxSlots];  // 0: [x][e], 1: [j][e]
  const double* v;      // [j][y]
  const uint8_t* jflag;
  const double* largest;
  const double* smallest;
  double* out;  // [x][y]
  double* lse;  // [x]: m + ln z of a normalised softmax row, or null
  unsigned long long* visited;
  unsigned* overflowed;
};

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Reductions over the 16 lanes of a half-warp (every lane of the warp calls).
__device__ __forceinline__ double half_max(double v) {
  for (int o = 8; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double half_min(double v) {
  for (int o = 8; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double half_sum(double v) {
  for (int o = 8; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ bool half_or(bool b) {
  int v = b;
  for (int o = 8; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v != 0;
}

struct RowState {
  double m[XT], z[XT], high[XT], light[XT], low[XT], rl[XT], rs[XT], resc[XT], lost[XT];
  long long terms[XT];
  int lo[XT], hi[XT];
  uint8_t sw[XT], sw_before[XT], pend[XT], spv[XT], check[XT];
};

constexpr int kStage = 32 * 65;  // doubles in one staged operand chunk (e rows of 64 + 1)
constexpr size_t kTileSmem = sizeof(double) * (XT * (JT + 1) + 2 * kStage) + sizeof(RowState);
constexpr size_t kUnshiftedSmem = sizeof(double) * 2 * kStage + sizeof(RowState);

// The guards of row r after its last tile (fused.rs:941-1013): whether the
// call overflowed, and the row's check of each output against the terms
// lost below the smallest normal (S.check, S.lost).
__device__ bool row_guards(RowState& S, int r, bool map, bool shifted, bool unnormalized) {
  const double NEG_INF = -INFINITY, POS_INF = INFINITY;
  const double normal = 2.0 * 2.2250738585072014e-308;
  bool over = false;
  const bool zp = !unnormalized;
  const double z = S.z[r], m = S.m[r];
  if (zp && !S.sw[r] && !isfinite(z)) over = true;
  S.check[r] = 0;
  auto weight = [&](double bound) { return map ? bound : shifted ? exp(bound - m) : exp(bound); };
  const double heaviest = weight(S.high[r]);
  if (!(S.sw[r] || S.high[r] == NEG_INF || heaviest == 0.0)) {
    const double lightest = weight(S.light[r]);
    const double largest = S.rl[r], smallest = S.rs[r];
    const double terms = 2.0 * (double)S.terms[r];
    bool finite = isfinite(__dmul_rn(__dmul_rn(heaviest, largest), terms));
    if (finite && zp) {
      const double quotient = __ddiv_rn(heaviest, fabs(z));
      finite = isfinite(quotient) && isfinite(__dmul_rn(__dmul_rn(quotient, largest), terms));
    }
    const double inverse = zp ? __ddiv_rn(1.0, fabs(z)) : 1.0;
    const double tiniest = 4.9406564584124654e-324;
    S.lost[r] = __dmul_rn(__dmul_rn(terms, tiniest), __dadd_rn(__dadd_rn(inverse, largest), 1.0));
    bool no_underflow = smallest == POS_INF;
    if (!no_underflow) {
      no_underflow = __dmul_rn(lightest, smallest) >= normal;
      if (no_underflow && zp) {
        const double quotient = __ddiv_rn(lightest, fabs(z));
        no_underflow = quotient >= normal && __dmul_rn(quotient, smallest) >= normal;
      }
    }
    if (!finite) over = true;
    else if (!no_underflow) S.check[r] = 1;
    if (S.low[r] != POS_INF) {
      const double lw = shifted ? exp(S.low[r] - m) : exp(S.low[r]);
      const bool ok = lw >= normal && (!zp || __ddiv_rn(lw, fabs(z)) >= normal);
      if (!ok) over = true;
    }
  }
  return over;
}

template <int DEPTH>
__global__ void __launch_bounds__(kThreads) fused_tiles(const TileArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  double(*blk)[JT + 1] = reinterpret_cast<double(*)[JT + 1]>(smem);
  double* stg = reinterpret_cast<double*>(smem + sizeof(double) * XT * (JT + 1));
  RowState& S = *reinterpret_cast<RowState*>(smem + sizeof(double) * (XT * (JT + 1) + 2 * kStage));
  __shared__ long long s_first, s_last;

  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int64_t x0 = (int64_t)blockIdx.x * XT;
  const int rows = (int)std::min<int64_t>(XT, p.nx - x0);
  const int64_t y0 = (int64_t)blockIdx.y * YC;
  const int ycount = p.ny > y0 ? (int)std::min<int64_t>(YC, p.ny - y0) : 0;
  const bool map = p.weight_expr != 0;
  const bool shifted = !map && p.shifted != 0;
  const bool unnormalized = p.normalizer == 2;
  const double NEG_INF = -INFINITY, POS_INF = INFINITY;

  if (t == 0) { s_first = p.nj; s_last = 0; }
  if (t < XT) {
    S.m[t] = shifted ? NEG_INF : 0.0;
    S.z[t] = 0.0;
    S.high[t] = NEG_INF;
    S.light[t] = POS_INF;
    S.low[t] = POS_INF;
    S.rl[t] = 0.0;
    S.rs[t] = POS_INF;
    S.terms[t] = 0;
    S.sw[t] = 0;
  }
  __syncthreads();
  if (t < rows) {
    int64_t lo, hi;
    allowed(p.mask, x0 + t, lo, hi);
    if (lo < hi) {
      atomicMin(&s_first, (long long)lo);
      atomicMax(&s_last, (long long)hi);
    }
  }
  __syncthreads();
  const int64_t first = s_first, last = s_last;

  double acc[4][4];
  for (int i = 0; i < 4; i++)
    for (int jj = 0; jj < 4; jj++) acc[i][jj] = 0.0;
  unsigned sv = 0;  // special_value bits of this thread's 16 outputs
  bool over = false;
  unsigned long long visited = 0;

  for (int64_t j0 = first - first % JT; j0 < last; j0 += JT) {
    const int width = (int)std::min<int64_t>(JT, p.nj - j0);
    // Each row's allowed positions within this tile, relative to j0.
    bool has = false;
    if (t < XT) {
      int lo = 0, hi = 0;
      if (t < rows) {
        int64_t l, h;
        allowed(p.mask, x0 + t, l, h);
        l = l < j0 ? j0 : (l > j0 + width ? j0 + width : l);
        h = h < j0 ? j0 : (h > j0 + width ? j0 + width : h);
        lo = (int)(l - j0);
        hi = (int)(h - j0);
      }
      S.lo[t] = lo;
      S.hi[t] = hi;
      S.pend[t] = 0;
      S.spv[t] = 0;
      has = lo < hi;
    }
    if (!__syncthreads_or(has)) continue;
    visited++;

    // Scores of the pair of tiles.
    double s[4][4];
    if (!p.score_expr) {
      for (int i = 0; i < 4; i++)
        for (int jj = 0; jj < 4; jj++) s[i][jj] = 0.0;
      double* qs = stg;            // [e][r], rows of 65
      double* ks = stg + kStage;   // [e][j]
      for (int64_t e0 = 0; e0 < p.ne; e0 += 32) {
        const int ec = (int)std::min<int64_t>(32, p.ne - e0);
        for (int idx = t; idx < XT * 32; idx += kThreads) {
          const int r = idx >> 5, e = idx & 31;
          qs[e * 65 + r] = (r < rows && e < ec) ? p.q[(x0 + r) * p.ne + e0 + e] : 0.0;
          ks[e * 65 + r] = (r < width && e < ec) ? p.k[(j0 + r) * p.ne + e0 + e] : 0.0;
        }
        __syncthreads();
        for (int e = 0; e < ec; e++) {
          double qv[4], kv[4];
          for (int i = 0; i < 4; i++) qv[i] = qs[e * 65 + ty + 16 * i];
          for (int jj = 0; jj < 4; jj++) kv[jj] = ks[e * 65 + tx + 16 * jj];
          for (int i = 0; i < 4; i++)
            for (int jj = 0; jj < 4; jj++) s[i][jj] = fma(qv[i], kv[jj], s[i][jj]);
        }
        __syncthreads();
      }
    } else if (p.score_shape == SCORE_NEG_SQUARED_DIFF) {
      // -power(a - b, 2) summed over E, a row's and a column's values per
      // slot loaded once for the thread's 4 rows and 4 columns.
      const double* ma = p.mats[p.shape_a];
      const double* mb = p.mats[p.shape_b];
      const bool a_row = p.side[p.shape_a] == 0, b_row = p.side[p.shape_b] == 0;
      for (int64_t e = 0; e < p.ne; e++) {
        double ar[4], ac[4], br[4], bc[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int r = ty + 16 * i, j = tx + 16 * i;
          const int64_t xr = (x0 + (r < rows ? r : 0)) * p.ne + e, jc = (j0 + (j < width ? j : 0)) * p.ne + e;
          ar[i] = a_row ? ma[xr] : 0.0;
          br[i] = b_row ? mb[xr] : 0.0;
          ac[i] = a_row ? 0.0 : ma[jc];
          bc[i] = b_row ? 0.0 : mb[jc];
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const double d = __dsub_rn(a_row ? ar[i] : ac[jj], b_row ? br[i] : bc[jj]);
            const double val = -__dmul_rn(d, d);
            s[i][jj] = e == 0 ? val : __dadd_rn(s[i][jj], val);
          }
      }
    } else {
      // One interpreter call site (a rolled loop through shared memory):
      // copies of it unrolled overflow the instruction cache.
      double slots[kMaxSlots];
      for (int q = 0; q < 16; q++) {
        const int r = ty + 16 * (q >> 2), j = tx + 16 * (q & 3);
        double acc_s = 0.0;
        if (r < rows && j < width) {
          for (int64_t e = 0; e < p.ne; e++) {
            for (int sl = 0; sl < p.n_slots; sl++)
              slots[sl] = p.side[sl] == 0 ? p.mats[sl][(x0 + r) * p.ne + e] : p.mats[sl][(j0 + j) * p.ne + e];
            const double val = eval_slots<DEPTH>(p.snodes, p.sn, slots);
            acc_s = e == 0 ? val : __dadd_rn(acc_s, val);
          }
        }
        blk[r][j] = acc_s;
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++) s[i][jj] = blk[ty + 16 * i][tx + 16 * jj];
      __syncwarp();
    }
    // Weights and the row state (fused.rs:811-909). A thread weighs its
    // 4 x 4 pairs (rows ty + 16 i, columns tx + 16 jj); a row's 64 columns
    // are the 16 threads of a half-warp, whose reductions run over lane
    // offsets 8, 4, 2, 1 (every lane takes part: rows outside the tile or
    // with no pair here reduce neutral values). The thread with tx = 0
    // keeps the row's state.
    double w[4][4];
    {
      double lgc[4], smc[4];
      uint8_t fc[4];
      #pragma unroll
      for (int jj = 0; jj < 4; jj++) {
        const int j = tx + 16 * jj;
        const bool live = j < width;
        fc[jj] = live ? p.jflag[j0 + j] : J_FINITE;
        lgc[jj] = live ? p.largest[j0 + j] : 0.0;
        smc[jj] = live ? p.smallest[j0 + j] : POS_INF;
      }
      #pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = ty + 16 * i;
        const bool row = r < rows;
        const int lo = row ? S.lo[r] : 0, hi = row ? S.hi[r] : 0;
        const bool active = lo < hi;  // the same for the half-warp
        bool in[4];
        #pragma unroll
        for (int jj = 0; jj < 4; jj++) in[jj] = tx + 16 * jj >= lo && tx + 16 * jj < hi;
        double lg = 0.0, sm = POS_INF;
        #pragma unroll
        for (int jj = 0; jj < 4; jj++) {
          lg = fmax(lg, in[jj] ? lgc[jj] : 0.0);
          sm = fmin(sm, in[jj] ? smc[jj] : POS_INF);
        }
        lg = half_max(lg);
        sm = half_min(sm);
        // State read by the half-warp before its tx = 0 thread writes it.
        const double m_old = row ? S.m[r] : 0.0;
        __syncwarp();
        if (map) {
          double ha = NEG_INF, la = POS_INF, sum = 0.0;
          bool bad = false;
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const double sc = s[i][jj];
            double x = 0.0;
            if (in[jj]) {
              if (p.weight_shape == WEIGHT_SIGMOID) x = __ddiv_rn(p.wc1, __dadd_rn(p.wc2, exp(-sc)));
              else if (p.weight_shape == WEIGHT_CAUCHY) x = __ddiv_rn(p.wc1, __dadd_rn(p.wc2, __dmul_rn(sc, sc)));
              else x = eval_score<DEPTH>(p.wnodes, p.wn, sc);
            }
            w[i][jj] = x;
            bad |= in[jj] && (!isfinite(x) || !(fc[jj] & J_FINITE));
            const double ax = fabs(x);
            ha = fmax(ha, in[jj] ? ax : NEG_INF);
            la = fmin(la, in[jj] && ax != 0.0 ? ax : POS_INF);
            sum += in[jj] ? x : 0.0;
          }
          ha = half_max(ha);
          la = half_min(la);
          sum = half_sum(sum);
          bad = half_or(bad);
          if (tx == 0 && active) {
            S.terms[r] += hi - lo;
            S.rl[r] = fmax(S.rl[r], lg);
            S.rs[r] = fmin(S.rs[r], sm);
            if (bad) over = true;
            S.high[r] = fmax(S.high[r], ha);
            S.light[r] = fmin(S.light[r], la);
            S.z[r] += sum;
          }
        } else {
          double sc[4];
          double hs = NEG_INF, ls = POS_INF, lows = POS_INF, mx = NEG_INF;
          bool any_nan = false, special_values = false;
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            double x = s[i][jj];
            if (in[jj]) {
              if (p.scale_kind == 1) x = x * p.scale_c;
              else if (p.scale_kind == 2) x = __ddiv_rn(x, p.scale_c);
            }
            sc[jj] = x;
            const bool fin = in[jj] && isfinite(x);
            hs = fmax(hs, fin ? x : NEG_INF);
            ls = fmin(ls, fin ? x : POS_INF);
            lows = fmin(lows, fin && (fc[jj] & J_INFINITE) ? x : POS_INF);
            any_nan |= in[jj] && isnan(x);
            mx = fmax(mx, in[jj] && !isnan(x) ? x : NEG_INF);
            special_values |= in[jj] && !(fc[jj] & J_FINITE);
          }
          hs = half_max(hs);
          ls = half_min(ls);
          lows = half_min(lows);
          if (shifted) {  // the same for the block: the running maximum's inputs
            mx = half_max(mx);
            any_nan = half_or(any_nan);
          }
          special_values = half_or(special_values);
          // The largest score so far, or NaN once any score is NaN.
          const double shift = shifted ? ((isnan(m_old) || any_nan) ? NAN : fmax(m_old, mx)) : 0.0;
          // Every score so far -inf: weights 0 here, and the row's state
          // past its score bounds stays.
          const bool none = shift == NEG_INF;
          double sum = 0.0;
          bool special_weights = false;
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const double x = in[jj] && !none ? exp(sc[jj] - shift) : 0.0;
            w[i][jj] = x;
            sum += x;
            special_weights |= in[jj] && !none && !isfinite(x);
          }
          sum = half_sum(sum);
          special_weights = half_or(special_weights);
          if (tx == 0 && active) {
            S.terms[r] += hi - lo;
            S.rl[r] = fmax(S.rl[r], lg);
            S.rs[r] = fmin(S.rs[r], sm);
            S.high[r] = fmax(S.high[r], hs);
            S.light[r] = fmin(S.light[r], ls);
            S.low[r] = fmin(S.low[r], lows);
            if (!none) {
              const double rescale = exp(m_old - shift);
              S.sw_before[r] = S.sw[r];
              if (shifted && rescale != 1.0) {
                // overflows(z, a, ...) before the rescale: z's part here,
                // a's by the threads that hold a.
                if (!S.sw[r] && !isfinite(S.z[r])) over = true;
                S.z[r] *= rescale;
                S.pend[r] = 1;
                S.resc[r] = rescale;
              }
              S.sw[r] |= special_weights;
              S.spv[r] = special_values;
              if (unnormalized && (special_weights || special_values)) over = true;
              S.z[r] += sum;
              S.m[r] = shift;
            }
          }
        }
        if (active)
          #pragma unroll
          for (int jj = 0; jj < 4; jj++)
            if (in[jj]) blk[r][tx + 16 * jj] = w[i][jj];
      }
    }
    __syncthreads();

    // The weighted values: a += w · v over each row's allowed span.
    double* vs = stg;  // [j][y], rows of 65
    const bool narrow = ycount <= kNarrow;
    for (int idx = t; idx < JT * YC; idx += kThreads) {
      const int j = idx >> 6, y = idx & 63;
      if (narrow && y >= ycount) continue;
      vs[j * 65 + y] = (j < width && y < ycount) ? p.v[(j0 + j) * p.ny + y0 + y] : 0.0;
    }
    __syncthreads();
    if (narrow) {
      // A few value columns: a row's weighted sum over the tile is the
      // half-warp's sum of its threads' four products, added to the output
      // held by the thread with tx = y (its acc[i][0]).
      #pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = ty + 16 * i;
        const bool row = r < rows;
        const int lo = row ? S.lo[r] : 0, hi = row ? S.hi[r] : 0;
        const bool active = lo < hi;
        if (active && tx < ycount && S.pend[r]) {
          const double rescale = S.resc[r];
          if (!S.sw_before[r] && !((sv >> (i * 4)) & 1) && !isfinite(acc[i][0])) over = true;
          acc[i][0] *= rescale;
        }
        for (int y = 0; y < ycount; y++) {
          double part = 0.0;
          bool special = false;
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const int j = tx + 16 * jj;
            const bool in = j >= lo && j < hi;
            const double vj = vs[j * 65 + y];
            part += in ? w[i][jj] * vj : 0.0;
            special |= in && !isfinite(vj);
          }
          part = half_sum(part);
          special = half_or(special);
          if (active && tx == y) {
            acc[i][0] += part;
            if (special) sv |= 1u << (i * 4);
          }
        }
      }
    } else {
      #pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = ty + 16 * i;
        if (r >= rows) continue;
        const int lo = S.lo[r], hi = S.hi[r];
        // A thread whose outputs tx + 16 jj are all past the chunk's holds none.
        if (lo >= hi || tx >= ycount) continue;
        if (S.pend[r]) {
          const double rescale = S.resc[r];
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) {
            const int y = tx + 16 * jj;
            if (y < ycount && !S.sw_before[r] && !((sv >> (i * 4 + jj)) & 1) && !isfinite(acc[i][jj])) over = true;
            acc[i][jj] *= rescale;
          }
        }
        for (int j = lo; j < hi; j++) {
          const double wt = blk[r][j];
          #pragma unroll
          for (int jj = 0; jj < 4; jj++) acc[i][jj] = fma(wt, vs[j * 65 + tx + 16 * jj], acc[i][jj]);
        }
        if (S.spv[r])
          for (int j = lo; j < hi; j++)
            if (!(p.jflag[j0 + j] & J_FINITE))
              #pragma unroll
              for (int jj = 0; jj < 4; jj++)
                if (!isfinite(vs[j * 65 + tx + 16 * jj])) sv |= 1u << (i * 4 + jj);
      }
    }
    __syncthreads();
  }

  // Normalisation and the row guards (fused.rs:941-1013).
  if (t < rows && row_guards(S, t, map, shifted, unnormalized)) over = true;
  __syncthreads();
  const double rounding = 2.220446049250313e-16 / 4.0;
  for (int i = 0; i < 4; i++) {
    const int r = ty + 16 * i;
    if (r >= rows) continue;
    const double z = S.z[r];
    const bool swr = S.sw[r] != 0;
    for (int jj = 0; jj < 4; jj++) {
      const int y = tx + 16 * jj;
      if (y >= ycount) continue;
      const bool spec = (sv >> (i * 4 + jj)) & 1;
      double a = acc[i][jj];
      if (unnormalized) {
        if (shifted && S.m[r] == NEG_INF) a = NAN;
      } else {
        if (!swr && !spec && !isfinite(a)) over = true;
        a = __ddiv_rn(a, z);
        if (z != 0.0 && !swr && !spec && !isfinite(a)) over = true;
      }
      if (S.check[r] && !spec && !(S.lost[r] <= rounding * fabs(a))) over = true;
      p.out[(x0 + r) * p.ny + y0 + y] = a;
    }
    if (p.lse && tx == 0 && blockIdx.y == 0 && !unnormalized && !map) p.lse[x0 + r] = S.m[r] + log(S.z[r]);
  }
  if (__syncthreads_or(over) && t == 0) atomicOr(p.overflowed, 1u);
  if (t == 0 && blockIdx.y == 0 && visited) atomicAdd(p.visited, visited);
}

// fused_tiles for exp weights without a shift (a smoother's exp(s / h))
// and at most kNarrow value columns. No weight then depends on another
// tile's scores, so no row needs its statistics before its last tile: a
// thread keeps its row's running statistics, weight sum, weighted sums and
// flags over all its tiles, and the four threads of a row combine them once
// at the end, where fused_tiles reduces over a half-warp at every tile. A
// thread owns row t % 64 and columns 16·(t / 64) .. + 15 of each 64 x 64
// tile of pairs. Scores are computed as fused_tiles computes them (the same
// operations in the same order, so the same bits); the sums add the same
// terms in another order (a thread's columns in order over the tiles, then
// the row's four threads in order). The row guards and outputs follow
// fused.rs:941-1013 as in fused_tiles.
// SHAPE: 0 product scores, 1 -power(a - b, 2) (SCORE_NEG_SQUARED_DIFF), 2 the
// interpreter.
// NY: the value columns the kernel sums at most (1 or kNarrow).
template <int DEPTH, int SHAPE, int NY>
__global__ void __launch_bounds__(kThreads, 2) fused_unshifted(const TileArgs p) {
  constexpr int CPT = JT / 4;          // columns a thread
  constexpr int RS = 6 + kNarrow;      // a thread's partials: z, high, light, low, largest, smallest, sums
  extern __shared__ __align__(16) unsigned char smem[];
  double* stg = reinterpret_cast<double*>(smem);  // staged q and k; after the last tile the partials
  RowState& S = *reinterpret_cast<RowState*>(smem + sizeof(double) * 2 * kStage);
  __shared__ long long s_first, s_last;
  __shared__ int s_lo[XT], s_hi[XT];
  __shared__ uint8_t s_fc[JT];
  __shared__ double s_lg[JT], s_sm[JT];
  __shared__ double vsm[JT * kNarrow];
  __shared__ long long s_terms[4][XT];
  __shared__ unsigned s_flags[4][XT];  // bit 0: a weight not finite; 1: a value not finite; 8 + y: column y's

  const int t = threadIdx.x, row = t % XT, cg = t / XT;
  const int64_t x0 = (int64_t)blockIdx.x * XT;
  const int rows = (int)std::min<int64_t>(XT, p.nx - x0);
  const int ycount = (int)std::min<int64_t>(NY, p.ny);
  const bool unnormalized = p.normalizer == 2;
  const double NEG_INF = -INFINITY, POS_INF = INFINITY;

  if (t == 0) { s_first = p.nj; s_last = 0; }
  __syncthreads();
  if (t < rows) {
    int64_t lo, hi;
    allowed(p.mask, x0 + t, lo, hi);
    if (lo < hi) {
      atomicMin(&s_first, (long long)lo);
      atomicMax(&s_last, (long long)hi);
    }
  }
  __syncthreads();
  const int64_t first = s_first, last = s_last;

  double z = 0.0, high = NEG_INF, light = POS_INF, low = POS_INF, rl = 0.0, rs = POS_INF;
  double acc[NY];
#pragma unroll
  for (int y = 0; y < NY; y++) acc[y] = 0.0;
  long long terms = 0;
  unsigned flags = 0;
  unsigned long long visited = 0;

  for (int64_t j0 = first - first % JT; j0 < last; j0 += JT) {
    const int width = (int)std::min<int64_t>(JT, p.nj - j0);
    bool has = false;
    if (t < XT) {
      int lo = 0, hi = 0;
      if (t < rows) {
        int64_t l, h;
        allowed(p.mask, x0 + t, l, h);
        l = l < j0 ? j0 : (l > j0 + width ? j0 + width : l);
        h = h < j0 ? j0 : (h > j0 + width ? j0 + width : h);
        lo = (int)(l - j0);
        hi = (int)(h - j0);
      }
      s_lo[t] = lo;
      s_hi[t] = hi;
      has = lo < hi;
      const bool live = t < width;
      s_fc[t] = live ? p.jflag[j0 + t] : J_FINITE;
      s_lg[t] = live ? p.largest[j0 + t] : 0.0;
      s_sm[t] = live ? p.smallest[j0 + t] : POS_INF;
    }
    for (int idx = t; idx < JT * ycount; idx += kThreads) {
      const int j = idx / ycount, y = idx % ycount;
      vsm[j * kNarrow + y] = j < width ? p.v[(j0 + j) * p.ny + y] : 0.0;
    }
    if (!__syncthreads_or(has)) continue;
    visited++;

    // Product and -power(a - b, 2) scores for the thread's 16 columns at
    // once; interpreted scores pair by pair in the weights' loop.
    double s[SHAPE == 2 ? 1 : CPT];
    if constexpr (SHAPE == 0) {
#pragma unroll
      for (int c = 0; c < CPT; c++) s[c] = 0.0;
      double* qs = stg;           // [e][r], rows of 65
      double* ks = stg + kStage;  // [e][j]
      for (int64_t e0 = 0; e0 < p.ne; e0 += 32) {
        const int ec = (int)std::min<int64_t>(32, p.ne - e0);
        for (int idx = t; idx < XT * 32; idx += kThreads) {
          const int r = idx >> 5, e = idx & 31;
          qs[e * 65 + r] = (r < rows && e < ec) ? p.q[(x0 + r) * p.ne + e0 + e] : 0.0;
          ks[e * 65 + r] = (r < width && e < ec) ? p.k[(j0 + r) * p.ne + e0 + e] : 0.0;
        }
        __syncthreads();
        for (int e = 0; e < ec; e++) {
          const double qv = qs[e * 65 + row];
#pragma unroll
          for (int c = 0; c < CPT; c++) s[c] = fma(qv, ks[e * 65 + cg * CPT + c], s[c]);
        }
        __syncthreads();
      }
    } else if constexpr (SHAPE == 1) {
      // -power(a - b, 2) summed over E.
      const double* ma = p.mats[p.shape_a];
      const double* mb = p.mats[p.shape_b];
      const bool a_row = p.side[p.shape_a] == 0, b_row = p.side[p.shape_b] == 0;
      const int64_t xr0 = (x0 + (row < rows ? row : 0)) * p.ne;
      for (int64_t e = 0; e < p.ne; e++) {
        const double ar = a_row ? ma[xr0 + e] : 0.0, br = b_row ? mb[xr0 + e] : 0.0;
#pragma unroll
        for (int c = 0; c < CPT; c++) {
          const int j = cg * CPT + c;
          const int64_t jc = (j0 + (j < width ? j : 0)) * p.ne + e;
          const double d = __dsub_rn(a_row ? ar : ma[jc], b_row ? br : mb[jc]);
          const double val = -__dmul_rn(d, d);
          s[c] = e == 0 ? val : __dadd_rn(s[c], val);
        }
      }
    }
    auto score = [&](int c) -> double {
      if constexpr (SHAPE != 2) {
        return s[c];
      } else {
        double slots[kMaxSlots];
        const int j = cg * CPT + c;
        double acc_s = 0.0;
        if (row < rows && j < width) {
          for (int64_t e = 0; e < p.ne; e++) {
            for (int sl = 0; sl < p.n_slots; sl++)
              slots[sl] = p.side[sl] == 0 ? p.mats[sl][(x0 + row) * p.ne + e] : p.mats[sl][(j0 + j) * p.ne + e];
            const double val = eval_slots<DEPTH>(p.snodes, p.sn, slots);
            acc_s = e == 0 ? val : __dadd_rn(acc_s, val);
          }
        }
        return acc_s;
      }
    };

    // Weights exp(scale(s)) on the row's allowed columns, and the row's
    // running state (fused.rs:811-909 with no shift).
    const int lo = s_lo[row], hi = s_hi[row];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
      const int j = cg * CPT + c;
      const bool in = j >= lo && j < hi;
      double x = score(c);
      if (in) {
        if (p.scale_kind == 1) x = x * p.scale_c;
        else if (p.scale_kind == 2) x = __ddiv_rn(x, p.scale_c);
      }
      const uint8_t fc = s_fc[j];
      const bool fin = in && isfinite(x);
      high = fmax(high, fin ? x : NEG_INF);
      light = fmin(light, fin ? x : POS_INF);
      low = fmin(low, fin && (fc & J_INFINITE) ? x : POS_INF);
      rl = fmax(rl, in ? s_lg[j] : 0.0);
      rs = fmin(rs, in ? s_sm[j] : POS_INF);
      const double w = in ? exp(x) : 0.0;
      z += w;
      terms += in;
      flags |= (in && !isfinite(w) ? 1u : 0u) | (in && !(fc & J_FINITE) ? 2u : 0u);
#pragma unroll
      for (int y = 0; y < NY; y++)
        if (y < ycount) {
          const double vj = vsm[j * kNarrow + y];
          acc[y] += in ? w * vj : 0.0;
          flags |= in && !isfinite(vj) ? 1u << (8 + y) : 0u;
        }
    }
    __syncthreads();
  }

  // The row's four threads' partials, combined in order.
  double* mine = stg + (cg * XT + row) * RS;
  mine[0] = z;
  mine[1] = high;
  mine[2] = light;
  mine[3] = low;
  mine[4] = rl;
  mine[5] = rs;
#pragma unroll
  for (int y = 0; y < NY; y++) mine[6 + y] = acc[y];
  s_terms[cg][row] = terms;
  s_flags[cg][row] = flags;
  __syncthreads();
  bool over = false;
  if (t < XT) {
    const int r = t;
    double* p0 = stg + r * RS;
    unsigned f = s_flags[0][r];
    long long n = s_terms[0][r];
    for (int g = 1; g < 4; g++) {
      const double* pg = stg + (g * XT + r) * RS;
      p0[0] += pg[0];
      p0[1] = fmax(p0[1], pg[1]);
      p0[2] = fmin(p0[2], pg[2]);
      p0[3] = fmin(p0[3], pg[3]);
      p0[4] = fmax(p0[4], pg[4]);
      p0[5] = fmin(p0[5], pg[5]);
      for (int y = 0; y < ycount; y++) p0[6 + y] += pg[6 + y];
      f |= s_flags[g][r];
      n += s_terms[g][r];
    }
    s_flags[0][r] = f;
    S.m[r] = 0.0;
    S.z[r] = p0[0];
    S.high[r] = p0[1];
    S.light[r] = p0[2];
    S.low[r] = p0[3];
    S.rl[r] = p0[4];
    S.rs[r] = p0[5];
    S.terms[r] = n;
    S.sw[r] = f & 1u;
    if (unnormalized && (f & 3u)) over = true;
    if (r < rows && row_guards(S, r, false, false, unnormalized)) over = true;
  }
  __syncthreads();
  const double rounding = 2.220446049250313e-16 / 4.0;
  for (int idx = t; idx < rows * ycount; idx += kThreads) {
    const int r = idx / ycount, y = idx % ycount;
    const double z_r = S.z[r];
    const bool swr = S.sw[r] != 0;
    const bool spec = (s_flags[0][r] >> (8 + y)) & 1u;
    double a = stg[r * RS + 6 + y];
    if (!unnormalized) {
      if (!swr && !spec && !isfinite(a)) over = true;
      a = __ddiv_rn(a, z_r);
      if (z_r != 0.0 && !swr && !spec && !isfinite(a)) over = true;
    }
    if (S.check[r] && !spec && !(S.lost[r] <= rounding * fabs(a))) over = true;
    p.out[(x0 + r) * p.ny + y] = a;
  }
  if (p.lse && !unnormalized && t < rows) p.lse[x0 + t] = S.m[t] + log(S.z[t]);
  if (__syncthreads_or(over) && t == 0) atomicOr(p.overflowed, 1u);
  if (t == 0 && visited) atomicAdd(p.visited, visited);
}

// The deepest stack a postfix expression reaches.
int stack_depth(const std::vector<ExprNode>& nodes) {
  int depth = 0, deepest = 0;
  for (const ExprNode& e : nodes) {
    if (e.kind == 0 || e.kind == 1) depth++;
    else if (e.kind != 2) depth--;
    deepest = std::max(deepest, depth);
  }
  return deepest;
}

// fused_tiles with a stack for expressions `depth` deep (parsed expressions
// are at most 60).
void launch_tiles(const TileArgs& a, int depth, dim3 grid, cudaStream_t s) {
  if (depth > 64) fail(EINFOLD_INVALID, "an expression deeper than 64");
  const char* general = std::getenv("EINFOLD_TILES_GENERAL");
  if (!a.weight_expr && !a.shifted && a.ny <= kNarrow && !(general && std::atoi(general) != 0)) {
    // Unshifted exp weights and few value columns: no per-tile reductions.
    // The interpreter's stack depth matters to its kernels only.
    const int shape = !a.score_expr ? 0 : (a.score_shape == SCORE_NEG_SQUARED_DIFF ? 1 : 2);
    const bool one = a.ny <= 1;
    auto kernel = shape == 0 ? (one ? fused_unshifted<8, 0, 1> : fused_unshifted<8, 0, kNarrow>)
                  : shape == 1 ? (one ? fused_unshifted<8, 1, 1> : fused_unshifted<8, 1, kNarrow>)
                               : (depth <= 8 ? fused_unshifted<8, 2, kNarrow> : fused_unshifted<64, 2, kNarrow>);
    EF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUnshiftedSmem));
    kernel<<<dim3(grid.x, 1), kThreads, kUnshiftedSmem, s>>>(a);
    EF_LAUNCH_CHECK();
    return;
  }
  auto kernel = depth <= 8 ? fused_tiles<8> : fused_tiles<64>;
  EF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem));
  kernel<<<grid, kThreads, kTileSmem, s>>>(a);
  EF_LAUNCH_CHECK();
}

// Each J position's values: whether all are finite, whether any is
// infinite, the largest finite magnitude (0 if none) and the smallest
// nonzero finite one (+inf if none) (fused.rs:371-385). A warp per J.
// With jlen (ragged batches of lnj positions), a position past its batch's
// length, which no row joins, is not read: it gets the statistics of zeros.
__global__ void value_stats(int64_t nj, int64_t ny, const double* __restrict__ v, uint8_t* __restrict__ flag,
                            double* __restrict__ largest, double* __restrict__ smallest, unsigned* nonfinite,
                            int64_t lnj = 1, const int64_t* __restrict__ jlen = nullptr) {
  const int lane = threadIdx.x & 31;
  for (int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nj;
       j += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    if (jlen && j % lnj >= jlen[j / lnj]) {
      if (lane == 0) {
        flag[j] = J_FINITE;
        largest[j] = 0.0;
        smallest[j] = INFINITY;
      }
      continue;
    }
    bool fin = true, inf = false;
    double lg = 0.0, sm = INFINITY;
    for (int64_t y = lane; y < ny; y += 32) {
      const double x = v[j * ny + y];
      if (!isfinite(x)) {
        fin = false;
        inf |= isinf(x);
      } else {
        const double a = fabs(x);
        lg = fmax(lg, a);
        if (a != 0.0) sm = fmin(sm, a);
      }
    }
    fin = __all_sync(0xffffffffu, fin);
    inf = __any_sync(0xffffffffu, inf);
    lg = warp_max(lg);
    sm = warp_min(sm);
    if (lane == 0) {
      if (!fin) atomicOr(nonfinite, 1u);
      flag[j] = (fin ? J_FINITE : 0) | (inf ? J_INFINITE : 0);
      largest[j] = lg;
      smallest[j] = sm;
    }
  }
}

// The pairs of 64 x 64 tiles that fused.rs:749-758 visits: for each X
// tile, the J tiles between its rows' first and last allowed position that
// some row's interval meets. A warp per X tile, a row per lane (two rows).
__global__ void count_tiles(int64_t nx, int64_t nj, Mask m, unsigned long long* visited) {
  const int lane = threadIdx.x & 31;
  unsigned long long local = 0;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t * XT < nx;
       t += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    int64_t lo[2], hi[2];
    long long first = nj, last = 0;
    for (int i = 0; i < 2; i++) {
      const int64_t x = t * XT + lane + 32 * i;
      lo[i] = hi[i] = 0;
      if (x < nx) allowed(m, x, lo[i], hi[i]);
      if (lo[i] < hi[i]) {
        first = min(first, (long long)lo[i]);
        last = max(last, (long long)hi[i]);
      }
    }
    for (int o = 16; o; o >>= 1) {
      first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
      last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
    }
    for (long long j0 = first - first % JT; j0 < last; j0 += JT) {
      const long long j1 = min(j0 + JT, (long long)nj);
      const bool meets = (lo[0] < hi[0] && lo[0] < j1 && hi[0] > j0) || (lo[1] < hi[1] && lo[1] < j1 && hi[1] > j0);
      if (__any_sync(0xffffffffu, meets)) local++;
    }
  }
  if (lane == 0 && local) atomicAdd(visited, local);
}

// Scatters a column's rows into matrix[row][col]; a repeated cell sets *dup.
__global__ void place_kernel(Role rows_r, Role cols_r, int64_t n, int64_t ncols, const double* __restrict__ vals,
                             double* __restrict__ mat, unsigned* __restrict__ held, unsigned* dup) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cell = role_position(rows_r, i) * ncols + role_position(cols_r, i);
    const unsigned bit = 1u << (cell & 31);
    if (atomicOr(&held[cell >> 5], bit) & bit) atomicOr(dup, 1u);
    mat[cell] = vals[i];
  }
}

// Output rows: x has one if it is allowed some J position.
__global__ void row_flags(int64_t nx, int64_t nj, Mask m, uint8_t* __restrict__ flags) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < nx; x += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo, hi;
    allowed(m, x, lo, hi);
    flags[x] = nj > 0 && lo < hi;
  }
}

__global__ void emit_rows(int64_t nx, int64_t ny, const uint8_t* __restrict__ flags,
                          const int64_t* __restrict__ row_index, OutKeys keys, const int64_t* __restrict__ xtab,
                          const int64_t* __restrict__ ytab, const double* __restrict__ out,
                          double* __restrict__ val_out) {
  // A thread per cell (x, y) of the row-major placed output.
  const int64_t cells = nx * ny;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = ny == 1 ? c : c / ny, y = c - x * ny;
    if (!flags[x]) continue;
    const int64_t o = row_index[x] * ny + y;
    for (int k = 0; k < keys.n; k++)
      store_key(keys.out[k], keys.width[k], o, keys.key[k].in_x ? xtab[(int64_t)k * nx + x] : ytab[(int64_t)k * ny + y]);
    val_out[o] = out[c];
  }
}

struct Placement {
  int operand;                 // 0 q, 1 k, 2 v
  const std::vector<int>* rows;
  const std::vector<int>* cols;
  int column;
};

std::optional<uint64_t> size_of(const std::vector<int>& dims, const std::vector<int64_t>& extent) {
  uint64_t n = 1;
  for (int d : dims)
    if (!checked_mul(n, (uint64_t)extent[d], &n)) return std::nullopt;
  return n;
}

}  // namespace

// A pipeline's roles, mask and placed matrices (fused.rs:151-345, 624-664).
struct PlacedPipeline {
  std::vector<int> ws, xs, es, js, ys;  // xs and js lead with ws
  Mask mask;
  std::vector<std::pair<int, int>> read;  // the producer's columns, (operand, column)
  std::vector<DeviceBuffer<double>> matrices;  // per read column, then the values
  std::vector<int64_t> extent;
  uint64_t nx = 0, ne = 0, nj = 0, ny = 0;
  // Ragged groups (the reference declines them): per batch, the X and J
  // positions present, as host vectors and device arrays; empty when every
  // batch is complete.
  std::vector<int64_t> xlen, jlen;
  DeviceBuffer<int64_t> xlen_dev, jlen_dev;
};

// Rows of a placed matrix: 0 no cell held, 1 every cell, 2 some.
__global__ void row_presence(const unsigned* __restrict__ held, int64_t rows, int64_t cols, uint8_t* __restrict__ state) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
    int64_t n = 0;
    for (int64_t c = r * cols; c < (r + 1) * cols; c++) n += (held[c >> 5] >> (c & 31)) & 1u;
    state[r] = n == 0 ? 0 : (n == cols ? 1 : 2);
  }
}

// The roles, conditions and placement of a pipeline. Where an operand
// misses cells, its batches are taken as ragged groups when every batch's
// present positions along X (for q) and J (for k and v, the same for both)
// are a prefix 0 .. length - 1 with every cell of those rows present, and
// `ragged_ok`; otherwise the pipeline declines, as the reference's
// placement does for any missing cell.
PlacedPipeline place_pipeline(Context& ctx, const PipelineD& p, const Relation& q, const Relation& k,
                              const Relation& v, bool ragged_ok) {
  cudaStream_t s = ctx.stream;
  PlacedPipeline P;
  const FoldD& pr = p.producer;
  if (pr.operands.size() != 2) decline("a pipeline's producer of other than two operands");
  const OperandD &op_q = pr.operands[0], &op_k = pr.operands[1], &values = p.values;
  const int own = pr.n_dims(), n = own + (int)p.equality.size();
  auto output = [&](int d) { return std::find(p.outputs.begin(), p.outputs.end(), d) != p.outputs.end(); };
  std::vector<int>&ws = P.ws, &xs = P.xs, &es = P.es, &js = P.js, &ys = P.ys;
  for (int d = 0; d < own; d++) {
    const bool hq = op_q.holds(d), hk = op_k.holds(d), produced = pr.output_of(d) >= 0, out = output(d),
               hv = values.holds(d);
    if (hq && hk && produced && out && hv) ws.push_back(d);
    else if (hq && !hk && produced && out && !hv) xs.push_back(d);
    else if (hq && hk && !produced && !out && !hv) es.push_back(d);
    else if (!hq && hk && produced && !out && hv) js.push_back(d);
    else decline("a dimension of no pipeline role");
  }
  for (int d = own; d < n; d++) {
    if (!output(d)) decline("a pipeline that sums its own dimension away");
    ys.push_back(d);
  }
  Mask& mask = P.mask;
  for (auto& c : pr.conditions) {
    if (xs.size() != 1 || js.size() != 1) decline("a condition without one X and one J dimension");
    ConditionD m;
    if (c.left == xs[0] && c.right == js[0]) m = c;
    else if (c.left == js[0] && c.right == xs[0]) {
      auto mm = c.mirrored();
      if (!mm) decline("a condition whose mirror overflows");
      m = *mm;
    } else {
      decline("a condition on other dimensions");
    }
    if (mask.n == kMaxMask) decline("more than 8 conditions");
    mask.cmp[mask.n] = m.cmp;
    mask.off[mask.n] = m.offset;
    mask.n++;
  }
  const std::vector<int> local_xs = xs, local_js = js;
  xs.insert(xs.begin(), ws.begin(), ws.end());
  js.insert(js.begin(), ws.begin(), ws.end());

  // The producer's columns: each operand's factor, or what its expression reads.
  std::vector<std::pair<int, int>>& read = P.read;
  if (!pr.row_expr) {
    if (op_q.factor < 0 || op_k.factor < 0) decline("a product's operand without a factor");
    read = {{0, op_q.factor}, {1, op_k.factor}};
  } else {
    read = pr.row_columns();
    std::sort(read.begin(), read.end());
    read.erase(std::unique(read.begin(), read.end()), read.end());
    bool reads0 = false, reads1 = false;
    for (auto& rc : read) {
      reads0 |= rc.first == 0;
      reads1 |= rc.first == 1;
      if (rc.first > 1) decline("an expression reading a third operand");
    }
    if (!reads0 || !reads1) decline("an expression that doesn't read both operands");
    if ((int)read.size() > kMaxSlots) decline("an expression reading more than 8 columns");
  }
  std::vector<Placement> placements;
  for (auto& rc : read) placements.push_back(rc.first == 0 ? Placement{0, &xs, &es, rc.second} : Placement{1, &js, &es, rc.second});
  placements.push_back(Placement{2, &js, &ys, values.factor});
  const OperandD* ops[3] = {&op_q, &op_k, &values};
  const Relation* rels[3] = {&q, &k, &v};

  // Keys and extents, each operand's staged once.
  std::vector<int64_t>& extent = P.extent;
  extent.assign((size_t)n, 0);
  std::optional<StagedKeys> staged[3];
  for (auto& pl : placements) {
    if (staged[pl.operand]) continue;
    staged[pl.operand] = stage_keys(ctx, *ops[pl.operand], *rels[pl.operand]);
    const OperandD& op = *ops[pl.operand];
    for (size_t i = 0; i < op.keys.size(); i++)
      extent[op.keys[i].dim] = std::max(extent[op.keys[i].dim], staged[pl.operand]->extent[i]);
  }
  auto nx_ = size_of(xs, extent), ne_ = size_of(es, extent), nj_ = size_of(js, extent), ny_ = size_of(ys, extent);
  auto lnx_ = size_of(local_xs, extent), lnj_ = size_of(local_js, extent);
  if (!nx_ || !ne_ || !nj_ || !ny_ || !lnx_ || !lnj_) decline("an extent product that overflows");
  P.nx = *nx_;
  P.ne = *ne_;
  P.nj = *nj_;
  P.ny = *ny_;
  mask.lnx = (int64_t)std::max<uint64_t>(*lnx_, 1);
  mask.lnj = (int64_t)*lnj_;
  ctx.phase("fused: keys");

  // Placement (fused.rs:624-664): exactly one non-NULL row per cell, or
  // ragged groups.
  bool ragged = false;
  std::vector<std::vector<uint8_t>> presence;  // per placement: each row's state
  for (auto& pl : placements) {
    const Relation& r = *rels[pl.operand];
    const OperandD& op = *ops[pl.operand];
    auto rows_n = size_of(*pl.rows, extent), cols_n = size_of(*pl.cols, extent);
    if (!rows_n || !cols_n) decline("an extent product that overflows");
    uint64_t cells = 0;
    if (!checked_mul(*rows_n, *cols_n, &cells)) decline("an extent product that overflows");
    uint64_t total = 0;
    for (auto& b : r.batches) total += (uint64_t)b.rows;
    if (cells >= UINT32_MAX || total > cells) decline("an operand without one row per cell");
    const bool complete = total == cells;
    if (!complete && !ragged_ok) decline("an operand without one row per cell");
    const Field& f = r.fields[pl.column];
    if (f.dictionary || f.kind != Kind::Float64) decline("a column that isn't DOUBLE");
    for (auto& b : r.batches)
      if (b.columns[pl.column].nulls() > 0) decline("a NULL factor");
    DeviceColumn col = stage_column(ctx, r, pl.column, false);
    DeviceBuffer<double> mat((size_t)std::max<uint64_t>(cells, 1), s);
    DeviceBuffer<unsigned> held((size_t)std::max<uint64_t>((cells + 31) / 32, 1), s);
    DeviceBuffer<unsigned> dup(1, s);
    held.zero();
    dup.zero();
    if (!complete) mat.zero();  // missing cells (of ragged groups' padding) hold zeros
    if (total) {
      const Role rr = role_of(*pl.rows, op, *staged[pl.operand], extent);
      const Role cr = role_of(*pl.cols, op, *staged[pl.operand], extent);
      place_kernel<<<blocks_for((int64_t)total, 256), 256, 0, s>>>(rr, cr, (int64_t)total, (int64_t)*cols_n,
                                                                   (const double*)col.ptr(), mat.get(), held.get(),
                                                                   dup.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
    unsigned d = 0;
    EF_CUDA(cudaMemcpyAsync(&d, dup.get(), 4, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    if (d) decline("an operand with a repeated cell");
    std::vector<uint8_t> state;
    if (!complete) {
      ragged = true;
      DeviceBuffer<uint8_t> st((size_t)std::max<uint64_t>(*rows_n, 1), s);
      row_presence<<<blocks_for(*rows_n, 256), 256, 0, s>>>(held.get(), (int64_t)*rows_n, (int64_t)*cols_n, st.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
      state.resize((size_t)*rows_n);
      if (*rows_n) EF_CUDA(cudaMemcpyAsync(state.data(), st.get(), (size_t)*rows_n, cudaMemcpyDeviceToHost, s));
      EF_CUDA(cudaStreamSynchronize(s));
    }
    presence.push_back(std::move(state));
    P.matrices.push_back(std::move(mat));
  }
  uint64_t out_cells = 0;
  if (!checked_mul(P.nx, P.ny, &out_cells) || out_cells >= UINT32_MAX) decline("an output of 2^32 cells or more");
  if (ragged) {
    // Ragged groups: per batch, a prefix of present rows along X (q's
    // matrices) and along J (k's and v's, the same prefix).
    if (pr.row_expr) decline("ragged groups with a row expression");
    const int64_t W = mask.lnx > 0 ? (int64_t)P.nx / mask.lnx : 0;
    if (W * mask.lnx != (int64_t)P.nx || W * mask.lnj != (int64_t)P.nj) decline("ragged groups that aren't batches");
    auto lengths = [&](const std::vector<uint8_t>& st, int64_t per, std::vector<int64_t>& len) -> bool {
      std::vector<int64_t> got((size_t)W, 0);
      for (int64_t w = 0; w < W; w++) {
        int64_t l = 0;
        while (l < per && (st.empty() || st[(size_t)(w * per + l)] == 1)) l++;
        for (int64_t r = l; r < per; r++)
          if (!st.empty() && st[(size_t)(w * per + r)] != 0) return false;
        got[(size_t)w] = l;
      }
      if (len.empty()) len = got;
      return len == got;
    };
    for (size_t i = 0; i < placements.size(); i++) {
      const bool along_x = placements[i].operand == 0;
      if (!lengths(presence[i], along_x ? mask.lnx : mask.lnj, along_x ? P.xlen : P.jlen))
        decline("an operand without one row per cell");
    }
    P.xlen_dev.allocate((size_t)std::max<int64_t>(W, 1), s);
    P.jlen_dev.allocate((size_t)std::max<int64_t>(W, 1), s);
    if (W) {
      EF_CUDA(cudaMemcpyAsync(P.xlen_dev.get(), P.xlen.data(), (size_t)W * 8, cudaMemcpyHostToDevice, s));
      EF_CUDA(cudaMemcpyAsync(P.jlen_dev.get(), P.jlen.data(), (size_t)W * 8, cudaMemcpyHostToDevice, s));
    }
    mask.xlen = P.xlen_dev.get();
    mask.jlen = P.jlen_dev.get();
  }
  ctx.phase("fused: place");
  return P;
}

FoldOutput fused_pipeline(Context& ctx, const PipelineD& p, const Relation& q, const Relation& k, const Relation& v,
                          const std::vector<Field>& schema, const einfold_options& o, Budget& budget) {
  (void)budget;  // the tile path asks no budget (fused.rs:151-489)
  cudaStream_t s = ctx.stream;
  const FoldD& pr = p.producer;
  PlacedPipeline P = place_pipeline(ctx, p, q, k, v, true);
  const std::vector<int>&xs = P.xs, &ys = P.ys;
  const std::vector<std::pair<int, int>>& read = P.read;
  std::vector<DeviceBuffer<double>>& matrices = P.matrices;
  const std::vector<int64_t>& extent = P.extent;
  const uint64_t nx = P.nx, ne = P.ne, nj = P.nj, ny = P.ny;
  const Mask mask = P.mask;
  uint64_t out_cells = nx * ny;
  (void)out_cells;

  DeviceBuffer<uint8_t> jflag((size_t)std::max<uint64_t>(nj, 1), s);
  DeviceBuffer<double> largest((size_t)std::max<uint64_t>(nj, 1), s), smallest((size_t)std::max<uint64_t>(nj, 1), s);
  DeviceBuffer<unsigned> nonfinite(1, s);
  nonfinite.zero();
  if (nj) {
    value_stats<<<blocks_for((int64_t)nj * 32, 256), 256, 0, s>>>((int64_t)nj, (int64_t)ny, matrices.back().get(),
                                                                  jflag.get(), largest.get(), smallest.get(),
                                                                  nonfinite.get(), mask.lnj, mask.jlen);
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  unsigned v_nonfinite = 0;
  EF_CUDA(cudaMemcpyAsync(&v_nonfinite, nonfinite.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));

  // Expressions, with column nodes pointing at their slots.
  std::vector<ExprNode> snodes = pr.row, wnodes = p.weight;
  for (auto& e : snodes)
    if (e.kind == 0) {
      const auto it = std::find(read.begin(), read.end(), std::make_pair(e.a, e.b));
      e.a = (int)(it - read.begin());
    }
  for (auto& e : wnodes)
    if (e.kind == 0) e.a = 0;
  DeviceBuffer<ExprNode> dnodes(std::max<size_t>(snodes.size() + wnodes.size(), 1), s);
  if (!snodes.empty())
    EF_CUDA(cudaMemcpyAsync(dnodes.get(), snodes.data(), snodes.size() * sizeof(ExprNode), cudaMemcpyHostToDevice, s));
  if (!wnodes.empty())
    EF_CUDA(cudaMemcpyAsync(dnodes.get() + snodes.size(), wnodes.data(), wnodes.size() * sizeof(ExprNode),
                            cudaMemcpyHostToDevice, s));

  TileArgs a{};
  a.nx = (int64_t)nx;
  a.ne = (int64_t)ne;
  a.nj = (int64_t)nj;
  a.ny = (int64_t)ny;
  a.mask = mask;
  a.weight_expr = p.weight_expr;
  a.scale_kind = p.scale_kind;
  a.scale_c = p.scale_c;
  a.shifted = p.shift == 1;
  a.normalizer = p.normalizer;
  a.wnodes = dnodes.get() + snodes.size();
  a.wn = (int)wnodes.size();
  a.score_expr = pr.row_expr;
  if (!pr.row_expr) {
    a.q = matrices[0].get();
    a.k = matrices[1].get();
  } else {
    a.snodes = dnodes.get();
    a.sn = (int)snodes.size();
    a.n_slots = (int)read.size();
    for (size_t i = 0; i < read.size(); i++) {
      a.mats[i] = matrices[i].get();
      a.side[i] = read[i].first;
    }
  }
  // Expressions of the shapes the kernel computes without the interpreter
  // (binary ops 0 add, 1 sub, 2 mul, 3 div, 4 pow; unary 0 neg, 2 exp).
  auto node = [](const ExprNode& e, int kind, int op) { return e.kind == kind && e.a == op; };
  if (pr.row_expr && snodes.size() == 6 && snodes[0].kind == 0 && snodes[1].kind == 0 && node(snodes[2], 3, 1) &&
      snodes[3].kind == 1 && snodes[3].value == 2.0 && node(snodes[4], 3, 4) && node(snodes[5], 2, 0)) {
    a.score_shape = SCORE_NEG_SQUARED_DIFF;
    a.shape_a = snodes[0].a;
    a.shape_b = snodes[1].a;
  }
  if (p.weight_expr && wnodes.size() == 7 && wnodes[0].kind == 1 && wnodes[1].kind == 1 && wnodes[2].kind == 0 &&
      node(wnodes[5], 3, 0) && node(wnodes[6], 3, 3)) {
    if (node(wnodes[3], 2, 0) && node(wnodes[4], 2, 2)) a.weight_shape = WEIGHT_SIGMOID;
    else if (wnodes[3].kind == 0 && node(wnodes[4], 3, 2)) a.weight_shape = WEIGHT_CAUCHY;
    a.wc1 = wnodes[0].value;
    a.wc2 = wnodes[1].value;
  }
  a.v = matrices.back().get();
  a.jflag = jflag.get();
  a.largest = largest.get();
  a.smallest = smallest.get();
  DeviceBuffer<double> out((size_t)std::max<uint64_t>(out_cells, 1), s);
  DeviceBuffer<unsigned long long> visited(1, s);
  DeviceBuffer<unsigned> overflowed(1, s);
  visited.zero();
  overflowed.zero();
  a.out = out.get();
  a.visited = visited.get();
  a.overflowed = overflowed.get();
  const uint64_t x_tiles = (nx + XT - 1) / XT;
  // The split form on the tensor cores, where it applies: product scores, a
  // softmax shifted by the kept maximum, an average, finite operands.
  bool split_done = false;
  const int64_t batches_w = mask.lnx > 0 ? (int64_t)nx / mask.lnx : 0;
  if (o.precision == 0 && !pr.row_expr && !p.weight_expr && p.shift == 1 && p.normalizer != 2 && !v_nonfinite &&
      nx > 0 && nj > 0 && ny > 0 && batches_w * mask.lnx == (int64_t)nx && batches_w * mask.lnj == (int64_t)nj) {
    AttentionProblem ap;
    ap.q = matrices[0].get();
    ap.k = matrices[1].get();
    ap.v = matrices.back().get();
    ap.batches = batches_w;
    ap.lnx = mask.lnx;
    ap.lnj = mask.lnj;
    ap.ne = (int64_t)ne;
    ap.ny = (int64_t)ny;
    ap.mask = mask;
    ap.scale_kind = p.scale_kind;
    ap.scale_c = p.scale_c;
    ap.largest = largest.get();
    ap.smallest = smallest.get();
    ap.out = out.get();
    ap.xlen_host = P.xlen;
    ap.jlen_host = P.jlen;
    const int slices = o.slices > 0 ? o.slices : 6;
    const AttentionOutcome r = attention_split(ctx, ap, slices, s);
    if (r == ATTENTION_GUARDED) decline("a sum that overflowed or may have underflowed");
    if (r == ATTENTION_DONE) {
      split_done = true;
      count_tiles<<<blocks_for(x_tiles * 32, 256), 256, 0, s>>>((int64_t)nx, (int64_t)nj, mask, visited.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
  }
  if (!split_done && !pr.row_expr && !p.weight_expr && p.shift == 1 && p.normalizer == 0 && !v_nonfinite &&
      nx > 0 && nj > 0 && ny > 0 && batches_w * mask.lnx == (int64_t)nx && batches_w * mask.lnj == (int64_t)nj &&
      !fp64_tiles_requested()) {
    // The FP64 form on the FP64 tensor pipe, for an attention-shaped
    // pipeline the split form didn't take (precision = fp64, or scores it
    // can't bound).
    AttentionProblem ap;
    ap.q = matrices[0].get();
    ap.k = matrices[1].get();
    ap.v = matrices.back().get();
    ap.batches = batches_w;
    ap.lnx = mask.lnx;
    ap.lnj = mask.lnj;
    ap.ne = (int64_t)ne;
    ap.ny = (int64_t)ny;
    ap.mask = mask;
    ap.scale_kind = p.scale_kind;
    ap.scale_c = p.scale_c;
    ap.largest = largest.get();
    ap.smallest = smallest.get();
    ap.out = out.get();
    const AttentionOutcome r = attention_f64_mma(ctx, ap, s);
    if (r == ATTENTION_GUARDED) decline("a sum that overflowed or may have underflowed");
    if (r == ATTENTION_DONE) {
      split_done = true;
      count_tiles<<<blocks_for(x_tiles * 32, 256), 256, 0, s>>>((int64_t)nx, (int64_t)nj, mask, visited.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
  }
  if (x_tiles && !split_done) {
    const dim3 grid((unsigned)x_tiles, (unsigned)std::max<uint64_t>((ny + YC - 1) / YC, 1));
    launch_tiles(a, std::max(stack_depth(snodes), stack_depth(wnodes)), grid, s);
    ctx.kernels++;
  }
  unsigned long long n_visited = 0;
  unsigned of = 0;
  EF_CUDA(cudaMemcpyAsync(&n_visited, visited.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&of, overflowed.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("fused: tiles");
  if (of) decline("a sum that overflowed or may have underflowed");

  // The pairs of tiles that share a batch (fused.rs:386-397).
  // The batch of a tile's first row advances with the tiles (a division
  // only for a tile whose rows reach past that batch).
  uint64_t tile_pairs = 0;
  const uint64_t lnx = (uint64_t)mask.lnx, lnj = (uint64_t)mask.lnj;
  uint64_t w0 = 0, next_batch = lnx;  // x0's batch and the first row past it
  for (uint64_t t = 0; t < x_tiles; t++) {
    const uint64_t x0 = t * XT, x1 = std::min<uint64_t>((t + 1) * XT, nx);
    while (x0 >= next_batch) {
      w0++;
      next_batch += lnx;
    }
    const uint64_t w1 = x1 - 1 < next_batch ? w0 : (x1 - 1) / lnx;
    const uint64_t start = w0 * lnj, end = w1 * lnj + lnj;
    tile_pairs += (end + JT - 1) / JT - start / JT;
  }

  // The rows: every y for each x with an allowed J position, in order.
  DeviceBuffer<uint8_t> flags((size_t)std::max<uint64_t>(nx, 1), s);
  DeviceBuffer<int64_t> row_index((size_t)std::max<uint64_t>(nx, 1), s);
  if (nx) {
    row_flags<<<blocks_for((int64_t)nx, 256), 256, 0, s>>>((int64_t)nx, (int64_t)nj, mask, flags.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  const int64_t n_rows = exclusive_scan_flags(ctx, flags.get(), (int64_t)nx, row_index.get());
  const int64_t n_out = n_rows * (int64_t)ny;
  OutKeys okeys;
  if (p.outputs.size() > (size_t)kMaxDims) decline("more than 8 outputs");
  for (size_t i = 0; i < p.outputs.size(); i++) {
    const int d = p.outputs[i];
    const bool in_x = std::find(xs.begin(), xs.end(), d) != xs.end();
    const std::vector<int>& role = in_x ? xs : ys;
    const size_t slot = (size_t)(std::find(role.begin(), role.end(), d) - role.begin());
    int64_t stride = 1;
    for (size_t e = slot + 1; e < role.size(); e++) stride *= extent[role[e]];
    okeys.key[okeys.n] = KeyAt{in_x ? 1 : 0, stride, std::max<int64_t>(extent[d], 1)};
    okeys.width[okeys.n] = width_of(schema[i].kind);
    okeys.n++;
  }
  DeviceBuffer<int64_t> xtab((size_t)std::max<uint64_t>(okeys.n * nx, 1), s),
      ytab((size_t)std::max<uint64_t>(okeys.n * ny, 1), s);
  if (nx) key_tables<<<blocks_for((int64_t)nx, 256), 256, 0, s>>>((int64_t)nx, okeys, 1, xtab.get());
  if (ny) key_tables<<<blocks_for((int64_t)ny, 256), 256, 0, s>>>((int64_t)ny, okeys, 0, ytab.get());
  ctx.kernels += 2;
  std::vector<DeviceBuffer<uint8_t>> key_dev;
  for (int i = 0; i < okeys.n; i++) {
    key_dev.emplace_back((size_t)(n_out ? n_out * okeys.width[i] : 1), s);
    okeys.out[i] = key_dev.back().get();
  }
  DeviceBuffer<double> vals((size_t)(n_out ? n_out : 1), s);
  if (n_out) {
    emit_rows<<<blocks_for((uint64_t)nx * ny, 256), 256, 0, s>>>((int64_t)nx, (int64_t)ny, flags.get(),
                                                                  row_index.get(), okeys, xtab.get(), ytab.get(),
                                                                  out.get(), vals.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  OutBatch ob;
  ob.rows = n_out;
  for (size_t i = 0; i < p.outputs.size(); i++) {
    OutColumn c;
    c.format = schema[i].format;
    c.name = schema[i].name;
    c.kind = schema[i].kind;
    c.nullable = schema[i].nullable;
    c.length = n_out;
    c.values = result_buffer(ctx, key_dev[i], (size_t)(n_out * okeys.width[i]), o.result_on_device);
    ob.columns.push_back(std::move(c));
  }
  OutColumn val;
  val.format = "g";
  val.kind = Kind::Float64;
  val.name = schema.back().name;
  val.nullable = schema.back().nullable;
  val.length = n_out;
  val.values = result_buffer(ctx, vals, (size_t)n_out * 8, o.result_on_device);
  ob.columns.push_back(std::move(val));
  EF_CUDA(cudaStreamSynchronize(s));
  FoldOutput result;
  result.algorithm = EINFOLD_ALG_FUSED;
  result.batches.push_back(std::move(ob));
  result.tiles_visited = n_visited;
  result.tiles = tile_pairs;
  ctx.phase("fused: result");
  return result;
}

namespace {

// Rows of a placed matrix that hold an operand's cells: all of them, or, in
// ragged groups, row r of batch r / per when r % per < len[r / per].
__global__ void length_flags(int64_t rows, int64_t per, const int64_t* __restrict__ len, uint8_t* __restrict__ flags) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x)
    flags[r] = !len || r % per < len[r / per];
}

// One batch of rows from a placed matrix [rows][cols]: a row per cell of the
// present rows, in order, with `op`'s key columns (as `fields` types them)
// recomputed from the cell's position, then the cell's value.
OutBatch emit_matrix(Context& ctx, const OperandD& op, const std::vector<Field>& fields,
                     const std::vector<int>& row_dims, const std::vector<int>& col_dims,
                     const std::vector<int64_t>& extent, const double* mat, int64_t rows, int64_t cols,
                     int64_t per, const int64_t* len, bool on_device) {
  cudaStream_t s = ctx.stream;
  DeviceBuffer<uint8_t> flags((size_t)std::max<int64_t>(rows, 1), s);
  DeviceBuffer<int64_t> row_index((size_t)std::max<int64_t>(rows, 1), s);
  if (rows) {
    length_flags<<<blocks_for((uint64_t)rows, 256), 256, 0, s>>>(rows, per, len, flags.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  const int64_t n_rows = exclusive_scan_flags(ctx, flags.get(), rows, row_index.get());
  const int64_t n_out = n_rows * cols;
  if (op.keys.size() > (size_t)kMaxDims) decline("more than 8 keys");
  OutKeys okeys;
  for (auto& key : op.keys) {
    const int d = key.dim;
    const bool in_x = std::find(row_dims.begin(), row_dims.end(), d) != row_dims.end();
    const std::vector<int>& role = in_x ? row_dims : col_dims;
    const size_t slot = (size_t)(std::find(role.begin(), role.end(), d) - role.begin());
    int64_t stride = 1;
    for (size_t e = slot + 1; e < role.size(); e++) stride *= extent[role[e]];
    okeys.key[okeys.n] = KeyAt{in_x ? 1 : 0, stride, std::max<int64_t>(extent[d], 1)};
    okeys.width[okeys.n] = width_of(fields[key.col].kind);
    okeys.n++;
  }
  DeviceBuffer<int64_t> xtab((size_t)std::max<int64_t>(okeys.n * rows, 1), s),
      ytab((size_t)std::max<int64_t>(okeys.n * cols, 1), s);
  if (rows) key_tables<<<blocks_for((uint64_t)rows, 256), 256, 0, s>>>(rows, okeys, 1, xtab.get());
  if (cols) key_tables<<<blocks_for((uint64_t)cols, 256), 256, 0, s>>>(cols, okeys, 0, ytab.get());
  ctx.kernels += 2;
  std::vector<DeviceBuffer<uint8_t>> key_dev;
  for (int i = 0; i < okeys.n; i++) {
    key_dev.emplace_back((size_t)(n_out ? n_out * okeys.width[i] : 1), s);
    okeys.out[i] = key_dev.back().get();
  }
  DeviceBuffer<double> vals((size_t)(n_out ? n_out : 1), s);
  if (n_out) {
    emit_rows<<<blocks_for((uint64_t)rows * cols, 256), 256, 0, s>>>(rows, cols, flags.get(), row_index.get(), okeys,
                                                                      xtab.get(), ytab.get(), mat, vals.get());
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  OutBatch ob;
  ob.rows = n_out;
  for (int i = 0; i < okeys.n; i++) {
    const Field& f = fields[op.keys[i].col];
    OutColumn c;
    c.format = f.format;
    c.name = f.name;
    c.kind = f.kind;
    c.nullable = f.nullable;
    c.length = n_out;
    c.values = result_buffer(ctx, key_dev[i], (size_t)(n_out * okeys.width[i]), on_device);
    ob.columns.push_back(std::move(c));
  }
  OutColumn val;
  val.format = "g";
  val.kind = Kind::Float64;
  val.name = "grad";
  val.nullable = true;
  val.length = n_out;
  val.values = result_buffer(ctx, vals, (size_t)n_out * 8, on_device);
  ob.columns.push_back(std::move(val));
  return ob;
}

}  // namespace

std::vector<Field> gradient_schema(const OperandD& op, const std::vector<Field>& fields) {
  std::vector<Field> out;
  for (auto& key : op.keys) out.push_back(fields[key.col]);
  Field g;
  g.format = "g";
  g.kind = Kind::Float64;
  g.nullable = true;
  g.name = "grad";
  out.push_back(g);
  return out;
}

GradientOutput pipeline_backward(Context& ctx, const PipelineD& p, const Relation& q, const Relation& k,
                                 const Relation& v, const Relation& d_out, const einfold_options& o) {
  cudaStream_t s = ctx.stream;
  const FoldD& pr = p.producer;
  if (pr.row_expr || p.weight_expr || p.shift != 1 || p.normalizer != 0 || p.scale_kind == 2)
    decline("a backward pass only for product scores, exp(s - MAX(s)) weights, scaled by one or times c, "
            "normalised over the kept groups");
  PlacedPipeline P = place_pipeline(ctx, p, q, k, v, true);
  const uint64_t nx = P.nx, ne = P.ne, nj = P.nj, ny = P.ny;
  const int64_t W = P.mask.lnx > 0 ? (int64_t)nx / P.mask.lnx : 0;
  if (W * P.mask.lnx != (int64_t)nx || W * P.mask.lnj != (int64_t)nj) decline("groups that aren't batches");
  if (P.matrices.size() != 3) decline("a producer reading more than one column an operand");
  // d_out: the result's keys (p.outputs, in order) and the gradient of each
  // result row, placed as out is, [x][y]; rows of no d_out row have 0.
  const int n_out_cols = (int)p.outputs.size();
  if ((int)d_out.fields.size() != n_out_cols + 1) fail(EINFOLD_INVALID, "d_out needs the result's key columns and one gradient column");
  const Field& gf = d_out.fields[(size_t)n_out_cols];
  if (gf.dictionary || gf.kind != Kind::Float64) fail(EINFOLD_INVALID, "d_out's gradient column must be DOUBLE");
  OperandD dop;
  for (int i = 0; i < n_out_cols; i++) dop.keys.push_back(KeyD{p.outputs[(size_t)i], i});
  dop.factor = n_out_cols;
  StagedKeys dk = stage_keys(ctx, dop, d_out);
  for (size_t i = 0; i < dop.keys.size(); i++)
    if (dk.extent[i] > P.extent[(size_t)dop.keys[i].dim]) decline("a d_out row of no result row");
  uint64_t cells = 0;
  if (!checked_mul(nx, ny, &cells) || cells >= UINT32_MAX) decline("an output of 2^32 cells or more");
  DeviceBuffer<double> g_out((size_t)std::max<uint64_t>(cells, 1), s);
  g_out.zero();
  {
    int64_t rows = 0;
    for (auto& b : d_out.batches) rows += b.rows;
    for (auto& b : d_out.batches)
      if (b.columns[(size_t)n_out_cols].nulls() > 0) decline("a NULL gradient");
    DeviceColumn col = stage_column(ctx, d_out, n_out_cols, false);
    DeviceBuffer<unsigned> held((size_t)std::max<uint64_t>((cells + 31) / 32, 1), s);
    DeviceBuffer<unsigned> dup(1, s);
    held.zero();
    dup.zero();
    if (rows) {
      const Role rr = role_of(P.xs, dop, dk, P.extent);
      const Role cr = role_of(P.ys, dop, dk, P.extent);
      place_kernel<<<blocks_for((uint64_t)rows, 256), 256, 0, s>>>(rr, cr, rows, (int64_t)ny, (const double*)col.ptr(),
                                                                   g_out.get(), held.get(), dup.get());
      ctx.kernels++;
      EF_LAUNCH_CHECK();
    }
    unsigned d = 0;
    EF_CUDA(cudaMemcpyAsync(&d, dup.get(), 4, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    if (d) decline("d_out with a repeated row");
  }
  // The forward pass again, for out and the rows' log-sum-exp.
  AttentionProblem ap;
  ap.q = P.matrices[0].get();
  ap.k = P.matrices[1].get();
  ap.v = P.matrices[2].get();
  ap.batches = W;
  ap.lnx = P.mask.lnx;
  ap.lnj = P.mask.lnj;
  ap.ne = (int64_t)ne;
  ap.ny = (int64_t)ny;
  ap.mask = P.mask;
  ap.scale_kind = p.scale_kind;
  ap.scale_c = p.scale_c;
  ap.xlen_host = P.xlen;
  ap.jlen_host = P.jlen;
  DeviceBuffer<double> out((size_t)std::max<uint64_t>(cells, 1), s), lse((size_t)std::max<uint64_t>(nx, 1), s);
  out.zero();
  lse.zero();
  ap.out = out.get();
  ap.lse = lse.get();
  if (attention_forward(ctx, ap, o.precision, o.slices, s) == ATTENTION_GUARDED)
    decline("a sum that overflowed or may have underflowed");
  AttentionGradients g;
  g.f = ap;
  g.out = out.get();
  g.lse = lse.get();
  g.d_out = g_out.get();
  DeviceBuffer<double> dq((size_t)std::max<uint64_t>(nx * ne, 1), s), dkm((size_t)std::max<uint64_t>(nj * ne, 1), s),
      dv((size_t)std::max<uint64_t>(nj * ny, 1), s);
  dq.zero();
  dkm.zero();
  dv.zero();
  g.d_q = dq.get();
  g.d_k = dkm.get();
  g.d_v = dv.get();
  Budget budget;
  budget.o = &o;
  g.budget = &budget;
  attention_backward(ctx, g, o.precision, s);
  ctx.phase("fused backward: gradients");
  GradientOutput r;
  const OperandD* ops[3] = {&pr.operands[0], &pr.operands[1], &p.values};
  const Relation* rels[3] = {&q, &k, &v};
  const double* mats[3] = {dq.get(), dkm.get(), dv.get()};
  const std::vector<int>* rdims[3] = {&P.xs, &P.js, &P.js};
  const std::vector<int>* cdims[3] = {&P.es, &P.es, &P.ys};
  const uint64_t nrows[3] = {nx, nj, nj}, ncols[3] = {ne, ne, ny};
  for (int i = 0; i < 3; i++) {
    const bool along_x = i == 0;
    const int64_t* len = P.xlen.empty() ? nullptr : (along_x ? P.xlen_dev.get() : P.jlen_dev.get());
    r.schemas[i] = gradient_schema(*ops[i], rels[i]->fields);
    r.batches[i].push_back(emit_matrix(ctx, *ops[i], rels[i]->fields, *rdims[i], *cdims[i], P.extent, mats[i],
                                       (int64_t)nrows[i], (int64_t)ncols[i], along_x ? P.mask.lnx : P.mask.lnj, len,
                                       o.result_on_device != 0));
  }
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("fused backward: result");
  return r;
}

AttentionOutcome attention_forward(Context& ctx, AttentionProblem p, int precision, int slices, cudaStream_t s) {
  const int64_t nx = p.batches * p.lnx, nj = p.batches * p.lnj;
  if (nx == 0 || p.ny == 0) return ATTENTION_DONE;
  DeviceBuffer<uint8_t> jflag((size_t)std::max<int64_t>(nj, 1), s);
  DeviceBuffer<double> largest((size_t)std::max<int64_t>(nj, 1), s), smallest((size_t)std::max<int64_t>(nj, 1), s);
  DeviceBuffer<unsigned> nonfinite(1, s);
  nonfinite.zero();
  if (nj) {
    value_stats<<<blocks_for(nj * 32, 256), 256, 0, s>>>(nj, p.ny, p.v, jflag.get(), largest.get(), smallest.get(),
                                                         nonfinite.get(), p.lnj, p.mask.jlen);
    ctx.kernels++;
    EF_LAUNCH_CHECK();
  }
  unsigned v_nonfinite = 0;
  EF_CUDA(cudaMemcpyAsync(&v_nonfinite, nonfinite.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  p.largest = largest.get();
  p.smallest = smallest.get();
  if (precision == 0 && !v_nonfinite && nj > 0) {
    const AttentionOutcome r = attention_split(ctx, p, slices > 0 ? slices : 6, s);
    if (r != ATTENTION_INELIGIBLE) return r;
  }
  if (!v_nonfinite && nj > 0 && !fp64_tiles_requested()) {
    const AttentionOutcome r = attention_f64_mma(ctx, p, s);
    if (r != ATTENTION_INELIGIBLE) return r;
  }
  TileArgs a{};
  a.nx = nx;
  a.ne = p.ne;
  a.nj = nj;
  a.ny = p.ny;
  a.mask = p.mask;
  a.scale_kind = p.scale_kind;
  a.scale_c = p.scale_c;
  a.shifted = 1;
  a.normalizer = 0;
  a.q = p.q;
  a.k = p.k;
  a.v = p.v;
  a.jflag = jflag.get();
  a.largest = largest.get();
  a.smallest = smallest.get();
  a.out = p.out;
  a.lse = p.lse;
  DeviceBuffer<unsigned long long> visited(1, s);
  DeviceBuffer<unsigned> overflowed(1, s);
  visited.zero();
  overflowed.zero();
  a.visited = visited.get();
  a.overflowed = overflowed.get();
  const dim3 grid((unsigned)((nx + XT - 1) / XT), (unsigned)((p.ny + YC - 1) / YC));
  launch_tiles(a, 0, grid, s);
  ctx.kernels++;
  unsigned of = 0;
  EF_CUDA(cudaMemcpyAsync(&of, overflowed.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("attention: fp64 tiles");
  return of ? ATTENTION_GUARDED : ATTENTION_DONE;
}

}  // namespace ef
