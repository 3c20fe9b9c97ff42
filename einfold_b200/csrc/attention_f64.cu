// The FP64 form of the attention forward pass on the FP64 tensor pipe: the
// pipeline einfold_pipeline runs for product scores, weights exp(s - m) with
// m the row's largest score, and an average normalised by the weights' sum
// (fused.rs:694-1019), for finite operands, with q·k and w·v as FP64
// mma.sync (m16n8k8) products and the online softmax in FP64 registers.
//
// A block takes 64 query rows of one batch (four warps of 16 rows) and 64
// value columns, and walks the batch's key tiles of 32 that its rows may
// join (tiles no row joins are never loaded). Per tile, each warp computes
// its 16 x 32 scores (S = Q·Kᵀ from shared memory), masks them by each row's
// allowed interval, rescales its running sums by exp(m_old - m_new), and
// adds P·V for its 16 rows. A row's four lanes exchange maxima by shuffles.
// The P fragments feed the second product from the accumulator registers:
// column 2t (2t + 1) of a score tile is taken as column t (t + 4) of the
// product's A operand, and V's rows are read in the same order, so no lane
// exchanges its scores. K and V tiles arrive by cp.async into two stages.
//
// Guards: the reference's overflow test and Bounds::hold (fused.rs:1024-1086)
// per row, as the split form applies them: the heaviest weight is 1, the
// lightest exp(min s - m), the values' bounds from the rows' allowed ranges.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "attention.cuh"
#include "fastexp.cuh"
#include "ptx.cuh"

namespace ef {

// EINFOLD_FP64_TILES=1 keeps the FP64 form on the CUDA cores' tile kernels.
bool fp64_tiles_requested() {
  static const bool on = [] {
    const char* e = std::getenv("EINFOLD_FP64_TILES");
    return e && e[0] == '1';
  }();
  return on;
}

namespace {

constexpr int FM = 64;   // query rows a block: four warps of 16
constexpr int FN = 32;   // keys a tile
constexpr int FY = 64;   // value columns a block
constexpr int VS = 66;   // the shared-memory stride of V's rows, in doubles (conflict-free fragment reads)
constexpr int kF64Threads = 128;
constexpr int kMaxFeatures = 128;

struct F64Args {
  const double* q;
  const double* k;
  const double* v;
  double* out;
  double* lse;
  int64_t lnx, lnj, ne, ny;
  Mask mask;
  int scale_kind;
  double scale_c;
  const double* rl;  // each row's largest and smallest nonzero value magnitude (Bounds::hold)
  const double* rs;
  const double* exp_table;
  int* status;  // bit 0: a guard fired
  unsigned long long* pairs;  // tile pairs (64 x 32) computed
  int stride;   // the shared-memory stride of q's and k's rows, in doubles
};

__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double a2, double a3, double b0,
                                     double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(ptx::smem_u32(dst)), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ASYNC: q's and k's rows (ne) and v's (ny) of even length and 16-byte
// aligned operands, so that tiles move in 16-byte cp.async copies; else
// element by element.
template <bool ASYNC>
__global__ void __launch_bounds__(kF64Threads, 2) attn_fwd_f64(const F64Args a) {
  extern __shared__ __align__(16) double sm[];
  const int stride = a.stride;
  double* sQ = sm;                       // [FM][stride]
  double* sK = sQ + FM * stride;         // [2][FN][stride]
  double* sV = sK + 2 * FN * stride;     // [2][FN][VS]
  __shared__ double texp[64];
  __shared__ long long span[2];
  __shared__ long long lo_s[FM], hi_s[FM];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int64_t w = blockIdx.y;
  const int64_t x0 = (int64_t)blockIdx.x * FM;
  const int y0 = blockIdx.z * FY;
  const int64_t r_base = w * a.lnx, c_base = w * a.lnj;
  const int ne8 = (int)((a.ne + 7) & ~7LL);
  if (tid < 64) texp[tid] = a.exp_table[tid];
  if (tid == 0) {
    span[0] = LLONG_MAX;
    span[1] = LLONG_MIN;
  }
  __syncthreads();
  if (tid < FM) {
    const int64_t xl = x0 + tid;
    int64_t lo = 0, hi = 0;
    if (xl < a.lnx) {
      allowed(a.mask, r_base + xl, lo, hi);
      lo -= c_base;
      hi -= c_base;
    }
    if (lo >= hi) lo = hi = 0;
    lo_s[tid] = lo;
    hi_s[tid] = hi;
    if (lo < hi) {
      atomicMin(&span[0], lo);
      atomicMax(&span[1], hi);
    }
  }
  for (int i = tid; i < FM * ne8; i += kF64Threads) {
    const int r = i / ne8, c = i - r * ne8;
    const int64_t xl = x0 + r;
    sQ[r * stride + c] = (xl < a.lnx && c < a.ne) ? a.q[(r_base + xl) * a.ne + c] : 0.0;
  }
  __syncthreads();
  const long long first = span[0], last = span[1];
  const int64_t t0 = first < last ? first / FN : 0;
  const int n_tiles = first < last ? (int)((last + FN - 1) / FN - t0) : 0;
  if (tid == 0 && n_tiles > 0) atomicAdd(a.pairs, (unsigned long long)n_tiles);

  // Tile `it`'s keys and values into stage `b` (zeros past the batch's keys,
  // the features and the value columns).
  auto load = [&](int it, int b) {
    const int64_t j0 = (t0 + it) * FN;
    double* k_s = sK + b * FN * stride;
    double* v_s = sV + b * FN * VS;
    if (ASYNC) {
      const int kc = ne8 / 2;  // 16-byte chunks of a key row
      for (int i = tid; i < FN * kc; i += kF64Threads) {
        const int r = i / kc, c = 2 * (i - r * kc);
        const bool in = j0 + r < a.lnj && c < a.ne;
        const double* src = in ? a.k + (c_base + j0 + r) * a.ne + c : a.k;
        cp_async16(k_s + r * stride + c, src, in ? 16 : 0);
      }
      for (int i = tid; i < FN * (FY / 2); i += kF64Threads) {
        const int r = i / (FY / 2), c = 2 * (i - r * (FY / 2));
        const bool in = j0 + r < a.lnj && y0 + c < a.ny;
        const double* src = in ? a.v + (c_base + j0 + r) * a.ny + y0 + c : a.v;
        cp_async16(v_s + r * VS + c, src, in ? 16 : 0);
      }
    } else {
      for (int i = tid; i < FN * ne8; i += kF64Threads) {
        const int r = i / ne8, c = i - r * ne8;
        k_s[r * stride + c] = (j0 + r < a.lnj && c < a.ne) ? a.k[(c_base + j0 + r) * a.ne + c] : 0.0;
      }
      for (int i = tid; i < FN * FY; i += kF64Threads) {
        const int r = i / FY, c = i - r * FY;
        v_s[r * VS + c] = (j0 + r < a.lnj && y0 + c < a.ny) ? a.v[(c_base + j0 + r) * a.ny + y0 + c] : 0.0;
      }
    }
  };

  const int r0 = warp * 16 + g, r1 = r0 + 8;  // this lane's two rows
  const long long lo0 = lo_s[r0], hi0 = hi_s[r0], lo1 = lo_s[r1], hi1 = hi_s[r1];
  double o[FY / 8][4];
#pragma unroll
  for (int n = 0; n < FY / 8; n++) o[n][0] = o[n][1] = o[n][2] = o[n][3] = 0.0;
  double m[2] = {-INFINITY, -INFINITY}, l[2] = {0.0, 0.0}, light[2] = {INFINITY, INFINITY};
  const double c_times = a.scale_kind == 1 ? a.scale_c : 1.0;

  if (n_tiles > 0) {
    load(0, 0);
    cp_commit();
  }
  for (int it = 0; it < n_tiles; it++) {
    const int b = it & 1;
    if (it + 1 < n_tiles) {
      load(it + 1, b ^ 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const double* k_s = sK + b * FN * stride;
    const double* v_s = sV + b * FN * VS;
    // Scores: this warp's 16 rows against the tile's 32 keys.
    double s[FN / 8][4];
#pragma unroll
    for (int n = 0; n < FN / 8; n++) s[n][0] = s[n][1] = s[n][2] = s[n][3] = 0.0;
    for (int kk = 0; kk < ne8; kk += 8) {
      const double a0 = sQ[r0 * stride + kk + t], a1 = sQ[r1 * stride + kk + t];
      const double a2 = sQ[r0 * stride + kk + t + 4], a3 = sQ[r1 * stride + kk + t + 4];
#pragma unroll
      for (int n = 0; n < FN / 8; n++) {
        const double* kr = k_s + (n * 8 + g) * stride + kk;
        dmma(s[n], a0, a1, a2, a3, kr[t], kr[t + 4]);
      }
    }
    // Scale, mask, the rows' maxima over the tile.
    const long long j0 = (t0 + it) * FN;
    double mx[2] = {-INFINITY, -INFINITY};
#pragma unroll
    for (int n = 0; n < FN / 8; n++)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const long long j = j0 + n * 8 + 2 * t + (i & 1);
        const bool row1 = i >= 2;
        const bool ok = row1 ? (j >= lo1 && j < hi1) : (j >= lo0 && j < hi0);
        double x = a.scale_kind == 2 ? __ddiv_rn(s[n][i], a.scale_c) : s[n][i] * c_times;
        s[n][i] = ok ? x : -INFINITY;
        mx[row1] = fmax(mx[row1], s[n][i]);
        if (ok) light[row1] = fmin(light[row1], x);
      }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      mx[h] = fmax(mx[h], __shfl_xor_sync(0xffffffffu, mx[h], 1));
      mx[h] = fmax(mx[h], __shfl_xor_sync(0xffffffffu, mx[h], 2));
    }
    double alpha[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const double mn = fmax(m[h], mx[h]);
      alpha[h] = (m[h] == mn) ? 1.0 : (m[h] == -INFINITY ? 0.0 : exp_tang(m[h] - mn, texp));
      m[h] = mn;
      l[h] *= alpha[h];
    }
#pragma unroll
    for (int n = 0; n < FN / 8; n++)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int h = i >= 2;
        const double p = s[n][i] == -INFINITY ? 0.0 : exp_tang(s[n][i] - m[h], texp);
        s[n][i] = p;
        l[h] += p;
      }
#pragma unroll
    for (int n = 0; n < FY / 8; n++) {
      o[n][0] *= alpha[0];
      o[n][1] *= alpha[0];
      o[n][2] *= alpha[1];
      o[n][3] *= alpha[1];
    }
    // out += P · V: score column 2t (2t + 1) of key group kk is the A
    // operand's column t (t + 4), and V's rows are read in that order.
#pragma unroll
    for (int kk = 0; kk < FN / 8; kk++) {
      const double* v0 = v_s + (kk * 8 + 2 * t) * VS;
      const double* v1 = v0 + VS;
#pragma unroll
      for (int n = 0; n < FY / 8; n++) dmma(o[n], s[kk][0], s[kk][2], s[kk][1], s[kk][3], v0[n * 8 + g], v1[n * 8 + g]);
    }
    __syncthreads();  // the stage is free for tile it + 2
  }

  // The rows' sums of weights over their four lanes; normalise, guard, store.
#pragma unroll
  for (int h = 0; h < 2; h++) {
    l[h] += __shfl_xor_sync(0xffffffffu, l[h], 1);
    l[h] += __shfl_xor_sync(0xffffffffu, l[h], 2);
    light[h] = fmin(light[h], __shfl_xor_sync(0xffffffffu, light[h], 1));
    light[h] = fmin(light[h], __shfl_xor_sync(0xffffffffu, light[h], 2));
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = h ? r1 : r0;
    const int64_t xl = x0 + r;
    const long long lo = h ? lo1 : lo0, hi = h ? hi1 : hi0;
    if (xl >= a.lnx || lo >= hi) continue;
    const double z = l[h];
    // Bounds::hold (fused.rs:1058-1086) with the heaviest weight 1.
    const double rl = a.rl[r_base + xl], rs = a.rs[r_base + xl];
    bool over = !(z <= 1.7976931348623157e308);
    const double normal = 2.0 * 2.2250738585072014e-308;
    const double lightest = exp(light[h] - m[h]);
    const double t2 = 2.0 * (double)(hi - lo);
    bool finite = isfinite(rl * t2);
    if (finite) {
      const double quotient = 1.0 / fabs(z);
      finite = isfinite(quotient) && isfinite(quotient * rl * t2);
    }
    const double lost = (t2 * 4.9406564584124654e-324) * ((1.0 / fabs(z) + rl) + 1.0);
    bool no_underflow = rs == INFINITY;
    if (!no_underflow) {
      no_underflow = lightest * rs >= normal;
      if (no_underflow) {
        const double quotient = lightest / fabs(z);
        no_underflow = quotient >= normal && quotient * rs >= normal;
      }
    }
    if (!finite) over = true;
    const double rounding = 2.220446049250313e-16 / 4.0;
    double* orow = a.out + (r_base + xl) * a.ny;
#pragma unroll
    for (int n = 0; n < FY / 8; n++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int64_t y = (int64_t)y0 + n * 8 + 2 * t + e;
        if (y >= a.ny) continue;
        const double acc = o[n][2 * h + e];
        if (!isfinite(acc)) over = true;
        const double val = __ddiv_rn(acc, z);
        if (!isfinite(val)) over = true;
        if (!no_underflow && !(lost <= rounding * fabs(val))) over = true;
        orow[y] = val;
      }
    if (t == 0 && a.lse && y0 == 0) a.lse[r_base + xl] = m[h] + log(z);
    if (over) atomicOr(a.status, 1);
  }
}

// Whether every value is finite, and the largest magnitude (as the bits of
// a non-negative double, which order as the values do).
__global__ void finite_max(const double* __restrict__ x, int64_t n, int* bad, unsigned long long* largest) {
  bool ok = true;
  double mx = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    ok &= isfinite(v);
    mx = fmax(mx, fabs(v));
  }
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (!__all_sync(0xffffffffu, ok) && (threadIdx.x & 31) == 0) atomicOr(bad, 1);
  if ((threadIdx.x & 31) == 0 && mx > 0.0) atomicMax(largest, (unsigned long long)__double_as_longlong(mx));
}

// ---- The backward pass on the FP64 tensor pipe -----------------------------
//
// Two kernels, as FlashAttention-2's backward: one with keys as rows (128 a
// block, eight warps of 16) walking the query tiles of 32 its keys are
// joined by, recomputing S^T = K·Q^T, P^T = exp(S^T - lse), dP^T = V·dO^T and
// dS^T = P^T (dP^T - D), and summing dV += P^T·dO and dK += dS^T·Q in
// registers; one with queries as rows walking their key tiles, recomputing
// S, P, dP and dS and summing dQ += dS·K. P and dS feed the second products
// from the accumulators (column 2t, 2t + 1 as the A operand's t, t + 4; the
// B operand's rows read in that order). Every output row is summed by one
// block, in tile order: no atomics. For d, dv <= 64.

constexpr int BR = 128;  // rows a block: eight warps of 16
constexpr int BC = 32;   // columns (queries or keys) a tile
constexpr int kBwdThreads = 256;
constexpr int RS = 68;   // shared-memory stride of the blocks' own rows
constexpr int CS = 66;   // shared-memory stride of a tile's rows

struct F64BwdArgs {
  const double* a1;  // rows' operand of the first product (k or q), [w·lr + r][d1]
  const double* a2;  // rows' operand of the second (v or d_out), [w·lr + r][d2]
  const double* b1;  // tiles' operand of the first (q or k), [w·lc + c][d1]
  const double* b2;  // tiles' operand of the second (d_out or v), [w·lc + c][d2]
  const double* lse;  // per query
  const double* dd;   // D per query
  double* out1;  // kv: d_v [rows][d2]; q: d_q [rows][d1]
  double* out2;  // kv: d_k [rows][d1]
  int64_t lr, lc, d1, d2;
  Mask mask;  // rows' allowed columns
  double scale;
  const double* exp_table;
  int keys_rows;  // 1: rows are keys (lse, D per column); 0: rows are queries
};

// Rows [r0, r0 + n) of a row-major matrix of `cols` columns into shared
// memory at `stride`, zeros past `valid` rows and `cols` columns, `width`
// (a multiple of 8) columns wide.
template <bool ASYNC>
__device__ __forceinline__ void load_rows(double* dst, int stride, const double* src, int64_t r0, int n, int64_t valid,
                                          int64_t cols, int width) {
  if (ASYNC) {
    const int kc = width / 2;
    for (int i = threadIdx.x; i < n * kc; i += kBwdThreads) {
      const int r = i / kc, c = 2 * (i - r * kc);
      const bool in = r0 + r < valid && c < cols;
      cp_async16(dst + r * stride + c, in ? src + (r0 + r) * cols + c : src, in ? 16 : 0);
    }
  } else {
    for (int i = threadIdx.x; i < n * width; i += kBwdThreads) {
      const int r = i / width, c = i - r * width;
      dst[r * stride + c] = (r0 + r < valid && c < cols) ? src[(r0 + r) * cols + c] : 0.0;
    }
  }
}

// KV: rows are keys (out1 = d_v, out2 = d_k); else rows are queries (out1 = d_q).
template <bool KV, bool ASYNC>
__global__ void __launch_bounds__(kBwdThreads, 1) attn_bwd_f64(const F64BwdArgs a) {
  extern __shared__ __align__(16) double sm[];
  double* sA1 = sm;                  // [BR][RS]
  double* sA2 = sA1 + BR * RS;       // [BR][RS]
  double* sB = sA2 + BR * RS;        // [2][b1 | b2] tiles, [BC][CS] each
  double* sLD = sB + 4 * BC * CS;    // [2][lse | D] of the tile's columns (KV)
  __shared__ double texp[64];
  __shared__ long long span[2];
  __shared__ long long lo_s[BR], hi_s[BR];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int64_t w = blockIdx.y;
  const int64_t x0 = (int64_t)blockIdx.x * BR;
  const int64_t r_base = w * a.lr, c_base = w * a.lc;
  const int w1 = (int)((a.d1 + 7) & ~7LL), w2 = (int)((a.d2 + 7) & ~7LL);
  if (tid < 64) texp[tid] = a.exp_table[tid];
  if (tid == 0) {
    span[0] = LLONG_MAX;
    span[1] = LLONG_MIN;
  }
  __syncthreads();
  if (tid < BR) {
    const int64_t xl = x0 + tid;
    int64_t lo = 0, hi = 0;
    if (xl < a.lr) {
      allowed(a.mask, r_base + xl, lo, hi);
      lo -= c_base;
      hi -= c_base;
    }
    if (lo >= hi) lo = hi = 0;
    lo_s[tid] = lo;
    hi_s[tid] = hi;
    if (lo < hi) {
      atomicMin(&span[0], lo);
      atomicMax(&span[1], hi);
    }
  }
  load_rows<ASYNC>(sA1, RS, a.a1 + r_base * a.d1, x0, BR, a.lr, a.d1, w1);
  load_rows<ASYNC>(sA2, RS, a.a2 + r_base * a.d2, x0, BR, a.lr, a.d2, w2);
  if (ASYNC) cp_commit();
  __syncthreads();
  const long long first = span[0], last = span[1];
  const int64_t t0 = first < last ? first / BC : 0;
  const int n_tiles = first < last ? (int)((last + BC - 1) / BC - t0) : 0;

  auto load = [&](int it, int b) {
    const int64_t j0 = (t0 + it) * BC;
    double* b1 = sB + b * 2 * BC * CS;
    double* b2 = b1 + BC * CS;
    load_rows<ASYNC>(b1, CS, a.b1 + c_base * a.d1, j0, BC, a.lc, a.d1, w1);
    load_rows<ASYNC>(b2, CS, a.b2 + c_base * a.d2, j0, BC, a.lc, a.d2, w2);
    if (KV && tid < 2 * BC) {
      // The tile's queries' lse and D.
      const int c = tid & (BC - 1);
      const int64_t q = j0 + c;
      const double* srcp = tid < BC ? a.lse : a.dd;
      sLD[b * 2 * BC + tid] = q < a.lc ? srcp[c_base + q] : 0.0;
    }
  };

  const int r0 = warp * 16 + g, r1 = r0 + 8;
  const long long lo0 = lo_s[r0], hi0 = hi_s[r0], lo1 = lo_s[r1], hi1 = hi_s[r1];
  // Queries as rows: their own lse and D.
  double lse_r[2] = {0.0, 0.0}, dd_r[2] = {0.0, 0.0};
  if (!KV) {
    if (x0 + r0 < a.lr) {
      lse_r[0] = a.lse[r_base + x0 + r0];
      dd_r[0] = a.dd[r_base + x0 + r0];
    }
    if (x0 + r1 < a.lr) {
      lse_r[1] = a.lse[r_base + x0 + r1];
      dd_r[1] = a.dd[r_base + x0 + r1];
    }
  }
  double o1[8][4], o2[8][4];  // KV: d_v, d_k; else d_q in o1
#pragma unroll
  for (int n = 0; n < 8; n++)
#pragma unroll
    for (int i = 0; i < 4; i++) o1[n][i] = o2[n][i] = 0.0;

  if (n_tiles > 0) {
    load(0, 0);
    if (ASYNC) cp_commit();
  }
  for (int it = 0; it < n_tiles; it++) {
    const int b = it & 1;
    if (it + 1 < n_tiles) {
      load(it + 1, b ^ 1);
      if (ASYNC) {
        cp_commit();
        cp_wait<1>();
      }
    } else if (ASYNC) {
      cp_wait<0>();
    }
    __syncthreads();
    const double* b1 = sB + b * 2 * BC * CS;
    const double* b2 = b1 + BC * CS;
    const double* ld = sLD + b * 2 * BC;
    double s[BC / 8][4], dp[BC / 8][4];
#pragma unroll
    for (int n = 0; n < BC / 8; n++)
#pragma unroll
      for (int i = 0; i < 4; i++) s[n][i] = dp[n][i] = 0.0;
    for (int kk = 0; kk < w1; kk += 8) {
      const double x0a = sA1[r0 * RS + kk + t], x1a = sA1[r1 * RS + kk + t];
      const double x2a = sA1[r0 * RS + kk + t + 4], x3a = sA1[r1 * RS + kk + t + 4];
#pragma unroll
      for (int n = 0; n < BC / 8; n++) {
        const double* br = b1 + (n * 8 + g) * CS + kk;
        dmma(s[n], x0a, x1a, x2a, x3a, br[t], br[t + 4]);
      }
    }
    for (int kk = 0; kk < w2; kk += 8) {
      const double x0a = sA2[r0 * RS + kk + t], x1a = sA2[r1 * RS + kk + t];
      const double x2a = sA2[r0 * RS + kk + t + 4], x3a = sA2[r1 * RS + kk + t + 4];
#pragma unroll
      for (int n = 0; n < BC / 8; n++) {
        const double* br = b2 + (n * 8 + g) * CS + kk;
        dmma(dp[n], x0a, x1a, x2a, x3a, br[t], br[t + 4]);
      }
    }
    // P = exp(scale·s - lse) on allowed pairs, dS = P (dP - D).
    const long long j0 = (t0 + it) * BC;
#pragma unroll
    for (int n = 0; n < BC / 8; n++)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int c = n * 8 + 2 * t + (i & 1);
        const long long j = j0 + c;
        const bool row1 = i >= 2;
        const bool ok = row1 ? (j >= lo1 && j < hi1) : (j >= lo0 && j < hi0);
        const double lse = KV ? ld[c] : lse_r[row1];
        const double dd = KV ? ld[BC + c] : dd_r[row1];
        // Pairs outside the mask weigh nothing, whatever lse and D hold there
        // (rows that join no key have neither).
        const double p = ok ? exp_tang(a.scale * s[n][i] - lse, texp) : 0.0;
        s[n][i] = p;
        dp[n][i] = ok ? p * (dp[n][i] - dd) : 0.0;
      }
    // KV: d_v += P^T·dO (o1), d_k += dS^T·Q (o2); else d_q += dS·K (o1).
#pragma unroll
    for (int kk = 0; kk < BC / 8; kk++) {
      if (KV) {
        const double* v0 = b2 + (kk * 8 + 2 * t) * CS;
        const double* v1 = v0 + CS;
#pragma unroll
        for (int n = 0; n < 8; n++)
          if (n * 8 < w2) dmma(o1[n], s[kk][0], s[kk][2], s[kk][1], s[kk][3], v0[n * 8 + g], v1[n * 8 + g]);
      }
      const double* k0 = b1 + (kk * 8 + 2 * t) * CS;
      const double* k1 = k0 + CS;
#pragma unroll
      for (int n = 0; n < 8; n++)
        if (n * 8 < w1) {
          if (KV) dmma(o2[n], dp[kk][0], dp[kk][2], dp[kk][1], dp[kk][3], k0[n * 8 + g], k1[n * 8 + g]);
          else dmma(o1[n], dp[kk][0], dp[kk][2], dp[kk][1], dp[kk][3], k0[n * 8 + g], k1[n * 8 + g]);
        }
    }
    __syncthreads();
  }
  // Store: rows of this block (zeros for rows that join nothing).
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int64_t xl = x0 + (h ? r1 : r0);
    if (xl >= a.lr) continue;
#pragma unroll
    for (int n = 0; n < 8; n++)
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int64_t c = n * 8 + 2 * t + e;
        if (KV) {
          if (c < a.d2) a.out1[(r_base + xl) * a.d2 + c] = o1[n][2 * h + e];
          if (c < a.d1) a.out2[(r_base + xl) * a.d1 + c] = a.scale * o2[n][2 * h + e];
        } else if (c < a.d1) {
          a.out1[(r_base + xl) * a.d1 + c] = a.scale * o1[n][2 * h + e];
        }
      }
  }
}

}  // namespace

AttentionOutcome attention_f64_mma(Context& ctx, const AttentionProblem& p, cudaStream_t s) {
  const int64_t W = p.batches, nx = W * p.lnx, nj = W * p.lnj;
  if (p.ne <= 0 || p.ne > kMaxFeatures || W > 65535 || p.ny <= 0 || fp64_tiles_requested()) return ATTENTION_INELIGIBLE;
  if ((p.ny + FY - 1) / FY > 65535) return ATTENTION_INELIGIBLE;
  // Finite q and k (v's finiteness the caller's statistics give): non-finite
  // scores take the FP64 tile kernel, which keeps their NaN and infinity rules.
  // And no score near overflow: |s| <= ne · max|q| · max|k| (times the scale).
  DeviceBuffer<int> flags(2, s);
  DeviceBuffer<unsigned long long> largest(2, s);
  flags.zero();
  largest.zero();
  finite_max<<<blocks_for((uint64_t)(nx * p.ne), 256), 256, 0, s>>>(p.q, nx * p.ne, flags.get(), largest.get());
  finite_max<<<blocks_for((uint64_t)(nj * p.ne), 256), 256, 0, s>>>(p.k, nj * p.ne, flags.get(), largest.get() + 1);
  ctx.kernels += 2;
  EF_LAUNCH_CHECK();
  int bad = 0;
  unsigned long long mq_bits = 0, mk_bits = 0;
  EF_CUDA(cudaMemcpyAsync(&bad, flags.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&mq_bits, largest.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&mk_bits, largest.get() + 1, 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  if (bad) return ATTENTION_INELIGIBLE;
  double mq, mk;
  std::memcpy(&mq, &mq_bits, 8);
  std::memcpy(&mk, &mk_bits, 8);
  const double scale = p.scale_kind == 1 ? std::fabs(p.scale_c) : (p.scale_kind == 2 ? 1.0 / std::fabs(p.scale_c) : 1.0);
  if (!(mq * mk * (double)p.ne * std::max(scale, 1.0) < 1e300)) return ATTENTION_INELIGIBLE;

  DeviceBuffer<double> bounds((size_t)(2 * nx + 2 * ((nj + 63) / 64) + 1), s);
  double* rl = bounds.get();
  double* rs = rl + nx;
  double* bmax = rs + nx;
  double* bmin = bmax + (nj + 63) / 64;
  if (nj) block_extrema<<<blocks_for((uint64_t)((nj + 63) / 64) * 32, 256), 256, 0, s>>>(nj, p.largest, p.smallest,
                                                                                         bmax, bmin);
  row_value_bounds<<<blocks_for((uint64_t)nx, 256), 256, 0, s>>>(nx, p.mask, p.largest, p.smallest, bmax, bmin, rl,
                                                                 rs);
  ctx.kernels += 2;
  F64Args a{};
  a.q = p.q;
  a.k = p.k;
  a.v = p.v;
  a.out = p.out;
  a.lse = p.lse;
  a.lnx = p.lnx;
  a.lnj = p.lnj;
  a.ne = p.ne;
  a.ny = p.ny;
  a.mask = p.mask;
  a.scale_kind = p.scale_kind;
  a.scale_c = p.scale_c;
  a.rl = rl;
  a.rs = rs;
  a.exp_table = exp_table(ctx.device);
  a.status = flags.get() + 1;
  DeviceBuffer<unsigned long long> pairs(1, s);
  pairs.zero();
  a.pairs = pairs.get();
  const int ne8 = (int)((p.ne + 7) & ~7LL);
  a.stride = ne8 + 4;
  const size_t smem = (size_t)(FM * a.stride + 2 * FN * a.stride + 2 * FN * VS) * sizeof(double);
  const bool async = p.ne % 2 == 0 && p.ny % 2 == 0 && (((uintptr_t)p.k | (uintptr_t)p.v) & 15) == 0;
  const dim3 grid((unsigned)((p.lnx + FM - 1) / FM), (unsigned)W, (unsigned)((p.ny + FY - 1) / FY));
  if (async) {
    EF_CUDA(cudaFuncSetAttribute(attn_fwd_f64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attn_fwd_f64<true><<<grid, kF64Threads, smem, s>>>(a);
  } else {
    EF_CUDA(cudaFuncSetAttribute(attn_fwd_f64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attn_fwd_f64<false><<<grid, kF64Threads, smem, s>>>(a);
  }
  EF_LAUNCH_CHECK();
  ctx.kernels++;
  int st = 0;
  EF_CUDA(cudaMemcpyAsync(&st, flags.get() + 1, 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("attention: fp64 mma");
  return (st & 1) ? ATTENTION_GUARDED : ATTENTION_DONE;
}

}  // namespace ef

namespace ef {

bool backward_f64_mma(Context& ctx, const AttentionGradients& g, const Mask& keys_mask, const double* dd,
                      cudaStream_t s) {
  const AttentionProblem& f = g.f;
  const int64_t W = f.batches;
  if (f.ne <= 0 || f.ne > 64 || f.ny <= 0 || f.ny > 64 || W > 65535) return false;
  if (fp64_tiles_requested()) return false;
  const double scale = f.scale_kind == 1 ? f.scale_c : 1.0;
  if (f.scale_kind == 2) return false;
  const size_t smem = (size_t)(2 * BR * RS + 4 * BC * CS + 4 * BC) * sizeof(double);
  const bool async = f.ne % 2 == 0 && f.ny % 2 == 0 &&
                     (((uintptr_t)f.q | (uintptr_t)f.k | (uintptr_t)f.v | (uintptr_t)g.d_out) & 15) == 0;
  F64BwdArgs kv{};
  kv.a1 = f.k;
  kv.a2 = f.v;
  kv.b1 = f.q;
  kv.b2 = g.d_out;
  kv.lse = g.lse;
  kv.dd = dd;
  kv.out1 = g.d_v;
  kv.out2 = g.d_k;
  kv.lr = f.lnj;
  kv.lc = f.lnx;
  kv.d1 = f.ne;
  kv.d2 = f.ny;
  kv.mask = keys_mask;
  kv.scale = scale;
  kv.exp_table = exp_table(ctx.device);
  kv.keys_rows = 1;
  F64BwdArgs qa = kv;
  qa.a1 = f.q;
  qa.a2 = g.d_out;
  qa.b1 = f.k;
  qa.b2 = f.v;
  qa.out1 = g.d_q;
  qa.out2 = nullptr;
  qa.lr = f.lnx;
  qa.lc = f.lnj;
  qa.mask = f.mask;
  qa.keys_rows = 0;
  auto launch = [&](auto kvtag, auto asynctag, const F64BwdArgs& args) {
    constexpr bool KVT = decltype(kvtag)::value, AS = decltype(asynctag)::value;
    EF_CUDA(cudaFuncSetAttribute(attn_bwd_f64<KVT, AS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid((unsigned)((args.lr + BR - 1) / BR), (unsigned)W);
    if (args.lr > 0) attn_bwd_f64<KVT, AS><<<grid, kBwdThreads, smem, s>>>(args);
    EF_LAUNCH_CHECK();
    ctx.kernels++;
  };
  if (async) {
    launch(std::true_type{}, std::true_type{}, kv);
    launch(std::false_type{}, std::true_type{}, qa);
  } else {
    launch(std::true_type{}, std::false_type{}, kv);
    launch(std::false_type{}, std::false_type{}, qa);
  }
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("attention backward: fp64 mma");
  return true;
}

}  // namespace ef
