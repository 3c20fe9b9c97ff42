// The backward pass of an attention-shaped pipeline: the gradients of the
// forward pass's average with respect to q, k and v, with the scores
// recomputed tile by tile from the saved log-sum-exp rather than stored.
//
// One kernel shape serves the three gradients. A CTA owns 128 rows of one
// batch and walks the column tiles of 64 its rows may pair with; per tile
//   s  = scale · (A1_r · B1_c)                  (product 1)
//   p  = exp(s - lse_x) on allowed pairs, else 0
//   dp = A2_r · B2_c, ds = p · (dp - D_x)       (product 2; not for d_v)
//   out_r += Σ_c w_rc · B3_c,  w = p (d_v) or ds (d_k, d_q)
// with x the query of the pair and D_x = Σ_y d_out_xy · out_xy:
//   d_v: rows keys,    A1 = k, B1 = q,                         B3 = d_out
//   d_k: rows keys,    A1 = k, B1 = q, A2 = v,     B2 = d_out, B3 = q
//   d_q: rows queries, A1 = q, B1 = k, A2 = d_out, B2 = v,     B3 = k
// (d_k and d_q then times scale). Each output row is summed by one CTA in
// column order: no atomics, the same bits on every run.
//
// The split form runs every product on tcgen05 kind::i8 over six int8
// digit planes, as the forward pass does, into TMEM columns 0..383; the
// weights w are cut into digits under a power of two per row and tile, and
// the rows' FP64 sums live in TMEM columns 384..511. Sixteen epilogue warps
// take a quarter of the columns each. The FP64 form runs the same tiles on
// the CUDA cores.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cmath>
#include <type_traits>

#include "attention.cuh"
#include "fastexp.cuh"
#include "gemm.cuh"
#include "levels.cuh"
#include "ptx.cuh"

namespace ef {
namespace {

using namespace ptx;

enum GradMode { GRAD_V = 0, GRAD_K = 1, GRAD_Q = 2 };

constexpr int GM = 128, GJ = 64, GY = 64;
constexpr int kEpi = 512;
constexpr int kGradThreads = 64 + kEpi;
constexpr int kSumCol = 384;
constexpr int kMaxSmem = 232448;
constexpr int S = 6;

template <int MODE>
struct GradShape {
  static constexpr bool kTwo = MODE != GRAD_V;
  static constexpr int kA1 = S * GM * 64;            // rows' digits, product 1 (64 B of features)
  static constexpr int kA2 = kTwo ? S * GM * 64 : 0;  // rows' digits, product 2
  static constexpr int kB1 = S * GJ * 64;            // per stage
  static constexpr int kB2 = kTwo ? S * GJ * 64 : 0;
  static constexpr int kB3 = S * GY * 64;
  static constexpr int kE = 2 * GJ * 4;              // the columns' exponents of products 1 and 2
  // Rows of keys: the columns' (queries') lse, and for d_k their D.
  static constexpr int kL = (MODE == GRAD_V ? 1 : (MODE == GRAD_K ? 2 : 0)) * GJ * 8;
  static constexpr int kP = S * GM * 64;
  static constexpr int kAux = 8192;
  static constexpr int kFixed = kA1 + kA2 + kP + kAux + 1024;
  static constexpr int kStage = (kB1 + kB2 + kB3 + kE + kL + 1023) / 1024 * 1024;
  static constexpr int kStages = kFixed + 2 * kStage <= kMaxSmem ? 2 : 1;
  static constexpr int kSmem = kFixed + kStages * kStage;
  static_assert(kSmem <= kMaxSmem, "the tiles must fit in shared memory");
};

struct GradArgs {
  Mask mask;  // the columns each row may pair with
  int64_t lr, lc, lr_pad, lc_pad, dy, dy_pad;
  int y0;
  double scale, out_factor;
  const int32_t* e_a1;  // [w][lr_pad]
  const int32_t* e_b1;  // [w][lc_pad]
  const int32_t* e_a2;
  const int32_t* e_b2;
  const int32_t* e_b3;  // [w][dy_pad]
  const double* lse;    // per query: [w·lq + x]
  const double* dd;     // D per query
  const double* lse_pad;  // the same, [w][lq_pad] (zeros past lq), for stages of keys' rows
  const double* dd_pad;
  const double* exp_table;
  double* out;  // [w·lr + r][dy]
  int* status;
  unsigned long long* tiles;
  int w0;  // the first batch of this launch (blockIdx.y counts from it)
  int reverse;  // row blocks from the last one (whose rows join the most columns) down
  // The d_k kernel's exports for the tile kernels (null: none), only for
  // the tiles some pair of is allowed: P's digit tiles as the d_v kernel cuts
  // them, [tile][S][128 rows][64 B] in the MMA's 64-byte swizzle, with their
  // rows' powers of two [tile][128], a key block's tiles from p_off[batch ·
  // n_rb + block] - p_base on, one a query tile it joins; and dS in tiles of
  // 128 queries by 64 keys, [tile][128][64], a query block's from
  // dq_off[batch · n_qb + block] - dq_base on, one a key tile from
  // dq_ct0[...] on (dq_n of them). Batches count from the launch's first.
  uint8_t* p_tiles;
  int32_t* p_exp;
  double* ds_out;
  const int64_t* p_off;
  const int64_t* dq_off;
  const int32_t* dq_ct0;
  const int32_t* dq_n;
  int64_t p_base, dq_base;
  int64_t n_rb, n_qb;  // key blocks and query blocks of a batch
};

constexpr int kPTile = S * GM * 64;  // bytes of one tile of weight digits

// FAST: every pair of row and column exponents of products 1 and 2 sums to
// a normal double's power of two.
template <int MODE, bool FAST>
__global__ void __launch_bounds__(kGradThreads, 1)
    grad_split(const __grid_constant__ CUtensorMap ta1, const __grid_constant__ CUtensorMap tb1,
               const __grid_constant__ CUtensorMap ta2, const __grid_constant__ CUtensorMap tb2,
               const __grid_constant__ CUtensorMap tb3, const GradArgs a) {
  using Sh = GradShape<MODE>;
  constexpr bool kTwo = Sh::kTwo;
  constexpr int CW = 16;  // columns per epilogue thread
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA1 = smem;
  uint8_t* sA2 = sA1 + Sh::kA1;
  uint8_t* sP = sA2 + Sh::kA2;
  uint8_t* sB = sP + Sh::kP;  // stages of [B1 | B2 | B3 | exponents]
  uint8_t* aux = sB + Sh::kStages * Sh::kStage;
  uint64_t* bars = (uint64_t*)aux;
  uint64_t* a_full = bars + 0;
  uint64_t* kv_full = bars + 1;   // [2]
  uint64_t* kv_empty = bars + 3;  // [2]
  uint64_t* s1_full = bars + 5;
  uint64_t* t1_free = bars + 6;
  uint64_t* s2_full = bars + 7;
  uint64_t* p_full = bars + 8;
  uint64_t* o_full = bars + 9;
  uint64_t* tmem_free = bars + 10;
  uint32_t* tmem_slot = (uint32_t*)(bars + 16);
  int* failed = (int*)(tmem_slot + 1);
  long long* span = (long long*)(tmem_slot + 4);
  int* row_lo = (int*)(aux + 256);
  int* row_hi = row_lo + GM;
  int* e3_s = row_hi + GM;               // [64]
  double* texp = (double*)(aux + 2048);  // [64]
  int* red = (int*)(aux + 4096);         // [4][128] the quarters' exponents
  int* redp = (int*)(aux + 6144);        // [4][128] the same for P (d_k's export)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rt = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int w = a.w0 + (int)blockIdx.y;
  const int64_t r_base = (int64_t)w * a.lr, c_base = (int64_t)w * a.lc;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 11; i++) mbar_init(&bars[i], 1);
    // Each epilogue warp arrives on the barriers that free TMEM or shared memory.
    mbar_init(t1_free, kEpi / 32);
    mbar_init(p_full, kEpi / 32);
    mbar_init(tmem_free, kEpi / 32);
    *failed = 0;
    span[0] = LLONG_MAX;
    span[1] = LLONG_MIN;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < GM) {
    const int64_t rl = (int64_t)rt * GM + threadIdx.x;
    int lo = 0, hi = 0;
    if (rl < a.lr) {
      int64_t l, h;
      allowed(a.mask, r_base + rl, l, h);
      lo = (int)(l - c_base);
      hi = (int)(h - c_base);
      if (lo < hi) {
        atomicMin(&span[0], (long long)lo);
        atomicMax(&span[1], (long long)hi);
      }
    }
    row_lo[threadIdx.x] = lo;
    row_hi[threadIdx.x] = hi;
  } else if (threadIdx.x < GM + GY) {
    const int c = threadIdx.x - GM;
    e3_s[c] = a.y0 + c < a.dy_pad ? a.e_b3[(int64_t)w * a.dy_pad + a.y0 + c] : 0;
  } else if (threadIdx.x < GM + GY + 64) {
    texp[threadIdx.x - GM - GY] = a.exp_table[threadIdx.x - GM - GY];
  }
  __syncthreads();
  const uint32_t tmem = *tmem_slot;
  const long long first = span[0], last = span[1];
  const int ct0 = first < last ? (int)(first / GJ) : 0;
  const int n_tiles = first < last ? (int)((last + GJ - 1) / GJ) - ct0 : 0;
  if (threadIdx.x == 0 && n_tiles > 0) atomicAdd(a.tiles, (unsigned long long)n_tiles);

  if (warp == 0) {
    if (lane == 0 && n_tiles > 0) {
      prefetch_map(&ta1);
      prefetch_map(&tb1);
      prefetch_map(&tb3);
      mbar_expect_tx(a_full, (uint32_t)(Sh::kA1 + Sh::kA2));
      tma_load_3d(sA1, &ta1, a_full, 0, rt * GM, w * S);
      if (kTwo) tma_load_3d(sA2, &ta2, a_full, 0, rt * GM, w * S);
      int issued = 0;
      for (int it = 0; it < n_tiles; it++) {
        const int st = it % Sh::kStages;
        const uint32_t round = (uint32_t)(it / Sh::kStages);
        if (*(volatile int*)failed) break;
        if (!mbar_wait(&kv_empty[st], (round & 1) ^ 1)) {
          atomicOr(a.status, 2);
          *(volatile int*)failed = 1;
          break;
        }
        mbar_expect_tx(&kv_full[st], (uint32_t)(Sh::kB1 + Sh::kB2 + Sh::kB3 + (kTwo ? 2 : 1) * GJ * 4 + Sh::kL));
        const int cl0 = (ct0 + it) * GJ;
        uint8_t* stage = sB + st * Sh::kStage;
        int* es = (int*)(stage + Sh::kB1 + Sh::kB2 + Sh::kB3);
        tma_load_3d(stage, &tb1, &kv_full[st], 0, cl0, w * S);
        if (kTwo) tma_load_3d(stage + Sh::kB1, &tb2, &kv_full[st], 0, cl0, w * S);
        tma_load_3d(stage + Sh::kB1 + Sh::kB2, &tb3, &kv_full[st], cl0, a.y0, w * S);
        bulk_load(es, a.e_b1 + (int64_t)w * a.lc_pad + cl0, GJ * 4, &kv_full[st]);
        if (kTwo) bulk_load(es + GJ, a.e_b2 + (int64_t)w * a.lc_pad + cl0, GJ * 4, &kv_full[st]);
        if (MODE != GRAD_Q) {
          double* ls = (double*)(stage + Sh::kB1 + Sh::kB2 + Sh::kB3 + Sh::kE);
          bulk_load(ls, a.lse_pad + (int64_t)w * a.lc_pad + cl0, GJ * 8, &kv_full[st]);
          if (MODE == GRAD_K) bulk_load(ls + GJ, a.dd_pad + (int64_t)w * a.lc_pad + cl0, GJ * 8, &kv_full[st]);
        }
        issued = it + 1;
      }
      mbar_wait(a_full, 0);
      for (int it = std::max(0, issued - Sh::kStages); it < issued; it++)
        mbar_wait(&kv_full[it % Sh::kStages], (uint32_t)((it / Sh::kStages) & 1));
    }
  } else if (warp == 1) {
    if (lane == 0 && n_tiles > 0) {
      uint64_t* last_bar = nullptr;
      uint32_t last_parity = 0;
      bool ok = mbar_wait(a_full, 0);
      // D (+)= A · B over S digit planes, the level scheme of the forward pass.
      auto product = [&](uint32_t a_base, uint32_t b_base, int n) {
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
          for (int s = 1; s <= S; s++) {
            const int total = (S + 1 - s) * n;
#pragma unroll
            for (int nn0 = 0; nn0 < total; nn0 += 256) {
              const int nn = total - nn0 < 256 ? total - nn0 : 256;
              umma_i8(tmem + (uint32_t)((s - 1) * n + nn0), desc_sw64(a_base + (s - 1) * GM * 64 + kk * 32),
                      desc_sw64(b_base + nn0 * 64 + kk * 32), idesc_i8(GM, nn), (kk > 0 || s > 1) ? 1u : 0u);
            }
          }
      };
      for (int it = 0; ok && it < n_tiles; it++) {
        const int st = it % Sh::kStages;
        const uint32_t round = (uint32_t)(it / Sh::kStages);
        const uint32_t par = (uint32_t)(it & 1);
        ok = mbar_wait(&kv_full[st], round & 1) && (it == 0 || mbar_wait(tmem_free, par ^ 1));
        if (!ok || *(volatile int*)failed) break;
        tc_fence_after();
        const uint32_t stage = smem_u32(sB + st * Sh::kStage);
        product(smem_u32(sA1), stage, GJ);
        umma_commit(s1_full);
        last_bar = s1_full;
        last_parity = par;
        if (kTwo) {
          ok = mbar_wait(t1_free, par);
          if (!ok || *(volatile int*)failed) break;
          tc_fence_after();
          product(smem_u32(sA2), stage + Sh::kB1, GJ);
          umma_commit(s2_full);
          last_bar = s2_full;
        }
        ok = mbar_wait(p_full, par);
        if (!ok || *(volatile int*)failed) break;
        tc_fence_after();
        product(smem_u32(sP), stage + Sh::kB1 + Sh::kB2, GY);
        umma_commit(o_full);
        umma_commit(&kv_empty[st]);
        last_bar = o_full;
      }
      if (!ok) {
        atomicOr(a.status, 2);
        *(volatile int*)failed = 1;
      }
      if (last_bar) mbar_wait(last_bar, last_parity);
    }
  } else {
    // Epilogue: warp w reads TMEM lanes 32·(w % 4) .. +31 and a quarter of
    // the columns; the four warps of a lane quarter exchange row maxima over
    // their own named barrier, and each warp signals the MMA warp by itself.
    const int h = (warp - 2) >> 2;
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int64_t rl = (int64_t)rt * GM + r;
    const bool valid = rl < a.lr;
    const int lo = row_lo[r], hi = row_hi[r];
    // Column c of a tile starting at cl0 is allowed iff (unsigned)(cl0 + c - lo) < span.
    const unsigned span = (valid && lo < hi) ? (unsigned)(hi - lo) : 0u;
    const int e1r = valid ? a.e_a1[(int64_t)w * a.lr_pad + rl] : 0;
    const int e2r = (kTwo && valid) ? a.e_a2[(int64_t)w * a.lr_pad + rl] : 0;
    // A row of queries reads its own lse and D; a row of keys its columns'.
    const double lse_r = (MODE == GRAD_Q && valid) ? a.lse[r_base + rl] : 0.0;
    const double dd_r = (MODE == GRAD_Q && valid) ? a.dd[r_base + rl] : 0.0;
    const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
    const uint32_t sum_addr = lane_addr + (uint32_t)(kSumCol + h * 2 * CW);
    int e3lo = INT_MAX, e3hi = INT_MIN;
    for (int c = 0; c < GY; c++) {
      e3lo = min(e3lo, e3_s[c]);
      e3hi = max(e3hi, e3_s[c]);
    }
    auto wait = [&](uint64_t* bar, uint32_t parity) {
      if (*(volatile int*)failed) return;
      if (!mbar_wait(bar, parity)) {
        *(volatile int*)failed = 1;
        atomicOr(a.status, 2);
      }
    };
    for (int it = 0; it < n_tiles; it++) {
      const int st = it % Sh::kStages;
      const int cl0 = (ct0 + it) * GJ + h * CW;
      const uint8_t* stage = sB + st * Sh::kStage;
      const int* es = (const int*)(stage + Sh::kB1 + Sh::kB2 + Sh::kB3) + h * CW;
      const double* ls = (const double*)(stage + Sh::kB1 + Sh::kB2 + Sh::kB3 + Sh::kE) + h * CW;
      const uint32_t par = (uint32_t)(it & 1);
      const int off = cl0 - lo;
      wait(s1_full, par);
      tc_fence_after();
      double wv[CW];
#pragma unroll
      for (int c4 = 0; c4 < CW / 4; c4++) {
        int32_t L[S][4];
#pragma unroll
        for (int l = 0; l < S; l++) tmem_ld4(lane_addr + (uint32_t)(l * GJ + h * CW + c4 * 4), L[l]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int c = c4 * 4 + i;
          const double l = combine_levels_small<S, 4>(L, i);
          const double s = a.scale * (FAST ? l * pow2(e1r + es[c]) : scale2(l, e1r + es[c]));
          const double p = exp_weight(s - (MODE == GRAD_Q ? lse_r : ls[c]), texp, 0);
          wv[c] = (unsigned)(off + c) < span ? p : 0.0;
        }
      }
      if (kTwo) {
        // d_k's export of dS: into the d_q kernel's tile of this tile's query
        // block and the row's key tile, row (query) cl0 + c, the keys
        // contiguous; nothing for a key tile the query block's rows don't join
        // (every pair there is masked).
        double* ds_col = nullptr;
        if (MODE == GRAD_K && a.ds_out) {
          const int64_t qbi = (int64_t)blockIdx.y * a.n_qb + cl0 / GM;
          const int64_t kt = ((int64_t)rt * GM + r) / GJ - a.dq_ct0[qbi];
          if (kt >= 0 && kt < a.dq_n[qbi])
            ds_col = a.ds_out + ((a.dq_off[qbi] - a.dq_base + kt) * GM + cl0 % GM) * GJ + r % GJ;
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(t1_free);
        if (MODE == GRAD_K && a.p_tiles) {
          // While d_out·v runs: P's digits for the d_v tile kernel, cut as
          // that kernel's own epilogue would (W = p · 2^(8S - ep), ep the
          // row's exponent over these 64 columns), stored as swizzled rows.
          double mp = 0.0;
#pragma unroll
          for (int c = 0; c < CW; c++) mp = fmax(mp, wv[c]);
          redp[h * GM + r] = mp > 0.0 ? slice_exponent(mp) : INT_MIN;
          named_bar(2 + quarter, 128);
          int ep = max(max(redp[r], redp[GM + r]), max(redp[2 * GM + r], redp[3 * GM + r]));
          ep = ep == INT_MIN ? 0 : ep;
          const int shift = 8 * S - ep;
          const double f1 = pow2(shift >> 1), f2 = pow2(shift - (shift >> 1));
          const int64_t tile = a.p_off[(int64_t)blockIdx.y * a.n_rb + rt] - a.p_base + it;
          uint8_t* dst = a.p_tiles + tile * kPTile + sw64_offset((uint32_t)r, (uint32_t)(h * CW));
          uint32_t chunk[S][4];
#pragma unroll
          for (int c4 = 0; c4 < CW / 4; c4++) {
            double x[4];
#pragma unroll
            for (int i = 0; i < 4; i++) x[i] = wv[c4 * 4 + i] * f1 * f2;
            uint32_t planes[S];
            digit_planes4<S>(x, planes);
#pragma unroll
            for (int s = 0; s < S; s++) chunk[s][c4] = planes[s];
          }
#pragma unroll
          for (int s = 0; s < S; s++)
            *(uint4*)(dst + s * GM * 64) = make_uint4(chunk[s][0], chunk[s][1], chunk[s][2], chunk[s][3]);
          if (h == 0) a.p_exp[tile * GM + r] = ep;
        }
        wait(s2_full, par);
        tc_fence_after();
#pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          int32_t L[S][4];
#pragma unroll
          for (int l = 0; l < S; l++) tmem_ld4(lane_addr + (uint32_t)(l * GJ + h * CW + c4 * 4), L[l]);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int c = c4 * 4 + i;
            const double l = combine_levels_small<S, 4>(L, i);
            const double dp = FAST ? l * pow2(e2r + es[GJ + c]) : scale2(l, e2r + es[GJ + c]);
            const double t = wv[c] * (dp - (MODE == GRAD_Q ? dd_r : ls[GJ + c]));
            wv[c] = wv[c] != 0.0 ? t : 0.0;
            if (ds_col) ds_col[(int64_t)c * GJ] = wv[c];
          }
        }
      }
      // The row's power of two for this tile, over the four quarters.
      double mx = 0.0;
#pragma unroll
      for (int c = 0; c < CW; c++) mx = fmax(mx, fabs(wv[c]));
      red[h * GM + r] = mx > 0.0 ? slice_exponent(mx) : INT_MIN;
      named_bar(2 + quarter, 128);
      int ew = max(max(red[r], red[GM + r]), max(red[2 * GM + r], red[3 * GM + r]));
      ew = ew == INT_MIN ? 0 : ew;
      // The weights' digits: W = w · 2^(8S - ew), |W| < 2^(8S-2), the power
      // of two applied in two exact halves (8S - ew lies in [-978, 1119]).
      const int shift = 8 * S - ew;
      const double f1 = pow2(shift >> 1), f2 = pow2(shift - (shift >> 1));
      uint8_t* prow = sP + r * 64;
#pragma unroll
      for (int c4 = 0; c4 < CW / 4; c4++) {
        double x[4];
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] = wv[c4 * 4 + i] * f1 * f2;
        uint32_t planes[S];
        digit_planes4<S>(x, planes);
        const uint32_t off4 = sw64_offset((uint32_t)r, (uint32_t)(h * CW + c4 * 4)) - (uint32_t)r * 64;
#pragma unroll
        for (int s = 0; s < S; s++) *(uint32_t*)(prow + s * GM * 64 + off4) = planes[s];
      }
      fence_proxy_async();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(p_full);
      wait(o_full, par);
      tc_fence_after();
      // sums += this tile's levels · 2^(ew + e3): one rounding either way,
      // the power of two a normal double on the first path.
      auto add_levels = [&](auto normal) {
#pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          int32_t L[S][4];
#pragma unroll
          for (int l = 0; l < S; l++) tmem_ld4(lane_addr + (uint32_t)(l * GY + h * CW + c4 * 4), L[l]);
          uint32_t sum[8];
          if (it > 0) tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int e = ew + e3_s[h * CW + c4 * 4 + i];
            const double prev = it > 0 ? __hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]) : 0.0;
            const double l = combine_levels_small<S, 4>(L, i);
            const double v = decltype(normal)::value ? fma(l, pow2(e), prev) : prev + scale2(l, e);
            sum[2 * i] = (uint32_t)__double2loint(v);
            sum[2 * i + 1] = (uint32_t)__double2hiint(v);
          }
          tmem_st8(sum_addr + c4 * 8, sum);
        }
      };
      if (__all_sync(0xffffffffu, ew + e3lo >= -1022 && ew + e3hi <= 1023)) add_levels(std::true_type{});
      else add_levels(std::false_type{});
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_free);
    }
    // Every lane of the warp reads TMEM (the loads are warp-wide); the rows
    // past the batch's end write nothing.
    tc_fence_after();
    const bool store = valid && !*(volatile int*)failed;
    double* orow = a.out + (r_base + rl) * a.dy;
#pragma unroll
    for (int c4 = 0; c4 < CW / 4; c4++) {
      uint32_t sum[8];
      if (n_tiles > 0) {
        tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
        tmem_wait_ld();
      }
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int64_t y = (int64_t)a.y0 + h * CW + c4 * 4 + i;
        const double v = n_tiles > 0 ? __hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]) : 0.0;
        if (store && y < a.dy) orow[y] = a.out_factor * v;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// The d_v and d_q tiles from the weights the d_k kernel exported: one
// product a tile (the weights' digits against the columns' B3 digits) and
// the rows' sums, with no scores, exponentials or d_out·v recomputed. d_v
// reads P's digit tiles and their rows' powers of two as they are; d_q reads
// dS (query-major, four 128-byte-swizzled boxes of 16 keys a tile), applies
// the mask and cuts its digits under the row's power of two over the tile,
// as grad_split's epilogue does, so that both gradients come out with the
// same bits as there.
template <int MODE>
struct TileShape {
  static constexpr bool kQ = MODE == GRAD_Q;
  static constexpr int kDs = kQ ? GM * GJ * 8 : 0;  // one dS tile
  static constexpr int kDsBufs = kQ ? 2 : 0;        // d_q: dS tiles double-buffered
  static constexpr int kBufs = kQ ? 1 : 2;          // weight digit tiles (d_v: one a stage)
  static constexpr int kB3 = S * GY * 64;
  static constexpr int kStage = kB3 + (kQ ? 0 : 1024);  // B3, and for d_v the rows' exponents
  static constexpr int kStages = kQ ? 1 : 2;
  static constexpr int kAux = 8192;
  static constexpr int kSmem = kDsBufs * kDs + kBufs * kPTile + kStages * kStage + kAux + 1024;
  static_assert(kSmem <= kMaxSmem, "the tiles must fit in shared memory");
};

template <int MODE>
__global__ void __launch_bounds__(kGradThreads, 1)
    grad_tiles(const __grid_constant__ CUtensorMap tds, const __grid_constant__ CUtensorMap tb3, const GradArgs a) {
  using Sh = TileShape<MODE>;
  constexpr bool kQ = Sh::kQ;
  constexpr int CW = 16;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sDs = smem;  // d_q: [2] dS tiles
  uint8_t* sP = sDs + Sh::kDsBufs * Sh::kDs;
  uint8_t* sB = sP + Sh::kBufs * kPTile;  // stages of [B3 | rows' exponents]
  uint8_t* aux = sB + Sh::kStages * Sh::kStage;
  uint64_t* bars = (uint64_t*)aux;
  uint64_t* kv_full = bars + 0;   // [2] B3 stages (d_v: with the weights' tile)
  uint64_t* kv_empty = bars + 2;  // [2]
  uint64_t* ds_full = bars + 4;   // [2] d_q: dS tiles
  uint64_t* ds_empty = bars + 6;  // [2]
  uint64_t* p_full = bars + 8;
  uint64_t* o_full = bars + 9;
  uint64_t* tmem_free = bars + 10;
  uint32_t* tmem_slot = (uint32_t*)(bars + 16);
  int* failed = (int*)(tmem_slot + 1);
  long long* span = (long long*)(tmem_slot + 4);
  int* row_lo = (int*)(aux + 256);
  int* row_hi = row_lo + GM;
  int* e3_s = row_hi + GM;        // [64]
  int* red = (int*)(aux + 4096);  // [4][128]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rt = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
  const int w = a.w0 + (int)blockIdx.y;
  const int64_t r_base = (int64_t)w * a.lr, c_base = (int64_t)w * a.lc;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; i++) {
      mbar_init(&kv_full[i], 1);
      // d_v: the MMAs' commit and every epilogue warp (which reads the
      // stage's exponents) free a stage.
      mbar_init(&kv_empty[i], kQ ? 1 : 1 + kEpi / 32);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(&ds_full[i], 1);
      mbar_init(&ds_empty[i], kEpi / 32);
    }
    mbar_init(p_full, kEpi / 32);
    mbar_init(o_full, 1);
    mbar_init(tmem_free, kEpi / 32);
    *failed = 0;
    span[0] = LLONG_MAX;
    span[1] = LLONG_MIN;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < GM) {
    const int64_t rl = (int64_t)rt * GM + threadIdx.x;
    int lo = 0, hi = 0;
    if (rl < a.lr) {
      int64_t l, h;
      allowed(a.mask, r_base + rl, l, h);
      lo = (int)(l - c_base);
      hi = (int)(h - c_base);
      if (lo < hi) {
        atomicMin(&span[0], (long long)lo);
        atomicMax(&span[1], (long long)hi);
      }
    }
    row_lo[threadIdx.x] = lo;
    row_hi[threadIdx.x] = hi;
  } else if (threadIdx.x < GM + GY) {
    const int c = threadIdx.x - GM;
    e3_s[c] = a.y0 + c < a.dy_pad ? a.e_b3[(int64_t)w * a.dy_pad + a.y0 + c] : 0;
  }
  __syncthreads();
  const uint32_t tmem = *tmem_slot;
  const long long first = span[0], last = span[1];
  const int ct0 = first < last ? (int)(first / GJ) : 0;
  const int n_tiles = first < last ? (int)((last + GJ - 1) / GJ) - ct0 : 0;
  if (threadIdx.x == 0 && n_tiles > 0) atomicAdd(a.tiles, (unsigned long long)n_tiles);
  // d_v: this key block's P tiles; d_q: this query block's dS tiles.
  auto tile_of = [&](int it) {
    return kQ ? a.dq_off[(int64_t)blockIdx.y * a.n_qb + rt] - a.dq_base + it
              : a.p_off[(int64_t)blockIdx.y * a.n_rb + rt] - a.p_base + it;
  };

  if (warp == 0) {
    if (lane == 0 && n_tiles > 0) {
      prefetch_map(&tb3);
      if (kQ) prefetch_map(&tds);
      int issued = 0;
      for (int it = 0; it < n_tiles; it++) {
        const int st = it & 1;
        const uint32_t round = (uint32_t)(it >> 1);
        const int cl0 = (ct0 + it) * GJ;
        if (*(volatile int*)failed) break;
        bool ok;
        if (kQ) {
          // dS two tiles ahead; B3 (one stage) once the previous tile's MMAs are done.
          ok = mbar_wait(&ds_empty[st], (round & 1) ^ 1);
          if (ok) {
            mbar_expect_tx(&ds_full[st], (uint32_t)Sh::kDs);
            for (int j = 0; j < 4; j++)
              tma_load_3d(sDs + st * Sh::kDs + j * GM * 128, &tds, &ds_full[st], 16 * j, (int)(tile_of(it) * GM),
                          0);
          }
          ok = ok && (it == 0 || mbar_wait(&kv_empty[0], (uint32_t)((it - 1) & 1)));
          if (ok) {
            mbar_expect_tx(&kv_full[0], (uint32_t)Sh::kB3);
            tma_load_3d(sB, &tb3, &kv_full[0], cl0, a.y0, w * S);
          }
        } else {
          ok = mbar_wait(&kv_empty[st], (round & 1) ^ 1);
          if (ok) {
            uint8_t* stage = sB + st * Sh::kStage;
            mbar_expect_tx(&kv_full[st], (uint32_t)(Sh::kB3 + kPTile + GM * 4));
            tma_load_3d(stage, &tb3, &kv_full[st], cl0, a.y0, w * S);
            bulk_load(sP + st * kPTile, a.p_tiles + tile_of(it) * kPTile, kPTile, &kv_full[st]);
            bulk_load(stage + Sh::kB3, a.p_exp + tile_of(it) * GM, GM * 4, &kv_full[st]);
          }
        }
        if (!ok) {
          atomicOr(a.status, 2);
          *(volatile int*)failed = 1;
          break;
        }
        issued = it + 1;
      }
      // Copies still in flight complete before the CTA may exit.
      for (int it = std::max(0, issued - 2); it < issued; it++) {
        if (kQ) {
          mbar_wait(&ds_full[it & 1], (uint32_t)((it >> 1) & 1));
          if (it == issued - 1) mbar_wait(&kv_full[0], (uint32_t)(it & 1));
        } else {
          mbar_wait(&kv_full[it & 1], (uint32_t)((it >> 1) & 1));
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && n_tiles > 0) {
      int last = -1;  // the last tile whose MMAs were committed
      bool ok = true;
      for (int it = 0; ok && it < n_tiles; it++) {
        const int st = kQ ? 0 : (it & 1);
        const uint32_t par = (uint32_t)(it & 1);
        ok = mbar_wait(&kv_full[st], kQ ? par : (uint32_t)((it >> 1) & 1)) &&
             (it == 0 || mbar_wait(tmem_free, par ^ 1)) && (!kQ || mbar_wait(p_full, par));
        if (!ok || *(volatile int*)failed) break;
        tc_fence_after();
        const uint32_t a_base = smem_u32(sP + (kQ ? 0 : st * kPTile)), b_base = smem_u32(sB + st * Sh::kStage);
#pragma unroll
        for (int kk = 0; kk < 2; kk++)
#pragma unroll
          for (int s = 1; s <= S; s++) {
            const int total = (S + 1 - s) * GY;
#pragma unroll
            for (int nn0 = 0; nn0 < total; nn0 += 256) {
              const int nn = total - nn0 < 256 ? total - nn0 : 256;
              umma_i8(tmem + (uint32_t)((s - 1) * GY + nn0), desc_sw64(a_base + (s - 1) * GM * 64 + kk * 32),
                      desc_sw64(b_base + nn0 * 64 + kk * 32), idesc_i8(GM, nn), (kk > 0 || s > 1) ? 1u : 0u);
            }
          }
        umma_commit(o_full);
        umma_commit(&kv_empty[st]);
        last = it;
      }
      if (!ok) {
        atomicOr(a.status, 2);
        *(volatile int*)failed = 1;
      }
      // MMAs still running complete before TMEM is freed.
      if (last >= 0) mbar_wait(o_full, (uint32_t)(last & 1));
    }
  } else {
    const int h = (warp - 2) >> 2;
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int64_t rl = (int64_t)rt * GM + r;
    const bool valid = rl < a.lr;
    const int lo = row_lo[r], hi = row_hi[r];
    const unsigned span_r = (valid && lo < hi) ? (unsigned)(hi - lo) : 0u;
    const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
    const uint32_t sum_addr = lane_addr + (uint32_t)(kSumCol + h * 2 * CW);
    int e3lo = INT_MAX, e3hi = INT_MIN;
    for (int c = 0; c < GY; c++) {
      e3lo = min(e3lo, e3_s[c]);
      e3hi = max(e3hi, e3_s[c]);
    }
    auto wait = [&](uint64_t* bar, uint32_t parity) {
      if (*(volatile int*)failed) return;
      if (!mbar_wait(bar, parity)) {
        *(volatile int*)failed = 1;
        atomicOr(a.status, 2);
      }
    };
    for (int it = 0; it < n_tiles; it++) {
      const int st = it & 1;
      const uint32_t par = (uint32_t)(it & 1);
      wait(kQ ? &ds_full[st] : &kv_full[st], (uint32_t)((it >> 1) & 1));
      int ew;
      if (kQ) {
        // This row's 16 keys of the tile: box h, 128-byte row r, its 16-byte
        // chunks permuted by r mod 8.
        const uint8_t* row = sDs + st * Sh::kDs + h * GM * 128 + r * 128;
        const int off = (ct0 + it) * GJ + h * CW - lo;
        double wv[CW];
#pragma unroll
        for (int j = 0; j < CW / 2; j++) {
          const double2 v = *(const double2*)(row + ((j ^ (r & 7)) << 4));
          wv[2 * j] = (unsigned)(off + 2 * j) < span_r ? v.x : 0.0;
          wv[2 * j + 1] = (unsigned)(off + 2 * j + 1) < span_r ? v.y : 0.0;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&ds_empty[st]);
        double mx = 0.0;
#pragma unroll
        for (int c = 0; c < CW; c++) mx = fmax(mx, fabs(wv[c]));
        red[h * GM + r] = mx > 0.0 ? slice_exponent(mx) : INT_MIN;
        named_bar(2 + quarter, 128);
        ew = max(max(red[r], red[GM + r]), max(red[2 * GM + r], red[3 * GM + r]));
        ew = ew == INT_MIN ? 0 : ew;
        const int shift = 8 * S - ew;
        const double f1 = pow2(shift >> 1), f2 = pow2(shift - (shift >> 1));
        uint8_t* prow = sP + r * 64;
#pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          double x[4];
#pragma unroll
          for (int i = 0; i < 4; i++) x[i] = wv[c4 * 4 + i] * f1 * f2;
          uint32_t planes[S];
          digit_planes4<S>(x, planes);
          const uint32_t off4 = sw64_offset((uint32_t)r, (uint32_t)(h * CW + c4 * 4)) - (uint32_t)r * 64;
#pragma unroll
          for (int s = 0; s < S; s++) *(uint32_t*)(prow + s * GM * 64 + off4) = planes[s];
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(p_full);
      } else {
        ew = ((const int*)(sB + st * Sh::kStage + Sh::kB3))[r];
        __syncwarp();
        if (lane == 0) mbar_arrive(&kv_empty[st]);
      }
      wait(o_full, par);
      tc_fence_after();
      // sums += this tile's levels · 2^(ew + e3), as in grad_split.
      auto add_levels = [&](auto normal) {
#pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          int32_t L[S][4];
#pragma unroll
          for (int l = 0; l < S; l++) tmem_ld4(lane_addr + (uint32_t)(l * GY + h * CW + c4 * 4), L[l]);
          uint32_t sum[8];
          if (it > 0) tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int e = ew + e3_s[h * CW + c4 * 4 + i];
            const double prev = it > 0 ? __hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]) : 0.0;
            const double l = combine_levels_small<S, 4>(L, i);
            const double v = decltype(normal)::value ? fma(l, pow2(e), prev) : prev + scale2(l, e);
            sum[2 * i] = (uint32_t)__double2loint(v);
            sum[2 * i + 1] = (uint32_t)__double2hiint(v);
          }
          tmem_st8(sum_addr + c4 * 8, sum);
        }
      };
      if (__all_sync(0xffffffffu, ew + e3lo >= -1022 && ew + e3hi <= 1023)) add_levels(std::true_type{});
      else add_levels(std::false_type{});
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_free);
    }
    tc_fence_after();
    const bool store = valid && !*(volatile int*)failed;
    double* orow = a.out + (r_base + rl) * a.dy;
#pragma unroll
    for (int c4 = 0; c4 < CW / 4; c4++) {
      uint32_t sum[8];
      if (n_tiles > 0) {
        tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
        tmem_wait_ld();
      }
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int64_t y = (int64_t)a.y0 + h * CW + c4 * 4 + i;
        const double v = n_tiles > 0 ? __hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]) : 0.0;
        if (store && y < a.dy) orow[y] = a.out_factor * v;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// The same tiles in FP64 on the CUDA cores: 64 rows by 64 outputs per CTA,
// a 4 x 4 block of (row, output) per thread.
constexpr int FT = 64;
struct GradFp64Args {
  Mask mask;
  int64_t lr, lc, d1, d2, dy;  // rows, columns per batch; widths of products 1, 2 and the values
  double scale, out_factor;
  const double* a1;  // [w·lr + r][d1]
  const double* b1;  // [w·lc + c][d1]
  const double* a2;  // [w·lr + r][d2]
  const double* b2;  // [w·lc + c][d2]
  const double* b3;  // [w·lc + c][dy]
  const double* lse;
  const double* dd;
  double* out;  // [w·lr + r][dy]
};

constexpr size_t kFp64Smem = sizeof(double) * (FT * (FT + 1) + 2 * 32 * (FT + 1));

template <int MODE>
__global__ void __launch_bounds__(256) grad_fp64(const GradFp64Args a) {
  extern __shared__ __align__(16) unsigned char smem_fp64[];
  double(*blk)[FT + 1] = reinterpret_cast<double(*)[FT + 1]>(smem_fp64);
  double(*sa)[FT + 1] = reinterpret_cast<double(*)[FT + 1]>(smem_fp64 + sizeof(double) * FT * (FT + 1));
  double(*sb)[FT + 1] = sa + 32;
  __shared__ int s_lo[FT], s_hi[FT];
  __shared__ long long s_first, s_last;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int w = blockIdx.z;
  const int64_t r0 = (int64_t)blockIdx.x * FT, y0 = (int64_t)blockIdx.y * FT;
  const int64_t r_base = (int64_t)w * a.lr, c_base = (int64_t)w * a.lc;
  const int rows = (int)std::min<int64_t>(FT, a.lr - r0);
  if (t == 0) {
    s_first = LLONG_MAX;
    s_last = LLONG_MIN;
  }
  __syncthreads();
  if (t < FT) {
    int lo = 0, hi = 0;
    if (t < rows) {
      int64_t l, h;
      allowed(a.mask, r_base + r0 + t, l, h);
      lo = (int)(l - c_base);
      hi = (int)(h - c_base);
      if (lo < hi) {
        atomicMin(&s_first, (long long)lo);
        atomicMax(&s_last, (long long)hi);
      }
    }
    s_lo[t] = lo;
    s_hi[t] = hi;
  }
  __syncthreads();
  const long long first = s_first, last = s_last;
  double acc[4][4] = {};
  // Σ_e A[r][e] B[c][e] for this thread's 4 x 4 (row, column) pairs.
  auto product = [&](const double* A, const double* B, int64_t dk, int64_t c0, int width, double (&o)[4][4]) {
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) o[i][j] = 0.0;
    for (int64_t e0 = 0; e0 < dk; e0 += 32) {
      const int ec = (int)std::min<int64_t>(32, dk - e0);
      for (int idx = t; idx < FT * 32; idx += 256) {
        const int rr = idx >> 5, e = idx & 31;
        sa[e][rr] = (rr < rows && e < ec) ? A[(r_base + r0 + rr) * dk + e0 + e] : 0.0;
        sb[e][rr] = (rr < width && e < ec) ? B[(c_base + c0 + rr) * dk + e0 + e] : 0.0;
      }
      __syncthreads();
      for (int e = 0; e < ec; e++)
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) o[i][j] = fma(sa[e][ty + 16 * i], sb[e][tx + 16 * j], o[i][j]);
      __syncthreads();
    }
  };
  for (long long c0 = first < last ? first - first % FT : 0; c0 < last; c0 += FT) {
    const int width = (int)std::min<long long>(FT, a.lc - c0);
    double s[4][4];
    product(a.a1, a.b1, a.d1, c0, width, s);
    double dp[4][4];
    if (MODE != GRAD_V) product(a.a2, a.b2, a.d2, c0, width, dp);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        const int rr = ty + 16 * i, cc = tx + 16 * j;
        const int64_t cl = c0 + cc;
        double wgt = 0.0;
        if (rr < rows && cc < width && cl >= s_lo[rr] && cl < s_hi[rr]) {
          const int64_t xq = MODE == GRAD_Q ? r_base + r0 + rr : c_base + cl;
          wgt = exp(a.scale * s[i][j] - a.lse[xq]);
          if (MODE != GRAD_V) wgt = wgt * (dp[i][j] - a.dd[xq]);
        }
        blk[rr][cc] = wgt;
      }
    __syncthreads();
    for (int cc = 0; cc < width; cc++) {
      double bv[4];
      for (int j = 0; j < 4; j++) {
        const int64_t y = y0 + tx + 16 * j;
        bv[j] = y < a.dy ? a.b3[(c_base + c0 + cc) * a.dy + y] : 0.0;
      }
      for (int i = 0; i < 4; i++) {
        const double wgt = blk[ty + 16 * i][cc];
        for (int j = 0; j < 4; j++) acc[i][j] = fma(wgt, bv[j], acc[i][j]);
      }
    }
    __syncthreads();
  }
  for (int i = 0; i < 4; i++) {
    const int rr = ty + 16 * i;
    if (rr >= rows) continue;
    for (int j = 0; j < 4; j++) {
      const int64_t y = y0 + tx + 16 * j;
      if (y < a.dy) a.out[(r_base + r0 + rr) * a.dy + y] = a.out_factor * acc[i][j];
    }
  }
}

// D_x = Σ_y d_out[x][y] · out[x][y], a warp per row.
__global__ void row_dots(int64_t n, int64_t dv, const double* __restrict__ d_out, const double* __restrict__ out,
                         double* __restrict__ dd) {
  const int lane = threadIdx.x & 31;
  for (int64_t x = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < n;
       x += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    double s = 0.0;
    for (int64_t y = lane; y < dv; y += 32) s = fma(d_out[x * dv + y], out[x * dv + y], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) dd[x] = s;
  }
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Whether a batch's last rows join more columns than its first (causal
// queries do; causal keys as rows the other way round): the blocks with the
// most work then go first.
// Per block of 128 rows of each batch: the first column tile of 64 its rows
// may pair with and how many, as the backward kernels find them (the span
// of the rows' allowed intervals).
__global__ void export_plan(Mask m, int64_t lr, int64_t lc, int64_t batches, int64_t blocks, int32_t* __restrict__ ct0,
                            int32_t* __restrict__ n) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < batches * blocks;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t w = x / blocks, b = x - w * blocks;
    long long first = LLONG_MAX, last = LLONG_MIN;
    for (int64_t r = b * GM; r < min(lr, b * GM + GM); r++) {
      int64_t lo, hi;
      allowed(m, w * lr + r, lo, hi);
      lo -= w * lc;
      hi -= w * lc;
      if (lo < hi) {
        first = min(first, (long long)lo);
        last = max(last, (long long)hi);
      }
    }
    ct0[x] = first < last ? (int32_t)(first / GJ) : 0;
    n[x] = first < last ? (int32_t)((last + GJ - 1) / GJ - first / GJ) : 0;
  }
}

bool last_rows_longest(Mask m, int64_t rows) {
  if (rows <= 0) return true;
  m.xlen = m.jlen = nullptr;
  int64_t lo0, hi0, lo1, hi1;
  allowed(m, 0, lo0, hi0);
  allowed(m, rows - 1, lo1, hi1);
  return hi1 - lo1 >= hi0 - lo0;
}

// The mask of keys as rows: each condition x <cmp> j + off as j <cmp'> x - off.
Mask transposed(const Mask& m) {
  static const int mirror[4] = {2, 3, 0, 1};
  Mask t;
  t.n = m.n;
  for (int i = 0; i < m.n; i++) {
    if (m.off[i] == INT64_MIN) fail(EINFOLD_INVALID, "a condition offset of -2^63 has no mirror");
    t.cmp[i] = mirror[m.cmp[i]];
    t.off[i] = -m.off[i];
  }
  t.lnx = m.lnj > 0 ? m.lnj : 1;
  t.lnj = m.lnx;
  t.xlen = m.jlen;
  t.jlen = m.xlen;
  return t;
}

// One operand's digits: rows (or columns) sliced, with exponents.
struct Digits {
  int8_t* d = nullptr;
  int32_t* e = nullptr;
};

template <int MODE>
void launch_split(const CUtensorMap* maps, const GradArgs& args, dim3 grid, bool fast, cudaStream_t stream) {
  using Sh = GradShape<MODE>;
  if (fast) {
    EF_CUDA(cudaFuncSetAttribute(grad_split<MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem));
    grad_split<MODE, true><<<grid, kGradThreads, Sh::kSmem, stream>>>(maps[0], maps[1], maps[2], maps[3], maps[4],
                                                                       args);
  } else {
    EF_CUDA(cudaFuncSetAttribute(grad_split<MODE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem));
    grad_split<MODE, false><<<grid, kGradThreads, Sh::kSmem, stream>>>(maps[0], maps[1], maps[2], maps[3], maps[4],
                                                                        args);
  }
  EF_LAUNCH_CHECK();
}

template <int MODE>
void launch_tiles(const CUtensorMap& tds, const CUtensorMap& tb3, const GradArgs& args, dim3 grid,
                  cudaStream_t stream) {
  using Sh = TileShape<MODE>;
  EF_CUDA(cudaFuncSetAttribute(grad_tiles<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem));
  grad_tiles<MODE><<<grid, kGradThreads, Sh::kSmem, stream>>>(tds, tb3, args);
  EF_LAUNCH_CHECK();
}

// dst[w][x] = src[w·l + x] for x < l, 0 up to l_pad.
__global__ void pad_rows(const double* __restrict__ src, int64_t batches, int64_t l, int64_t l_pad,
                         double* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < batches * l_pad;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t w = i / l_pad, x = i - w * l_pad;
    dst[i] = x < l ? src[w * l + x] : 0.0;
  }
}

// The split backward; false if it doesn't apply or an operand isn't finite
// (nothing written).
bool backward_split(Context& ctx, const AttentionGradients& g, const double* dd, cudaStream_t s) {
  const AttentionProblem& f = g.f;
  const int64_t W = f.batches, lq = f.lnx, lk = f.lnj, d = f.ne, dv = f.ny;
  if (d > 64 || dv > 64 || d <= 0 || dv <= 0 || lq <= 0 || lk <= 0) return false;
  if (lq > (1 << 30) || lk > (1 << 30) || W > 65535) return false;
  const int64_t lq_pad = round_up(lq, GM), lk_pad = round_up(lk, GM);
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  // Row digits of q, k, v, d_out (64 B of features each) and column digits
  // of d_out, q, k (K-major along the batch's positions).
  const size_t rq = al((size_t)(W * S * lq_pad * 64)), rk = al((size_t)(W * S * lk_pad * 64));
  const size_t cq = al((size_t)(W * S * 64 * lq_pad)), ck = al((size_t)(W * S * 64 * lk_pad));
  const size_t eqs = al((size_t)(W * lq_pad) * 4), eks = al((size_t)(W * lk_pad) * 4), ecs = al((size_t)(W * 64) * 4);
  const size_t cm = al((size_t)(W * 64) * 8), lp = al((size_t)(W * lq_pad) * 8);
  const size_t total = 2 * rq + 2 * rk + 2 * cq + ck + 2 * eqs + 2 * eks + 3 * ecs + cm + 2 * lp + 256;
  DeviceBuffer<uint8_t> scratch(total, s);
  uint8_t* p = scratch.get();
  auto take = [&](size_t n) {
    uint8_t* q = p;
    p += n;
    return q;
  };
  Digits Qr{(int8_t*)take(rq), nullptr}, dOr{(int8_t*)take(rq), nullptr}, Kr{(int8_t*)take(rk), nullptr},
      Vr{(int8_t*)take(rk), nullptr}, dOc{(int8_t*)take(cq), nullptr}, Qc{(int8_t*)take(cq), nullptr},
      Kc{(int8_t*)take(ck), nullptr};
  Qr.e = (int32_t*)take(eqs);
  dOr.e = (int32_t*)take(eqs);
  Kr.e = (int32_t*)take(eks);
  Vr.e = (int32_t*)take(eks);
  dOc.e = (int32_t*)take(ecs);
  Qc.e = (int32_t*)take(ecs);
  Kc.e = (int32_t*)take(ecs);
  unsigned long long* colmax = (unsigned long long*)take(cm);
  double* lse_pad = (double*)take(lp);
  double* dd_pad = (double*)take(lp);
  // [0] slicing, [1] kernels, [2..7] tile pairs of the three kernels,
  // [8..15] (max e, max -e) of q's, k's, v's and d_out's rows
  int* status = (int*)take(256);
  unsigned long long* tiles = (unsigned long long*)(status + 2);
  EF_CUDA(cudaMemsetAsync(status, 0, 32, s));
  const int init[8] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN};
  EF_CUDA(cudaMemcpyAsync(status + 8, init, 32, cudaMemcpyHostToDevice, s));
  // Ragged batches: the padding rows are not read (their digits are zeros).
  const int64_t *xl = f.mask.xlen, *jl = f.mask.jlen;
  slice_rows_into(S, f.q, W, lq, d, d, lq_pad, 64, Qr.e, Qr.d, status, s, xl);
  slice_rows_into(S, g.d_out, W, lq, dv, dv, lq_pad, 64, dOr.e, dOr.d, status, s, xl);
  slice_rows_into(S, f.k, W, lk, d, d, lk_pad, 64, Kr.e, Kr.d, status, s, jl);
  slice_rows_into(S, f.v, W, lk, dv, dv, lk_pad, 64, Vr.e, Vr.d, status, s, jl);
  slice_cols_into(S, g.d_out, W, lq, dv, 64, lq_pad, colmax, dOc.e, dOc.d, status, s, xl);
  slice_cols_into(S, f.q, W, lq, d, 64, lq_pad, colmax, Qc.e, Qc.d, status, s, xl);
  slice_cols_into(S, f.k, W, lk, d, 64, lk_pad, colmax, Kc.e, Kc.d, status, s, jl);
  exponent_range(Qr.e, W * lq_pad, status + 8, s);
  exponent_range(Kr.e, W * lk_pad, status + 10, s);
  exponent_range(Vr.e, W * lk_pad, status + 12, s);
  exponent_range(dOr.e, W * lq_pad, status + 14, s);
  pad_rows<<<blocks_for((uint64_t)(W * lq_pad), 256), 256, 0, s>>>(g.lse, W, lq, lq_pad, lse_pad);
  pad_rows<<<blocks_for((uint64_t)(W * lq_pad), 256), 256, 0, s>>>(dd, W, lq, lq_pad, dd_pad);
  EF_LAUNCH_CHECK();
  ctx.kernels += 16;
  int sts[16];
  EF_CUDA(cudaMemcpyAsync(sts, status, 64, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  int st = sts[0];
  if (st & 1) return false;
  // Products 1 (q·k) and 2 (d_out·v) have normal powers of two 2^(e_r + e_c).
  const bool fast = (int64_t)sts[8] + sts[10] <= 1023 && (int64_t)sts[9] + sts[11] <= 1022 &&
                    (int64_t)sts[12] + sts[14] <= 1023 && (int64_t)sts[13] + sts[15] <= 1022;
  ctx.phase("attention backward: sliced");
  auto rows_map = [&](const Digits& x, int64_t rows_pad, int box) {
    return digit_planes_map(x.d, 64, rows_pad, W * S, box, S);
  };
  auto cols_map = [&](const Digits& x, int64_t k_pad) { return digit_planes_map(x.d, k_pad, 64, W * S, GY, S); };
  const Mask keys_mask = transposed(f.mask);
  const double* table = exp_table(ctx.device);
  GradArgs args[3];
  CUtensorMap mode_maps[3][5];
  for (int mode = 0; mode < 3; mode++) {
    GradArgs& a = args[mode];
    a = GradArgs{};
    CUtensorMap* maps = mode_maps[mode];
    const bool keys = mode != GRAD_Q;
    a.mask = keys ? keys_mask : f.mask;
    a.lr = keys ? lk : lq;
    a.lc = keys ? lq : lk;
    a.lr_pad = keys ? lk_pad : lq_pad;
    a.lc_pad = keys ? lq_pad : lk_pad;
    a.scale = f.scale_kind == 1 ? f.scale_c : 1.0;
    a.lse = g.lse;
    a.dd = dd;
    a.lse_pad = lse_pad;
    a.dd_pad = dd_pad;
    a.exp_table = table;
    a.status = status + 1;
    a.tiles = tiles + mode;
    if (mode == GRAD_V) {
      maps[0] = rows_map(Kr, lk_pad, GM);
      maps[1] = rows_map(Qr, lq_pad, GJ);
      maps[2] = maps[0];
      maps[3] = maps[1];
      maps[4] = cols_map(dOc, lq_pad);
      a.e_a1 = Kr.e;
      a.e_b1 = Qr.e;
      a.e_b3 = dOc.e;
      a.dy = dv;
      a.out = g.d_v;
      a.out_factor = 1.0;
    } else if (mode == GRAD_K) {
      maps[0] = rows_map(Kr, lk_pad, GM);
      maps[1] = rows_map(Qr, lq_pad, GJ);
      maps[2] = rows_map(Vr, lk_pad, GM);
      maps[3] = rows_map(dOr, lq_pad, GJ);
      maps[4] = cols_map(Qc, lq_pad);
      a.e_a1 = Kr.e;
      a.e_b1 = Qr.e;
      a.e_a2 = Vr.e;
      a.e_b2 = dOr.e;
      a.e_b3 = Qc.e;
      a.dy = d;
      a.out = g.d_k;
      a.out_factor = a.scale;
    } else {
      maps[0] = rows_map(Qr, lq_pad, GM);
      maps[1] = rows_map(Kr, lk_pad, GJ);
      maps[2] = rows_map(dOr, lq_pad, GM);
      maps[3] = rows_map(Vr, lk_pad, GJ);
      maps[4] = cols_map(Kc, lk_pad);
      a.e_a1 = Qr.e;
      a.e_b1 = Kr.e;
      a.e_a2 = dOr.e;
      a.e_b2 = Vr.e;
      a.e_b3 = Kc.e;
      a.dy = d;
      a.out = g.d_q;
      a.out_factor = a.scale;
    }
    a.dy_pad = 64;
    a.y0 = 0;
    a.n_rb = a.lr_pad / GM;
    a.reverse = last_rows_longest(a.mask, a.lr);
  }
  // The tile path: d_k first, exporting P's digits and dS; then d_v and d_q
  // from them, one product a tile each. The exports cover only the tiles
  // some pair of is allowed (export_plan counts them per block), 14 bytes a
  // pair of those. Batches go in chunks whose exports fit the export limit
  // (EINFOLD_BACKWARD_EXPORT_MB, 4096 by default): all in one when they fit,
  // else in chunks of at most half of it in two buffers, the chunks
  // alternating between the call's stream and the context's second stream,
  // so that one chunk's kernels run beside the other's and a chunk's last
  // wave of blocks leaves no SM idle. The buffers are freed at the end of
  // the call. A batch whose exports alone exceed half the limit takes the
  // three kernels that each recompute the scores.
  const int64_t n_kb = lk_pad / GM, n_qb = lq_pad / GM;
  static const size_t limit = [] {
    const char* e = std::getenv("EINFOLD_BACKWARD_EXPORT_MB");
    const long long mb = e ? std::atoll(e) : 4096;
    return (size_t)std::max(0ll, mb) << 20;
  }();
  DeviceBuffer<int32_t> plan((size_t)(2 * W * (n_kb + n_qb)), s);
  int32_t* pk_ct0 = plan.get();
  int32_t* pk_n = pk_ct0 + W * n_kb;
  int32_t* pq_ct0 = pk_n + W * n_kb;
  int32_t* pq_n = pq_ct0 + W * n_qb;
  export_plan<<<blocks_for((uint64_t)(W * n_kb), 128), 128, 0, s>>>(keys_mask, lk, lq, W, n_kb, pk_ct0, pk_n);
  export_plan<<<blocks_for((uint64_t)(W * n_qb), 128), 128, 0, s>>>(f.mask, lq, lk, W, n_qb, pq_ct0, pq_n);
  ctx.kernels += 2;
  EF_LAUNCH_CHECK();
  std::vector<int32_t> hk_n((size_t)(W * n_kb)), hq_n((size_t)(W * n_qb));
  EF_CUDA(cudaMemcpyAsync(hk_n.data(), pk_n, hk_n.size() * 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(hq_n.data(), pq_n, hq_n.size() * 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  // Each block's first tile (exclusive over all batches), and each batch's tiles.
  std::vector<int64_t> hp_off((size_t)(W * n_kb) + 1), hq_off((size_t)(W * n_qb) + 1);
  for (size_t x = 0; x < hk_n.size(); x++) hp_off[x + 1] = hp_off[x] + hk_n[x];
  for (size_t x = 0; x < hq_n.size(); x++) hq_off[x + 1] = hq_off[x] + hq_n[x];
  constexpr size_t kPBytes = (size_t)kPTile + GM * 4, kDsBytes = (size_t)GM * GJ * 8;
  auto bytes_of = [&](int64_t w0, int64_t w1) {
    const int64_t np = hp_off[(size_t)(w1 * n_kb)] - hp_off[(size_t)(w0 * n_kb)];
    const int64_t nq = hq_off[(size_t)(w1 * n_qb)] - hq_off[(size_t)(w0 * n_qb)];
    return al((size_t)np * kPTile) + al((size_t)np * GM * 4) + (size_t)nq * kDsBytes;
  };
  // The chunks and buffers under a limit: one chunk when every batch's
  // exports fit it, else chunks of at most half of it in two buffers; none
  // when one batch's exports exceed half of it.
  std::vector<std::pair<int64_t, int64_t>> chunks;
  int buffers = 1;
  auto plan_under = [&](size_t lim) {
    chunks.clear();
    buffers = 1;
    if (bytes_of(0, W) <= lim) {
      chunks.push_back({0, W});
      return;
    }
    buffers = 2;
    int64_t w0 = 0;
    while (w0 < W) {
      if (bytes_of(w0, w0 + 1) > lim / 2) {
        chunks.clear();
        return;
      }
      int64_t w1 = w0 + 1;
      while (w1 < W && bytes_of(w0, w1 + 1) <= lim / 2) w1++;
      chunks.push_back({w0, w1});
      w0 = w1;
    }
  };
  auto biggest_chunk = [&]() {
    size_t b = 0;
    for (auto& c : chunks) b = std::max(b, bytes_of(c.first, c.second));
    return std::max<size_t>(b, 256);
  };
  // With a budget, the plan's buffers are asked of it, and a refusal halves
  // the limit until a plan is granted or none is left.
  struct Granted {
    Budget* budget = nullptr;
    uint64_t bytes = 0;
    ~Granted() {
      if (budget && bytes) budget->release(bytes);
    }
  } granted;
  for (size_t lim = limit;; lim /= 2) {
    plan_under(lim);
    if (chunks.empty() || !g.budget) break;
    const uint64_t want = (uint64_t)buffers * biggest_chunk();
    if (g.budget->try_reserve(want)) {
      granted.budget = g.budget;
      granted.bytes = want;
      break;
    }
    if (lim == 0) {
      chunks.clear();
      break;
    }
  }
  (void)kPBytes;
  DeviceBuffer<int64_t> offs;
  if (!chunks.empty()) {
    offs.allocate(hp_off.size() + hq_off.size(), s);
    EF_CUDA(cudaMemcpyAsync(offs.get(), hp_off.data(), hp_off.size() * 8, cudaMemcpyHostToDevice, s));
    EF_CUDA(cudaMemcpyAsync(offs.get() + hp_off.size(), hq_off.data(), hq_off.size() * 8, cudaMemcpyHostToDevice, s));
  }
  const int64_t* p_off = offs.get();
  const int64_t* q_off = offs.get() + hp_off.size();
  DeviceBuffer<uint8_t> exports[2];
  cudaStream_t streams[2] = {s, s};
  cudaEvent_t e0, e1, joined = nullptr;
  EF_CUDA(cudaEventCreate(&e0));
  EF_CUDA(cudaEventCreate(&e1));
  EF_CUDA(cudaEventRecord(e0, s));
  if (!chunks.empty() && buffers == 2) {
    if (!ctx.aux) EF_CUDA(cudaStreamCreateWithFlags(&ctx.aux, cudaStreamNonBlocking));
    streams[1] = ctx.aux;
    EF_CUDA(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
    EF_CUDA(cudaEventRecord(joined, s));  // the slicing above, before the second stream starts
    EF_CUDA(cudaStreamWaitEvent(ctx.aux, joined, 0));
  }
  if (!chunks.empty()) {
    const size_t biggest = biggest_chunk();
    for (int b = 0; b < buffers; b++) exports[b].allocate(biggest, streams[b]);
    for (size_t c = 0; c < chunks.size(); c++) {
      const int b = (int)(c % (size_t)buffers);
      cudaStream_t st = streams[b];
      const int64_t w0 = chunks[c].first, w1 = chunks[c].second;
      const int64_t np = hp_off[(size_t)(w1 * n_kb)] - hp_off[(size_t)(w0 * n_kb)];
      const int64_t nq = hq_off[(size_t)(w1 * n_qb)] - hq_off[(size_t)(w0 * n_qb)];
      uint8_t* p_tiles = exports[b].get();
      int32_t* p_exp = (int32_t*)(p_tiles + al((size_t)np * kPTile));
      double* ds = (double*)((uint8_t*)p_exp + al((size_t)np * GM * 4));
      const CUtensorMap tds = f64_boxes_map(ds, GJ, std::max<int64_t>(nq, 1) * GM, 1, 16, GM);
      const unsigned wc = (unsigned)(w1 - w0);
      GradArgs k = args[GRAD_K], v = args[GRAD_V], q = args[GRAD_Q];
      for (GradArgs* g2 : {&k, &v, &q}) {
        g2->w0 = (int)w0;
        g2->p_tiles = p_tiles;
        g2->p_exp = p_exp;
        g2->p_off = p_off + w0 * n_kb;
        g2->p_base = hp_off[(size_t)(w0 * n_kb)];
        g2->dq_off = q_off + w0 * n_qb;
        g2->dq_ct0 = pq_ct0 + w0 * n_qb;
        g2->dq_n = pq_n + w0 * n_qb;
        g2->dq_base = hq_off[(size_t)(w0 * n_qb)];
        g2->n_rb = n_kb;
        g2->n_qb = n_qb;
      }
      k.ds_out = ds;
      launch_split<GRAD_K>(mode_maps[GRAD_K], k, dim3((unsigned)n_kb, wc), fast, st);
      launch_tiles<GRAD_V>(tds, mode_maps[GRAD_V][4], v, dim3((unsigned)n_kb, wc), st);
      launch_tiles<GRAD_Q>(tds, mode_maps[GRAD_Q][4], q, dim3((unsigned)n_qb, wc), st);
      ctx.kernels += 3;
    }
    if (joined) {
      EF_CUDA(cudaEventRecord(joined, ctx.aux));  // the second stream's chunks, before the call's stream goes on
      EF_CUDA(cudaStreamWaitEvent(s, joined, 0));
    }
  } else {
    for (int mode = 0; mode < 3; mode++) {
      const dim3 grid((unsigned)(args[mode].lr_pad / GM), (unsigned)W);
      if (mode == GRAD_V) launch_split<GRAD_V>(mode_maps[mode], args[mode], grid, fast, s);
      else if (mode == GRAD_K) launch_split<GRAD_K>(mode_maps[mode], args[mode], grid, fast, s);
      else launch_split<GRAD_Q>(mode_maps[mode], args[mode], grid, fast, s);
      ctx.kernels++;
    }
  }
  const int64_t chunk = chunks.empty() ? 0 : 1;
  EF_CUDA(cudaEventRecord(e1, s));
  unsigned long long pairs[3] = {};
  EF_CUDA(cudaMemcpyAsync(&st, status + 1, 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(pairs, tiles, 24, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (joined) cudaEventDestroy(joined);
  if (st & 2) fail(EINFOLD_TIMEOUT, "a bounded wait in the attention backward ran out");
  // Digit products executed: per pair of tiles, S(S+1)/2 digit pairs of a
  // 128 x 64 x 64 product, three for d_k, and for d_v and d_q one on the
  // tile path (else two and three).
  ctx.product_ms += ms;
  const double per = (S * (S + 1) / 2) * 2.0 * GM * GJ * 64;
  const double pv = chunk >= 1 ? 1.0 : 2.0, pq = chunk >= 1 ? 1.0 : 3.0;
  ctx.product_ops += per * (pv * (double)pairs[0] + 3.0 * (double)pairs[1] + pq * (double)pairs[2]);
  ctx.phase("attention backward: tiles");
  return true;
}

void backward_fp64(Context& ctx, const AttentionGradients& g, const double* dd, cudaStream_t s) {
  const AttentionProblem& f = g.f;
  const int64_t W = f.batches, lq = f.lnx, lk = f.lnj, d = f.ne, dv = f.ny;
  const Mask keys_mask = transposed(f.mask);
  for (int mode = 0; mode < 3; mode++) {
    GradFp64Args a{};
    const bool keys = mode != GRAD_Q;
    a.mask = keys ? keys_mask : f.mask;
    a.lr = keys ? lk : lq;
    a.lc = keys ? lq : lk;
    a.scale = f.scale_kind == 1 ? f.scale_c : 1.0;
    a.lse = g.lse;
    a.dd = dd;
    if (mode == GRAD_V) {
      a.a1 = f.k; a.b1 = f.q; a.d1 = d; a.b3 = g.d_out; a.dy = dv; a.out = g.d_v; a.out_factor = 1.0;
    } else if (mode == GRAD_K) {
      a.a1 = f.k; a.b1 = f.q; a.d1 = d; a.a2 = f.v; a.b2 = g.d_out; a.d2 = dv; a.b3 = f.q; a.dy = d;
      a.out = g.d_k; a.out_factor = a.scale;
    } else {
      a.a1 = f.q; a.b1 = f.k; a.d1 = d; a.a2 = g.d_out; a.b2 = f.v; a.d2 = dv; a.b3 = f.k; a.dy = d;
      a.out = g.d_q; a.out_factor = a.scale;
    }
    if (a.lr == 0 || a.dy == 0 || W == 0) continue;
    const dim3 grid((unsigned)((a.lr + FT - 1) / FT), (unsigned)((a.dy + FT - 1) / FT), (unsigned)W);
    if (mode == GRAD_V) {
      EF_CUDA(cudaFuncSetAttribute(grad_fp64<GRAD_V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFp64Smem));
      grad_fp64<GRAD_V><<<grid, 256, kFp64Smem, s>>>(a);
    } else if (mode == GRAD_K) {
      EF_CUDA(cudaFuncSetAttribute(grad_fp64<GRAD_K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFp64Smem));
      grad_fp64<GRAD_K><<<grid, 256, kFp64Smem, s>>>(a);
    } else {
      EF_CUDA(cudaFuncSetAttribute(grad_fp64<GRAD_Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFp64Smem));
      grad_fp64<GRAD_Q><<<grid, 256, kFp64Smem, s>>>(a);
    }
    EF_LAUNCH_CHECK();
    ctx.kernels++;
  }
  EF_CUDA(cudaStreamSynchronize(s));
  ctx.phase("attention backward: fp64 tiles");
}

}  // namespace

void attention_backward(Context& ctx, const AttentionGradients& g, int precision, cudaStream_t s) {
  const AttentionProblem& f = g.f;
  const int64_t W = f.batches, lq = f.lnx;
  if (W <= 0) return;
  if (W > 65535) fail(EINFOLD_INVALID, "more than 65535 batches");
  DeviceBuffer<double> dd((size_t)std::max<int64_t>(W * lq, 1), s);
  if (W * lq > 0) {
    row_dots<<<blocks_for((uint64_t)(W * lq) * 32, 256), 256, 0, s>>>(W * lq, f.ny, g.d_out, g.out, dd.get());
    EF_LAUNCH_CHECK();
    ctx.kernels++;
  }
  if (precision == 0 && backward_split(ctx, g, dd.get(), s)) return;
  if (backward_f64_mma(ctx, g, transposed(f.mask), dd.get(), s)) return;
  backward_fp64(ctx, g, dd.get(), s);
}

}  // namespace ef
