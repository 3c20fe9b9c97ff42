// The split forward pass of an attention-shaped pipeline on the B200: the
// tile of fused.rs:694-1019 for product scores, a softmax shifted by the
// running maximum and a normalised average, with both products on the
// tensor cores.
//
// A CTA owns 128 query rows of one batch and walks the batch's key tiles of
// 64 that its rows may join. Per tile:
//   1. q·k: the rows' and keys' S int8 digit planes (sliced once, staged by
//      TMA) multiply on tcgen05 kind::i8, each digit s of q against digits
//      1..S+1-s of k stacked along N, so that digit pair (s, t) accumulates
//      in TMEM columns (s + t - 2)·64: level l's exact int32 sum.
//   2. Sixteen epilogue warps read the levels (a row per TMEM lane, a
//      quarter of the columns per warp group), combine them in FP64 under
//      the row's and key's powers of two, apply the mask, update the running
//      maximum (shared between the quarters), and turn the weights
//      exp(s - m) in [0, 1] into S digit planes of a fixed scale 2^2,
//      written to shared memory in the MMA's 64-byte swizzle.
//   3. w·v: the weights' digits against v's column-scaled digits, the same
//      level scheme, into the same TMEM columns (q·k's levels were read).
//   4. The epilogue rescales the row's FP64 running sums and adds the
//      levels to them, in units of each value column's power of two (applied
//      once, at the end). The sums live in the 128 TMEM columns the six
//      slices' 384 level columns leave free, two 32-bit columns a value, so
//      that a thread's registers hold only its 16 scores.
// The four warps sharing a row exchange its maximum over a named barrier of
// their own; every other hand-off is an mbarrier each warp arrives on.
// A TMA producer warp double-buffers k and v tiles; an MMA warp issues both
// products. Every wait is bounded (2 s); on a timeout the kernel sets a
// status bit, waits for its copies and MMAs in flight, frees TMEM and
// returns.
//
// Launch forms: a block per (query tile, batch) item, or persistent blocks
// (one an SM) that claim the items of a work list in its order from a
// counter, keeping their barriers and TMEM across items: the barriers'
// phases count the block's key tiles and q loads since the launch.
//
// Accuracy: each operand value carries 8S - 2 bits under its row's (or
// column's) power of two, levels above S + 1 are dropped, and every level
// sum is exact, so a score's error is about ne · 2^(3-8S) · max|q| · max|k|
// and a weight's about 2^(1-8S): with S = 6, scores to ~1e-14 of their scale
// and averages to ~1e-14 of max|v|.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "attention.cuh"
#include "fastexp.cuh"
#include "gemm.cuh"
#include "levels.cuh"
#include "ptx.cuh"

namespace ef {
namespace {

using namespace ptx;

constexpr int AM = 128;  // query rows per CTA (TMEM lanes)
constexpr int AJ = 64;   // key positions per tile
constexpr int AY = 64;   // value columns per CTA
constexpr int kEpi = 512;     // 16 epilogue warps: a row per TMEM lane, a quarter of the columns each
constexpr int kAttnThreads = 64 + kEpi;
constexpr int kSumCol = 384;  // TMEM columns of the rows' FP64 running sums, two per value
constexpr int kMaxSmem = 232448;

template <int S, int KB>
struct AttnShape {
  static constexpr int kQ = KB * S * AM * 64;  // q digits [kb][s][128][64 B]
  static constexpr int kK = KB * S * AJ * 64;  // k digits per stage [kb][t][64][64 B]
  static constexpr int kV = S * AY * 64;       // v digits per stage [t][64 y][64 B of j]
  static constexpr int kP = S * AM * 64;       // weight digits [s][128][64 B of j]
  static constexpr int kAux = 8192;            // barriers, row spans, exponents, exchanges
  static constexpr int kFixed = kQ + kP + kAux + 1024;
  static constexpr int kStages = kFixed + 2 * (kK + kV) <= kMaxSmem ? 2 : 1;
  static constexpr int kSmem = kFixed + kStages * (kK + kV);
  static_assert(kSmem <= kMaxSmem, "the tiles must fit in shared memory");
  static_assert(S * 64 <= kSumCol, "the levels and the running sums must fit in TMEM");
};

struct AttnArgs {
  Mask mask;
  int64_t lnx, lnj, lnx_pad, lnj_pad, ny, ny_pad;
  int y0;
  int scale_kind;
  double scale_c;
  const int32_t* eq;  // [w][lnx_pad]
  const int32_t* ek;  // [w][lnj_pad]
  const int32_t* ev;  // [w][ny_pad]
  const double* rl;   // [w·lnx + x]: the largest magnitude of the values the row weighs
  const double* rs;   // and the smallest nonzero one (+inf if none)
  const double* exp_table;
  double* out;  // [w·lnx + x][ny]
  double* lse;  // [w·lnx + x] or null
  int* status;  // bit 0: a guard fired; bit 1: a wait ran out
  unsigned long long* tiles;  // (row tile, key tile) pairs computed
  const int2* items;  // a work list of (query tile, batch) items; null: the grid's (x: tile, y: batch)
  int n_items;
  // Persistent blocks: the next item of the list no block has claimed (zero
  // at the launch). Null: block i runs items[i].
  unsigned* next;
  int reverse;        // the grid's query tiles from the last one (whose rows join the most keys) down
};

// The S levels of this thread's 4 TMEM columns at `col`.
template <int S>
__device__ __forceinline__ void load_levels(uint32_t lane_addr, int col, int32_t (&L)[S][4]) {
#pragma unroll
  for (int l = 0; l < S; l++) tmem_ld4(lane_addr + (uint32_t)(l * 64 + col), L[l]);
  tmem_wait_ld();
}

template <int S, int KB>
__device__ __forceinline__ double level_sum(const int32_t (&L)[S][4], int i) {
  // Level sums of products over 64 values of k fit the int32 pairs.
  if constexpr (KB == 1) return combine_levels_small<S, 4>(L, i);
  else return combine_levels<S, 4>(L, i);
}

// FAST: every q row's and k row's exponents sum to at most 1023 and at
// least -1022, so a score's power of two is a normal double.
template <int S, int KB, bool FAST>
__global__ void __launch_bounds__(kAttnThreads, 1)
    attn_fwd_split(const __grid_constant__ CUtensorMap tq, const __grid_constant__ CUtensorMap tk,
                   const __grid_constant__ CUtensorMap tv, const AttnArgs a) {
  using Sh = AttnShape<S, KB>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sQ = smem;
  uint8_t* sP = sQ + Sh::kQ;
  uint8_t* sK = sP + Sh::kP;
  uint8_t* sV = sK + Sh::kStages * Sh::kK;
  uint8_t* aux = sV + Sh::kStages * Sh::kV;
  uint64_t* bars = (uint64_t*)aux;  // 16 barriers
  uint64_t* q_full = bars + 0;
  uint64_t* kv_full = bars + 1;   // [2]
  uint64_t* kv_empty = bars + 3;  // [2]
  uint64_t* qk_full = bars + 5;
  uint64_t* pv_full = bars + 6;
  uint64_t* p_full = bars + 7;
  uint64_t* tmem_free = bars + 8;
  uint32_t* tmem_slot = (uint32_t*)(bars + 16);
  int* failed = (int*)(tmem_slot + 1);
  int* item_slot = (int*)(tmem_slot + 2);         // the item the block runs next
  long long* span = (long long*)(tmem_slot + 4);  // first, last
  int* row_lo = (int*)(aux + 256);                // [128]
  int* row_hi = row_lo + AM;                      // [128]
  int* ev_s = row_hi + AM;                        // [64]
  int* ek_s = (int*)(aux + 1536);                 // [2][64], a stage's key exponents
  double* texp = (double*)(aux + 2048);           // [64]
  double* red = (double*)(aux + 4096);            // [4][128]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    mbar_init(q_full, 1);
    for (int i = 0; i < 2; i++) {
      mbar_init(&kv_full[i], 1);
      mbar_init(&kv_empty[i], 1);
    }
    mbar_init(qk_full, 1);
    mbar_init(pv_full, 1);
    mbar_init(p_full, kEpi / 32);  // each epilogue warp arrives
    mbar_init(tmem_free, kEpi / 32);
    *failed = 0;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  if (threadIdx.x < 64) texp[threadIdx.x] = a.exp_table[threadIdx.x];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  // The barriers' completed phases before the current item: one per key
  // tile (kv_full and kv_empty by stage) and one per q load.
  int tiles_before = 0, q_loads = 0;
  for (int round_ = 0;; round_++) {
    if (threadIdx.x == 0) {
      *item_slot = a.next ? (int)atomicAdd(a.next, 1u) : round_ == 0 ? 0 : INT_MAX;
      span[0] = LLONG_MAX;
      span[1] = LLONG_MIN;
    }
    __syncthreads();
    // Every thread reads the same item and failure flag: all leave together.
    const int item = *item_slot;
    if (*(volatile int*)failed || item >= (a.next ? a.n_items : 1)) break;
    // The longest rows of a causal mask first; work lists in their order.
    int xt, w;
    if (a.items) {
      const int2 wk = a.items[a.next ? item : (int)blockIdx.x];
      xt = wk.x;
      w = wk.y;
    } else {
      xt = a.reverse ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
      w = (int)blockIdx.y;
    }
    const int64_t x_base = (int64_t)w * a.lnx;
    // Each row's allowed keys, local to the batch.
    if (threadIdx.x < AM) {
      const int64_t xl = (int64_t)xt * AM + threadIdx.x;
      int lo = 0, hi = 0;
      if (xl < a.lnx) {
        int64_t l, h;
        allowed(a.mask, x_base + xl, l, h);
        lo = (int)(l - (int64_t)w * a.lnj);
        hi = (int)(h - (int64_t)w * a.lnj);
        if (lo < hi) {
          atomicMin(&span[0], (long long)lo);
          atomicMax(&span[1], (long long)hi);
        }
      }
      row_lo[threadIdx.x] = lo;
      row_hi[threadIdx.x] = hi;
    } else if (threadIdx.x < AM + AY) {
      const int c = threadIdx.x - AM;
      ev_s[c] = a.y0 + c < a.ny_pad ? a.ev[(int64_t)w * a.ny_pad + a.y0 + c] : 0;
    }
    __syncthreads();
    const long long first = span[0], last = span[1];
    const int jt0 = first < last ? (int)(first / AJ) : 0;
    const int n_tiles = first < last ? (int)((last + AJ - 1) / AJ) - jt0 : 0;
    if (threadIdx.x == 0 && n_tiles > 0) atomicAdd(a.tiles, (unsigned long long)n_tiles);

    if (warp == 0) {
      if (lane == 0 && n_tiles > 0) {
        // Producer: q's digits once, then k's and v's per tile, with the
        // keys' exponents.
        prefetch_map(&tq);
        prefetch_map(&tk);
        prefetch_map(&tv);
        mbar_expect_tx(q_full, (uint32_t)Sh::kQ);
        for (int kb = 0; kb < KB; kb++) tma_load_3d(sQ + kb * S * AM * 64, &tq, q_full, kb * 64, xt * AM, w * S);
        int issued = 0;
        for (int it = 0; it < n_tiles; it++) {
          const int g = tiles_before + it;
          const int st = g % Sh::kStages;
          const uint32_t round = (uint32_t)(g / Sh::kStages);
          if (*(volatile int*)failed) break;
          if (!mbar_wait(&kv_empty[st], (round & 1) ^ 1)) {
            atomicOr(a.status, 2);
            *(volatile int*)failed = 1;
            break;
          }
          mbar_expect_tx(&kv_full[st], (uint32_t)(Sh::kK + Sh::kV + AJ * 4));
          const int jl0 = (jt0 + it) * AJ;
          for (int kb = 0; kb < KB; kb++)
            tma_load_3d(sK + st * Sh::kK + kb * S * AJ * 64, &tk, &kv_full[st], kb * 64, jl0, w * S);
          tma_load_3d(sV + st * Sh::kV, &tv, &kv_full[st], jl0, a.y0, w * S);
          bulk_load(ek_s + st * AJ, a.ek + (int64_t)w * a.lnj_pad + jl0, AJ * 4, &kv_full[st]);
          issued = it + 1;
        }
        // Copies still in flight complete before the item ends.
        mbar_wait(q_full, (uint32_t)(q_loads & 1));
        for (int it = std::max(0, issued - Sh::kStages); it < issued; it++) {
          const int g = tiles_before + it;
          mbar_wait(&kv_full[g % Sh::kStages], (uint32_t)((g / Sh::kStages) & 1));
        }
      }
    } else if (warp == 1) {
      if (lane == 0 && n_tiles > 0) {
        // MMA issuer. The item's first tile needs no tmem_free: the block's
        // barrier between items follows the epilogue's last TMEM read.
        uint64_t* last_bar = nullptr;
        uint32_t last_parity = 0;
        bool ok = mbar_wait(q_full, (uint32_t)(q_loads & 1));
        for (int it = 0; ok && it < n_tiles; it++) {
          const int g = tiles_before + it;
          const int st = g % Sh::kStages;
          const uint32_t round = (uint32_t)(g / Sh::kStages);
          ok = mbar_wait(&kv_full[st], round & 1) && (it == 0 || mbar_wait(tmem_free, (uint32_t)((g - 1) & 1)));
          if (!ok || *(volatile int*)failed) break;
          tc_fence_after();
          const uint32_t q_base = smem_u32(sQ), k_base = smem_u32(sK + st * Sh::kK);
  #pragma unroll
          for (int kb = 0; kb < KB; kb++)
  #pragma unroll
            for (int kk = 0; kk < 2; kk++)
  #pragma unroll
              for (int s = 1; s <= S; s++) {
                const int total = (S + 1 - s) * AJ;
  #pragma unroll
                for (int nn0 = 0; nn0 < total; nn0 += 256) {
                  const int nn = total - nn0 < 256 ? total - nn0 : 256;
                  const uint64_t ad = desc_sw64(q_base + (kb * S + s - 1) * AM * 64 + kk * 32);
                  const uint64_t bd = desc_sw64(k_base + kb * S * AJ * 64 + nn0 * 64 + kk * 32);
                  umma_i8(tmem + (uint32_t)((s - 1) * AJ + nn0), ad, bd, idesc_i8(AM, nn),
                          (kb > 0 || kk > 0 || s > 1) ? 1u : 0u);
                }
              }
          umma_commit(qk_full);
          last_bar = qk_full;
          last_parity = (uint32_t)(g & 1);
          ok = mbar_wait(p_full, (uint32_t)(g & 1));
          if (!ok || *(volatile int*)failed) break;
          tc_fence_after();
          const uint32_t p_base = smem_u32(sP), v_base = smem_u32(sV + st * Sh::kV);
  #pragma unroll
          for (int kk = 0; kk < 2; kk++)
  #pragma unroll
            for (int s = 1; s <= S; s++) {
              const int total = (S + 1 - s) * AY;
  #pragma unroll
              for (int nn0 = 0; nn0 < total; nn0 += 256) {
                const int nn = total - nn0 < 256 ? total - nn0 : 256;
                const uint64_t ad = desc_sw64(p_base + (s - 1) * AM * 64 + kk * 32);
                const uint64_t bd = desc_sw64(v_base + nn0 * 64 + kk * 32);
                umma_i8(tmem + (uint32_t)((s - 1) * AY + nn0), ad, bd, idesc_i8(AM, nn), (kk > 0 || s > 1) ? 1u : 0u);
              }
            }
          umma_commit(pv_full);
          umma_commit(&kv_empty[st]);
          last_bar = pv_full;
          last_parity = (uint32_t)(g & 1);
        }
        if (!ok) {
          atomicOr(a.status, 2);
          *(volatile int*)failed = 1;
        }
        // MMAs still running complete before TMEM is freed.
        if (last_bar) mbar_wait(last_bar, last_parity);
      }
    } else {
      // Epilogue: warp w reads TMEM lanes 32·(w % 4) .. +31; warps 2..5 take
      // columns 0..15 of each tile and of the sums, 6..9 columns 16..31, and
      // so on. The four warps of a lane quarter exchange row maxima over their
      // own named barrier; each warp signals the MMA warp by itself.
      constexpr int CW = 16;  // columns per thread
      constexpr int kShift = 8 * S - 2;
      const int h = (warp - 2) >> 2;
      const int quarter = warp & 3;
      const int r = quarter * 32 + lane;
      const int64_t xl = (int64_t)xt * AM + r;
      const bool valid = xl < a.lnx;
      const int lo = row_lo[r], hi = row_hi[r];
      // Column c of a tile starting at jl0 is allowed iff (unsigned)(jl0 + c - lo) < span.
      const unsigned span = (valid && lo < hi) ? (unsigned)(hi - lo) : 0u;
      const int eqr = valid ? a.eq[(int64_t)w * a.lnx_pad + xl] : 0;
      const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
      const uint32_t sum_addr = lane_addr + (uint32_t)(kSumCol + h * 2 * CW);
      const double NEG_INF = -INFINITY;
      // z sums the weights times 2^(8S-2); the running sums are in units of
      // their columns' powers of two 2^(2 + ev).
      double m = NEG_INF, z = 0.0, light = INFINITY;
      auto wait = [&](uint64_t* bar, uint32_t parity) {
        if (*(volatile int*)failed) return;
        if (!mbar_wait(bar, parity)) {
          *(volatile int*)failed = 1;
          atomicOr(a.status, 2);
        }
      };
      for (int it = 0; it < n_tiles; it++) {
        const int g = tiles_before + it;
        const int jl0 = (jt0 + it) * AJ + h * CW;
        const int* eks = ek_s + (g % Sh::kStages) * AJ + h * CW;
        wait(qk_full, (uint32_t)(g & 1));
        tc_fence_after();
        double sc[CW];
  #pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          int32_t L[S][4];
          load_levels<S>(lane_addr, h * CW + c4 * 4, L);
  #pragma unroll
          for (int i = 0; i < 4; i++) {
            const int c = c4 * 4 + i;
            const double l = level_sum<S, KB>(L, i);
            sc[c] = FAST ? l * pow2(eqr + eks[c]) : scale2(l, eqr + eks[c]);
          }
        }
        if (a.scale_kind == 1) {
  #pragma unroll
          for (int c = 0; c < CW; c++) sc[c] *= a.scale_c;
        } else if (a.scale_kind == 2) {
  #pragma unroll
          for (int c = 0; c < CW; c++) sc[c] = __ddiv_rn(sc[c], a.scale_c);
        }
        // The mask, and the row's largest and smallest allowed scores.
        const int off = jl0 - lo;
        double mx = NEG_INF;
        if (__all_sync(0xffffffffu, off >= 0 && (unsigned)off + CW <= span)) {
  #pragma unroll
          for (int c = 0; c < CW; c++) {
            mx = fmax(mx, sc[c]);
            light = fmin(light, sc[c]);
          }
        } else {
  #pragma unroll
          for (int c = 0; c < CW; c++) {
            const bool in = (unsigned)(off + c) < span;
            light = fmin(light, in ? sc[c] : INFINITY);
            sc[c] = in ? sc[c] : NEG_INF;
            mx = fmax(mx, sc[c]);
          }
        }
        red[h * AM + r] = mx;
        named_bar(2 + quarter, 128);
        mx = fmax(fmax(red[r], red[AM + r]), fmax(red[2 * AM + r], red[3 * AM + r]));
        const double m_new = fmax(m, mx);
        double rescale = 1.0;
        if (m_new != m) {
          rescale = m == NEG_INF ? 0.0 : exp_tang(m - m_new, texp);
          z *= rescale;
          m = m_new;
        }
        // Weights and their digits: W = exp(s - m) · 2^(8S-2) < 2^(8S-2),
        // balanced base-256 digits, most significant first, four columns a
        // word.
        uint8_t* prow = sP + r * 64;
  #pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          double x[4];
  #pragma unroll
          for (int i = 0; i < 4; i++) {
            const double sv = sc[c4 * 4 + i];
            const double wt = exp_weight(sv - m, texp, kShift);
            x[i] = sv == NEG_INF ? 0.0 : wt;
            z += x[i];
          }
          uint32_t planes[S];
          digit_planes4<S>(x, planes);
          const uint32_t off4 = sw64_offset((uint32_t)r, (uint32_t)(h * CW + c4 * 4)) - (uint32_t)r * 64;
  #pragma unroll
          for (int s = 0; s < S; s++) *(uint32_t*)(prow + s * AM * 64 + off4) = planes[s];
        }
        fence_proxy_async();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(p_full);
        wait(pv_full, (uint32_t)(g & 1));
        tc_fence_after();
        // sums = sums · rescale + this tile's weighted values, four at a time.
  #pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          int32_t L[S][4];
          load_levels<S>(lane_addr, h * CW + c4 * 4, L);
          uint32_t sum[8];
          if (it > 0) {
            tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
            tmem_wait_ld();
          }
  #pragma unroll
          for (int i = 0; i < 4; i++) {
            const double l = combine_levels_small<S, 4>(L, i);
            const double v = it > 0 ? fma(__hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]), rescale, l) : l;
            sum[2 * i] = (uint32_t)__double2loint(v);
            sum[2 * i + 1] = (uint32_t)__double2hiint(v);
          }
          tmem_st8(sum_addr + c4 * 8, sum);
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(tmem_free);
      }
      if (n_tiles > 0) {
        // The four quarters' sums of weights and lightest scores (P's digits
        // are no longer read).
        double* xz = (double*)sP;
        double* xlg = xz + 4 * AM;
        xz[h * AM + r] = z;
        xlg[h * AM + r] = light;
        named_bar(2 + quarter, 128);
        z = ((xz[r] + xz[AM + r]) + (xz[2 * AM + r] + xz[3 * AM + r])) * pow2(-kShift);
        light = fmin(fmin(xlg[r], xlg[AM + r]), fmin(xlg[2 * AM + r], xlg[3 * AM + r]));
        tc_fence_after();
        double o[CW];
  #pragma unroll
        for (int c4 = 0; c4 < CW / 4; c4++) {
          uint32_t sum[8];
          tmem_ld8(sum_addr + c4 * 8, (int32_t*)sum);
          tmem_wait_ld();
  #pragma unroll
          for (int i = 0; i < 4; i++)
            o[c4 * 4 + i] = scale2(__hiloint2double((int)sum[2 * i + 1], (int)sum[2 * i]), 2 + ev_s[h * CW + c4 * 4 + i]);
        }
        if (valid && lo < hi && !*(volatile int*)failed) {
          // Bounds::hold (fused.rs:1058-1086): the heaviest weight is
          // exp(high - m) = 1, the row's largest score being m.
          const double rl = a.rl[x_base + xl], rs = a.rs[x_base + xl];
          bool over = !(z <= 1.7976931348623157e308);
          const double normal = 2.0 * 2.2250738585072014e-308;
          const double lightest = exp(light - m);
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
          double* orow = a.out + (x_base + xl) * a.ny;
  #pragma unroll
          for (int c = 0; c < CW; c++) {
            const int64_t y = (int64_t)a.y0 + h * CW + c;
            if (y >= a.ny) continue;
            if (!isfinite(o[c])) over = true;
            const double v = __ddiv_rn(o[c], z);
            if (!isfinite(v)) over = true;
            if (!no_underflow && !(lost <= rounding * fabs(v))) over = true;
            orow[y] = v;
          }
          if (h == 0 && a.lse && a.y0 == 0) a.lse[x_base + xl] = m + log(z);
          if (over) atomicOr(a.status, 1);
        }
      }
    }
    tiles_before += n_tiles;
    q_loads += n_tiles > 0 ? 1 : 0;
    // The item's TMEM reads and shared-memory uses end before the next
    // item's setup and MMAs.
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// The kernel variant for d <= 64 (KB 1) or <= 128 (KB 2), with or without
// the fast powers of two.
using AttnKernel = void (*)(CUtensorMap, CUtensorMap, CUtensorMap, AttnArgs);

AttnKernel attn_kernel(int kb, bool fast, int* smem) {
  *smem = kb == 1 ? AttnShape<6, 1>::kSmem : AttnShape<6, 2>::kSmem;
  if (kb == 1) return fast ? attn_fwd_split<6, 1, true> : attn_fwd_split<6, 1, false>;
  return fast ? attn_fwd_split<6, 2, true> : attn_fwd_split<6, 2, false>;
}

// How the (query tile, batch) items of a forward pass reach the SMs.
enum Schedule : int {
  kGridSchedule = 0,   // a block per item: the grid's order, or the work list's by key tiles
  kTilesSchedule = 1,  // persistent blocks claiming the items by key tiles, most first
  kBatchSchedule = 2,  // persistent, batch by batch (the most key tiles first), in a batch by key tiles
  kSchedules = 3,
};

// A problem's work lists (the items that join some key).
struct WorkLists {
  std::vector<int2> by_tiles, by_batch;
};

std::mutex g_work_lock;

// The schedules timed fastest, by padded shape and conditions (not by the
// ragged lengths, which a training loop may change at every step).
std::vector<int64_t> tuning_key(const AttentionProblem& p, int kb, bool fast) {
  std::vector<int64_t> key = {p.batches, p.lnx, p.lnj, p.ne, p.ny, kb, fast,
                              (int64_t)(!p.xlen_host.empty() || !p.jlen_host.empty()), p.mask.n};
  for (int i = 0; i < p.mask.n; i++) {
    key.push_back(p.mask.cmp[i]);
    key.push_back(p.mask.off[i]);
  }
  return key;
}
std::map<std::vector<int64_t>, int>& tuned_schedules() {
  static std::map<std::vector<int64_t>, int> tuned;
  return tuned;
}

// The work lists of a problem. Those of the last few shapes (lengths,
// extents, conditions) are kept: a training loop over the same batches
// asks for the same ones at every step.
std::shared_ptr<WorkLists> work_lists(const AttentionProblem& p) {
  std::vector<int64_t> key = {p.batches, p.lnx, p.lnj, p.ne, p.ny, p.mask.n, (int64_t)p.xlen_host.size(),
                              (int64_t)p.jlen_host.size()};
  for (int i = 0; i < p.mask.n; i++) {
    key.push_back(p.mask.cmp[i]);
    key.push_back(p.mask.off[i]);
  }
  key.insert(key.end(), p.xlen_host.begin(), p.xlen_host.end());
  key.insert(key.end(), p.jlen_host.begin(), p.jlen_host.end());
  static std::vector<std::pair<std::vector<int64_t>, std::shared_ptr<WorkLists>>> kept;  // most recent last
  {
    std::lock_guard<std::mutex> g(g_work_lock);
    for (size_t i = 0; i < kept.size(); i++)
      if (kept[i].first == key) {
        auto hit = kept[i];
        kept.erase(kept.begin() + (int64_t)i);
        kept.push_back(hit);
        return hit.second;
      }
  }
  Mask hm = p.mask;
  hm.xlen = p.xlen_host.empty() ? nullptr : p.xlen_host.data();
  hm.jlen = p.jlen_host.empty() ? nullptr : p.jlen_host.data();
  const bool ragged = hm.xlen || hm.jlen;
  // A query tile's key tiles (0: it joins none); without lengths every
  // batch has batch 0's.
  auto key_tiles = [&](int64_t w, int64_t xt) -> int64_t {
    const int64_t rows = hm.xlen ? hm.xlen[w] : p.lnx;
    int64_t first = INT64_MAX, last = INT64_MIN;
    for (int64_t r = xt * AM; r < std::min(rows, xt * AM + AM); r++) {
      int64_t lo, hi;
      allowed(hm, w * p.lnx + r, lo, hi);
      if (lo < hi) {
        first = std::min(first, lo - w * p.lnj);
        last = std::max(last, hi - w * p.lnj);
      }
    }
    return first < last ? (last + AJ - 1) / AJ - first / AJ : 0;
  };
  const int64_t n_xt = (p.lnx + AM - 1) / AM;
  std::vector<int64_t> first_batch;
  if (!ragged)
    for (int64_t xt = 0; xt < n_xt; xt++) first_batch.push_back(key_tiles(0, xt));
  std::vector<std::pair<int64_t, int2>> work;
  std::vector<std::pair<int64_t, int64_t>> batch_total;  // (key tiles, batch)
  for (int64_t w = 0; w < p.batches; w++) {
    int64_t total = 0;
    const int64_t rows = hm.xlen ? hm.xlen[w] : p.lnx;
    for (int64_t xt = 0; xt * AM < rows; xt++) {
      const int64_t n = ragged ? key_tiles(w, xt) : first_batch[(size_t)xt];
      if (n > 0) work.push_back({n, make_int2((int)xt, (int)w)});
      total += n;
    }
    batch_total.push_back({total, w});
  }
  auto most_first = [](const auto& a, const auto& b) { return a.first > b.first; };
  auto lists = std::make_shared<WorkLists>();
  std::stable_sort(work.begin(), work.end(), most_first);
  for (auto& x : work) lists->by_tiles.push_back(x.second);
  std::stable_sort(batch_total.begin(), batch_total.end(), most_first);
  std::vector<int64_t> place((size_t)p.batches);
  for (size_t i = 0; i < batch_total.size(); i++) place[(size_t)batch_total[i].second] = (int64_t)i;
  std::vector<int2> by_batch = lists->by_tiles;
  std::stable_sort(by_batch.begin(), by_batch.end(),
                   [&](const int2& a, const int2& b) { return place[(size_t)a.y] < place[(size_t)b.y]; });
  lists->by_batch = std::move(by_batch);
  std::lock_guard<std::mutex> g(g_work_lock);
  kept.emplace_back(std::move(key), lists);
  if (kept.size() > 8) kept.erase(kept.begin());
  return lists;
}

// EINFOLD_ATTENTION_SCHEDULE = grid | tiles | batches forces a schedule;
// unset, the first call of a shape times them all.
int forced_schedule() {
  const char* s = std::getenv("EINFOLD_ATTENTION_SCHEDULE");
  if (!s || !*s) return -1;
  if (!std::strcmp(s, "grid")) return kGridSchedule;
  if (!std::strcmp(s, "tiles")) return kTilesSchedule;
  if (!std::strcmp(s, "batches")) return kBatchSchedule;
  fail(EINFOLD_INVALID, "EINFOLD_ATTENTION_SCHEDULE is %s, not grid, tiles or batches", s);
  return -1;
}

// EINFOLD_GRAPHS=0 launches directly instead of through CUDA graphs.
bool graphs_enabled() {
  const char* s = std::getenv("EINFOLD_GRAPHS");
  return !(s && !std::strcmp(s, "0"));
}

template <class T>
void put(std::vector<uint8_t>& key, const T& v) {
  const uint8_t* b = (const uint8_t*)&v;
  key.insert(key.end(), b, b + sizeof v);
}

}  // namespace

// Each row's largest and smallest nonzero value magnitude over its allowed
// keys (the bounds of Bounds::hold), from blocks of 64 keys' extrema.
__global__ void block_extrema(int64_t nj, const double* __restrict__ largest, const double* __restrict__ smallest,
                              double* __restrict__ bmax, double* __restrict__ bmin) {
  const int lane = threadIdx.x & 31;
  for (int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b * 64 < nj;
       b += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    double mx = 0.0, mn = INFINITY;
    for (int64_t j = b * 64 + lane; j < min(nj, b * 64 + 64); j += 32) {
      mx = fmax(mx, largest[j]);
      mn = fmin(mn, smallest[j]);
    }
    for (int o = 16; o; o >>= 1) {
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if (lane == 0) {
      bmax[b] = mx;
      bmin[b] = mn;
    }
  }
}

__global__ void row_value_bounds(int64_t nx, Mask m, const double* __restrict__ largest,
                                 const double* __restrict__ smallest, const double* __restrict__ bmax,
                                 const double* __restrict__ bmin, double* __restrict__ rl, double* __restrict__ rs) {
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < nx; x += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo, hi;
    allowed(m, x, lo, hi);
    double mx = 0.0, mn = INFINITY;
    int64_t j = lo;
    for (; j < hi && (j & 63); j++) {
      mx = fmax(mx, largest[j]);
      mn = fmin(mn, smallest[j]);
    }
    for (; j + 64 <= hi; j += 64) {
      mx = fmax(mx, bmax[j >> 6]);
      mn = fmin(mn, bmin[j >> 6]);
    }
    for (; j < hi; j++) {
      mx = fmax(mx, largest[j]);
      mn = fmin(mn, smallest[j]);
    }
    rl[x] = mx;
    rs[x] = mn;
  }
}


AttentionOutcome attention_split(Context& ctx, const AttentionProblem& p, int slices, cudaStream_t stream) {
  // Six slices: their levels (384 TMEM columns) and the rows' FP64 sums
  // (128) fill TMEM.
  const int S = slices;
  if (S != 6) return ATTENTION_INELIGIBLE;
  const int KB = p.ne <= 64 ? 1 : (p.ne <= 128 ? 2 : 0);
  if (KB == 0) return ATTENTION_INELIGIBLE;
  if (p.batches <= 0 || p.lnx <= 0 || p.lnj <= 0 || p.ny <= 0) return ATTENTION_INELIGIBLE;
  if (p.lnx > (1 << 30) || p.lnj > (1 << 30) || p.batches > 65535 || p.batches * S > INT32_MAX) return ATTENTION_INELIGIBLE;
  const int64_t W = p.batches;
  const int64_t lnx_pad = round_up(p.lnx, AM), lnj_pad = round_up(p.lnj, AJ), d_pad = 64 * KB;
  const int64_t ny_pad = round_up(p.ny, AY);
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t szq = al((size_t)(W * S * lnx_pad * d_pad)), szk = al((size_t)(W * S * lnj_pad * d_pad)),
               szv = al((size_t)(W * S * ny_pad * lnj_pad));
  const size_t sze = al((size_t)(W * (lnx_pad + lnj_pad + ny_pad)) * 4), szc = al((size_t)(W * p.ny) * 8);
  DeviceBuffer<uint8_t> scratch(szq + szk + szv + sze + szc + 256, stream);
  uint8_t* b = scratch.get();
  int8_t* qd = (int8_t*)b;
  int8_t* kd = (int8_t*)(b + szq);
  int8_t* vd = (int8_t*)(b + szq + szk);
  int32_t* eq = (int32_t*)(b + szq + szk + szv);
  int32_t* ek = eq + W * lnx_pad;
  int32_t* ev = ek + W * lnj_pad;
  unsigned long long* colmax = (unsigned long long*)(b + szq + szk + szv + sze);
  // [0] slicing, [1] kernel, [2..3] max eq, max -eq, [4..5] max ek, max -ek,
  // [6..7] tile pairs
  int* status = (int*)(b + szq + szk + szv + sze + szc);
  unsigned long long* tiles = (unsigned long long*)(status + 6);
  EF_CUDA(cudaMemsetAsync(status, 0, 32, stream));
  const int init[4] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN};
  EF_CUDA(cudaMemcpyAsync(status + 2, init, 16, cudaMemcpyHostToDevice, stream));
  // Ragged batches: the padding rows are neither read nor given digits. A
  // padding query joins no key and a padding key no query, so their digits
  // only meet masked scores (weights exactly 0) in exact integer sums, and
  // their rows' exponents (0) still bound the scores.
  slice_rows_into(S, p.q, W, p.lnx, p.ne, p.ne, lnx_pad, d_pad, eq, qd, status, stream, p.mask.xlen,
                  p.mask.xlen != nullptr);
  slice_rows_into(S, p.k, W, p.lnj, p.ne, p.ne, lnj_pad, d_pad, ek, kd, status, stream, p.mask.jlen,
                  p.mask.jlen != nullptr);
  slice_cols_into(S, p.v, W, p.lnj, p.ny, ny_pad, lnj_pad, colmax, ev, vd, status, stream, p.mask.jlen);
  exponent_range(eq, W * lnx_pad, status + 2, stream);
  exponent_range(ek, W * lnj_pad, status + 4, stream);
  ctx.kernels += 6;
  int st[6];
  EF_CUDA(cudaMemcpyAsync(st, status, 24, cudaMemcpyDeviceToHost, stream));
  EF_CUDA(cudaStreamSynchronize(stream));
  ctx.phase("attention: sliced");
  // Every operand finite, and no score near overflow: |s| < ne · 2^(eq+ek-4).
  if (st[0] & 1) return ATTENTION_INELIGIBLE;
  if ((int64_t)st[2] + st[4] + 8 + (int64_t)std::ceil(std::log2((double)p.ne + 1)) > 1000) return ATTENTION_INELIGIBLE;
  // Scores' powers of two 2^(eq + ek) all normal doubles (the bound above
  // keeps eq + ek below 1000).
  const bool fast = (int64_t)st[3] + st[5] <= 1022;

  const CUtensorMap tq = digit_planes_map(qd, d_pad, lnx_pad, W * S, AM, S);
  const CUtensorMap tk = digit_planes_map(kd, d_pad, lnj_pad, W * S, AJ, S);
  const CUtensorMap tv = digit_planes_map(vd, lnj_pad, ny_pad, W * S, AY, S);
  AttnArgs args{};
  args.mask = p.mask;
  args.lnx = p.lnx;
  args.lnj = p.lnj;
  args.lnx_pad = lnx_pad;
  args.lnj_pad = lnj_pad;
  args.ny = p.ny;
  args.ny_pad = ny_pad;
  args.scale_kind = p.scale_kind;
  args.scale_c = p.scale_c;
  args.eq = eq;
  args.ek = ek;
  args.ev = ev;
  // The rows' value bounds for the guard, from blocks of 64 keys.
  const int64_t nx = W * p.lnx, nj = W * p.lnj;
  DeviceBuffer<double> bounds((size_t)(2 * nx + 2 * ((nj + 63) / 64)), stream);
  double* rl = bounds.get();
  double* rs = rl + nx;
  double* bmax = rs + nx;
  double* bmin = bmax + (nj + 63) / 64;
  block_extrema<<<blocks_for((uint64_t)((nj + 63) / 64) * 32, 256), 256, 0, stream>>>(nj, p.largest, p.smallest, bmax,
                                                                                     bmin);
  row_value_bounds<<<blocks_for((uint64_t)nx, 256), 256, 0, stream>>>(nx, p.mask, p.largest, p.smallest, bmax, bmin,
                                                                      rl, rs);
  EF_LAUNCH_CHECK();
  ctx.kernels += 2;
  args.rl = rl;
  args.rs = rs;
  args.exp_table = exp_table(ctx.device);
  args.out = p.out;
  args.lse = p.lse;
  args.status = status + 1;
  args.tiles = tiles;
  {
    // The query tiles whose rows join the most keys first: the last ones
    // under a causal mask, the first ones when the mask runs the other way.
    Mask m = p.mask;
    m.xlen = m.jlen = nullptr;
    int64_t lo0, hi0, lo1, hi1;
    allowed(m, 0, lo0, hi0);
    allowed(m, p.lnx - 1, lo1, hi1);
    args.reverse = hi1 - lo1 >= hi0 - lo0;
  }
  // The items that join some key, by key tiles and batch by batch.
  const std::shared_ptr<WorkLists> lists = work_lists(p);
  const int n_items = (int)lists->by_tiles.size();
  if (n_items == 0) return ATTENTION_DONE;
  const bool ragged = !p.xlen_host.empty() || !p.jlen_host.empty();
  const int n_y = (int)((p.ny + AY - 1) / AY);
  DeviceBuffer<int2> items((size_t)n_items * 2, stream);
  EF_CUDA(cudaMemcpyAsync(items.get(), lists->by_tiles.data(), (size_t)n_items * sizeof(int2),
                          cudaMemcpyHostToDevice, stream));
  EF_CUDA(cudaMemcpyAsync(items.get() + n_items, lists->by_batch.data(), (size_t)n_items * sizeof(int2),
                          cudaMemcpyHostToDevice, stream));
  DeviceBuffer<unsigned> counters((size_t)n_y, stream);
  int smem = 0;
  const AttnKernel kernel = attn_kernel(KB, fast, &smem);
  EF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int persistent_blocks = std::min(n_items, ctx.sm_count);
  // The tile phase under a schedule: a launch per block of 64 value columns
  // (persistent ones after zeroing their item counters).
  auto enqueue = [&](int schedule, cudaStream_t st) {
    AttnArgs ar = args;
    dim3 grid((unsigned)(lnx_pad / AM), (unsigned)W);
    if (schedule == kGridSchedule) {
      if (ragged) {
        ar.items = items.get();
        ar.n_items = n_items;
        grid = dim3((unsigned)n_items, 1);
      }
    } else {
      ar.items = items.get() + (schedule == kBatchSchedule ? n_items : 0);
      ar.n_items = n_items;
      grid = dim3((unsigned)persistent_blocks, 1);
      EF_CUDA(cudaMemsetAsync(counters.get(), 0, (size_t)n_y * sizeof(unsigned), st));
    }
    for (int yb = 0; yb < n_y; yb++) {
      ar.y0 = yb * AY;
      ar.next = schedule == kGridSchedule ? nullptr : counters.get() + yb;
      kernel<<<grid, kAttnThreads, smem, st>>>(tq, tk, tv, ar);
      EF_LAUNCH_CHECK();
    }
  };
  cudaEvent_t e0, e1;
  EF_CUDA(cudaEventCreate(&e0));
  EF_CUDA(cudaEventCreate(&e1));
  int schedule = forced_schedule();
  const std::vector<int64_t> tkey = tuning_key(p, KB, fast);
  if (schedule < 0) {
    std::lock_guard<std::mutex> g(g_work_lock);
    const auto it = tuned_schedules().find(tkey);
    if (it != tuned_schedules().end()) schedule = it->second;
  }
  if (schedule < 0) {
    // The first call of this shape: each schedule twice (the same results
    // each time), the fastest by its shorter run.
    float best = INFINITY;
    for (int sc = 0; sc < kSchedules; sc++) {
      for (int rep = 0; rep < 2; rep++) {
        EF_CUDA(cudaEventRecord(e0, stream));
        enqueue(sc, stream);
        EF_CUDA(cudaEventRecord(e1, stream));
        EF_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        EF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ctx.kernels += (uint64_t)n_y;
        if (ms < best) {
          best = ms;
          schedule = sc;
        }
      }
    }
    {
      std::lock_guard<std::mutex> g(g_work_lock);
      auto& tuned = tuned_schedules();
      if (tuned.size() >= 256) tuned.clear();
      tuned[tkey] = schedule;
    }
    EF_CUDA(cudaMemsetAsync(tiles, 0, sizeof(unsigned long long), stream));
  }
  EF_CUDA(cudaEventRecord(e0, stream));
  if (graphs_enabled()) {
    // Replayed while every argument of the launches is the same (pointers
    // included); else captured again and updated in place.
    std::vector<uint8_t> shape, key;
    put(shape, ctx.device);
    put(shape, KB);
    put(shape, fast);
    put(shape, schedule);
    put(shape, n_y);
    put(shape, ragged);
    put(shape, persistent_blocks);
    for (const void* ptr : {(const void*)scratch.get(), (const void*)items.get(), (const void*)counters.get(),
                            (const void*)rl, (const void*)p.out, (const void*)p.lse, (const void*)args.exp_table,
                            (const void*)p.mask.xlen, (const void*)p.mask.jlen})
      put(key, ptr);
    for (int64_t x : {W, p.lnx, p.lnj, p.ne, p.ny, lnx_pad, lnj_pad, ny_pad, (int64_t)n_items, (int64_t)p.scale_kind,
                      (int64_t)args.reverse, (int64_t)p.mask.n, p.mask.lnx, p.mask.lnj})
      put(key, x);
    put(key, p.scale_c);
    for (int i = 0; i < p.mask.n; i++) {
      put(key, p.mask.cmp[i]);
      put(key, p.mask.off[i]);
    }
    ctx.graph = ctx.graphs.run(shape, key, stream, [&](cudaStream_t st) { enqueue(schedule, st); });
  } else {
    enqueue(schedule, stream);
  }
  ctx.kernels += (uint64_t)n_y;
  ctx.schedule = schedule;
  EF_CUDA(cudaEventRecord(e1, stream));
  unsigned long long pairs = 0;
  EF_CUDA(cudaMemcpyAsync(st, status + 1, 4, cudaMemcpyDeviceToHost, stream));
  EF_CUDA(cudaMemcpyAsync(&pairs, tiles, 8, cudaMemcpyDeviceToHost, stream));
  EF_CUDA(cudaStreamSynchronize(stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // Digit products executed: per pair of tiles, S(S+1)/2 digit pairs of a
  // 128 x 64 x d_pad product (scores) and of a 128 x 64 x 64 one (values).
  ctx.product_ms += ms;
  ctx.product_ops += (double)pairs * (S * (S + 1) / 2) * 2.0 * AM * AJ * (double)(d_pad + AY);
  ctx.phase("attention: tiles");
  if (st[0] & 2) fail(EINFOLD_TIMEOUT, "a bounded wait in the attention kernel ran out");
  return (st[0] & 1) ? ATTENTION_GUARDED : ATTENTION_DONE;
}

}  // namespace ef
