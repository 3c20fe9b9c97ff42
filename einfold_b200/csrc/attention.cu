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
//   2. Eight epilogue warps read the levels (a row per TMEM lane, half the
//      columns per warp group), combine them in FP64 under the row's and
//      key's powers of two, apply the mask, update the running maximum
//      (shared between the two halves), rescale the running sums, and turn
//      the weights exp(s - m) in [0, 1] into S digit planes of a fixed scale
//      2^2, written to shared memory in the MMA's 64-byte swizzle.
//   3. w·v: the weights' digits against v's column-scaled digits, the same
//      level scheme, into the same TMEM columns (q·k's levels were read).
//   4. The epilogue adds the levels to its FP64 sums.
// A TMA producer warp double-buffers k and v tiles; an MMA warp issues both
// products. Every wait is bounded (2 s); on a timeout the kernel sets a
// status bit, waits for its copies and MMAs in flight, frees TMEM and
// returns.
//
// Accuracy: each operand value carries 8S - 2 bits under its row's (or
// column's) power of two, levels above S + 1 are dropped, and every level
// sum is exact, so a score's error is about ne · 2^(3-8S) · max|q| · max|k|
// and a weight's about 2^(1-8S): with S = 6, scores to ~1e-14 of their scale
// and averages to ~1e-14 of max|v|.
#include <algorithm>
#include <cmath>

#include "attention.cuh"
#include "gemm.cuh"
#include "ptx.cuh"

namespace ef {
namespace {

using namespace ptx;

constexpr int AM = 128;  // query rows per CTA (TMEM lanes)
constexpr int AJ = 64;   // key positions per tile
constexpr int AY = 64;   // value columns per CTA
constexpr int kEpi = 256;
constexpr int kAttnThreads = 64 + kEpi;
constexpr int kMaxSmem = 232448;

template <int S, int KB>
struct AttnShape {
  static constexpr int kQ = KB * S * AM * 64;  // q digits [kb][s][128][64 B]
  static constexpr int kK = KB * S * AJ * 64;  // k digits per stage [kb][t][64][64 B]
  static constexpr int kV = S * AY * 64;       // v digits per stage [t][64 y][64 B of j]
  static constexpr int kP = S * AM * 64;       // weight digits [s][128][64 B of j]
  static constexpr int kAux = 4096;            // barriers, row spans, exchanges, exponents
  static constexpr int kFixed = kQ + kP + kAux + 1024;
  static constexpr int kStages = kFixed + 2 * (kK + kV) <= kMaxSmem ? 2 : 1;
  static constexpr int kSmem = kFixed + kStages * (kK + kV);
  static_assert(kSmem <= kMaxSmem, "the tiles must fit in shared memory");
  static_assert(S * 64 <= 512, "the levels must fit in TMEM");
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
  const double* largest;
  const double* smallest;
  double* out;  // [w·lnx + x][ny]
  double* lse;  // [w·lnx + x] or null
  int* status;  // bit 0: a guard fired; bit 1: a wait ran out
  unsigned long long* tiles;  // (row tile, key tile) pairs computed
};

// The S levels of one TMEM column, combined: Σ_l L_l 2^{-8(l+2)}, in groups
// of three summed exactly in int64 and added from the smallest group up.
template <int S>
__device__ __forceinline__ double combine(const int32_t (&L)[S][8], int i) {
  double v = 0.0;
#pragma unroll
  for (int g = (S - 1) / 3; g >= 0; g--) {
    long long part = 0;
    const int l0 = 3 * g, l1 = (3 * g + 3 < S ? 3 * g + 3 : S);
#pragma unroll
    for (int l = l0; l < l1; l++) part = part * 256 + (long long)L[l][i];
    v += (double)part * pow2(-8 * (l1 + 1));
  }
  return v;
}

template <int S, int KB>
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
  long long* span = (long long*)(tmem_slot + 4);  // first, last
  int* row_lo = (int*)(aux + 256);                // [128]
  int* row_hi = row_lo + AM;                      // [128]
  int* ev_s = row_hi + AM;                        // [64]
  double* red = (double*)(aux + 2048);            // [2][128]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xt = (int)(gridDim.x - 1 - blockIdx.x);  // the longest rows of a causal mask first
  const int w = blockIdx.y;
  const int64_t x_base = (int64_t)w * a.lnx;

  if (threadIdx.x == 0) {
    mbar_init(q_full, 1);
    for (int i = 0; i < 2; i++) {
      mbar_init(&kv_full[i], 1);
      mbar_init(&kv_empty[i], 1);
    }
    mbar_init(qk_full, 1);
    mbar_init(pv_full, 1);
    mbar_init(p_full, 1);
    mbar_init(tmem_free, 1);
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
  const uint32_t tmem = *tmem_slot;
  const long long first = span[0], last = span[1];
  const int jt0 = first < last ? (int)(first / AJ) : 0;
  const int n_tiles = first < last ? (int)((last + AJ - 1) / AJ) - jt0 : 0;
  if (threadIdx.x == 0 && n_tiles > 0) atomicAdd(a.tiles, (unsigned long long)n_tiles);

  if (warp == 0) {
    if (lane == 0 && n_tiles > 0) {
      // Producer: q's digits once, then k's and v's per tile.
      prefetch_map(&tq);
      prefetch_map(&tk);
      prefetch_map(&tv);
      mbar_expect_tx(q_full, (uint32_t)Sh::kQ);
      for (int kb = 0; kb < KB; kb++) tma_load_3d(sQ + kb * S * AM * 64, &tq, q_full, kb * 64, xt * AM, w * S);
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
        mbar_expect_tx(&kv_full[st], (uint32_t)(Sh::kK + Sh::kV));
        const int jl0 = (jt0 + it) * AJ;
        for (int kb = 0; kb < KB; kb++)
          tma_load_3d(sK + st * Sh::kK + kb * S * AJ * 64, &tk, &kv_full[st], kb * 64, jl0, w * S);
        tma_load_3d(sV + st * Sh::kV, &tv, &kv_full[st], jl0, a.y0, w * S);
        issued = it + 1;
      }
      // Copies still in flight complete before the CTA may exit.
      mbar_wait(q_full, 0);
      for (int it = std::max(0, issued - Sh::kStages); it < issued; it++)
        mbar_wait(&kv_full[it % Sh::kStages], (uint32_t)((it / Sh::kStages) & 1));
    }
  } else if (warp == 1) {
    if (lane == 0 && n_tiles > 0) {
      // MMA issuer.
      uint64_t* last_bar = nullptr;
      uint32_t last_parity = 0;
      bool ok = mbar_wait(q_full, 0);
      for (int it = 0; ok && it < n_tiles; it++) {
        const int st = it % Sh::kStages;
        const uint32_t round = (uint32_t)(it / Sh::kStages);
        ok = mbar_wait(&kv_full[st], round & 1) && (it == 0 || mbar_wait(tmem_free, (uint32_t)((it - 1) & 1)));
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
        last_parity = (uint32_t)(it & 1);
        ok = mbar_wait(p_full, (uint32_t)(it & 1));
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
        last_parity = (uint32_t)(it & 1);
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
    // columns 0..31 of each tile, warps 6..9 columns 32..63.
    const int h = (warp - 2) >> 2;
    const int r = (warp & 3) * 32 + lane;
    const int64_t xl = (int64_t)xt * AM + r;
    const bool valid = xl < a.lnx;
    const int lo = row_lo[r], hi = row_hi[r];
    const int eqr = valid ? a.eq[(int64_t)w * a.lnx_pad + xl] : 0;
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const double NEG_INF = -INFINITY;
    double m = NEG_INF, z = 0.0, light = INFINITY, rl = 0.0, rs = INFINITY;
    long long terms = 0;
    double o[32];
#pragma unroll
    for (int c = 0; c < 32; c++) o[c] = 0.0;
    bool ok = true;
    for (int it = 0; it < n_tiles; it++) {
      const int jl0 = (jt0 + it) * AJ;
      ok = named_bar_and(1, kEpi, mbar_wait(qk_full, (uint32_t)(it & 1)));
      if (!ok) break;
      tc_fence_after();
      double sc[32];
#pragma unroll
      for (int c8 = 0; c8 < 4; c8++) {
        int32_t L[S][8];
#pragma unroll
        for (int l = 0; l < S; l++) tmem_ld8(lane_addr + (uint32_t)(l * AJ + h * 32 + c8 * 8), L[l]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int jl = jl0 + h * 32 + c8 * 8 + i;
          double s = scale2(combine<S>(L, i), eqr + a.ek[(int64_t)w * a.lnj_pad + jl]);
          if (a.scale_kind == 1) s = s * a.scale_c;
          else if (a.scale_kind == 2) s = __ddiv_rn(s, a.scale_c);
          sc[c8 * 8 + i] = s;
        }
      }
      // The row's allowed keys in this half tile, their largest score, and
      // the guard's statistics.
      double mx = NEG_INF;
#pragma unroll
      for (int c = 0; c < 32; c++) {
        const int jl = jl0 + h * 32 + c;
        if (valid && jl >= lo && jl < hi) {
          mx = fmax(mx, sc[c]);
          light = fmin(light, sc[c]);
          terms++;
          rl = fmax(rl, a.largest[(int64_t)w * a.lnj + jl]);
          rs = fmin(rs, a.smallest[(int64_t)w * a.lnj + jl]);
        } else {
          sc[c] = NEG_INF;
        }
      }
      red[h * AM + r] = mx;
      named_bar(1, kEpi);
      mx = fmax(mx, red[(1 - h) * AM + r]);
      const double m_new = fmax(m, mx);
      if (m_new != m) {
        const double rescale = m == NEG_INF ? 0.0 : exp(m - m_new);
        z *= rescale;
#pragma unroll
        for (int c = 0; c < 32; c++) o[c] *= rescale;
        m = m_new;
      }
      // Weights and their digits: W = w · 2^(8S-2) < 2^(8S-2), balanced
      // base-256 digits, most significant first.
      const double to_int = pow2(8 * S - 2);
#pragma unroll
      for (int c16 = 0; c16 < 2; c16++) {
        uint32_t wd[S][4];
#pragma unroll
        for (int s = 0; s < S; s++)
#pragma unroll
          for (int q = 0; q < 4; q++) wd[s][q] = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const double s0 = sc[c16 * 16 + i];
          const double wt = s0 == NEG_INF ? 0.0 : exp(s0 - m);
          z += wt;
          long long W = llrint(wt * to_int);
#pragma unroll
          for (int s = S - 1; s >= 0; s--) {
            const long long d = ((W + 128) & 255) - 128;
            wd[s][i >> 2] |= ((uint32_t)(d & 255)) << (8 * (i & 3));
            W = (W - d) >> 8;
          }
        }
#pragma unroll
        for (int s = 0; s < S; s++)
          *(uint4*)(sP + s * AM * 64 + sw64_offset((uint32_t)r, (uint32_t)((2 * h + c16) * 16))) =
              make_uint4(wd[s][0], wd[s][1], wd[s][2], wd[s][3]);
      }
      fence_proxy_async();
      tc_fence_before();
      named_bar(1, kEpi);
      if (warp == 2 && lane == 0) mbar_arrive(p_full);
      ok = named_bar_and(1, kEpi, mbar_wait(pv_full, (uint32_t)(it & 1)));
      if (!ok) break;
      tc_fence_after();
#pragma unroll
      for (int c8 = 0; c8 < 4; c8++) {
        int32_t L[S][8];
#pragma unroll
        for (int l = 0; l < S; l++) tmem_ld8(lane_addr + (uint32_t)(l * AY + h * 32 + c8 * 8), L[l]);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; i++) o[c8 * 8 + i] += scale2(combine<S>(L, i), 2 + ev_s[h * 32 + c8 * 8 + i]);
      }
      tc_fence_before();
      named_bar(1, kEpi);
      if (warp == 2 && lane == 0) mbar_arrive(tmem_free);
    }
    if (!ok) {
      if (warp == 2 && lane == 0) {
        atomicOr(a.status, 2);
        *(volatile int*)failed = 1;
      }
    } else if (n_tiles > 0) {
      // The two halves' sums and statistics (P's digits are no longer read).
      double* xz = (double*)sP;
      double* xl_ = xz + 2 * AM;
      double* xrl = xl_ + 2 * AM;
      double* xrs = xrl + 2 * AM;
      long long* xt_ = (long long*)(xrs + 2 * AM);
      xz[h * AM + r] = z;
      xl_[h * AM + r] = light;
      xrl[h * AM + r] = rl;
      xrs[h * AM + r] = rs;
      xt_[h * AM + r] = terms;
      named_bar(1, kEpi);
      const int o2 = (1 - h) * AM + r;
      z += xz[o2];
      light = fmin(light, xl_[o2]);
      rl = fmax(rl, xrl[o2]);
      rs = fmin(rs, xrs[o2]);
      terms += xt_[o2];
      if (valid && lo < hi) {
        // Bounds::hold (fused.rs:1058-1086): the heaviest weight is
        // exp(high - m) = 1, the row's largest score being m.
        bool over = !(z <= 1.7976931348623157e308);
        const double normal = 2.0 * 2.2250738585072014e-308;
        const double heaviest = 1.0, lightest = exp(light - m);
        const double t2 = 2.0 * (double)terms;
        bool finite = isfinite(heaviest * rl * t2);
        if (finite) {
          const double quotient = heaviest / fabs(z);
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
        for (int c = 0; c < 32; c++) {
          const int64_t y = (int64_t)a.y0 + h * 32 + c;
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
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

__global__ void exp_max(const int32_t* __restrict__ e, int64_t n, int* __restrict__ out) {
  int m = INT_MIN;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = max(m, e[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

template <int S, int KB>
void launch(const CUtensorMap& tq, const CUtensorMap& tk, const CUtensorMap& tv, const AttnArgs& args, dim3 grid,
            cudaStream_t stream) {
  using Sh = AttnShape<S, KB>;
  EF_CUDA(cudaFuncSetAttribute(attn_fwd_split<S, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem));
  attn_fwd_split<S, KB><<<grid, kAttnThreads, Sh::kSmem, stream>>>(tq, tk, tv, args);
  EF_LAUNCH_CHECK();
}

}  // namespace

AttentionOutcome attention_split(Context& ctx, const AttentionProblem& p, int slices, cudaStream_t stream) {
  const int S = slices;
  if (S != 6 && S != 7) return ATTENTION_INELIGIBLE;
  const int KB = p.ne <= 64 ? 1 : (p.ne <= 128 ? 2 : 0);
  if (KB == 0 || (S == 7 && KB == 2)) return ATTENTION_INELIGIBLE;
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
  // [0] slicing, [1] kernel, [2] max eq, [3] max ek, [4..5] tile pairs
  int* status = (int*)(b + szq + szk + szv + sze + szc);
  unsigned long long* tiles = (unsigned long long*)(status + 4);
  EF_CUDA(cudaMemsetAsync(status, 0, 24, stream));
  const int init[2] = {INT_MIN, INT_MIN};
  EF_CUDA(cudaMemcpyAsync(status + 2, init, 8, cudaMemcpyHostToDevice, stream));
  slice_rows_into(S, p.q, W, p.lnx, p.ne, p.ne, lnx_pad, d_pad, eq, qd, status, stream);
  slice_rows_into(S, p.k, W, p.lnj, p.ne, p.ne, lnj_pad, d_pad, ek, kd, status, stream);
  slice_cols_into(S, p.v, W, p.lnj, p.ny, ny_pad, lnj_pad, colmax, ev, vd, status, stream);
  exp_max<<<blocks_for((uint64_t)(W * lnx_pad), 256), 256, 0, stream>>>(eq, W * lnx_pad, status + 2);
  exp_max<<<blocks_for((uint64_t)(W * lnj_pad), 256), 256, 0, stream>>>(ek, W * lnj_pad, status + 3);
  ctx.kernels += 6;
  int st[4];
  EF_CUDA(cudaMemcpyAsync(st, status, 16, cudaMemcpyDeviceToHost, stream));
  EF_CUDA(cudaStreamSynchronize(stream));
  ctx.phase("attention: sliced");
  // Every operand finite, and no score near overflow: |s| < ne · 2^(eq+ek-4).
  if (st[0] & 1) return ATTENTION_INELIGIBLE;
  if ((int64_t)st[2] + st[3] + 8 + (int64_t)std::ceil(std::log2((double)p.ne + 1)) > 1000) return ATTENTION_INELIGIBLE;

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
  args.largest = p.largest;
  args.smallest = p.smallest;
  args.out = p.out;
  args.lse = p.lse;
  args.status = status + 1;
  args.tiles = tiles;
  const dim3 grid((unsigned)(lnx_pad / AM), (unsigned)W);
  cudaEvent_t e0, e1;
  EF_CUDA(cudaEventCreate(&e0));
  EF_CUDA(cudaEventCreate(&e1));
  EF_CUDA(cudaEventRecord(e0, stream));
  for (int64_t y0 = 0; y0 < p.ny; y0 += AY) {
    args.y0 = (int)y0;
    if (S == 6 && KB == 1) launch<6, 1>(tq, tk, tv, args, grid, stream);
    else if (S == 6) launch<6, 2>(tq, tk, tv, args, grid, stream);
    else launch<7, 1>(tq, tk, tv, args, grid, stream);
    ctx.kernels++;
  }
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
