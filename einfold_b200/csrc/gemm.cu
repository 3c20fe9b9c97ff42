// Dense products on the B200: the split product on the tensor cores
// (tcgen05 kind::i8, operands staged by TMA, level accumulators in TMEM),
// and the FP64 product on the CUDA cores in the reference's order.
//
// The split product. Each row of A (and of BT, a column of B) is scaled by a
// power of two 2^e with |x / 2^e| < 1/4, rounded to 8S fractional bits, and
// written as S balanced base-256 digits in [-128, 127], most significant
// first: x ≈ 2^e Σ_s d_s 2^{-8s}. A product a·b is then 2^{e+f} Σ_{s,t}
// d_s g_t 2^{-8(s+t)}; the terms of level l = s + t ≤ S + 1 are kept (the
// others are below the rounding of the digits), and each level's sum over k
// is an exact int32 accumulation on the tensor cores while S·k·2^14 < 2^31.
// One MMA per digit s of A covers every digit t ≤ S + 1 - s of B at once: the
// B tile holds B's digits stacked along N, and the MMA's accumulator starts
// at TMEM column (s - 1)·64, so that the product of digits s and t lands in
// column (s + t - 2)·64 + j: level l's accumulator. The epilogue reads the S
// levels, combines them in FP64 from the smallest up, and scales by 2^{e+f}.
// Integer sums are exact, so the result doesn't depend on the tiling, the
// order of the MMAs, or the number of SMs.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <climits>
#include <mutex>
#include <type_traits>

#include "gemm.cuh"
#include "levels.cuh"
#include "ptx.cuh"

namespace ef {
namespace {

using namespace ptx;

constexpr int BM = 128;  // rows of A per tile (TMEM lanes)
constexpr int BN = 64;   // columns of C per tile (per level)
constexpr int BK = 64;   // bytes (int8 values) of k per pipeline stage
constexpr int kThreads = 192;
constexpr int kGroup = 8;                    // tile rows per raster group

// 2^{-8l}.
__device__ __forceinline__ double exp2_neg8(int l) { return pow2(-8 * l); }

// Instruction descriptor of the split product: M = BM.
__host__ __device__ constexpr uint32_t idesc_i8(int n) { return ptx::idesc_i8(BM, n); }

template <int S>
struct SplitShape {
  static constexpr int kASlab = BM * BK;
  static constexpr int kBSlab = BN * BK;
  static constexpr int kStage = S * (kASlab + kBSlab);
  static constexpr int kStagesFit = (220 * 1024) / kStage;
  static constexpr int kStages = kStagesFit > 4 ? 4 : kStagesFit;
  static constexpr int kSmem = kStages * kStage + 1024 + 256;
  // TMEM columns: S levels of BN int32 columns, rounded up to a power of two.
  static constexpr uint32_t kTmemCols = S * BN <= 128 ? 128 : (S * BN <= 256 ? 256 : 512);
  static_assert(kStages >= 2, "two pipeline stages must fit");
};

template <int S>
__global__ void __launch_bounds__(kThreads, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
                      const int32_t* __restrict__ ea, const int32_t* __restrict__ eb, double* __restrict__ c,
                      int m, int n, int m_pad, int n_pad, int kb0, int k_blocks, int tiles_m, int tiles_n,
                      int accumulate, int* status) {
  using Sh = SplitShape<S>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + Sh::kStages * S * Sh::kASlab;
  uint64_t* full = (uint64_t*)(sB + Sh::kStages * S * Sh::kBSlab);
  uint64_t* empty = full + Sh::kStages;
  uint64_t* done = empty + Sh::kStages;
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  int* failed = (int*)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int w = blockIdx.y;
  // Grouped raster: kGroup tile rows share each tile column in turn, so the
  // CTAs on the GPU at once read a compact block of A's and B's digits.
  const int tile = blockIdx.x;
  const int per_group = kGroup * tiles_n;
  const int first_m = (tile / per_group) * kGroup;
  const int group_rows = min(tiles_m - first_m, kGroup);
  const int tm = first_m + (tile % per_group) % group_rows;
  const int tn = (tile % per_group) / group_rows;
  const int m0 = tm * BM, n0 = tn * BN;

  if (threadIdx.x == 0) {
    for (int i = 0; i < Sh::kStages; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    *failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, Sh::kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // Producer: one 3D TMA load per operand per stage brings all S digits.
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tma_a) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tma_b) : "memory");
    for (int kb = 0; kb < k_blocks; kb++) {
      const int st = kb % Sh::kStages;
      const uint32_t round = (uint32_t)(kb / Sh::kStages);
      if (!mbar_wait(&empty[st], (round & 1) ^ 1)) {
        atomicOr(status, 2);
        *failed = 1;
        break;
      }
      mbar_expect_tx(&full[st], (uint32_t)Sh::kStage);
      const int kc = (kb0 + kb) * BK;
      tma_load_3d(sA + st * S * Sh::kASlab, &tma_a, &full[st], kc, m0, w * S);
      tma_load_3d(sB + st * S * Sh::kBSlab, &tma_b, &full[st], kc, n0, w * S);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer.
    for (int kb = 0; kb < k_blocks; kb++) {
      const int st = kb % Sh::kStages;
      const uint32_t round = (uint32_t)(kb / Sh::kStages);
      if (!mbar_wait(&full[st], round & 1)) {
        atomicOr(status, 2);
        *failed = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a_base = smem_u32(sA + st * S * Sh::kASlab);
      const uint32_t b_base = smem_u32(sB + st * S * Sh::kBSlab);
#pragma unroll
      for (int kk = 0; kk < BK / 32; kk++) {
#pragma unroll
        for (int s = 1; s <= S; s++) {
          const int total = (S + 1 - s) * BN;
#pragma unroll
          for (int nn0 = 0; nn0 < total; nn0 += 256) {
            const int nn = total - nn0 < 256 ? total - nn0 : 256;
            const uint64_t ad = desc_sw64(a_base + (s - 1) * Sh::kASlab + kk * 32);
            const uint64_t bd = desc_sw64(b_base + nn0 * BK + kk * 32);
            const uint32_t acc = (kb > 0 || kk > 0 || s > 1) ? 1u : 0u;
            umma_i8(tmem + (uint32_t)((s - 1) * BN + nn0), ad, bd, idesc_i8(nn), acc);
          }
        }
      }
      umma_commit(&empty[st]);
    }
    // Signals the epilogue once every MMA issued so far has completed.
    umma_commit(done);
  } else if (warp >= 2) {
    // Epilogue: warp w reads TMEM lanes 32·(w % 4) .. +31, one row per thread.
    const bool ok = mbar_wait(done, 0, true);
    tc_fence_after();
    if (!ok) atomicOr(status, 2);
    const int q = warp & 3;
    const int r = m0 + q * 32 + lane;
    const bool run = ok && !*failed && k_blocks > 0;
    const int er = run && r < m ? ea[(int64_t)w * m_pad + r] : 0;
    double* crow = c + ((int64_t)w * m + r) * (int64_t)n;
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
    for (int chunk = 0; chunk < BN / 16; chunk++) {
      int32_t acc[S][16];
      if (run) {
#pragma unroll
        for (int l = 0; l < S; l++) tmem_ld16(lane_addr + (uint32_t)(l * BN + chunk * 16), acc[l]);
        tmem_wait_ld();
      }
      if (run && r < m) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int col = n0 + chunk * 16 + j;
          if (col >= n) continue;
          // Levels 2.. S+1 in groups of three, each summed exactly in int64
          // (|level| < 2^31, so three of them shifted by 8 bits fit in 2^48),
          // then converted once and added from the smallest group up.
          double v = 0.0;
#pragma unroll
          for (int g = (S - 1) / 3; g >= 0; g--) {
            long long part = 0;
            const int l0 = 3 * g, l1 = (3 * g + 3 < S ? 3 * g + 3 : S);
#pragma unroll
            for (int l = l0; l < l1; l++) part = part * 256 + (long long)acc[l][j];
            // part carries levels l0+2 .. l1+1, its last at weight 2^{-8(l1+1)}.
            v += (double)part * exp2_neg8(l1 + 1);
          }
          const int e = er + eb[(int64_t)w * n_pad + col];
          double x = (e > -960 && e < 960) ? v * pow2(e) : ldexp(v, e);
          if (accumulate) x += crow[col];
          crow[col] = x;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, Sh::kTmemCols);
  }
}

// Slices rows of x [batches][rows][k] (leading dimension ld): for each row,
// the exponent e with max|x| < 2^(e-2) (0 for a row of zeros), then the S
// digits of x / 2^e, written to digits[(w·S + s)][r][k] for r < rows_pad and
// k < k_pad (zeros beyond). One block per row: the second pass over a row
// reads it from L2. Status bit 1 if a value isn't finite.
template <int S>
__global__ void __launch_bounds__(256) slice_rows(const double* __restrict__ x, int64_t batches, int64_t rows,
                                                  int64_t k, int64_t ld, int64_t rows_pad, int64_t k_pad,
                                                  int32_t* __restrict__ e_out, int8_t* __restrict__ digits,
                                                  int* status, const int64_t* __restrict__ lens) {
  __shared__ double red[8];
  __shared__ int ex_s;
  const int64_t slab = rows_pad * k_pad;
  for (int64_t g = blockIdx.x; g < batches * rows_pad; g += gridDim.x) {
    const int64_t w = g / rows_pad, r = g % rows_pad;
    const double* row = x + (w * rows + r) * ld;
    const bool live = r < rows && (!lens || r < lens[w]);
    double m = 0.0;
    bool bad = false;
    if (live) {
      for (int64_t i = threadIdx.x; i < k; i += blockDim.x) {
        const double v = fabs(row[i]);
        bad |= !(v <= 1.7976931348623157e308);
        m = fmax(m, v);
      }
    }
    if (bad) atomicOr(status, 1);
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) mm = fmax(mm, red[i]);
      int ex = 0;
      if (mm > 0.0 && mm <= 1.7976931348623157e308) {
        frexp(mm, &ex);
        ex += 2;
      }
      ex_s = ex;
      e_out[g] = ex;
    }
    __syncthreads();
    const int shift = 8 * S - ex_s;
    // Four consecutive values per thread: a warp reads 1 KB of the row and
    // writes 128 contiguous bytes of each digit plane.
    for (int64_t q4 = threadIdx.x; q4 < k_pad / 4; q4 += blockDim.x) {
      uint32_t word[S];
#pragma unroll
      for (int s = 0; s < S; s++) word[s] = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int64_t kk = q4 * 4 + j;
        double v = (live && kk < k) ? row[kk] : 0.0;
        if (!(fabs(v) <= 1.7976931348623157e308)) v = 0.0;
        long long X = llrint(ldexp(v, shift));
#pragma unroll
        for (int s = S - 1; s >= 0; s--) {
          const long long d = ((X + 128) & 255) - 128;
          word[s] |= ((uint32_t)(d & 255)) << (8 * j);
          X = (X - d) >> 8;
        }
      }
#pragma unroll
      for (int s = 0; s < S; s++)
        *(uint32_t*)(digits + (w * S + s) * slab + r * k_pad + q4 * 4) = word[s];
    }
    __syncthreads();
  }
}

// The same cut for rows of at most 128 values (attention's features): a
// warp per row, four consecutive values per lane, the same digits.
template <int S>
__global__ void __launch_bounds__(256) slice_short_rows(const double* __restrict__ x, int64_t batches, int64_t rows,
                                                        int64_t k, int64_t ld, int64_t rows_pad, int64_t k_pad,
                                                        int32_t* __restrict__ e_out, int8_t* __restrict__ digits,
                                                        int* status, const int64_t* __restrict__ lens,
                                                        bool skip_padding) {
  const int lane = threadIdx.x & 31;
  const int64_t slab = rows_pad * k_pad;
  for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < batches * rows_pad;
       g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t w = g / rows_pad, r = g % rows_pad;
    const double* row = x + (w * rows + r) * ld;
    const bool live = r < rows && (!lens || r < lens[w]);
    double v[4];
    double m = 0.0;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int64_t kk = lane * 4 + j;
      v[j] = (live && kk < k) ? row[kk] : 0.0;
      const double a = fabs(v[j]);
      bad |= !(a <= 1.7976931348623157e308);
      m = fmax(m, a);
    }
    if (bad) atomicOr(status, 1);
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int ex = 0;
    if (m > 0.0 && m <= 1.7976931348623157e308) {
      frexp(m, &ex);
      ex += 2;
    }
    if (lane == 0) e_out[g] = ex;
    if constexpr (S <= 6) {
      // The digits from the bytes of the rounded values (digit_planes4:
      // round to nearest, ties to even, as llrint below), x · 2^(8S - ex) in
      // two exact factors. Rows past their length keep their old digits
      // when the caller never reads them (skip_padding).
      if (lane * 4 < k_pad && (live || !skip_padding)) {
        const int shift = 8 * S - ex;
        const double f1 = ptx::pow2(shift >> 1), f2 = ptx::pow2(shift - (shift >> 1));
        double xs[4];
#pragma unroll
        for (int j = 0; j < 4; j++) xs[j] = (fabs(v[j]) <= 1.7976931348623157e308 ? v[j] : 0.0) * f1 * f2;
        uint32_t planes[S];
        digit_planes4<S>(xs, planes);
#pragma unroll
        for (int s = 0; s < S; s++) *(uint32_t*)(digits + (w * S + s) * slab + r * k_pad + lane * 4) = planes[s];
      }
      continue;
    }
    if (lane * 4 < k_pad && (live || !skip_padding)) {
      const int shift = 8 * S - ex;
      uint32_t word[S];
#pragma unroll
      for (int s = 0; s < S; s++) word[s] = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double vv = fabs(v[j]) <= 1.7976931348623157e308 ? v[j] : 0.0;
        long long X = llrint(ldexp(vv, shift));
#pragma unroll
        for (int s = S - 1; s >= 0; s--) {
          const long long d = ((X + 128) & 255) - 128;
          word[s] |= ((uint32_t)(d & 255)) << (8 * j);
          X = (X - d) >> 8;
        }
      }
#pragma unroll
      for (int s = 0; s < S; s++) *(uint32_t*)(digits + (w * S + s) * slab + r * k_pad + lane * 4) = word[s];
    }
  }
}

// Rows of at most 64 values (k_pad == 64), for S <= 6: half a warp per row,
// four values a lane loaded 16 bytes at a time, the digits cut from the
// bytes of the rounded values (digit_planes4: round to nearest, ties to
// even, as llrint, so the same digits as slice_short_rows).
template <int S>
__global__ void __launch_bounds__(256) slice_half_warp_rows(const double* __restrict__ x, int64_t batches,
                                                            int64_t rows, int64_t k, int64_t ld, int64_t rows_pad,
                                                            int32_t* __restrict__ e_out, int8_t* __restrict__ digits,
                                                            int* status, const int64_t* __restrict__ lens,
                                                            bool skip_padding) {
  constexpr int64_t kPad = 64;
  const int lane = threadIdx.x & 31, l16 = lane & 15, half = lane >> 4;
  const int64_t slab = rows_pad * kPad, total = batches * rows_pad;
  // Both halves of a warp take their loop steps together (the shuffles are warp-wide).
  for (int64_t gp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; gp * 2 < total;
       gp += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t g = gp * 2 + half;
    const int64_t w = g / rows_pad, r = g % rows_pad;
    const bool live = g < total && r < rows && (!lens || r < lens[w]);
    const double* row = x + (w * rows + r) * ld;
    const int64_t c0 = (int64_t)l16 * 4;
    double v[4];
    if (live && c0 + 3 < k && ((((uintptr_t)(row + c0)) & 15) == 0)) {
      const double2 a = *(const double2*)(row + c0), b = *(const double2*)(row + c0 + 2);
      v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) v[j] = (live && c0 + j < k) ? row[c0 + j] : 0.0;
    }
    double m = 0.0;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double a = fabs(v[j]);
      bad |= !(a <= 1.7976931348623157e308);
      m = fmax(m, a);
      if (!(a <= 1.7976931348623157e308)) v[j] = 0.0;
    }
    if (bad) atomicOr(status, 1);
    for (int o = 8; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int ex = 0;
    if (m > 0.0 && m <= 1.7976931348623157e308) {
      frexp(m, &ex);
      ex += 2;
    }
    if (g < total) {
      if (l16 == 0) e_out[g] = ex;
      // x · 2^(8S - ex) in two exact factors (8S - ex may leave the normal range).
      const int shift = 8 * S - ex;
      const double f1 = ptx::pow2(shift >> 1), f2 = ptx::pow2(shift - (shift >> 1));
      double xs[4];
#pragma unroll
      for (int j = 0; j < 4; j++) xs[j] = v[j] * f1 * f2;
      uint32_t planes[S];
      digit_planes4<S>(xs, planes);
      if (live || !skip_padding)
#pragma unroll
        for (int s2 = 0; s2 < S; s2++) *(uint32_t*)(digits + (w * S + s2) * slab + r * kPad + c0) = planes[s2];
    }
  }
}

// Launches the row slicer that suits the row length.
template <int S>
void launch_slice_rows(const double* x, int64_t batches, int64_t rows, int64_t k, int64_t ld, int64_t rows_pad,
                       int64_t k_pad, int32_t* e_out, int8_t* digits, int* status, cudaStream_t stream,
                       const int64_t* lens = nullptr, bool skip_padding = false) {
  if constexpr (S <= 6) {
    if (k_pad == 64) {
      slice_half_warp_rows<S><<<blocks_for((uint64_t)(batches * rows_pad) * 16, 256), 256, 0, stream>>>(
          x, batches, rows, k, ld, rows_pad, e_out, digits, status, lens, skip_padding);
      return;
    }
  }
  if (k_pad <= 128)
    slice_short_rows<S><<<blocks_for((uint64_t)(batches * rows_pad) * 32, 256), 256, 0, stream>>>(
        x, batches, rows, k, ld, rows_pad, k_pad, e_out, digits, status, lens, skip_padding);
  else
    slice_rows<S><<<blocks_for((uint64_t)(batches * rows_pad), 1, 148 * 8), 256, 0, stream>>>(
        x, batches, rows, k, ld, rows_pad, k_pad, e_out, digits, status, lens);
}

// The largest magnitude of each column of x [batches][k][n] (row-major):
// blocks of rows reduce apart and combine with an atomic max on the bits
// (non-negative doubles order as their bits). Status bit 1 if a value isn't
// finite. `colmax` must start at zero.
__global__ void col_max(const double* __restrict__ x, int64_t batches, int64_t k, int64_t n,
                        unsigned long long* __restrict__ colmax, int* status, const int64_t* __restrict__ lens) {
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t w = blockIdx.z;
  const int64_t rows_per = (k + gridDim.y - 1) / gridDim.y;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per, r1 = min(lens ? min(k, lens[w]) : k, r0 + rows_per);
  if (col >= n) return;
  // Eight rows at a time into independent maxima, so that eight loads are
  // in flight per thread.
  double mx[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  bool bad = false;
  const double* p = x + w * k * n + col;
  int64_t r = r0;
  for (; r + 8 <= r1; r += 8) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const double v = fabs(p[(r + i) * n]);
      bad |= !(v <= 1.7976931348623157e308);
      mx[i] = fmax(mx[i], v);
    }
  }
  for (; r < r1; r++) {
    const double v = fabs(p[r * n]);
    bad |= !(v <= 1.7976931348623157e308);
    mx[0] = fmax(mx[0], v);
  }
  const double m = fmax(fmax(fmax(mx[0], mx[1]), fmax(mx[2], mx[3])), fmax(fmax(mx[4], mx[5]), fmax(mx[6], mx[7])));
  if (bad) atomicOr(status, 1);
  if (m > 0.0) atomicMax(&colmax[w * n + col], (unsigned long long)__double_as_longlong(m));
}

// The S digits of each column of x [batches][k][n] under its column's
// exponent, written K-major: digits[(w·S + s)][col][kk] for col < n_pad and
// kk < k_pad. A 64 x 64 tile is staged in shared memory, read along n and
// cut along k; each thread cuts 16 values of k of one column.
template <int S>
__global__ void __launch_bounds__(256) col_digits(const double* __restrict__ x, int64_t k, int64_t n, int64_t n_pad,
                                                  int64_t k_pad, const unsigned long long* __restrict__ colmax,
                                                  int32_t* __restrict__ e_out, int8_t* __restrict__ digits,
                                                  const int64_t* __restrict__ lens) {
  __shared__ double tile[64][65];
  const int64_t w = blockIdx.z;
  const int64_t k0 = (int64_t)blockIdx.y * 64, n0 = (int64_t)blockIdx.x * 64;
  const double* X = x + w * k * n;
  const int64_t kl = lens ? min(k, lens[w]) : k;
  for (int i = threadIdx.x; i < 64 * 64; i += 256) {
    const int kr = i / 64, nc = i % 64;
    const int64_t gk = k0 + kr, gn = n0 + nc;
    double v = (gk < kl && gn < n) ? X[gk * n + gn] : 0.0;
    if (!(fabs(v) <= 1.7976931348623157e308)) v = 0.0;
    tile[kr][nc] = v;
  }
  __syncthreads();
  const int nl = threadIdx.x / 4, kc = threadIdx.x % 4;
  const int64_t col = n0 + nl;
  if (col >= n_pad) return;
  int ex = 0;
  if (col < n) {
    const double mm = __longlong_as_double((long long)colmax[w * n + col]);
    if (mm > 0.0) {
      frexp(mm, &ex);
      ex += 2;
    }
  }
  if (blockIdx.y == 0 && kc == 0) e_out[w * n_pad + col] = ex;
  const int shift = 8 * S - ex;
  uint32_t word[S][4];
  if constexpr (S <= 6) {
    // The bytes of the rounded values (round to nearest, ties to even, as
    // llrint), the power of two in two exact factors.
    const double f1 = ptx::pow2(shift >> 1), f2 = ptx::pow2(shift - (shift >> 1));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double xs[4];
#pragma unroll
      for (int i = 0; i < 4; i++) xs[i] = tile[kc * 16 + q * 4 + i][nl] * f1 * f2;
      uint32_t planes[S];
      digit_planes4<S>(xs, planes);
#pragma unroll
      for (int s = 0; s < S; s++) word[s][q] = planes[s];
    }
  } else {
#pragma unroll
    for (int s = 0; s < S; s++)
#pragma unroll
      for (int q = 0; q < 4; q++) word[s][q] = 0;
#pragma unroll
    for (int j = 0; j < 16; j++) {
      long long X2 = llrint(ldexp(tile[kc * 16 + j][nl], shift));
#pragma unroll
      for (int s = S - 1; s >= 0; s--) {
        const long long d = ((X2 + 128) & 255) - 128;
        word[s][j >> 2] |= ((uint32_t)(d & 255)) << (8 * (j & 3));
        X2 = (X2 - d) >> 8;
      }
    }
  }
  const int64_t slab = n_pad * k_pad;
#pragma unroll
  for (int s = 0; s < S; s++) {
    uint4* dst = (uint4*)(digits + (w * S + s) * slab + col * k_pad + k0 + kc * 16);
    *dst = make_uint4(word[s][0], word[s][1], word[s][2], word[s][3]);
  }
}

// FP64 product in k order. 64x64 tiles, 256 threads, 4x4 cells each.
template <bool FMA>
__global__ void __launch_bounds__(256) fp64_gemm_kernel(const double* __restrict__ a, const uint32_t* __restrict__ held,
                                                        const double* __restrict__ b, double* __restrict__ c,
                                                        int64_t m, int64_t n, int64_t k, int64_t zblock) {
  constexpr int T = 64, KT = 16;
  __shared__ double As[KT][T + 1];
  __shared__ double Bs[KT][T + 1];
  __shared__ uint8_t Hs[KT][T + 4];
  const int64_t w = blockIdx.z;
  const double* A = a + w * m * k;
  const double* B = b + w * k * n;
  double* C = c + w * m * n;
  const int64_t r0 = (int64_t)blockIdx.y * T, c0 = (int64_t)blockIdx.x * T;
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  double part[4][4], out[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) part[i][j] = out[i][j] = 0.0;
  for (int64_t k0 = 0; k0 < k; k0 += KT) {
    for (int idx = threadIdx.x; idx < T * KT; idx += 256) {
      const int row = idx / KT, kk = idx % KT;
      const int64_t gr = r0 + row, gk = k0 + kk;
      const bool in = gr < m && gk < k;
      As[kk][row] = in ? A[gr * k + gk] : 0.0;
      const int64_t cell = (w * m + gr) * k + gk;
      Hs[kk][row] = in ? (held ? (uint8_t)(((held[cell >> 4] >> ((cell & 15) * 2)) & 3) == 2) : (uint8_t)1)
                       : (uint8_t)0;
    }
    for (int idx = threadIdx.x; idx < T * KT; idx += 256) {
      const int kk = idx / T, col = idx % T;
      const int64_t gc = c0 + col, gk = k0 + kk;
      Bs[kk][col] = (gc < n && gk < k) ? B[gk * n + gc] : 0.0;
    }
    __syncthreads();
    const int kt = (int)((k - k0) < KT ? (k - k0) : KT);
    for (int kk = 0; kk < kt; kk++) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const double av = As[kk][tr * 4 + i];
        const bool h = Hs[kk][tr * 4 + i] != 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double bv = Bs[kk][tc * 4 + j];
          if (FMA) {
            if (h) part[i][j] = fma(av, bv, part[i][j]);
          } else {
            const double p = h ? __dmul_rn(av, bv) : 0.0;
            part[i][j] = __dadd_rn(part[i][j], p);
          }
        }
      }
      if (zblock > 0 && (k0 + kk + 1) % zblock == 0) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) {
            out[i][j] = __dadd_rn(out[i][j], part[i][j]);
            part[i][j] = 0.0;
          }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int64_t gr = r0 + tr * 4 + i;
    if (gr >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int64_t gc = c0 + tc * 4 + j;
      if (gc >= n) continue;
      double v = part[i][j];
      if (zblock > 0) v = (k % zblock != 0) ? __dadd_rn(out[i][j], part[i][j]) : out[i][j];
      C[gr * n + gc] = v;
    }
  }
}

__global__ void transpose_kernel(const double* __restrict__ b, double* __restrict__ bt, int64_t rows, int64_t cols) {
  __shared__ double tile[32][33];
  const int64_t w = blockIdx.z;
  const double* B = b + w * rows * cols;
  double* BT = bt + w * rows * cols;
  const int64_t x0 = (int64_t)blockIdx.x * 32, y0 = (int64_t)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int64_t r = y0 + i, cc = x0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < rows && cc < cols) ? B[r * cols + cc] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int64_t cc = x0 + i, r = y0 + threadIdx.x;
    if (cc < cols && r < rows) BT[cc * rows + r] = tile[threadIdx.x][i];
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  if (!fn) fail(EINFOLD_DEVICE, "cuTensorMapEncodeTiled is unavailable");
  return fn;
}

// A 3D int8 tensor map over digits [planes][rows][k_pad], boxes of
// (64 B of k, box_rows, S planes), 64-byte swizzle.
CUtensorMap digit_map(const int8_t* digits, int64_t k_pad, int64_t rows, int64_t planes, int box_rows, int S) {
  CUtensorMap map;
  cuuint64_t dims[3] = {(cuuint64_t)k_pad, (cuuint64_t)rows, (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)k_pad, (cuuint64_t)(k_pad * rows)};
  cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, (cuuint32_t)S};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)digits, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(EINFOLD_DEVICE, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return map;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Scratch the split product needs beyond its inputs and output.
struct SplitScratch {
  int8_t* da;                   // A's digits [batches·S][m_pad][k_pad]
  int8_t* db;                   // B's digits [batches·S][n_pad][k_pad]
  int32_t* ea;                  // A's row exponents [batches][m_pad]
  int32_t* eb;                  // B's column exponents [batches][n_pad]
  unsigned long long* colmax;   // B's column maxima [batches][n] (natural B only)
  int* status;
};

struct SplitDims {
  int64_t m_pad, n_pad, k_pad;
};

SplitDims split_dims(int64_t m, int64_t n, int64_t k) {
  return {round_up(m, BM), round_up(n, BN), round_up(k > 0 ? k : 1, BK)};
}

// Bytes of each scratch array, 256-byte aligned, in SplitScratch order.
void split_scratch_sizes(int S, int64_t batches, int64_t m, int64_t n, int64_t k, size_t sz[6]) {
  SplitDims d = split_dims(m, n, k);
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  sz[0] = al((size_t)(batches * S * d.m_pad * d.k_pad));
  sz[1] = al((size_t)(batches * S * d.n_pad * d.k_pad));
  sz[2] = al((size_t)(batches * d.m_pad) * 4);
  sz[3] = al((size_t)(batches * d.n_pad) * 4);
  sz[4] = al((size_t)(batches * n) * 8);
  sz[5] = 256;
}

// The product with scratch already in place: slices both operands, runs the
// tensor-core kernel over k in chunks, and returns the status word. Allocates
// nothing. `timed` records CUDA events around the product kernels.
template <int S>
int split_run(Context& ctx, const double* a, const double* b, bool b_natural, double* c, int64_t batches, int64_t m,
              int64_t n, int64_t k, const SplitScratch& sc, cudaStream_t stream, bool timed) {
  using Sh = SplitShape<S>;
  const SplitDims d = split_dims(m, n, k);
  const int64_t m_pad = d.m_pad, n_pad = d.n_pad, k_pad = d.k_pad;
  EF_CUDA(cudaMemsetAsync(sc.status, 0, sizeof(int), stream));
  launch_slice_rows<S>(a, batches, m, k, k, m_pad, k_pad, sc.ea, sc.da, sc.status, stream);
  if (b_natural) {
    EF_CUDA(cudaMemsetAsync(sc.colmax, 0, (size_t)(batches * n) * 8, stream));
    const unsigned splits = (unsigned)std::min<int64_t>(64, (k + 127) / 128);
    col_max<<<dim3((unsigned)((n + 255) / 256), splits, (unsigned)batches), 256, 0, stream>>>(b, batches, k, n,
                                                                                             sc.colmax, sc.status,
                                                                                             nullptr);
    col_digits<S><<<dim3((unsigned)(n_pad / 64), (unsigned)(k_pad / 64), (unsigned)batches), 256, 0, stream>>>(
        b, k, n, n_pad, k_pad, sc.colmax, sc.eb, sc.db, nullptr);
    ctx.kernels += 2;
  } else {
    launch_slice_rows<S>(b, batches, n, k, k, n_pad, k_pad, sc.eb, sc.db, sc.status, stream);
    ctx.kernels++;
  }
  EF_LAUNCH_CHECK();
  ctx.kernels++;
  ctx.phase("split: sliced");
  CUtensorMap ta = digit_map(sc.da, k_pad, m_pad, batches * S, BM, S);
  CUtensorMap tb = digit_map(sc.db, k_pad, n_pad, batches * S, BN, S);
  EF_CUDA(cudaFuncSetAttribute(split_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::kSmem));
  // Each level's int32 sum is exact while S·kc·2^14 < 2^31: long k runs in
  // chunks whose FP64 results are added.
  const int64_t k_blocks = k_pad / BK;
  const int64_t chunk_blocks = ((int64_t)1 << 31) / ((int64_t)S << 14) / BK;
  const int tiles_m = (int)(m_pad / BM), tiles_n = (int)(n_pad / BN);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    EF_CUDA(cudaEventCreate(&e0));
    EF_CUDA(cudaEventCreate(&e1));
    EF_CUDA(cudaEventRecord(e0, stream));
  }
  for (int64_t kb0 = 0; kb0 < k_blocks; kb0 += chunk_blocks) {
    const int kbs = (int)std::min<int64_t>(chunk_blocks, k_blocks - kb0);
    dim3 grid((unsigned)(tiles_m * tiles_n), (unsigned)batches);
    split_gemm_kernel<S><<<grid, kThreads, Sh::kSmem, stream>>>(ta, tb, sc.ea, sc.eb, c, (int)m, (int)n, (int)m_pad,
                                                                 (int)n_pad, (int)kb0, kbs, tiles_m, tiles_n,
                                                                 kb0 > 0 ? 1 : 0, sc.status);
    EF_LAUNCH_CHECK();
    ctx.kernels++;
  }
  if (timed) EF_CUDA(cudaEventRecord(e1, stream));
  int st = 0;
  EF_CUDA(cudaMemcpyAsync(&st, sc.status, sizeof(int), cudaMemcpyDeviceToHost, stream));
  EF_CUDA(cudaStreamSynchronize(stream));
  if (timed) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // Digit products executed: S(S+1)/2 pairs of an (m_pad x k_pad) by
    // (k_pad x n_pad) int8 product, 2 ops per multiply-add.
    ctx.product_ms += ms;
    ctx.product_ops += 2.0 * (double)batches * (double)m_pad * (double)n_pad * (double)k_pad * (S * (S + 1) / 2);
  }
  return st;
}

void check_status(int st) {
  if (st & 1) fail(EINFOLD_INVALID, "the split product was given a value that isn't finite");
  if (st & 2) fail(EINFOLD_TIMEOUT, "a bounded wait in the split product ran out");
}

template <int S>
void split_gemm_s(Context& ctx, const double* a, const double* b, bool b_natural, double* c, int64_t batches,
                  int64_t m, int64_t n, int64_t k, cudaStream_t stream) {
  size_t sz[6];
  split_scratch_sizes(S, batches, m, n, k, sz);
  size_t total = 0;
  for (size_t x : sz) total += x;
  DeviceBuffer<uint8_t> scratch(total, stream);
  uint8_t* p = scratch.get();
  SplitScratch sc;
  sc.da = (int8_t*)p; p += sz[0];
  sc.db = (int8_t*)p; p += sz[1];
  sc.ea = (int32_t*)p; p += sz[2];
  sc.eb = (int32_t*)p; p += sz[3];
  sc.colmax = (unsigned long long*)p; p += sz[4];
  sc.status = (int*)p;
  check_status(split_run<S>(ctx, a, b, b_natural, c, batches, m, n, k, sc, stream, true));
}

template <class F>
void dispatch_slices(int slices, F&& f) {
  switch (slices) {
    case 2: f(std::integral_constant<int, 2>()); break;
    case 3: f(std::integral_constant<int, 3>()); break;
    case 4: f(std::integral_constant<int, 4>()); break;
    case 5: f(std::integral_constant<int, 5>()); break;
    case 6: f(std::integral_constant<int, 6>()); break;
    case 7: f(std::integral_constant<int, 7>()); break;
    default: fail(EINFOLD_INVALID, "slices must be 2 to 7, not %d", slices);
  }
}

}  // namespace

void split_gemm(Context& ctx, const double* a, const double* b, bool b_natural, double* c, int64_t batches,
                int64_t m, int64_t n, int64_t k, int slices, cudaStream_t stream) {
  if (batches <= 0 || m <= 0 || n <= 0) return;
  if (m > INT32_MAX / 2 || n > INT32_MAX / 2 || batches > 65535) fail(EINFOLD_INVALID, "a product too large");
  if (k <= 0) {
    EF_CUDA(cudaMemsetAsync(c, 0, (size_t)(batches * m * n) * sizeof(double), stream));
    return;
  }
  dispatch_slices(slices, [&](auto S) { split_gemm_s<decltype(S)::value>(ctx, a, b, b_natural, c, batches, m, n, k, stream); });
}

__global__ void exponent_range_kernel(const int32_t* __restrict__ e, int64_t n, int* __restrict__ out) {
  int hi = INT_MIN, lo = INT_MIN;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    hi = max(hi, e[i]);
    lo = max(lo, -e[i]);
  }
  for (int o = 16; o; o >>= 1) {
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    lo = max(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, hi);
    atomicMax(out + 1, lo);
  }
}

void exponent_range(const int32_t* e, int64_t n, int* out, cudaStream_t stream) {
  if (n <= 0) return;
  exponent_range_kernel<<<blocks_for((uint64_t)n, 256), 256, 0, stream>>>(e, n, out);
  EF_LAUNCH_CHECK();
}

void slice_rows_into(int S, const double* x, int64_t batches, int64_t rows, int64_t k, int64_t ld, int64_t rows_pad,
                     int64_t k_pad, int32_t* e_out, int8_t* digits, int* status, cudaStream_t stream,
                     const int64_t* lens, bool skip_padding) {
  if (batches <= 0 || rows_pad <= 0) return;
  dispatch_slices(S, [&](auto SS) {
    launch_slice_rows<decltype(SS)::value>(x, batches, rows, k, ld, rows_pad, k_pad, e_out, digits, status, stream,
                                           lens, skip_padding);
  });
  EF_LAUNCH_CHECK();
}

void slice_cols_into(int S, const double* x, int64_t batches, int64_t k, int64_t n, int64_t n_pad, int64_t k_pad,
                     unsigned long long* colmax, int32_t* e_out, int8_t* digits, int* status, cudaStream_t stream,
                     const int64_t* lens) {
  if (batches <= 0 || n_pad <= 0 || k_pad <= 0) return;
  if (n_pad % 64 || k_pad % 64) fail(EINFOLD_INVALID, "column digits need multiples of 64");
  EF_CUDA(cudaMemsetAsync(colmax, 0, (size_t)(batches * n) * 8, stream));
  if (n > 0 && k > 0) {
    const unsigned splits = (unsigned)std::min<int64_t>(64, (k + 127) / 128);
    col_max<<<dim3((unsigned)((n + 255) / 256), splits, (unsigned)batches), 256, 0, stream>>>(x, batches, k, n, colmax,
                                                                                             status, lens);
  }
  dispatch_slices(S, [&](auto SS) {
    col_digits<decltype(SS)::value><<<dim3((unsigned)(n_pad / 64), (unsigned)(k_pad / 64), (unsigned)batches), 256, 0,
                                      stream>>>(x, k, n, n_pad, k_pad, colmax, e_out, digits, lens);
  });
  EF_LAUNCH_CHECK();
}

CUtensorMap digit_planes_map(const int8_t* digits, int64_t k_pad, int64_t rows, int64_t planes, int box_rows,
                             int box_planes) {
  return digit_map(digits, k_pad, rows, planes, box_rows, box_planes);
}

CUtensorMap f64_boxes_map(const double* x, int64_t cols, int64_t rows, int64_t batches, int box_cols, int box_rows) {
  if (box_cols * 8 > 128) fail(EINFOLD_INVALID, "a 128-byte-swizzled box holds at most 16 doubles a row");
  CUtensorMap map;
  cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)batches};
  cuuint64_t strides[2] = {(cuuint64_t)(cols * 8), (cuuint64_t)(cols * rows * 8)};
  cuuint32_t box[3] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)x, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(EINFOLD_DEVICE, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return map;
}

void fp64_gemm(Context& ctx, const double* a, const uint32_t* held, const double* b, double* c, int64_t batches,
               int64_t m, int64_t n, int64_t k, int64_t /*batch_of_row*/, int64_t zblock, bool fused_multiply_add,
               cudaStream_t stream) {
  if (batches <= 0 || m <= 0 || n <= 0) return;
  dim3 grid((unsigned)((n + 63) / 64), (unsigned)((m + 63) / 64), (unsigned)batches);
  if (fused_multiply_add)
    fp64_gemm_kernel<true><<<grid, 256, 0, stream>>>(a, held, b, c, m, n, k, 0);
  else
    fp64_gemm_kernel<false><<<grid, 256, 0, stream>>>(a, held, b, c, m, n, k, zblock);
  EF_LAUNCH_CHECK();
  ctx.kernels++;
}

void transpose(const double* b, double* bt, int64_t batches, int64_t rows, int64_t cols, cudaStream_t stream) {
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32), (unsigned)batches);
  transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(b, bt, rows, cols);
  EF_LAUNCH_CHECK();
}

// ---- The split product for callers that can't allocate ----------------

namespace {

// Scratch for einfold_split_gemm_static: every device that loads the library
// holds these 64 MiB until the process exits.
constexpr size_t kStaticScratchBytes = (size_t)64 << 20;
__device__ __align__(256) uint8_t g_split_scratch[kStaticScratchBytes];

std::mutex g_static_lock;
struct StaticBase {
  void* context = nullptr;  // the CUDA context the address belongs to
  void* ptr = nullptr;
};
StaticBase g_static_base[64];

// The calling thread's current CUDA context (the driver's cuCtxGetCurrent,
// reached through the runtime's entry-point query).
void* current_context() {
  typedef int (*GetCurrent)(void**);
  static GetCurrent fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (GetCurrent)p;
  });
  if (!fn) fail(EINFOLD_DEVICE, "cuCtxGetCurrent is unavailable");
  void* c = nullptr;
  if (fn(&c) != 0) fail(EINFOLD_DEVICE, "cuCtxGetCurrent failed");
  return c;
}

// The array's device address in the current context of `device`. Host code
// can't use the array's name as an address: the first call in a context
// looks the address up with cudaGetSymbolAddress and keeps it with the
// context's handle; a new context on the device (after cudaDeviceReset, say,
// which reloads the module at another address) looks it up again.
uint8_t* static_scratch(int device) {
  if (device < 0 || device >= 64) fail(EINFOLD_INVALID, "device %d out of range", device);
  void* ctx = current_context();
  if (!ctx) {
    // No context yet on this thread: the device's primary context, as the
    // runtime would make current at its first call that needs one.
    EF_CUDA(cudaSetDevice(device));
    ctx = current_context();
    if (!ctx) fail(EINFOLD_DEVICE, "no current CUDA context");
  }
  std::lock_guard<std::mutex> lock(g_static_lock);
  StaticBase& b = g_static_base[device];
  if (b.context != ctx || !b.ptr) {
    void* p = nullptr;
    EF_CUDA(cudaGetSymbolAddress(&p, g_split_scratch));
    b.context = ctx;
    b.ptr = p;
  }
  return (uint8_t*)b.ptr;
}

// The scratch a product needs, saturating instead of wrapping: sizes whose
// product would overflow 64 bits compare as larger than any array.
uint64_t static_scratch_needed(int S, int64_t batches, int64_t m, int64_t n, int64_t k) {
  const SplitDims d = split_dims(m, n, k);
  auto al = [](uint64_t x) { return sat_add(x, 255) & ~(uint64_t)255; };
  const uint64_t bs = sat_mul((uint64_t)batches, (uint64_t)S);
  uint64_t t = al(sat_mul(sat_mul(bs, (uint64_t)d.m_pad), (uint64_t)d.k_pad));
  t = sat_add(t, al(sat_mul(sat_mul(bs, (uint64_t)d.n_pad), (uint64_t)d.k_pad)));
  t = sat_add(t, al(sat_mul(sat_mul((uint64_t)batches, (uint64_t)d.m_pad), 4)));
  t = sat_add(t, al(sat_mul(sat_mul((uint64_t)batches, (uint64_t)d.n_pad), 4)));
  t = sat_add(t, al(sat_mul(sat_mul((uint64_t)batches, (uint64_t)n), 8)));
  return sat_add(t, 256);
}

}  // namespace

}  // namespace ef

extern "C" int32_t einfold_split_gemm_static(const double* a, const double* b, double* c, int64_t batches, int64_t m,
                                             int64_t n, int64_t k, int32_t b_transposed, int32_t slices,
                                             void* stream, char* message, int32_t message_len) {
  using namespace ef;
  try {
    int device = 0;
    EF_CUDA(cudaGetDevice(&device));
    uint8_t* base = static_scratch(device);
    const int S = slices ? slices : kDefaultSlices;
    if (S < kMinSlices || S > kMaxSlices) fail(EINFOLD_INVALID, "slices must be 2 to 7, not %d", S);
    if (batches < 0 || m < 0 || n < 0 || k < 0) fail(EINFOLD_INVALID, "negative sizes");
    cudaStream_t s = (cudaStream_t)stream;
    if (batches == 0 || m == 0 || n == 0) return EINFOLD_OK;
    if (m > INT32_MAX / 2 || n > INT32_MAX / 2 || batches > 65535) fail(EINFOLD_INVALID, "a product too large");
    if (k == 0) {
      EF_CUDA(cudaMemsetAsync(c, 0, (size_t)(batches * m * n) * sizeof(double), s));
      EF_CUDA(cudaStreamSynchronize(s));
      return EINFOLD_OK;
    }
    if (k > INT64_MAX / 2) fail(EINFOLD_INVALID, "a product too large");
    const uint64_t need = static_scratch_needed(S, batches, m, n, k);
    if (need > kStaticScratchBytes)
      fail(EINFOLD_INVALID,
           "this product needs %llu bytes of scratch, more than the %zu einfold_split_gemm_static holds; "
           "use einfold_split_gemm", (unsigned long long)need, kStaticScratchBytes);
    // Within the array, so every size below fits in 64 bits.
    size_t sz[6];
    split_scratch_sizes(S, batches, m, n, k, sz);
    SplitScratch sc;
    uint8_t* p = base;
    sc.da = (int8_t*)p; p += sz[0];
    sc.db = (int8_t*)p; p += sz[1];
    sc.ea = (int32_t*)p; p += sz[2];
    sc.eb = (int32_t*)p; p += sz[3];
    sc.colmax = (unsigned long long*)p; p += sz[4];
    sc.status = (int*)p;
    Context local;  // no stream or pool of its own: the caller's stream, nothing allocated
    local.device = device;
    local.stream = s;
    int st = 0;
    dispatch_slices(S, [&](auto SS) {
      st = split_run<decltype(SS)::value>(local, a, b, b_transposed == 0, c, batches, m, n, k, sc, s, false);
    });
    check_status(st);
    return EINFOLD_OK;
  } catch (const Failure& f) {
    if (message && message_len > 0) std::snprintf(message, (size_t)message_len, "%s", f.what());
    return f.status;
  }
}
