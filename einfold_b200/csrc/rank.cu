// Ranking keys by their bytes on the device: the discrimination algorithm's
// first step (crates/einfold-kernels/src/discriminate.rs:103-156 `radix`,
// :212-235 `ranks`, :280-292 `ranks_of_words`).
//
// Keys are W 64-bit words each, most significant word first, ordered as
// unsigned integers. A stable LSD radix sort of (key, row) pairs runs one
// 8-bit pass per byte that varies between keys (constant bytes are skipped,
// as the reference skips them), then each row's rank is the number of
// distinct keys before its own, and first[r] the smallest row holding rank r
// (the first of its run, as the sort is stable).
//
// One pass: the keys are cut into as many chunks as blocks fit on the GPU at
// once. An upsweep counts each chunk's digits; one exclusive scan of the
// digit-major table gives each (digit, chunk) its first output position; a
// downsweep block then sorts its chunk tile by tile: each key ranked among
// equal digits of its warp with __match_any_sync in row order, warps combined
// in shared memory, the tile reordered by digit in shared memory and written
// out run by run, contiguously. No block waits on another. Every pass is
// stable, so the result is the reference's bit for bit.
#include <cub/cub.cuh>

#include <cstdlib>

#include "ptx.cuh"
#include "rank.cuh"
#include "stage.cuh"

namespace ef {

void thrust_iota(Context& ctx, uint32_t* out, int64_t n, cudaStream_t s);

namespace {

constexpr int kThreads = 256;

template <int W>
__global__ void or_and_words(const uint64_t* __restrict__ keys, int64_t n, int64_t ld, unsigned long long* __restrict__ acc) {
  unsigned long long o[W], a[W];
#pragma unroll
  for (int w = 0; w < W; w++) { o[w] = 0; a[w] = ~0ull; }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int w = 0; w < W; w++) {
      const unsigned long long k = keys[(int64_t)w * ld + i];
      o[w] |= k;
      a[w] &= k;
    }
#pragma unroll
  for (int w = 0; w < W; w++) {
    for (int s = 16; s; s >>= 1) {
      o[w] |= __shfl_xor_sync(0xffffffffu, o[w], s);
      a[w] &= __shfl_xor_sync(0xffffffffu, a[w], s);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicOr(&acc[2 * w], o[w]);
      atomicAnd(&acc[2 * w + 1], a[w]);
    }
  }
}

// Upsweep of one pass: the digit counts of each chunk of consecutive keys,
// written digit-major (table[d·chunks + c]) so that one exclusive scan gives
// every (digit, chunk)'s first output position, stably.
// gridDim.y blocks share a chunk, each counting a slice of it and adding
// into the table, which starts at zero.
__global__ void __launch_bounds__(kThreads) chunk_counts(const uint64_t* __restrict__ kw, int64_t n, int shift,
                                                         int64_t chunk, int chunks,
                                                         unsigned long long* __restrict__ table) {
  __shared__ unsigned int h[8][256];
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < 8 * 256; i += kThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const int64_t c = blockIdx.x;
  const int64_t slice = (chunk + gridDim.y - 1) / gridDim.y;
  const int64_t lo = c * chunk + blockIdx.y * slice, hi = min(min(n, c * chunk + chunk), lo + slice);
  for (int64_t i = lo + tid; i < hi; i += kThreads) atomicAdd(&h[warp][(kw[i] >> shift) & 255], 1u);
  __syncthreads();
  unsigned int t = 0;
#pragma unroll
  for (int w = 0; w < 8; w++) t += h[w][tid];
  if (t) atomicAdd(&table[(int64_t)tid * chunks + c], (unsigned long long)t);
}

constexpr int kCountSplit = 4;  // blocks counting each chunk

// Downsweep of one pass: block c sorts its chunk tile by tile, each key
// ranked among equal digits in row order, its destination its digit's
// running offset plus that rank. Within a warp, item i of every lane is
// matched with __match_any_sync; each group's first lane stores the group's
// size as a byte in counts[warp][digit][i], and a lane's rank among its warp's
// equal digits is the sum of the bytes of items before its own (at most
// 7·32, one 64-bit load and two dp4a) plus its place in its group: no item
// waits on another's result. Tiles arrive by TMA bulk copies into two shared-memory stages, the
// next one in flight while the current one is ranked; each stage is then
// reused to reorder its tile by digit, and the tile is written out run by
// run, contiguously.
template <int W, int ITEMS>
__global__ void __launch_bounds__(kThreads) chunk_scatter(const uint64_t* __restrict__ kin,
                                                          const uint32_t* __restrict__ vin,
                                                          uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                          int64_t n, int64_t ldi, int64_t ldo, int word, int shift,
                                                          int64_t chunk, int chunks,
                                                          const long long* __restrict__ offsets, int* err) {
  constexpr int TILE = kThreads * ITEMS;
  constexpr int WARPS = kThreads / 32;
  constexpr int STAGE = TILE * (8 * W + 4);
  extern __shared__ __align__(128) uint8_t smem[];
  static_assert(ITEMS <= 8, "a digit's counts of the warp's items fill one 64-bit word");
  // Byte i: item i's group size; then (low word) the warp's first place
  // among the tile's keys of the digit.
  __shared__ __align__(16) uint64_t counts[WARPS][256];
  __shared__ long long running[256];
  __shared__ long long dbase[256];  // a digit's destination minus its first place in the tile
  __shared__ __align__(8) uint64_t bar[2];
  typedef cub::BlockScan<unsigned int, kThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t c = blockIdx.x;
  const int64_t lo = c * chunk, hi = min(n, lo + chunk);
  const int64_t tiles = (hi - lo + TILE - 1) / TILE;
  running[tid] = offsets[(int64_t)tid * chunks + c];
  const unsigned lt_mask = (1u << lane) - 1u;
  auto skeys = [&](int s) { return (uint64_t*)(smem + s * STAGE); };
  auto svals = [&](int s) { return (uint32_t*)(smem + s * STAGE + TILE * 8 * W); };
  // Issues tile t's copies into stage t & 1: whole 16-byte multiples by TMA,
  // a ragged tail of the array's last tile by the waiting threads.
  auto issue = [&](int64_t t) {
    const int s = (int)(t & 1);
    const int64_t base = lo + t * TILE;
    const int64_t count = min((int64_t)TILE, hi - base);
    const int64_t bulk = count & ~(int64_t)3;
    const uint32_t bytes = (uint32_t)(bulk * 8 * W + (vin ? bulk * 4 : 0));
    ptx::mbar_expect_tx(&bar[s], bytes);
    if (bulk) {
      for (int w = 0; w < W; w++)
        ptx::bulk_load(skeys(s) + w * TILE, kin + (int64_t)w * ldi + base, (uint32_t)(bulk * 8), &bar[s]);
      if (vin) ptx::bulk_load(svals(s), vin + base, (uint32_t)(bulk * 4), &bar[s]);
    }
  };
  if (tid == 0) {
    ptx::mbar_init(&bar[0], 1);
    ptx::mbar_init(&bar[1], 1);
    ptx::mbar_fence_init();
    if (tiles > 0) issue(0);
    if (tiles > 1) issue(1);
  }
  __syncthreads();
  for (int64_t t = 0; t < tiles; t++) {
    const int s = (int)(t & 1);
    const int64_t base = lo + t * TILE;
    const int64_t count = min((int64_t)TILE, hi - base);
    const int64_t bulk = count & ~(int64_t)3;
    if (!ptx::mbar_wait(&bar[s], (uint32_t)((t >> 1) & 1), true)) atomicOr(err, 1);
    // This warp's byte counts start at zero (its own 2 KB; no other warp reads them yet).
#pragma unroll
    for (int i = 0; i < 256 / 32; i++) counts[warp][i * 32 + lane] = 0;
    __syncwarp();
    uint64_t key[ITEMS][W];
    uint32_t val[ITEMS];
    int digit[ITEMS];
    unsigned int local[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const int off = warp * 32 * ITEMS + i * 32 + lane;
      if (off < count) {
        const bool in_smem = off < bulk;
#pragma unroll
        for (int w = 0; w < W; w++) key[i][w] = in_smem ? skeys(s)[w * TILE + off] : kin[(int64_t)w * ldi + base + off];
        val[i] = vin ? (in_smem ? svals(s)[off] : vin[base + off]) : (uint32_t)(base + off);
        uint64_t wd = key[i][0];
#pragma unroll
        for (int w = 1; w < W; w++)
          if (word == w) wd = key[i][w];
        digit[i] = (int)((wd >> shift) & 255);
      } else {
        digit[i] = 256;
      }
    }
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const int d = digit[i];
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const unsigned below = __popc(peers & lt_mask);
      if (d < 256 && below == 0) ((uint8_t*)&counts[warp][d])[i] = (uint8_t)__popc(peers);
      local[i] = below;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const int d = digit[i];
      if (i > 0 && d < 256) {
        const uint64_t c = counts[warp][d] & ((1ull << (8 * i)) - 1);  // items before i
        local[i] += (unsigned)__dp4a((int)(uint32_t)c, 0x01010101, __dp4a((int)(uint32_t)(c >> 32), 0x01010101, 0));
      }
    }
    __syncthreads();  // every item read out of the stage; every warp's counts complete
    unsigned int total = 0;
#pragma unroll
    for (int w = 0; w < WARPS; w++) {
      const uint64_t c = counts[w][tid];
      // The warp's count of this digit, up to 256: the bytes summed in 32 bits.
      const unsigned cnt = (unsigned)__dp4a((int)(uint32_t)c, 0x01010101, __dp4a((int)(uint32_t)(c >> 32), 0x01010101, 0));
      counts[w][tid] = total;
      total += cnt;
    }
    unsigned int ex;
    Scan(tmp).ExclusiveSum(total, ex);
    // Each warp's first place among the tile's keys of this digit, and the
    // digit's destination base, so that each key needs one lookup.
#pragma unroll
    for (int w = 0; w < WARPS; w++) counts[w][tid] += ex;
    dbase[tid] = running[tid] - (long long)ex;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const int d = digit[i];
      if (d < 256) {
        const unsigned pos = (unsigned)counts[warp][d] + local[i];
#pragma unroll
        for (int w = 0; w < W; w++) skeys(s)[w * TILE + pos] = key[i][w];
        svals(s)[pos] = val[i];
      }
    }
    __syncthreads();
    for (int j = tid; j < count; j += kThreads) {
      const uint64_t wd = skeys(s)[word * TILE + j];
      const int d = (int)((wd >> shift) & 255);
      const long long dst = dbase[d] + j;
#pragma unroll
      for (int w = 0; w < W; w++) kout[(int64_t)w * ldo + dst] = skeys(s)[w * TILE + j];
      if (vout) vout[dst] = svals(s)[j];
    }
    __syncthreads();  // the stage is free again
    running[tid] += total;
    if (tid == 0 && t + 2 < tiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(t + 2);
    }
  }
}

// ---- One-sweep passes --------------------------------------------------
//
// The histograms of every byte of the keys come from one read of them; each
// pass is then one kernel. A block claims the next tile of keys from a
// counter (so every earlier tile's block is already running), ranks its keys
// among equal digits as the chunked downsweep does, publishes its per-digit
// counts, and finds how many keys of each digit the earlier tiles hold by
// looking back over their published counts (decoupled look-back): a tile
// whose own offsets are known publishes them as inclusive prefixes, and a
// look-back stops at the first prefix it meets. Waits are bounded. The
// stable order, and so every rank, is the chunked passes' exactly.

constexpr uint32_t kFlagAgg = 1u << 30, kFlagPre = 2u << 30, kValue = (1u << 30) - 1;
// Up to this many keys, the rank array (4 bytes a key) stays in L2 and ranks
// are scattered straight to their rows.
constexpr int64_t kScatterInL2 = (int64_t)1 << 22;

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
  asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Counts of every byte value at every byte position of the keys (word-major
// W words), added into hist[8W][256] (zero on entry).
template <int W>
__global__ void __launch_bounds__(kThreads) byte_histograms(const uint64_t* __restrict__ keys, int64_t n, int64_t ld,
                                                            unsigned long long* __restrict__ hist) {
  __shared__ unsigned int h[8 * W][256];
  for (int i = threadIdx.x; i < 8 * W * 256; i += kThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
#pragma unroll
    for (int w = 0; w < W; w++) {
      const uint64_t k = __ldcs(&keys[(int64_t)w * ld + i]);
#pragma unroll
      for (int b = 0; b < 8; b++) atomicAdd(&h[8 * w + b][(k >> (8 * b)) & 255], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * W * 256; i += kThreads) {
    const unsigned int c = (&h[0][0])[i];
    if (c) atomicAdd(&hist[i], (unsigned long long)c);
  }
}

// One pass, one tile of 256·ITEMS keys a block. The tile arrives in shared
// memory by bulk copies (one a key word and one for the row numbers, whole
// 16-byte multiples; a ragged tail of the last tile is read directly), so
// that a block's loads take no load slots of its warps; its keys and row
// numbers stay there, and each lane keeps only its items' digits and places
// in registers (item i of a lane is key warp·32·ITEMS + 32i + lane of the
// tile), so that three blocks fit an SM. As soon as they arrive, the tile's count of each
// digit (shared-memory atomics) is published, so that later tiles'
// look-backs can pass this one while it ranks. Each warp then ranks its
// items among equal digits in order: eight ballots over a digit's bits (and
// a ninth for the padding past the last key) give each lane the lanes that
// hold its digit, for every item before any counter is touched, and a
// per-warp counter of each digit in shared memory, item by item, gives the
// group its first place, so a key's place among its warp's equal digits
// counts every earlier key of the warp. The warps' counters then become
// offsets (digit by digit, over the warps), a block scan gives each digit's
// first place in the tile, and the look-back each digit's keys in earlier
// tiles, reading four earlier tiles' words at a time. The keys are
// reordered by digit through the first key word's stage, a word at a time
// (read from the stage into registers first) and then the row numbers, and
// written out as runs of consecutive destinations. Key words (ldi) and row numbers start 16-byte aligned.
template <int W, int ITEMS, int MIN_BLOCKS>
__global__ void __launch_bounds__(kThreads, MIN_BLOCKS) onesweep_pass(const uint64_t* __restrict__ kin,
                                                             const uint32_t* __restrict__ vin,
                                                             uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                             int64_t n, int64_t ldi, int64_t ldo, int word, int shift,
                                                             const uint32_t* __restrict__ digit_start,
                                                             uint32_t* __restrict__ status,
                                                             unsigned int* __restrict__ tile_counter, int* err) {
  constexpr int TILE = kThreads * ITEMS;
  constexpr int WARPS = kThreads / 32;
  static_assert(TILE <= 65535, "a tile's places fit 16 bits");
  extern __shared__ __align__(128) uint8_t smem[];
  uint64_t* kstage = (uint64_t*)smem;               // [W][TILE]: the tile's key words
  uint32_t* vstage = (uint32_t*)(kstage + W * TILE);  // [TILE]: its row numbers
  uint8_t* sdig = (uint8_t*)(vstage + TILE);        // [TILE]: the reordered keys' digits
  uint64_t* xbuf = kstage;                          // [TILE]: one word of the reordered keys, or the rows
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint16_t wcount[WARPS][256];         // per warp: a digit's keys so far, then its offset
  __shared__ uint16_t dstart[256];                // a digit's first place in the tile
  __shared__ long long dbase[256];                // a digit's destination minus its first place
  __shared__ unsigned int hcount[256];            // the tile's keys of each digit
  __shared__ unsigned int s_tile;
  typedef cub::BlockScan<unsigned int, kThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    s_tile = atomicAdd(tile_counter, 1u);
    ptx::mbar_init(&bar, 1);
    ptx::mbar_fence_init();
  }
#pragma unroll
  for (int d = lane; d < 256; d += 32) wcount[warp][d] = 0;
  hcount[tid] = 0;
  __syncthreads();
  const int64_t t = s_tile;
  const int64_t base = t * TILE;
  const int64_t count = min((int64_t)TILE, n - base);
  const unsigned lt_mask = (1u << lane) - 1u;
  const int kb = (int)(count & ~(int64_t)1);               // keys the bulk copies bring
  const int vb = vin ? (int)(count & ~(int64_t)3) : 0;     // row numbers they bring
  if (tid == 0) {
    ptx::mbar_expect_tx(&bar, (uint32_t)(kb * 8 * W + vb * 4));
    if (kb)
#pragma unroll
      for (int w = 0; w < W; w++) ptx::bulk_load(kstage + w * TILE, kin + (int64_t)w * ldi + base, (uint32_t)(kb * 8), &bar);
    if (vb) ptx::bulk_load(vstage, vin + base, (uint32_t)(vb * 4), &bar);
  }
  if (!ptx::mbar_wait(&bar, 0)) {
    // The copies didn't land in time: fail the sort, and wait once more for
    // them before the block's shared memory goes.
    atomicOr(err, 1);
    ptx::mbar_wait(&bar, 0);
  }

  // Keys and row numbers stay in the stage until the reorder reads them.
  uint32_t dp[ITEMS];  // digit (bits 16..24; 256: no key) and place among the warp's equal digits (bits 0..15)
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const int off = warp * 32 * ITEMS + i * 32 + lane;
    uint32_t d = 256;
    if (off < count) {
      const uint64_t wd = off < kb ? kstage[word * TILE + off] : kin[(int64_t)word * ldi + base + off];
      d = (uint32_t)((wd >> shift) & 255);
    }
    dp[i] = d << 16;
  }
  // The tile's count of each digit, published at once (thread tid owns
  // digit tid): tile 0's counts are its inclusive prefixes.
#pragma unroll
  for (int i = 0; i < ITEMS; i++)
    if ((dp[i] >> 16) < 256) atomicAdd(&hcount[dp[i] >> 16], 1u);
  __syncthreads();
  const unsigned int total = hcount[tid];
  uint32_t* my = status + t * 256 + tid;
  st_volatile(my, (t == 0 ? kFlagPre : kFlagAgg) | total);
  // The lanes holding each item's digit (256 marks no key).
  unsigned peers[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const uint32_t d = dp[i] >> 16;
    unsigned m = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; b++) {
      const bool bit = (d >> b) & 1u;
      const unsigned set = __ballot_sync(0xffffffffu, bit);
      m &= bit ? set : ~set;
    }
    peers[i] = m;
  }
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const uint32_t d = dp[i] >> 16;
    const unsigned c = d < 256 ? wcount[warp][d] : 0u;
    __syncwarp();
    if (d < 256 && (peers[i] & lt_mask) == 0) wcount[warp][d] = (uint16_t)(c + __popc(peers[i]));
    dp[i] |= c + __popc(peers[i] & lt_mask);
    __syncwarp();
  }
  __syncthreads();
  {
    unsigned int acc = 0;
#pragma unroll
    for (int w = 0; w < WARPS; w++) {
      const unsigned c = wcount[w][tid];
      wcount[w][tid] = (uint16_t)acc;
      acc += c;
    }
  }
  unsigned int ex;
  Scan(tmp).ExclusiveSum(total, ex);
  // The look-back, four earlier tiles' words at a time, in order: a count
  // is added, a prefix ends it, and a word not yet published is read again
  // (flags only go from none to count to prefix, so an early read of a
  // count stays valid).
  unsigned int before = 0;
  if (t > 0) {
    constexpr int kWindow = 4;
    int64_t tt = t - 1;
    uint64_t start = 0;
    bool failed = false;
    while (true) {
      uint32_t v[kWindow];
#pragma unroll
      for (int k = 0; k < kWindow; k++) v[k] = tt - k >= 0 ? ld_volatile(status + (tt - k) * 256 + tid) : 0u;
      bool done = false;
      int used = 0;
#pragma unroll
      for (int k = 0; k < kWindow; k++) {
        if (done || used < k || tt - k < 0) continue;
        const uint32_t flag = v[k] & ~kValue;
        if (flag == 0) continue;
        before += v[k] & kValue;
        used = k + 1;
        if (flag == kFlagPre) done = true;
      }
      if (done) break;
      if (used == 0) {
        if (!start) start = ptx::now_ns();
        else if (ptx::now_ns() - start > ptx::kWaitNs) {
          failed = true;
          break;
        }
      }
      tt -= used;
    }
    if (failed) atomicOr(err, 1);
    st_volatile(my, kFlagPre | (before + total));
  }
  dstart[tid] = (uint16_t)ex;
  dbase[tid] = (long long)digit_start[tid] + (long long)before - (long long)ex;
  __syncthreads();
  // Each item's place in the reordered tile.
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const uint32_t d = dp[i] >> 16;
    if (d < 256) {
      const uint32_t pos = (uint32_t)dstart[d] + wcount[warp][d] + (dp[i] & 0xffffu);
      dp[i] = (d << 16) | pos;
      sdig[pos] = (uint8_t)d;
    }
  }
#pragma unroll
  for (int w = 0; w <= W; w++) {
    // Word w of the keys (w < W), then the rows, through the one buffer
    // (word 0's stage: its keys are read before any is overwritten).
    if (w < W) {
      uint64_t kw[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; i++) {
        const int off = warp * 32 * ITEMS + i * 32 + lane;
        if ((dp[i] >> 16) < 256) kw[i] = off < kb ? kstage[w * TILE + off] : kin[(int64_t)w * ldi + base + off];
      }
      if (w == 0) __syncthreads();
#pragma unroll
      for (int i = 0; i < ITEMS; i++)
        if ((dp[i] >> 16) < 256) xbuf[dp[i] & 0xffffu] = kw[i];
    } else {
#pragma unroll
      for (int i = 0; i < ITEMS; i++)
        if ((dp[i] >> 16) < 256) {
          const int off = warp * 32 * ITEMS + i * 32 + lane;
          ((uint32_t*)xbuf)[dp[i] & 0xffffu] =
              vin ? (off < vb ? vstage[off] : vin[base + off]) : (uint32_t)(base + off);
        }
    }
    __syncthreads();
    for (int j = tid; j < count; j += kThreads) {
      const long long dst = dbase[sdig[j]] + j;
      if (w < W) __stcs(&kout[(int64_t)w * ldo + dst], xbuf[j]);
      else __stcs(&vout[dst], ((const uint32_t*)xbuf)[j]);
    }
    __syncthreads();
  }
}

// The ranks from the sorted pairs: a key heads its run when it differs from
// the one before it; its run's rank is the number of heads before it. Tiles
// are claimed in order and the heads counted before each tile come from a
// look-back over the earlier tiles' counts, as in the passes. Each thread
// takes ITEMS consecutive positions. rank[row] is written for every row and
// first[r] by the head of run r; *distinct gets the number of runs.
template <int W, int ITEMS>
__global__ void __launch_bounds__(kThreads) rank_runs(const uint64_t* __restrict__ keys, int64_t ld,
                                                      const uint32_t* __restrict__ rows, int64_t n,
                                                      uint32_t* __restrict__ status,
                                                      unsigned int* __restrict__ tile_counter,
                                                      uint32_t* __restrict__ rank, uint32_t* __restrict__ first,
                                                      unsigned long long* __restrict__ distinct, int* err) {
  constexpr int TILE = kThreads * ITEMS;
  typedef cub::BlockScan<unsigned int, kThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned int s_tile, s_before;
  const int tid = threadIdx.x;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const int64_t t = s_tile;
  const int64_t p0 = t * TILE + (int64_t)tid * ITEMS;
  unsigned int heads = 0;
  unsigned int hmask = 0;
  uint32_t r[ITEMS];
  {
    uint64_t prev[W];
#pragma unroll
    for (int w = 0; w < W; w++) prev[w] = p0 > 0 && p0 - 1 < n ? keys[(int64_t)w * ld + p0 - 1] : 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const int64_t p = p0 + i;
      if (p < n) {
        bool h = p == 0;
#pragma unroll
        for (int w = 0; w < W; w++) {
          const uint64_t k = keys[(int64_t)w * ld + p];
          h |= k != prev[w];
          prev[w] = k;
        }
        r[i] = rows[p];
        if (h) {
          hmask |= 1u << i;
          heads++;
        }
      }
    }
  }
  unsigned int ex, total;
  Scan(tmp).ExclusiveSum(heads, ex, total);
  if (tid == 0) {
    uint32_t* my = status + t;
    unsigned int before = 0;
    if (t == 0) {
      st_volatile(my, kFlagPre | total);
    } else {
      st_volatile(my, kFlagAgg | total);
      int64_t tt = t - 1;
      uint64_t start = 0;
      while (true) {
        const uint32_t v = ld_volatile(status + tt);
        const uint32_t flag = v & ~kValue;
        if (flag == 0) {
          if (!start) start = ptx::now_ns();
          else if (ptx::now_ns() - start > ptx::kWaitNs) {
            atomicOr(err, 1);
            break;
          }
          continue;
        }
        before += v & kValue;
        if (flag == kFlagPre || tt == 0) break;
        tt--;
      }
      st_volatile(my, kFlagPre | (before + total));
    }
    s_before = before;
    if ((t + 1) * TILE >= n) *distinct = (unsigned long long)(before + total);
  }
  __syncthreads();
  unsigned int cur = s_before + ex;
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const int64_t p = p0 + i;
    if (p < n) {
      if (hmask >> i & 1u) {
        first[cur] = r[i];
        cur++;
      }
      rank[r[i]] = cur - 1;
    }
  }
}

// The ranks of the sorted pairs when the rank array is too large for L2:
// each tile of sorted positions (claimed in order; it arrives in shared
// memory by bulk copies) finds its keys' run heads and ranks (ballots count
// the heads before each position within a warp, the warps' counts give the
// tile's own, published at once, and a look-back by one warp over 32 earlier
// tiles' counts at a time gives its first rank), writes first[r] for its
// heads, and partitions its (row, rank) pairs by bucket = row >> bshift, each
// bucket's pairs of all tiles in one contiguous region (bucket b holds
// exactly the rows [b << bshift, (b + 1) << bshift) of the n, so its region's
// start is known; a look-back over the earlier tiles' bucket counts, four
// tiles at a time, gives this tile's place in it). The order of pairs within
// a bucket is of no consequence: scatter_ranks then writes rank[row] for each
// pair, and the pairs of one bucket, read in order, fall in one rank range of
// 2^bshift rows that stays in L2 while it is written. Item i of a lane is
// position warp·32·ITEMS + 32i + lane of the tile; the rows stay in shared
// memory and a lane keeps only its items' ranks and bucket slots, so that
// three blocks fit an SM.
constexpr int kBuckets = 256;
template <int W>
constexpr int part_items() { return W == 1 ? 20 : (W == 2 ? 8 : (W == 3 ? 6 : 4)); }

// Sums a value over a warp.
__device__ __forceinline__ unsigned int warp_sum(unsigned int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int W, int ITEMS>
__global__ void __launch_bounds__(kThreads, 3) rank_partition(const uint64_t* __restrict__ keys, int64_t ld,
                                                              const uint32_t* __restrict__ rows, int64_t n, int bshift,
                                                              uint32_t* __restrict__ head_status,
                                                              uint32_t* __restrict__ bucket_status,
                                                              unsigned int* __restrict__ tile_counter,
                                                              uint64_t* __restrict__ pairs, uint32_t* __restrict__ first,
                                                              unsigned long long* __restrict__ distinct, int* err) {
  constexpr int TILE = kThreads * ITEMS;
  constexpr int WARPS = kThreads / 32;
  typedef cub::BlockScan<unsigned int, kThreads> Scan;
  __shared__ typename Scan::TempStorage tmp;
  extern __shared__ __align__(128) uint8_t smem[];
  uint64_t* kstage = (uint64_t*)smem;                 // [W][TILE]: the tile's key words; then its reordered pairs
  uint32_t* rstage = (uint32_t*)(kstage + W * TILE);  // [TILE]: its rows
  uint64_t* spairs = kstage;
  __shared__ __align__(8) uint64_t bar;
  __shared__ unsigned int s_tile, s_before;
  __shared__ unsigned int wheads[WARPS];      // each warp's heads
  __shared__ unsigned int cnt[kBuckets];      // this tile's pairs of each bucket
  __shared__ unsigned int at[kBuckets];       // a bucket's first slot in the tile's reordered pairs
  __shared__ long long dbase[kBuckets];       // a bucket's destination minus its first slot in the tile
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  if (tid == 0) {
    s_tile = atomicAdd(tile_counter, 1u);
    ptx::mbar_init(&bar, 1);
    ptx::mbar_fence_init();
  }
  cnt[tid] = 0;
  __syncthreads();
  const int64_t t = s_tile;
  const int64_t base = t * TILE;
  const int count = (int)min((int64_t)TILE, n - base);
  const int kb = count & ~1, rb = count & ~3;  // keys and rows the bulk copies bring
  if (tid == 0) {
    ptx::mbar_expect_tx(&bar, (uint32_t)(kb * 8 * W + rb * 4));
    if (kb)
#pragma unroll
      for (int w = 0; w < W; w++) ptx::bulk_load(kstage + w * TILE, keys + (int64_t)w * ld + base, (uint32_t)(kb * 8), &bar);
    if (rb) ptx::bulk_load(rstage, rows + base, (uint32_t)(rb * 4), &bar);
  }
  if (!ptx::mbar_wait(&bar, 0)) {
    // The copies didn't land in time: fail the sort, and wait once more for
    // them before the block's shared memory goes.
    atomicOr(err, 1);
    ptx::mbar_wait(&bar, 0);
  }
  auto key_at = [&](int j, int w) -> uint64_t {
    return j < kb ? kstage[w * TILE + j] : keys[(int64_t)w * ld + base + j];
  };
  auto row_at = [&](int j) -> uint32_t { return j < rb ? rstage[j] : rows[base + j]; };
  // Heads, and the heads at or before each item within the warp (the rows
  // stay in the stage).
  uint32_t hrank[ITEMS];  // that count (bit 31: the item is a head); then the item's rank
  unsigned int wcount = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const int j = warp * 32 * ITEMS + i * 32 + lane;
    bool h = false;
    if (j < count) {
      h = base + j == 0;
#pragma unroll
      for (int w = 0; w < W; w++) {
        const uint64_t prev = j > 0 ? key_at(j - 1, w) : (base > 0 ? keys[(int64_t)w * ld + base - 1] : 0);
        h |= key_at(j, w) != prev;
      }
    }
    const unsigned heads = __ballot_sync(0xffffffffu, h);
    hrank[i] = (wcount + __popc(heads & lt_mask) + (h ? 1u : 0u)) | (h ? 0x80000000u : 0u);
    wcount += __popc(heads);
  }
  if (lane == 0) wheads[warp] = wcount;
  __syncthreads();
  unsigned int woff = 0, total = 0;
#pragma unroll
  for (int w = 0; w < WARPS; w++) {
    woff += w < warp ? wheads[w] : 0u;
    total += wheads[w];
  }
  // The heads before this tile: published at once, then a look-back by
  // warp 0 over 32 earlier tiles' counts at a time (flags only go from none
  // to count to prefix, so an early read of a count stays valid).
  if (warp == 0) {
    uint32_t* my = head_status + t;
    if (lane == 0) st_volatile(my, (t == 0 ? kFlagPre : kFlagAgg) | total);
    unsigned int before = 0;
    if (t > 0) {
      int64_t tt = t - 1;
      uint64_t start = 0;
      while (true) {
        const int64_t idx = tt - lane;
        const uint32_t v = idx >= 0 ? ld_volatile(head_status + idx) : kFlagPre;
        const uint32_t flag = v & ~kValue;
        const unsigned waiting = __ballot_sync(0xffffffffu, flag == 0);
        const unsigned prefix = __ballot_sync(0xffffffffu, flag == kFlagPre);
        const int f0 = waiting ? __ffs(waiting) - 1 : 32, p = prefix ? __ffs(prefix) - 1 : 32;
        if (p < f0) {
          before += warp_sum(lane <= p ? v & kValue : 0u);
          break;
        }
        before += warp_sum(lane < f0 ? v & kValue : 0u);
        tt -= f0;
        if (f0 == 0) {
          // Lane 0's clock decides, so that the warp leaves together.
          if (!start) start = ptx::now_ns();
          if (__shfl_sync(0xffffffffu, ptx::now_ns() - start > ptx::kWaitNs ? 1 : 0, 0)) {
            if (lane == 0) atomicOr(err, 1);
            break;
          }
        }
      }
      if (lane == 0) st_volatile(my, kFlagPre | (before + total));
    }
    if (lane == 0) {
      s_before = before;
      if (base + TILE >= n) *distinct = (unsigned long long)(before + total);
    }
  }
  __syncthreads();
  // Ranks; first rows; the pairs' bucket counts.
  const unsigned int first_rank = s_before + woff;
  uint32_t slot[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const int j = warp * 32 * ITEMS + i * 32 + lane;
    if (j < count) {
      const uint32_t ri = row_at(j);
      const unsigned int rk = first_rank + (hrank[i] & 0x7fffffffu) - 1u;
      if (hrank[i] >> 31) first[rk] = ri;
      hrank[i] = rk;
      slot[i] = atomicAdd(&cnt[ri >> bshift], 1u);
    }
  }
  __syncthreads();
  const unsigned int mine = cnt[tid];
  const int64_t bucket_rows = (int64_t)1 << bshift;
  uint32_t* bst = bucket_status + t * kBuckets + tid;
  st_volatile(bst, (t == 0 ? kFlagPre : kFlagAgg) | mine);
  unsigned int bex;
  Scan(tmp).ExclusiveSum(mine, bex);
  unsigned int bbefore = 0;
  if (t > 0) {
    constexpr int kWindow = 4;
    int64_t tt = t - 1;
    uint64_t start = 0;
    bool failed = false;
    while (true) {
      uint32_t v[kWindow];
#pragma unroll
      for (int k = 0; k < kWindow; k++) v[k] = tt - k >= 0 ? ld_volatile(bucket_status + (tt - k) * kBuckets + tid) : 0u;
      bool done = false;
      int used = 0;
#pragma unroll
      for (int k = 0; k < kWindow; k++) {
        if (done || used < k || tt - k < 0) continue;
        const uint32_t flag = v[k] & ~kValue;
        if (flag == 0) continue;
        bbefore += v[k] & kValue;
        used = k + 1;
        if (flag == kFlagPre) done = true;
      }
      if (done) break;
      if (used == 0) {
        if (!start) start = ptx::now_ns();
        else if (ptx::now_ns() - start > ptx::kWaitNs) {
          failed = true;
          break;
        }
      }
      tt -= used;
    }
    if (failed) atomicOr(err, 1);
    st_volatile(bst, kFlagPre | (bbefore + mine));
  }
  at[tid] = bex;
  dbase[tid] = (long long)tid * bucket_rows + (long long)bbefore - (long long)bex;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const int j = warp * 32 * ITEMS + i * 32 + lane;
    if (j < count) {
      const uint32_t ri = row_at(j);
      spairs[at[ri >> bshift] + slot[i]] = ((uint64_t)ri << 32) | hrank[i];
    }
  }
  __syncthreads();
  for (int j = tid; j < count; j += kThreads) {
    const uint64_t x = spairs[j];
    const int b = (int)((uint32_t)(x >> 32) >> bshift);
    __stcs(&pairs[dbase[b] + j], x);
  }
}

__global__ void scatter_ranks(const uint64_t* __restrict__ pairs, int64_t n, uint32_t* __restrict__ rank) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t x = __ldcs(&pairs[i]);
    rank[(uint32_t)(x >> 32)] = (uint32_t)x;
  }
}

template <int W>
__global__ void head_flags(const uint64_t* __restrict__ keys, int64_t n, int64_t ld, uint8_t* __restrict__ head) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    bool h = i == 0;
    if (!h)
#pragma unroll
      for (int w = 0; w < W; w++) h |= keys[(int64_t)w * ld + i] != keys[(int64_t)w * ld + i - 1];
    head[i] = h;
  }
}

__global__ void finish_ranks(const uint8_t* __restrict__ head, const int64_t* __restrict__ before,
                             const uint32_t* __restrict__ rows, int64_t n, uint32_t* __restrict__ rank,
                             uint32_t* __restrict__ first) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = before[i] + head[i] - 1;
    rank[rows[i]] = (uint32_t)r;
    if (head[i]) first[r] = rows[i];
  }
}

// One stable pass of the LSD sort over n (key, row) pairs on byte `shift`
// of key word `word`: digit counts per chunk, one scan, the downsweep. With
// vin null the rows are the positions; with vout null they aren't written.
template <int W>
void radix_pass(Context& ctx, const uint64_t* kin, int64_t ldi, const uint32_t* vin, uint64_t* kout, int64_t ldo,
                uint32_t* vout, int64_t n, int word, int shift, int* err, cudaStream_t s) {
  constexpr int ITEMS = W == 1 ? 8 : (W == 2 ? 6 : 4);
  constexpr int TILE = kThreads * ITEMS;
  // Chunks: as many as blocks resident at once, each a whole number of tiles.
  int per_sm = 0;
  const size_t smem = 2 * (size_t)TILE * (8 * W + 4);
  EF_CUDA(cudaFuncSetAttribute(chunk_scatter<W, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  EF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chunk_scatter<W, ITEMS>, kThreads, smem));
  int64_t chunks = (int64_t)std::max(1, per_sm) * ctx.sm_count;
  const int64_t chunk = ((n + chunks - 1) / chunks + TILE - 1) / TILE * TILE;
  chunks = (n + chunk - 1) / chunk;
  DeviceBuffer<unsigned long long> table((size_t)(256 * chunks), s);
  DeviceBuffer<long long> offsets((size_t)(256 * chunks), s);
  size_t temp = 0;
  EF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, table.get(), offsets.get(), (int)(256 * chunks), s));
  DeviceBuffer<uint8_t> scan_tmp(temp ? temp : 1, s);
  EF_CUDA(cudaMemsetAsync(table.get(), 0, (size_t)(256 * chunks) * 8, s));
  chunk_counts<<<dim3((unsigned)chunks, kCountSplit), kThreads, 0, s>>>(kin + (int64_t)word * ldi, n, shift, chunk,
                                                                        (int)chunks, table.get());
  EF_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.get(), temp, table.get(), offsets.get(), (int)(256 * chunks), s));
  chunk_scatter<W, ITEMS><<<(unsigned)chunks, kThreads, smem, s>>>(kin, vin, kout, vout, n, ldi, ldo, word, shift,
                                                                   chunk, (int)chunks, offsets.get(), err);
  EF_LAUNCH_CHECK();
  ctx.kernels += 3;
}

// The one-sweep ranking (n < 2^30, so that a status word holds a count
// and its flag): one read of the keys for every byte's histogram, one kernel
// per pass over the bytes that vary, and one for the ranks.
template <int W>
int64_t rank_keys_onesweep(Context& ctx, const uint64_t* keys, int64_t n, int64_t ld, uint32_t* rank,
                           uint32_t* first, cudaStream_t s, uint32_t* sorted_rows) {
  constexpr int ITEMS = W == 1 ? 20 : (W == 2 ? 8 : (W == 3 ? 6 : 4));
  constexpr int MIN_BLOCKS = 3;
  constexpr int TILE = kThreads * ITEMS;
  constexpr int RITEMS = 8;
  constexpr int RTILE = kThreads * RITEMS;
  const int64_t tiles = (n + TILE - 1) / TILE;
  const int64_t rtiles = (n + RTILE - 1) / RTILE;
  // The passes' bulk copies read 16-byte aligned words: copy keys that aren't.
  DeviceBuffer<uint64_t> aligned;
  if (((uintptr_t)keys & 15) || (W > 1 && (ld & 1))) {
    const int64_t lda = (n + 1) & ~(int64_t)1;
    aligned.allocate((size_t)(W * lda), s);
    EF_CUDA(cudaMemcpy2DAsync(aligned.get(), (size_t)lda * 8, keys, (size_t)ld * 8, (size_t)n * 8, W,
                              cudaMemcpyDeviceToDevice, s));
    keys = aligned.get();
    ld = lda;
  }
  DeviceBuffer<unsigned long long> hist((size_t)(8 * W * 256), s);
  hist.zero();
  byte_histograms<W><<<blocks_for((uint64_t)n, kThreads, (unsigned)ctx.sm_count * 8u), kThreads, 0, s>>>(keys, n, ld,
                                                                                                       hist.get());
  ctx.kernels++;
  EF_LAUNCH_CHECK();
  std::vector<unsigned long long> h((size_t)(8 * W * 256));
  EF_CUDA(cudaMemcpyAsync(h.data(), hist.get(), h.size() * 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  // Passes: the least significant byte of the last word first; a byte whose
  // values are all one (a bin holds every key) is skipped.
  std::vector<int> pw, ps;
  std::vector<uint32_t> starts;
  for (int w = W - 1; w >= 0; w--)
    for (int b = 0; b < 8; b++) {
      const unsigned long long* c = &h[(size_t)(8 * w + b) * 256];
      bool varies = true;
      for (int d = 0; d < 256; d++)
        if (c[d] == (unsigned long long)n) varies = false;
      if (!varies) continue;
      pw.push_back(w);
      ps.push_back(8 * b);
      uint32_t acc = 0;
      for (int d = 0; d < 256; d++) {
        starts.push_back(acc);
        acc += (uint32_t)c[d];
      }
    }
  const int passes = (int)pw.size();
  DeviceBuffer<uint32_t> dstart((size_t)std::max(1, passes) * 256, s);
  if (passes) EF_CUDA(cudaMemcpyAsync(dstart.get(), starts.data(), starts.size() * 4, cudaMemcpyHostToDevice, s));
  constexpr int PTILE = kThreads * part_items<W>();
  const int64_t status_words = std::max(tiles * 256, std::max(rtiles, (n + PTILE - 1) / PTILE));
  DeviceBuffer<uint32_t> status((size_t)status_words, s);
  DeviceBuffer<unsigned int> counters((size_t)passes + 1, s);
  counters.zero();
  DeviceBuffer<int> err(1, s);
  err.zero();
  DeviceBuffer<uint64_t> kb[2];
  DeviceBuffer<uint32_t> vb[2];
  const uint64_t* cur_k = keys;
  int64_t cur_ld = ld;
  const uint32_t* cur_v = nullptr;
  const size_t smem = (size_t)TILE * (8 * W + 4 + 1);
  if (passes) {
    const int64_t ldb = (n + 1) & ~(int64_t)1;
    for (int b = 0; b < 2; b++) {
      kb[b].allocate((size_t)(W * ldb), s);
      vb[b].allocate((size_t)n, s);
    }
    EF_CUDA(cudaFuncSetAttribute(onesweep_pass<W, ITEMS, MIN_BLOCKS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (int p = 0; p < passes; p++) {
      EF_CUDA(cudaMemsetAsync(status.get(), 0, (size_t)tiles * 256 * 4, s));
      onesweep_pass<W, ITEMS, MIN_BLOCKS><<<(unsigned)tiles, kThreads, smem, s>>>(
          cur_k, cur_v, kb[p & 1].get(), vb[p & 1].get(), n, cur_ld, ldb, pw[p], ps[p], dstart.get() + p * 256,
          status.get(), counters.get() + p, err.get());
      ctx.kernels++;
      cur_k = kb[p & 1].get();
      cur_ld = ldb;
      cur_v = vb[p & 1].get();
    }
    EF_LAUNCH_CHECK();
  }
  DeviceBuffer<uint32_t> identity;
  if (!cur_v) {
    identity.allocate((size_t)n, s);
    thrust_iota(ctx, identity.get(), n, s);
    cur_v = identity.get();
  }
  DeviceBuffer<unsigned long long> distinct(1, s);
  // The finish's per-tile head counts start unpublished (either finish's tiles).
  EF_CUDA(cudaMemsetAsync(status.get(), 0, (size_t)std::max(rtiles, (n + PTILE - 1) / PTILE) * 4, s));
  if (n <= kScatterInL2) {
    // The rank array fits in L2: its scattered writes merge there.
    rank_runs<W, RITEMS><<<(unsigned)rtiles, kThreads, 0, s>>>(cur_k, cur_ld, cur_v, n, status.get(),
                                                               counters.get() + passes, rank, first, distinct.get(),
                                                               err.get());
    ctx.kernels++;
  } else {
    // Ranks partitioned by the rows' high bits, then scattered bucket by bucket.
    int bshift = 0;
    while ((((int64_t)1 << bshift) * kBuckets) < n) bshift++;
    const int64_t ptiles = (n + PTILE - 1) / PTILE;
    DeviceBuffer<uint32_t> bstatus((size_t)(ptiles * kBuckets), s);
    DeviceBuffer<uint64_t> pairs((size_t)n, s);
    EF_CUDA(cudaMemsetAsync(bstatus.get(), 0, (size_t)(ptiles * kBuckets) * 4, s));
    const size_t psmem = (size_t)PTILE * (8 * W + 4);
    EF_CUDA(cudaFuncSetAttribute(rank_partition<W, part_items<W>()>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)psmem));
    rank_partition<W, part_items<W>()><<<(unsigned)ptiles, kThreads, psmem, s>>>(
        cur_k, cur_ld, cur_v, n, bshift, status.get(), bstatus.get(), counters.get() + passes, pairs.get(), first,
        distinct.get(), err.get());
    scatter_ranks<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(pairs.get(), n, rank);
    ctx.kernels += 2;
  }
  EF_LAUNCH_CHECK();
  if (sorted_rows) EF_CUDA(cudaMemcpyAsync(sorted_rows, cur_v, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  unsigned long long k = 0;
  int e = 0;
  EF_CUDA(cudaMemcpyAsync(&k, distinct.get(), 8, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaMemcpyAsync(&e, err.get(), 4, cudaMemcpyDeviceToHost, s));
  EF_CUDA(cudaStreamSynchronize(s));
  if (e) fail(EINFOLD_TIMEOUT, "a bounded wait in the radix sort ran out");
  return (int64_t)k;
}

template <int W>
int64_t rank_keys_w(Context& ctx, const uint64_t* keys, int64_t n, int64_t ld, uint32_t* rank, uint32_t* first,
                    cudaStream_t s, uint32_t* sorted_rows) {
  if (n <= 0) return 0;
  // TMA bulk copies read 16-byte aligned words: copy keys that aren't.
  DeviceBuffer<uint64_t> aligned;
  if (((uintptr_t)keys & 15) || (W > 1 && (ld & 1))) {
    const int64_t lda = (n + 1) & ~(int64_t)1;
    aligned.allocate((size_t)(W * lda), s);
    EF_CUDA(cudaMemcpy2DAsync(aligned.get(), (size_t)lda * 8, keys, (size_t)ld * 8, (size_t)n * 8, W,
                              cudaMemcpyDeviceToDevice, s));
    keys = aligned.get();
    ld = lda;
  }
  if (n >= (int64_t)UINT32_MAX) fail(EINFOLD_COMPUTE, "ranking at most 2^32 - 1 rows together");
  DeviceBuffer<unsigned long long> acc(2 * W, s);
  {
    std::vector<unsigned long long> init(2 * W);
    for (int w = 0; w < W; w++) { init[2 * w] = 0; init[2 * w + 1] = ~0ull; }
    EF_CUDA(cudaMemcpyAsync(acc.get(), init.data(), init.size() * 8, cudaMemcpyHostToDevice, s));
    or_and_words<W><<<blocks_for(n, 256), 256, 0, s>>>(keys, n, ld, acc.get());
    ctx.kernels++;
    std::vector<unsigned long long> got(2 * W);
    EF_CUDA(cudaMemcpyAsync(got.data(), acc.get(), got.size() * 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    init = got;
    // Passes: least significant byte of the last word first; bytes no key varies in are skipped.
    std::vector<int> pw, ps;
    for (int w = W - 1; w >= 0; w--)
      for (int sh = 0; sh < 64; sh += 8)
        if (((init[2 * w] ^ init[2 * w + 1]) >> sh) & 0xff) {
          pw.push_back(w);
          ps.push_back(sh);
        }
    const int passes = (int)pw.size();
    DeviceBuffer<uint64_t> kb[2];
    DeviceBuffer<uint32_t> vb[2];
    const uint64_t* cur_k = keys;
    int64_t cur_ld = ld;
    const uint32_t* cur_v = nullptr;
    DeviceBuffer<int> err(1, s);
    err.zero();
    if (passes) {
      const int64_t ldb = (n + 1) & ~(int64_t)1;
      for (int b = 0; b < 2; b++) {
        kb[b].allocate((size_t)(W * ldb), s);
        vb[b].allocate((size_t)n, s);
      }
      for (int p = 0; p < passes; p++) {
        radix_pass<W>(ctx, cur_k, cur_ld, cur_v, kb[p & 1].get(), ldb, vb[p & 1].get(), n, pw[p], ps[p], err.get(), s);
        cur_k = kb[p & 1].get();
        cur_ld = ldb;
        cur_v = vb[p & 1].get();
      }
    }
    DeviceBuffer<uint32_t> identity;
    if (!cur_v) {
      // No byte varies: every key is the same; rows stay in order.
      identity.allocate((size_t)n, s);
      thrust_iota(ctx, identity.get(), n, s);
      cur_v = identity.get();
    }
    DeviceBuffer<uint8_t> head((size_t)n, s);
    DeviceBuffer<int64_t> before((size_t)n, s);
    head_flags<W><<<blocks_for(n, 256), 256, 0, s>>>(cur_k, n, cur_ld, head.get());
    ctx.kernels++;
    const int64_t distinct = exclusive_scan_flags(ctx, head.get(), n, before.get());
    finish_ranks<<<blocks_for(n, 256), 256, 0, s>>>(head.get(), before.get(), cur_v, n, rank, first);
    ctx.kernels++;
    if (sorted_rows) EF_CUDA(cudaMemcpyAsync(sorted_rows, cur_v, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    EF_LAUNCH_CHECK();
    int e = 0;
    EF_CUDA(cudaMemcpyAsync(&e, err.get(), 4, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    if (e) fail(EINFOLD_TIMEOUT, "a bounded wait in the radix sort ran out");
    return distinct;
  }
}

}  // namespace

__global__ void iota_kernel(uint32_t* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

void thrust_iota(Context& ctx, uint32_t* out, int64_t n, cudaStream_t s) {
  iota_kernel<<<blocks_for(n, 256), 256, 0, s>>>(out, n);
  ctx.kernels++;
}

int64_t rank_keys(Context& ctx, const uint64_t* keys, int words, int64_t n, int64_t ld, uint32_t* rank,
                  uint32_t* first, cudaStream_t s, uint32_t* sorted_rows) {
  if (n <= 0) return 0;
  // The one-sweep passes below 2^30 keys (a status word's count); the
  // chunked passes beyond, or when EINFOLD_RANK_CHUNKED is set.
  static const bool chunked = std::getenv("EINFOLD_RANK_CHUNKED") != nullptr;
  if (n < ((int64_t)1 << 30) && !chunked) {
    switch (words) {
      case 1: return rank_keys_onesweep<1>(ctx, keys, n, ld, rank, first, s, sorted_rows);
      case 2: return rank_keys_onesweep<2>(ctx, keys, n, ld, rank, first, s, sorted_rows);
      case 3: return rank_keys_onesweep<3>(ctx, keys, n, ld, rank, first, s, sorted_rows);
      case 4: return rank_keys_onesweep<4>(ctx, keys, n, ld, rank, first, s, sorted_rows);
      default: fail(EINFOLD_INVALID, "keys of %d words", words);
    }
  }
  switch (words) {
    case 1: return rank_keys_w<1>(ctx, keys, n, ld, rank, first, s, sorted_rows);
    case 2: return rank_keys_w<2>(ctx, keys, n, ld, rank, first, s, sorted_rows);
    case 3: return rank_keys_w<3>(ctx, keys, n, ld, rank, first, s, sorted_rows);
    case 4: return rank_keys_w<4>(ctx, keys, n, ld, rank, first, s, sorted_rows);
    default: fail(EINFOLD_INVALID, "keys of %d words", words);
  }
}

}  // namespace ef
